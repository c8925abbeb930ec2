"""The C ABI without a GPU: the libraries load, every symbol declared in
include/*.h is exported, argument errors are returned (never trapped) before
any device work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from wind_b200 import _capi, lib, networks as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(wind_\w+|cudaIntegrate\w+)\s*\(",
                                 src, flags=re.M)))


def test_libwind_exports_every_declared_symbol():
    names = _declared("wind.h")
    assert "wind_integrate" in names and "wind_integrate_batch_noalloc" in names
    dll = C.CDLL(lib.library_path())
    for n in names:
        assert hasattr(dll, n), f"{n} declared in include/wind.h but not exported"


@pytest.mark.parametrize("net", ["nr_test", "katz96", "stifftrig"])
@pytest.mark.parametrize("method", ["sie", "rk2"])
def test_legacy_libraries_export_reference_symbol(net, method):
    assert _declared("wind_legacy.h") == ["cudaIntegrateSIE", "cudaIntegrateSystem"]
    fn = lib.legacy(net, method)  # looks up _Z19cudaIntegrateSystemffiPfS_iiff
    assert fn is not None


@pytest.mark.parametrize("net", ["nr_test", "katz96", "stifftrig"])
def test_sie_host_libraries_export_reference_symbol(net):
    fn = lib.legacy_host(net)  # looks up _Z16cudaIntegrateSIEffiPfS_iiff
    assert fn is not None


def test_global_entry_argument_errors():
    w = lib.load()
    wl = W.workload_mixed_class(5, 2, dt=1e-3)
    ns = _capi.network_struct(wl.net)
    y = wl.y0.copy()
    o = lib.options("sie", "gje_f64", "gold")
    tot, t = C.c_int64(0), C.c_double(0.0)
    # mass action is outside the SIE_host variant's scope
    assert w.wind_integrate_global(C.byref(o), C.byref(ns), 0.0, 1e-3, 1, y.ctypes.data, 2, 1e-8,
                                   1e-6, C.byref(tot), C.byref(t), _capi.MEM_HOST,
                                   None) == _capi.WIND_ERR_UNSUPPORTED
    k = W.workload_katz96(2)
    ks = _capi.network_struct(k.net)
    yk = k.y0.copy()
    for bad in (dict(method=_capi.METHODS["rk2"]), dict(solver=7)):
        ob = lib.options("sie", "gje_f64", "gold")
        for f, v in bad.items():
            setattr(ob, f, v)
        assert w.wind_integrate_global(C.byref(ob), C.byref(ks), 0.0, 1.0, 1, yk.ctypes.data, 2,
                                       1e-8, 1e-6, C.byref(tot), C.byref(t), _capi.MEM_HOST,
                                       None) == _capi.WIND_ERR_ARGUMENT
    assert w.wind_integrate_global(C.byref(o), C.byref(ks), 0.0, 1.0, 0, yk.ctypes.data, 2, 1e-8,
                                   1e-6, C.byref(tot), C.byref(t), _capi.MEM_HOST,
                                   None) == _capi.WIND_ERR_ARGUMENT
    # tiled networks are integrated by wind_integrate, not by the shared-step variant
    kt = W.tile_workload(k, 3)
    ts = _capi.network_struct(kt.net)
    yt = kt.y0.copy()
    assert w.wind_integrate_global(C.byref(o), C.byref(ts), 0.0, 1.0, 1, yt.ctypes.data, 2, 1e-8,
                                   1e-6, C.byref(tot), C.byref(t), _capi.MEM_HOST,
                                   None) == _capi.WIND_ERR_UNSUPPORTED


def test_defaults_and_strings():
    w = lib.load()
    o = _capi.WindOptions()
    w.wind_default_options(C.byref(o))
    assert (o.method, o.solver, o.controller, o.spec_width) == (0, 0, 0, 0)
    assert b"sm_100a" in w.wind_version()
    assert w.wind_status_string(1) == b"invalid argument"


def _call(net, y, **kw):
    w = lib.load()
    o = lib.options(**kw)
    ns = _capi.network_struct(net)
    return w.wind_integrate(C.byref(o), C.byref(ns), 0.0, 1.0, 1, y.ctypes.data if y is not None else None,
                            net.nsys, 1e-6, 1e-6, None, None, None, _capi.MEM_HOST, None)


def test_argument_errors_are_returned():
    net = W.nr_test(4)
    y = np.ones((4, 2))
    w = lib.load()
    o = lib.options()
    o.method = 7
    ns = _capi.network_struct(net)
    assert w.wind_integrate(C.byref(o), C.byref(ns), 0.0, 1.0, 1, y.ctypes.data, 4, 1e-6, 1e-6,
                            None, None, None, 0, None) == _capi.WIND_ERR_ARGUMENT
    # wrong equation count for the builtin network (not a whole number of tiles)
    bad = W.Network(W.NET_NR_TEST, 3, 4, constants=net.constants)
    assert _call(bad, y) == _capi.WIND_ERR_ARGUMENT
    kc = W.workload_katz96(4).net.constants
    assert _call(W.Network(W.NET_KATZ96, 12, 4, constants=kc), np.ones((4, 12))) == \
        _capi.WIND_ERR_ARGUMENT
    # more tiles than the tiled kernel holds
    assert _call(W.Network(W.NET_KATZ96, 5 * 65, 4, constants=kc), np.ones((4, 325))) == \
        _capi.WIND_ERR_UNSUPPORTED
    # missing constants
    bad = W.Network(W.NET_KATZ96, 5, 4)
    assert _call(bad, np.ones((4, 5))) == _capi.WIND_ERR_ARGUMENT
    # unknown network kind
    bad = W.Network(99, 2, 4, constants=net.constants)
    assert _call(bad, y) == _capi.WIND_ERR_ARGUMENT
    # null state with systems to integrate
    assert _call(net, None) == _capi.WIND_ERR_ARGUMENT
    # bad memory flag
    assert w.wind_integrate(C.byref(lib.options()), C.byref(ns), 0.0, 1.0, 1, y.ctypes.data, 4,
                            1e-6, 1e-6, None, None, None, 5, None) == _capi.WIND_ERR_ARGUMENT
    # n_integration_steps < 1
    assert w.wind_integrate(C.byref(lib.options()), C.byref(ns), 0.0, 1.0, 0, y.ctypes.data, 4,
                            1e-6, 1e-6, None, None, None, 0, None) == _capi.WIND_ERR_ARGUMENT


def test_zero_systems_is_a_no_op():
    net = W.nr_test(0)
    assert _call(net, np.ones((0, 2))) == _capi.WIND_OK
    w = lib.load()
    assert w.wind_integrate_batch(C.byref(lib.options()), None, 0, None) == _capi.WIND_OK


def test_sim_and_tensor_core_options_are_checked_before_any_work():
    """The fixed-step SIM method is accepted by wind_integrate only, and the
    tensor-core solver value is in range; both are rejected by the batch and
    serving entry points before anything is launched."""
    w = lib.load()
    o = lib.options("sim", "lu_f64", "gold")
    assert o.method == _capi.METHOD_SIM
    # batch entry points reject the method (no groups are read)
    assert w.wind_integrate_batch(C.byref(o), None, 0, None) == _capi.WIND_ERR_ARGUMENT
    o = lib.options("sie", "mixed_tc", "gold")
    assert o.solver == _capi.SOLVER_MIXED_TC
    o.solver = _capi.SOLVER_MIXED_TC + 1
    net = W.nr_test(4)
    ns = _capi.network_struct(net)
    y = np.ones((4, 2))
    assert w.wind_integrate(C.byref(o), C.byref(ns), 0.0, 1.0, 1, y.ctypes.data, 4, 1e-6, 1e-6,
                            None, None, None, 0, None) == _capi.WIND_ERR_ARGUMENT
