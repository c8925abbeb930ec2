"""CPU tests of the runtime plug-in compiler (NVRTC runs without a GPU):
the reference-contract plug-in sources compile for sm_100a, a broken
source is an argument error carrying the compiler's message, and the size
limits are checked before anything runs."""
import os

import numpy as np
import pytest

from wind_b200 import _capi, lib

HERE = os.path.dirname(os.path.abspath(__file__))
PLUGINS = os.path.join(os.path.dirname(HERE), "oracle", "plugins")


def source(name):
    with open(os.path.join(PLUGINS, name)) as fh:
        return fh.read()


@pytest.mark.parametrize("name,n,nc,opts", [
    ("nr_test_gold.c", 2, 4, ""),
    ("katz96_tiled_gold.c", 15, 10, "-DNTILE=3"),
    ("mass_action_gold.c", 12, 5 * 30 + 144, "-DMA_N=12 -DMA_R=30 -DMA_LINEAR=1"),
])
def test_reference_contract_sources_compile(name, n, nc, opts):
    p = lib.Plugin(source(name), n, nc, opts)
    assert p.handle
    p.close()


def test_compile_error_is_reported():
    bad = ("#include \"ode_gold.h\"\n"
           "void calculate_dydt(float t, float* y, float* c, float* f, int n) { f[0] = nope; }\n"
           "void calculate_jacobian(float* y, float* c, float* J) {}\n")
    with pytest.raises(lib.WindError) as e:
        lib.Plugin(bad, 2, 1)
    assert e.value.code == _capi.WIND_ERR_ARGUMENT
    assert "nope" in str(e.value)


def test_plugin_limits():
    w = lib.load()
    h = lib.C.c_void_p()
    src = source("nr_test_gold.c").encode()
    assert w.wind_plugin_create(src, 65, 4, None, lib.C.byref(h), None, 0) == _capi.WIND_ERR_UNSUPPORTED
    assert w.wind_plugin_create(src, 0, 4, None, lib.C.byref(h), None, 0) == _capi.WIND_ERR_ARGUMENT
    assert w.wind_plugin_create(None, 2, 4, None, lib.C.byref(h), None, 0) == _capi.WIND_ERR_ARGUMENT
    p = lib.Plugin(source("nr_test_gold.c"), 2, 4)
    y = np.ones((3, 2))
    o = lib.options("sie", "lu_f64")
    # the plug-in path is the reference's Gauss-Jordan algorithm only
    assert w.wind_integrate_plugin(lib.C.byref(o), p.handle, 0.0, 1.0, 1, np.ones((3, 4)).ctypes.data,
                                   y.ctypes.data, 3, 1e-8, 1e-6, None, None, None, 0,
                                   None) == _capi.WIND_ERR_UNSUPPORTED
    assert w.wind_integrate_plugin(lib.C.byref(lib.options()), p.handle, 0.0, 1.0, 1, None,
                                   y.ctypes.data, 3, 1e-8, 1e-6, None, None, None, 0,
                                   None) == _capi.WIND_ERR_ARGUMENT
    assert w.wind_integrate_plugin(lib.C.byref(lib.options()), None, 0.0, 1.0, 1, None,
                                   y.ctypes.data, 3, 1e-8, 1e-6, None, None, None, 0,
                                   None) == _capi.WIND_ERR_ARGUMENT
    p.close()
