"""The SIE_host variant on the GPU: one step shared by every system
(wind_integrate_global, and the mangled cudaIntegrateSIE drop-in of
lib/<network>/sie_host.so), against the oracle's restatement of its
controller (cuda/SIE_host/harness_kernel.cu:248-425)."""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests.helpers import mixed_err
from wind_b200 import lib, networks as W

pytestmark = pytest.mark.gpu


def _cases():
    k = W.workload_katz96(300, seed=51, atol=1e-8, rtol=1e-6)
    # the shared step doubles after every accept and the loop gives up after
    # 9 refinements, so these start from small steps (as its callers must)
    k = W.Workload(k.net, k.y0, 0.0, 1e3, k.atol, k.rtol, 100, 1, "katz96")
    nr = W.workload_nr(200, seed=52)
    nr = W.Workload(nr.net, nr.y0, 0.0, 0.01, nr.atol, nr.rtol, 1000, 1, "nr")
    trig = W.Workload(W.stifftrig(64), np.tile([0.0, 1.0], (64, 1)).astype(np.float64), 0.0, 0.05,
                      1e-6, 1e-6, 1000, 1, "stifftrig")
    return [k, nr, trig]


CASES = _cases()


@pytest.mark.parametrize("wl", CASES, ids=[c.label for c in CASES])
def test_global_gje_bitexact(cuda_device, wl):
    y_o = wl.y0.copy()
    tot_o, t_o = O.restated_global(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol,
                                   wl.n_integration_steps)
    y_g = wl.y0.copy()
    tot_g, t_g = lib.integrate_global(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "gje_f64",
                                      wl.n_integration_steps)
    assert np.array_equal(y_g, y_o)
    assert tot_g == tot_o and t_g == t_o
    assert t_o == wl.tend


@pytest.mark.parametrize("solver", ["lu_f64", "mixed"])
@pytest.mark.parametrize("wl", CASES, ids=[c.label for c in CASES])
def test_global_fast_solvers_close(cuda_device, wl, solver):
    y_o = wl.y0.copy()
    _, t_o = O.restated_global(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol,
                               wl.n_integration_steps)
    y_g = wl.y0.copy()
    _, t_g = lib.integrate_global(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, solver,
                                  wl.n_integration_steps)
    assert t_g == t_o
    assert mixed_err(y_g, y_o, wl.atol) <= 1e-5


def test_global_gives_up_like_the_reference(cuda_device):
    """An unreachable tolerance: 9 refinements, then the loop stops with the
    state untouched (harness_kernel.cu:289)."""
    wl = W.workload_katz96(40, seed=53)
    y = wl.y0.copy()
    tot, t = lib.integrate_global(wl.net, y, 0.0, 1e13, 1e-30, 1e-30)
    assert t == 0.0 and np.array_equal(y, wl.y0) and tot == 9 * 3 * 40


def test_cudaIntegrateSIE_dropin(cuda_device):
    """The mangled SIE_host entry on float32 host arrays equals the oracle's
    restatement run on the same float32 inputs, rounded to float32."""
    wl = CASES[0]
    fn = lib.legacy_host("katz96")
    c32 = wl.net.constants.astype(np.float32)
    y32 = wl.y0.astype(np.float32)
    tnow, tend = np.float32(wl.tnow), np.float32(wl.tend)
    atol, rtol = np.float32(wl.atol), np.float32(wl.rtol)
    net64 = W.Network(wl.net.kind, wl.net.n_eq, wl.net.nsys, constants=c32.astype(np.float64))
    y_o = y32.astype(np.float64)
    tot_o, _ = O.restated_global(net64, y_o, float(tnow), float(tend), float(atol), float(rtol),
                                 wl.n_integration_steps)
    y_in = np.ascontiguousarray(y32.copy())
    ret = fn(tnow, tend, wl.n_integration_steps, c32.ctypes.data, y_in.ctypes.data, wl.net.nsys,
             wl.net.n_eq, atol, rtol)
    assert ret == tot_o
    assert np.array_equal(y_in, y_o.astype(np.float32))
