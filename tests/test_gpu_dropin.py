"""The drop-in libraries and the device-resident output loop, on the GPU.

* lib/<network>/{sie,rk2}.so export the reference's mangled
  cudaIntegrateSystem and are called exactly as python/ode_systems/
  ode_base.py:441-469 calls them (float32 host arrays, in-place update, int
  step total).  The state runs in FP64 with the reference GPU kernel's
  controller; results must equal the oracle (DEVICE semantics) on the same
  float32 inputs, rounded back to float32.
* the golden vectors of the reference's own CPU integrator, on the GPU with
  GOLD semantics, bit for bit.
* wind_integrate_output_steps (CUDA-graph outer loop) equals one
  wind_integrate call per output interval, and the NR test's exact solution.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests.test_oracle import NAMES, golden_case
from wind_b200 import lib, networks as W

pytestmark = pytest.mark.gpu


def _legacy_case(net):
    if net == "katz96":
        wl = W.workload_katz96(64, seed=21)
        return W.Workload(wl.net, wl.y0, 0.0, 1e10, 1e-6, 1e-4, 1, 1)
    if net == "nr_test":
        wl = W.workload_nr(32, seed=22)
        return W.Workload(wl.net, wl.y0, 0.0, 0.005, 1e-8, 1e-6, 1, 1)
    return W.Workload(W.stifftrig(8), np.tile([0.0, 1.0], (8, 1)).astype(np.float64), 0.0, 0.25,
                      1e-6, 1e-6, 1, 1)


@pytest.mark.parametrize("method", ["sie", "rk2"])
@pytest.mark.parametrize("net", ["nr_test", "katz96", "stifftrig"])
def test_legacy_entry_matches_oracle(cuda_device, net, method):
    wl = _legacy_case(net)
    if method == "rk2" and net == "katz96":
        wl = W.Workload(wl.net, wl.y0, 0.0, 1e6, 1e-4, 1e-4, 1, 1)
    fn = lib.legacy(net, method)
    f32 = np.float32
    c32 = np.ascontiguousarray(wl.net.constants.astype(f32))
    y32 = np.ascontiguousarray(wl.y0.astype(f32))
    y_in = y32.copy()  # the call updates y32 in place
    S, N = y32.shape
    nsteps = fn(f32(wl.tnow), f32(wl.tend), 1, c32.ctypes.data, y32.ctypes.data, S, N,
                f32(wl.atol), f32(wl.rtol))
    # the oracle on exactly what the drop-in saw: float32 inputs widened
    net64 = W.Network(wl.net.kind, N, S, constants=c32.astype(np.float64))
    y_o = y_in.astype(np.float64)
    tot, _, _ = O.restated(net64, y_o, float(f32(wl.tnow)), float(f32(wl.tend)),
                           float(f32(wl.atol)), float(f32(wl.rtol)), method, "device")
    assert np.array_equal(y32, y_o.astype(f32))
    assert nsteps == tot


@pytest.mark.parametrize("name", NAMES)
def test_golden_vectors_on_gpu(cuda_device, name):
    wl, method, y_ref, tot_ref = golden_case(name)
    y = wl.y0.copy()
    tot, st, _ = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, method, "gje_f64",
                               "gold", wl.n_integration_steps)
    assert np.array_equal(y, y_ref)
    assert tot == tot_ref


def test_output_steps_graph_equals_calls(cuda_device):
    wl = W.workload_nr(256, seed=3)
    y_graph = wl.y0.copy()
    out, steps = lib.integrate_output_steps(wl.net, y_graph, 0.0, 0.2, wl.atol, wl.rtol, 20)
    y = wl.y0.copy()
    t, dt = 0.0, 0.2 / 20
    assert np.array_equal(out[0], wl.y0)
    for k in range(20):
        tot, _, _ = lib.integrate(wl.net, y, t, t + dt, wl.atol, wl.rtol)
        assert np.array_equal(out[k + 1], y)
        assert steps[k] == tot
        t += dt
    assert np.array_equal(y_graph, y)


def test_nr_config_against_exact_solution(cuda_device):
    """1024 NR systems, t = 0..1 in 100 output steps, rtol 1e-6 / atol 1e-8."""
    wl = W.workload_nr(1024)
    y = wl.y0.copy()
    out, steps = lib.integrate_output_steps(wl.net, y, 0.0, 1.0, wl.atol, wl.rtol, 100)
    exact = W.nr_analytic(wl.y0, 1.0)
    rel = np.max(np.abs(y - exact) / np.abs(exact))
    assert rel < 1e-4, rel  # first-order SIE at rtol 1e-6
    assert steps.sum() > 0
