"""GPU parity of the semi-implicit midpoint method (WIND_METHOD_SIM,
python/pysolvers/sim.py:36-90) through the C ABI: against the golden vectors
of the reference's own sim.py and against the oracle, at the FP64 bar."""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import sim_cases as SC
from wind_b200 import _capi, lib, networks as W

pytestmark = pytest.mark.gpu

CASES = SC.load()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_sim_matches_reference_and_oracle(cuda_device, case):
    name, net, y0, dt, m, y_ref = case
    y = y0.copy()
    tot, st, ns = lib.integrate(net, y, 0.0, m * dt, 1e-8, 1e-6, "sim", "lu_f64", "gold", m)
    assert SC.rel_err(y, y_ref) < SC.TOL
    y_o = y0.copy()
    O.restated_sim(net, y_o, 0.0, m * dt, m)
    assert SC.rel_err(y, y_o) < SC.TOL
    assert tot == net.nsys * (m + 1)
    assert np.all(ns == m + 1) and np.all(st == 0)


@pytest.mark.parametrize("which", ["katz96", "dense32", "ma16"])
def test_sim_batch_vs_oracle(cuda_device, which):
    """Batches that fill the persistent grid several times over."""
    if which == "katz96":
        wl = W.workload_katz96(20000, seed=310)
        dt, m = 5e7, 40
    elif which == "dense32":
        wl = W.workload_dense(600, first=4096)
        dt, m = 1e-4, 30
    else:
        wl = W.workload_mixed_class(16, 3000, seed=311, dt=1.0)
        dt, m = 1e-5, 40
    y = wl.y0.copy()
    tot, st, ns = lib.integrate(wl.net, y, 0.0, m * dt, 1e-8, 1e-6, "sim", "auto", "gold", m)
    y_o = wl.y0.copy()
    O.restated_sim(wl.net, y_o, 0.0, m * dt, m)
    fin = np.isfinite(y_o).all(axis=1)
    assert fin.mean() > 0.99
    assert SC.rel_err_systemwise(y[fin], y_o[fin]) < SC.TOL
    assert tot == wl.net.nsys * (m + 1)


def test_sim_device_arrays_and_timeout(cuda_device):
    """Device-memory call; a tiny device deadline stops a long run with the
    TIMEOUT bit on every system (no fault: the kernel checks the clock)."""
    import torch
    wl = W.workload_katz96(4096, seed=312)
    d = {"constants": torch.from_numpy(wl.net.constants).to(cuda_device)}
    y = torch.from_numpy(wl.y0.copy()).to(cuda_device)
    tot, st, ns = lib.integrate(wl.net, y, 0.0, 1e9, 1e-8, 1e-6, "sim", "lu_f64", "gold", 10,
                                device_arrays=d)
    y_o = wl.y0.copy()
    O.restated_sim(wl.net, y_o, 0.0, 1e9, 10)
    assert SC.rel_err_systemwise(y.cpu().numpy(), y_o) < SC.TOL
    y2 = wl.y0.copy()
    _, st2, ns2 = lib.integrate(wl.net, y2, 0.0, 1e9, 1e-8, 1e-6, "sim", "lu_f64", "gold",
                                2_000_000, timeout_s=1e-4)
    assert np.all(st2 & _capi.SYS_TIMEOUT)
    assert np.all(ns2 < 2_000_001)


def test_sim_unsupported_shapes(cuda_device):
    k = W.workload_katz96(8, seed=313)
    y = k.y0.copy()
    with pytest.raises(lib.WindError) as e:
        lib.integrate(k.net, y, 0.0, 1e8, 1e-8, 1e-6, "sim", "gje_f64", "gold", 4)
    assert e.value.code == _capi.WIND_ERR_UNSUPPORTED
    big = W.workload_mixed_class(64, 2, seed=314, dt=1.0)
    with pytest.raises(lib.WindError) as e:
        lib.integrate(big.net, big.y0.copy(), 0.0, 1e-4, 1e-8, 1e-6, "sim", "lu_f64", "gold", 4)
    assert e.value.code == _capi.WIND_ERR_UNSUPPORTED
    with pytest.raises(lib.WindError) as e:
        lib.integrate_batch([k], method="sim", solver="lu_f64", controller="gold")
    assert e.value.code == _capi.WIND_ERR_ARGUMENT


def test_sim_output_steps_equal_consecutive_calls(cuda_device):
    """wind_integrate_output_steps with SIM: each output interval is one
    m-step call, the same as consecutive wind_integrate calls."""
    wl = W.workload_katz96(512, seed=315)
    y = wl.y0.copy()
    traj, steps = lib.integrate_output_steps(wl.net, y, 0.0, 3e8, 1e-8, 1e-6, 3, 8, "sim",
                                             "lu_f64", "gold")
    y_c = wl.y0.copy()
    for k in range(3):
        lib.integrate(wl.net, y_c, k * 1e8, (k + 1) * 1e8, 1e-8, 1e-6, "sim", "lu_f64", "gold", 8)
        assert np.array_equal(traj[k + 1], y_c)
    assert np.array_equal(y, y_c)
    assert np.all(steps == 512 * 9)
