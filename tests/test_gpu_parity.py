"""GPU parity: the CUDA integrators against the CPU oracle, through the C ABI.

* GJE_F64 (the reference algorithm) must be bit-identical to the FP64
  restatement -- state, per-system substep counts and the total -- for both
  controller semantics and both methods, every network, every speculative
  width.
* LU_F64 and MIXED must stay within the stated tolerance of the FP64 oracle.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests.helpers import small_workloads, rk2_variant, mixed_err
from wind_b200 import lib, networks as W

pytestmark = pytest.mark.gpu

CASES = small_workloads()


def _ids(cases):
    return [c.label for c in cases]


@pytest.mark.parametrize("ctrl", ["gold", "device"])
@pytest.mark.parametrize("wl", CASES, ids=_ids(CASES))
def test_sie_gje_bitexact(cuda_device, wl, ctrl):
    y_o = wl.y0.copy()
    tot_o, st_o, n_o = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", ctrl,
                                  wl.n_integration_steps, threads=8)
    y_g = wl.y0.copy()
    tot_g, st_g, n_g = lib.integrate(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie",
                                     "gje_f64", ctrl, wl.n_integration_steps)
    assert np.array_equal(y_g, y_o), f"max diff {np.max(np.abs(y_g - y_o))}"
    assert np.array_equal(n_g, n_o)
    assert tot_g == tot_o
    assert np.array_equal(st_g, st_o)


@pytest.mark.parametrize("ctrl", ["gold", "device"])
@pytest.mark.parametrize("wl", CASES[:4], ids=_ids(CASES[:4]))
def test_rk2_bitexact(cuda_device, wl, ctrl):
    wl = rk2_variant(wl)
    y_o = wl.y0.copy()
    tot_o, st_o, n_o = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "rk2", ctrl,
                                  wl.n_integration_steps, threads=8)
    y_g = wl.y0.copy()
    tot_g, st_g, n_g = lib.integrate(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "rk2",
                                     "gje_f64", ctrl, wl.n_integration_steps)
    assert np.array_equal(y_g, y_o)
    assert np.array_equal(n_g, n_o)
    assert tot_g == tot_o


@pytest.mark.parametrize("width", [1, 2, 4, 8, 16, 32])
def test_speculative_width_identical(cuda_device, width):
    wl = CASES[1]  # katz96
    y_o = wl.y0.copy()
    tot_o, _, n_o = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "device")
    y_g = wl.y0.copy()
    tot_g, _, n_g = lib.integrate(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie",
                                  "gje_f64", "device", spec_width=width)
    assert np.array_equal(y_g, y_o)
    assert np.array_equal(n_g, n_o)


@pytest.mark.parametrize("solver", ["lu_f64", "mixed"])
@pytest.mark.parametrize("wl", CASES, ids=_ids(CASES))
def test_fast_solvers_close(cuda_device, wl, solver):
    """LU_F64 / MIXED vs the FP64 oracle: |err| <= 1e-5 * max(|y|, atol)."""
    y_o = wl.y0.copy()
    O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "device", threads=8)
    y_g = wl.y0.copy()
    lib.integrate(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver, "device")
    assert mixed_err(y_g, y_o, wl.atol) <= 1e-5


def test_batch_matches_single_calls(cuda_device):
    """wind_integrate_batch (several shapes at once) equals one call per shape."""
    groups = [CASES[1]] + [c for c in CASES if c.net.kind == W.NET_MASS_ACTION][:2]
    got = lib.integrate_batch(groups, "sie", "gje_f64", "device")
    for (yg, sg, ng), wl in zip(got, groups):
        y = wl.y0.copy()
        lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "gje_f64", "device")
        assert np.array_equal(yg, y)
