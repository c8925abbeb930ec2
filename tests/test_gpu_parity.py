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


CTA = __import__("tests.helpers", fromlist=["cta_workloads"]).cta_workloads()


@pytest.mark.parametrize("ctrl", ["gold", "device"])
@pytest.mark.parametrize("wl", CTA, ids=_ids(CTA))
def test_cta_gje_bitexact(cuda_device, wl, ctrl):
    y_o = wl.y0.copy()
    tot_o, st_o, n_o = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", ctrl,
                                  threads=8)
    y_g = wl.y0.copy()
    tot_g, st_g, n_g = lib.integrate(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie",
                                     "gje_f64", ctrl)
    assert np.array_equal(y_g, y_o), f"max diff {np.max(np.abs(y_g - y_o))}"
    assert np.array_equal(n_g, n_o) and tot_g == tot_o


@pytest.mark.parametrize("wl", CTA, ids=_ids(CTA))
def test_cta_rk2_bitexact(cuda_device, wl):
    wl = rk2_variant(wl)
    y_o = wl.y0.copy()
    tot_o, _, n_o = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "rk2", "device")
    y_g = wl.y0.copy()
    tot_g, _, n_g = lib.integrate(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "rk2",
                                  "gje_f64", "device")
    assert np.array_equal(y_g, y_o) and tot_g == tot_o


@pytest.mark.parametrize("solver", ["lu_f64", "mixed"])
@pytest.mark.parametrize("wl", CTA, ids=_ids(CTA))
def test_cta_fast_solvers_close(cuda_device, wl, solver):
    y_o = wl.y0.copy()
    O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "device", threads=8)
    y_g = wl.y0.copy()
    lib.integrate(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver, "device")
    assert mixed_err(y_g, y_o, wl.atol) <= 1e-5


@pytest.mark.parametrize("nsys", [1, 3, 40, 5000])
def test_lane_speculation_counts(cuda_device, nsys):
    """Batch sizes from 1 to thousands exercise every team size of the
    lane kernel's helpers; results must stay identical to the serial loop."""
    wl = W.workload_katz96(nsys, seed=41, atol=1e-8, rtol=1e-6)
    wl = W.Workload(wl.net, wl.y0, 0.0, 1e10, wl.atol, wl.rtol, 1, 1, "k")
    y_o = wl.y0.copy()
    tot_o, _, n_o = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "device",
                               threads=8)
    y_g = wl.y0.copy()
    tot_g, _, n_g = lib.integrate(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie",
                                  "gje_f64", "device")
    assert np.array_equal(y_g, y_o) and np.array_equal(n_g, n_o)


def test_bad_species_index_is_reported(cuda_device):
    """A species index >= N is caught by the kernel's bounds check: the
    system is flagged and left untouched, the others integrate normally."""
    import torch
    wl = [c for c in CASES if c.net.kind == W.NET_MASS_ACTION and c.net.linear is None][0]
    net = wl.net.subset(slice(0, 4))
    sp = net.species.copy()
    sp[2, 0, 1] = net.n_eq + 3
    dev = torch.device("cuda", 0)
    arrays = {"rates": torch.from_numpy(net.rates).to(dev),
              "species": torch.from_numpy(sp).to(dev)}
    y = torch.from_numpy(wl.y0[:4].copy()).to(dev)
    _, status, _ = lib.integrate(net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, device_arrays=arrays)
    torch.cuda.synchronize()
    st = status.cpu().numpy()
    assert st[2] & 32 and (st[[0, 1, 3]] == 0).all()
    assert np.array_equal(y.cpu().numpy()[2], wl.y0[2])


@pytest.mark.parametrize("solver", ["gje_f64", "lu_f64", "mixed"])
def test_mixed_size_single_launch(cuda_device, solver):
    """Mass-action groups of N = 5, 16, 32, 40, 64 (plus a builtin group) in
    one wind_integrate_batch call: the mass-action groups share ONE
    persistent launch; every system's result equals its own single call."""
    groups = [c for c in CASES if c.net.kind == W.NET_MASS_ACTION and c.net.linear is None]
    groups += [CTA[0], CTA[2], CASES[1]]
    got = lib.integrate_batch(groups, "sie", solver, "device")
    n0 = lib.launch_count()
    lib.integrate_batch(groups, "sie", solver, "device")
    assert lib.launch_count() - n0 == 2  # one mixed-size launch + one lane launch
    for (yg, sg, ng), wl in zip(got, groups):
        y = wl.y0.copy()
        _, st, n = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver,
                                 "device")
        assert np.array_equal(yg, y), wl.label
        assert np.array_equal(ng, n) and np.array_equal(sg, st)


def test_cta_mixed_fallback_flag(cuda_device):
    """MIXED inverts N > 32 systems by Gauss-Jordan without pivoting.  Here
    (I - hJ)[0][0] of the first full step is exactly zero (no reaction
    touches species 0 and h L[0][0] = 1), so that inverse cannot be formed:
    the substep is redone with the pivoted Gauss-Jordan inverse, the system
    carries WIND_SYS_REFINE_FALLBACK, and its result is the FP64 LU path's.
    Species 0 and 1 are coupled through L so the matrix stays nonsingular."""
    rng = np.random.default_rng(7)
    n, s, dt = 40, 4, 1e-3
    net = W.random_mass_action(rng, s, n - 1, 80, 1e-3, 1e-1)
    net.species = (net.species + 1).astype(np.uint16)  # species 1..N-1 only
    net.n_eq = n
    lin = np.zeros((s, n, n), np.float32)
    for k in range(s):
        lin[k] = -np.eye(n, dtype=np.float32)
        lin[k, 0, 0] = np.float32(1.0 / dt)
        lin[k, 0, 1] = lin[k, 1, 0] = np.float32(1.0)
    net.linear = lin
    y0 = rng.uniform(0.5, 1.0, (s, n))
    y_lu, y_mx = y0.copy(), y0.copy()
    _, st_lu, _ = lib.integrate(net, y_lu, 0.0, dt, 1e-8, 1e-6, "sie", "lu_f64", "device")
    _, st_mx, _ = lib.integrate(net, y_mx, 0.0, dt, 1e-8, 1e-6, "sie", "mixed", "device")
    st_lu, st_mx = np.asarray(st_lu), np.asarray(st_mx)
    assert not (st_lu & 8).any()
    assert (st_mx & 8).all()
    assert np.isfinite(y_mx).all()
    assert mixed_err(y_mx, y_lu, 1e-8) <= 1e-5
