"""Parity at the benchmark configurations, and the per-system failure status
on every kernel family (GPU).

* config 3 -- the dense N = 32 network (seed 2) over the full dt = 1 at atol
  1e-8 / rtol 1e-6: LU_F64 and MIXED against the FP64 oracle on the first
  systems of the benchmark batch;
* config 4 -- every size class of the mixed-size batch (N = 5, 16, 32, 64,
  157; seed 3; dt = 1) through wind_integrate_batch (one persistent launch),
  against golden outputs of the FP64 oracle (tests/golden/config4.npz, made
  by tests/golden/make_config_golden.py: one 157-species system takes the
  oracle about ten minutes);
* configs 1 and 2 -- LU_F64 against the 1e-10 relative bar of the plain FP64
  path;
* failure detection -- a device deadline that has passed, an attempt budget
  of 2 and a NaN initial state make each kernel family report TIMEOUT,
  MAX_ATTEMPTS and NONFINITE per system, with the other systems of the
  launch unaffected.  No fault or trap is involved: the kernels check and
  return.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as O
from tests.helpers import mixed_err
from wind_b200 import _capi, lib, networks as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
THREADS = os.cpu_count() or 1
SYS_NONFINITE, SYS_MAX_ATTEMPTS, SYS_TIMEOUT = 1, 2, 16


# ---- config 3 --------------------------------------------------------------
@pytest.fixture(scope="module")
def dense32():
    wl = W.workload_dense(24)
    y_o = wl.y0.copy()
    _, st, steps = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "gold",
                              threads=THREADS)
    assert st.max() == 0 and steps.min() > 10000  # the stiff interval it is quoted on
    return wl, y_o


@pytest.mark.parametrize("solver", ["lu_f64", "mixed"])
def test_config3_dense32_full_interval(cuda_device, dense32, solver):
    wl, y_o = dense32
    y = wl.y0.copy()
    _, st, _ = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver, "gold")
    err = mixed_err(y, y_o, wl.atol)
    assert err <= 1e-5, f"{solver}: max rel err {err:.3e} vs the FP64 oracle"
    assert (st & ~8).max() == 0


@pytest.mark.parametrize("solver", ["gje_f64", "lu_f64", "mixed"])
def test_config3_divergent_system_flagged(cuda_device, solver):
    """System 42 of the dense batch blows up in finite time under the
    reference algorithm (the oracle ends non-finite); every solver flags it
    NONFINITE, and the finite system integrated in the same launch keeps the
    oracle's result."""
    wl = W.workload_dense(1, first=42)
    y_o = wl.y0.copy()
    _, st_o, _ = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "gold")
    assert not np.isfinite(y_o).all() and st_o[0] & SYS_NONFINITE
    w0 = W.workload_dense(1, first=0)
    y0_o = w0.y0.copy()
    O.restated(w0.net, y0_o, w0.tnow, w0.tend, w0.atol, w0.rtol, "sie", "gold")
    both = W.Workload(W._cat_networks([w0.net, wl.net], slice(0, 2)),
                      np.concatenate([w0.y0, wl.y0]), wl.tnow, wl.tend, wl.atol, wl.rtol, 1, 1,
                      "dense32")
    y = both.y0.copy()
    _, st, _ = lib.integrate(both.net, y, both.tnow, both.tend, both.atol, both.rtol, "sie",
                             solver, "gold")
    assert st[1] & SYS_NONFINITE and not np.isfinite(y[1]).all()
    assert (st[0] & ~8) == 0
    if solver == "gje_f64":
        assert np.array_equal(y[0], y0_o[0])
    else:
        assert mixed_err(y[:1], y0_o, wl.atol) <= 1e-5


# ---- config 4 --------------------------------------------------------------
@pytest.fixture(scope="module")
def config4():
    g = np.load(os.path.join(HERE, "golden", "config4.npz"))
    groups, want, sens = [], [], []
    for n in W.MIXED_SIZES:
        y_ref = g[f"n{n}_y"]
        wl = W.workload_mixed_class(n, y_ref.shape[0], seed=3, dt=1.0, atol=1e-8, rtol=1e-6)
        assert np.array_equal(wl.y0, g[f"n{n}_y0"]), "workload generator drifted from the fixture"
        groups.append(wl)
        want.append(y_ref)
        sens.append(g[f"n{n}_sensitive"])
    return groups, want, sens


@pytest.fixture(scope="module")
def config4_gpu(cuda_device, config4):
    groups, _, _ = config4
    return {s: lib.integrate_batch(groups, "sie", s, "gold") for s in ("lu_f64", "mixed")}


@pytest.mark.parametrize("solver", ["lu_f64", "mixed"])
def test_config4_all_sizes_one_launch(cuda_device, config4, config4_gpu, solver):
    """Every size class in one persistent launch against the FP64 oracle.
    Systems the fixture marks sensitive (multistable: a 1e-14 perturbation of
    the solves moves them to another steady state) are compared with the
    plain FP64 path's result instead, which sits on the same branch."""
    groups, want, sens = config4
    for gi, ((y, st, n), wl, y_ref, sv) in enumerate(zip(config4_gpu[solver], groups, want, sens)):
        ok = ~sv
        err = mixed_err(y[ok], y_ref[ok], wl.atol)
        assert err <= 1e-5, f"N={wl.net.n_eq} {solver}: max rel err {err:.3e} vs the FP64 oracle"
        if sv.any() and solver == "mixed":
            y_lu = config4_gpu["lu_f64"][gi][0]
            err = mixed_err(y[sv], y_lu[sv], wl.atol)
            assert err <= 1e-5, f"N={wl.net.n_eq}: sensitive systems, MIXED vs LU_F64 {err:.3e}"
        assert (st & ~8).max() == 0
    assert sum(int(v.sum()) for v in sens) <= 2  # the fixture holds a handful at most


def test_config4_gje_matches_oracle_small_classes(cuda_device, config4):
    """The reference algorithm, bit for bit, on the classes the oracle
    integrates quickly (N = 5, 16) in the same one-launch batch."""
    groups, want, _ = config4
    small = [(wl, y) for wl, y in zip(groups, want) if wl.net.n_eq <= 16]
    got = lib.integrate_batch([wl for wl, _ in small], "sie", "gje_f64", "gold")
    for (y, st, n), (wl, y_ref) in zip(got, small):
        assert np.array_equal(y, y_ref), f"N={wl.net.n_eq}: GJE_F64 differs from the oracle"


# ---- configs 1 and 2: the plain FP64 path at 1e-10 ------------------------------
def test_config1_nr_lu_f64_1e10(cuda_device):
    wl = W.workload_nr(1024)
    out_o = wl.y0.copy()
    out_g = wl.y0.copy()
    dt = (wl.tend - wl.tnow) / wl.n_output_steps
    for k in range(wl.n_output_steps):
        t0 = wl.tnow + k * dt
        O.restated(wl.net, out_o, t0, t0 + dt, wl.atol, wl.rtol, "sie", "device", threads=THREADS)
        lib.integrate(wl.net, out_g, t0, t0 + dt, wl.atol, wl.rtol, "sie", "lu_f64", "device")
    err = float(np.max(np.abs(out_g - out_o) / np.abs(out_o)))
    assert err <= 1e-10, f"NR LU_F64 max rel err {err:.3e}"


def test_config2_katz96_lu_f64_1e10(cuda_device):
    wl = W.workload_katz96(2048, atol=1e-8, rtol=1e-6)
    y_o = wl.y0.copy()
    O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "device", threads=THREADS)
    y_g = wl.y0.copy()
    lib.integrate(wl.net, y_g, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "lu_f64", "device")
    err = mixed_err(y_g, y_o, wl.atol)
    assert err <= 1e-10, f"Katz96 LU_F64 max rel err {err:.3e}"


# ---- failure detection on every kernel family ------------------------------
def _families():
    k96 = W.workload_katz96(12, seed=70, atol=1e-8, rtol=1e-6)
    k96 = W.Workload(k96.net, k96.y0, 0.0, 1e11, k96.atol, k96.rtol, 1, 1, "lane_katz96")
    ma16 = W.workload_mixed_class(16, 12, seed=71, dt=1e-3, atol=1e-8, rtol=1e-6)
    ma64 = W.workload_mixed_class(64, 4, seed=72, dt=1e-4, atol=1e-6, rtol=1e-4)
    return [(k96, "lu_f64"), (k96, "gje_f64"), (ma16, "gje_f64"), (ma16, "lu_f64"),
            (ma16, "mixed"), (ma64, "lu_f64"), (ma64, "mixed"), (ma64, "gje_f64")]


FAM = _families()
FAM_IDS = [f"{wl.label}-{s}" for wl, s in FAM]


@pytest.mark.parametrize("wl,solver", FAM, ids=FAM_IDS)
def test_status_timeout(cuda_device, wl, solver):
    """A device deadline of 1 ns passes within the first attempts (the
    global timer ticks about every microsecond): every system stops with
    TIMEOUT, well short of the interval, and the call returns normally."""
    y = wl.y0.copy()
    _, st, n = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver, "device",
                             timeout_s=1e-9)
    assert np.all(st & SYS_TIMEOUT), st
    y_full = wl.y0.copy()
    _, _, n_full = lib.integrate(wl.net, y_full, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver,
                                 "device")
    assert n.sum() < n_full.sum()


@pytest.mark.parametrize("wl,solver", FAM, ids=FAM_IDS)
def test_status_max_attempts(cuda_device, wl, solver):
    """An attempt budget of 2: systems that need more stop with MAX_ATTEMPTS
    after exactly 2 attempts (6 substeps); the oracle with the same budget
    flags the same systems."""
    y = wl.y0.copy()
    _, st, n = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver, "device",
                             max_attempts=2)
    y_o = wl.y0.copy()
    _, st_o, n_o = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "device",
                              max_attempts=2, threads=THREADS)
    assert np.any(st & SYS_MAX_ATTEMPTS)
    assert np.array_equal(st & SYS_MAX_ATTEMPTS, st_o & SYS_MAX_ATTEMPTS)
    assert np.all(n[(st & SYS_MAX_ATTEMPTS) != 0] == 6)
    if solver == "gje_f64":
        assert np.array_equal(y, y_o) and np.array_equal(st, st_o)


@pytest.mark.parametrize("wl,solver", FAM, ids=FAM_IDS)
def test_status_nonfinite_isolated(cuda_device, wl, solver):
    """A NaN in one system's initial state: that system ends NONFINITE, every
    other system of the launch ends exactly as in a launch without it."""
    bad = 1
    y0 = wl.y0.copy()
    y0[bad, 0] = np.nan
    y = y0.copy()
    _, st, _ = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver, "device")
    assert st[bad] & SYS_NONFINITE
    clean = wl.y0.copy()
    _, st_c, _ = lib.integrate(wl.net, clean, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", solver,
                               "device")
    keep = np.arange(wl.net.nsys) != bad
    assert np.array_equal(y[keep], clean[keep])
    assert np.array_equal(st[keep], st_c[keep])


def test_status_in_one_launch_batch(cuda_device):
    """The same three failures inside wind_integrate_batch (one persistent
    launch over several sizes): a NaN system in one group, the others clean."""
    groups = [W.workload_mixed_class(n, 6, seed=73, dt=1e-4, atol=1e-8, rtol=1e-6)
              for n in (5, 32, 64)]
    ref = lib.integrate_batch(groups, "sie", "mixed", "device")
    groups[1].y0[2, 3] = np.nan
    got = lib.integrate_batch(groups, "sie", "mixed", "device")
    for gi, ((y, st, _), (y_r, st_r, _)) in enumerate(zip(got, ref)):
        if gi == 1:
            assert st[2] & SYS_NONFINITE
            keep = np.arange(6) != 2
            assert np.array_equal(y[keep], y_r[keep])
        else:
            assert np.array_equal(y, y_r) and np.array_equal(st, st_r)
