"""CPU tests of the oracle (test infrastructure): pinned against the golden
vectors made by the reference's own CPU integrator, against the reference
build itself when it is present, and against known answers."""
import os

import numpy as np
import pytest

from oracle import pyoracle as O
from wind_b200 import networks as W

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = np.load(os.path.join(HERE, "golden", "golden.npz"))
NAMES = sorted({k.split("/")[0] for k in GOLDEN.files})


def golden_case(name):
    meta = GOLDEN[f"{name}/meta"]
    kind, n = int(meta[0]), int(meta[1])
    arr = {k: GOLDEN[f"{name}/{k}"] for k in ("constants", "rates", "species", "linear")
           if f"{name}/{k}" in GOLDEN.files}
    y0 = GOLDEN[f"{name}/y0"]
    net = W.Network(kind, n, y0.shape[0], **arr)
    wl = W.Workload(net, y0, meta[2], meta[3], meta[4], meta[5], int(meta[6]), 1, name)
    return wl, str(GOLDEN[f"{name}/method"]), GOLDEN[f"{name}/y"], int(meta[7])


@pytest.mark.parametrize("name", NAMES)
def test_restatement_matches_golden(name):
    """GOLD semantics reproduce the reference c_baseline bit for bit."""
    wl, method, y_ref, tot_ref = golden_case(name)
    y = wl.y0.copy()
    tot, st, _ = O.restated(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, method, "gold",
                            wl.n_integration_steps)
    assert np.array_equal(y, y_ref), f"max diff {np.max(np.abs(y - y_ref))}"
    assert tot == tot_ref
    assert st.max() == 0


def _random_cases():
    rng = np.random.default_rng(7)
    k = W.workload_katz96(24, seed=9)
    yield "katz96", "sie", W.Workload(k.net, k.y0, 0.0, 1e12, 1e-7, 1e-5, 1, 1)
    yield "katz96", "rk2", W.Workload(k.net, k.y0, 0.0, 3e6, 1e-4, 1e-4, 1, 1)
    nr = W.workload_nr(8, seed=5)
    yield "nr", "sie", W.Workload(nr.net, nr.y0, 0.0, 0.003, 1e-8, 1e-6, 2, 1)
    for n, r, lin in ((5, 50, False), (16, 160, False), (32, 64, True)):
        net = W.random_mass_action(rng, 3, n, r, 1e-3, 1e1)
        if lin:
            net.linear = W.dense_linear(rng, 3, n, 1e-2, 1e4)
        y0 = rng.uniform(0, 1, (3, n))
        yield net.name, "sie", W.Workload(net, y0, 0.0, 1e-4, 1e-6, 1e-4, 1, 1)


@pytest.mark.parametrize("case", list(_random_cases()), ids=lambda c: f"{c[0]}-{c[1]}")
def test_restatement_matches_reference_build(case):
    name, method, wl = case
    if not O.reference_available(wl.net, method):
        pytest.skip("oracle/_ref not built (reference sources absent)")
    y_o, y_r = wl.y0.copy(), wl.y0.copy()
    tot_o, _, _ = O.restated(wl.net, y_o, wl.tnow, wl.tend, wl.atol, wl.rtol, method, "gold",
                             wl.n_integration_steps)
    tot_r = O.reference(wl.net, y_r, wl.tnow, wl.tend, wl.atol, wl.rtol, method,
                        wl.n_integration_steps)
    assert np.array_equal(y_o, y_r)
    assert tot_o == tot_r


def test_nr_analytic_known_answer():
    """NR test against its exact solution (python/ode_systems/NR_test.py:72-77
    generalised to any initial condition) over t = 0..0.2 in 20 outputs."""
    wl = W.workload_nr(8, seed=0)
    y = wl.y0.copy()
    t = 0.0
    for _ in range(20):
        O.restated(wl.net, y, t, t + 0.01, 1e-10, 1e-8, "rk2", "device")
        t += 0.01
    exact = W.nr_analytic(wl.y0, t)
    assert np.max(np.abs(y - exact) / np.abs(exact)) < 1e-6


def test_katz96_conserves_hydrogen():
    """The H total y0+y1 is an invariant of the Katz96 RHS and the H block of
    its Jacobian has zero column sums, so SIE conserves it to rounding.  (The
    He total is not conserved by SIE: the reference Jacobian's J[13] = J[12]
    (cuda/ode_system/ode_gold.c:79) breaks the zero column sum of the He
    block; parity keeps that behaviour.)"""
    wl = W.workload_katz96(64, seed=3)
    y = wl.y0.copy()
    O.restated(wl.net, y, 0.0, 1e12, 1e-8, 1e-6, "sie", "device", threads=4)
    assert np.allclose(y[:, 0] + y[:, 1], 1.0, rtol=0, atol=1e-12)


def test_oracle_edge_cases():
    wl = W.workload_katz96(4, seed=1)
    # empty range
    y = wl.y0.copy()
    tot, _, _ = O.restated(wl.net.subset(slice(0, 0)), y[:0], 0.0, 1.0, 1e-3, 1e-3)
    assert tot == 0
    # tnow == tend: nothing happens
    y = wl.y0.copy()
    tot, st, _ = O.restated(wl.net, y, 5.0, 5.0, 1e-3, 1e-3)
    assert tot == 0 and np.array_equal(y, wl.y0)
    # attempt budget
    y = wl.y0.copy()
    tot, st, n = O.restated(wl.net, y, 0.0, 1e13, 1e-10, 1e-10, max_attempts=3)
    assert (n <= 9).all() and (st & 2).any()
    # non-finite initial condition is reported, not trapped
    y = wl.y0.copy()
    y[1, 0] = np.nan
    tot, st, _ = O.restated(wl.net, y, 0.0, 1e10, 1e-3, 1e-3)
    assert st[1] & 1 and st[0] == 0


def test_global_controller_nr_known_answer():
    """The SIE_host controller (one step shared by all systems) restated.  It
    gives up after 9 consecutive refinements, so its callers start from a
    small step: with 1000 initial steps per output interval the NR test over
    t = 0..1 in 100 intervals reaches every interval's end and tracks the
    exact solution (first-order SIE at rtol 1e-6); every attempt counts 3
    substeps per system."""
    wl = W.workload_nr(64)
    y = wl.y0.copy()
    dt = (wl.tend - wl.tnow) / wl.n_output_steps
    total = 0
    for k in range(wl.n_output_steps):
        tot, t_reached = O.restated_global(wl.net, y, wl.tnow + k * dt, wl.tnow + (k + 1) * dt,
                                           wl.atol, wl.rtol, 1000)
        assert t_reached >= wl.tnow + (k + 1) * dt * (1 - 1e-12)
        assert tot % (3 * wl.net.nsys) == 0
        total += tot
    exact = W.nr_analytic(wl.y0, wl.tend)
    assert np.max(np.abs(y - exact) / np.abs(exact)) < 1e-4
    assert total > 0


def test_global_controller_gives_up_after_nine_refinements():
    """With a tolerance no step can meet, the shared-step loop stops after 9
    consecutive refinements (harness_kernel.cu:289): 10 attempts, the state
    untouched and the time not advanced."""
    wl = W.workload_katz96(4, seed=12)
    y = wl.y0.copy()
    tot, t_reached = O.restated_global(wl.net, y, 0.0, 1e13, 1e-30, 1e-30)
    assert t_reached == 0.0
    assert np.array_equal(y, wl.y0)
    assert tot == 9 * 3 * 4


def test_dense_workload_diverges_under_the_reference_algorithm():
    """System 42 of the seed-2 dense N=32 workload blows up in finite time at
    dt = 1 (its random two-body reactions dominate the linear decay): the
    restated reference algorithm ends non-finite and flags it, as does the
    reference's own c_baseline build; system 0 stays finite."""
    for s, finite in ((0, True), (42, False)):
        wl = W.workload_dense(1, first=s)
        y = wl.y0.copy()
        _, st, ns = O.restated(wl.net, y, 0.0, 1.0, 1e-8, 1e-6, "sie", "gold")
        assert bool(np.isfinite(y).all()) == finite
        assert (int(st[0]) & 1) == (0 if finite else 1)
        if O.reference_available(wl.net):
            yr = wl.y0.copy()
            tot = O.reference(wl.net, yr, 0.0, 1.0, 1e-8, 1e-6, "sie")
            assert bool(np.isfinite(yr).all()) == finite
            if finite:
                assert np.array_equal(yr, y) and tot == int(ns[0])


def test_tiled_identical_tiles_equal_the_untiled_network():
    """Ntile identical copies (the reference's tileEquations) integrate as the
    one untiled system does: the block-diagonal elimination of the full
    matrix leaves every tile on the untiled trajectory, with the same substep
    counts."""
    k = W.workload_katz96(6, seed=104)
    base = W.Workload(k.net, k.y0, 0.0, 1e12, 1e-8, 1e-6, 1, 1)
    for method in ("sie", "rk2"):
        y1 = base.y0.copy()
        _, _, n1 = O.restated(base.net, y1, 0.0, 1e12 if method == "sie" else 1e6, 1e-8, 1e-6,
                              method, "gold")
        t = W.tile_workload(base, 4)
        yt = t.y0.copy()
        _, _, nt = O.restated(t.net, yt, 0.0, 1e12 if method == "sie" else 1e6, 1e-8, 1e-6,
                              method, "gold")
        assert np.array_equal(yt, np.tile(y1, (1, 4)))
        assert np.array_equal(nt, n1)


def test_tiled_network_arguments():
    k = W.katz96_rates(np.array([1e4]), np.array([1.0]), np.array([1e-13]))
    bad = W.Network(W.NET_KATZ96, 7, 1, constants=k)  # not a multiple of 5
    with pytest.raises(ValueError):
        O.restated(bad, np.zeros((1, 7)), 0.0, 1.0, 1e-8, 1e-6)
    with pytest.raises(ValueError):
        W.tile_network(W.tile_network(W.nr_test(1), 2), 2)
    assert W.tile_network(W.nr_test(3), 5).name == "nr_test_t5"
