"""Workload generators: seeded, shaped as the configurations describe."""
import numpy as np

from wind_b200 import networks as W


def test_seeded_and_deterministic():
    a, b = W.workload_katz96(100), W.workload_katz96(100)
    assert np.array_equal(a.net.constants, b.net.constants)
    c, d = W.workload_dense(3), W.workload_dense(3)
    assert np.array_equal(c.net.linear, d.net.linear) and np.array_equal(c.y0, d.y0)


def test_katz96_rates():
    wl = W.workload_katz96(1000)
    c = wl.net.constants
    assert c.shape == (1000, 10) and np.all(np.isfinite(c)) and np.all(c >= 0)
    # photo rates: Gamma_gamma,He0 / Gamma_gamma,H0 fixed at 3.7e-12/4.4e-11
    assert np.allclose(c[:, 4] / c[:, 1], 3.7e-12 / 4.4e-11)
    assert np.allclose(wl.y0[:, 3], W.Y_HELIUM)


def test_dense_linear_is_stable_symmetric():
    rng = np.random.default_rng(0)
    L = W.dense_linear(rng, 4, 8, 1e-2, 1e2).astype(np.float64)
    assert np.allclose(L, np.transpose(L, (0, 2, 1)), atol=1e-4)
    ev = np.linalg.eigvalsh(L)
    assert ev.max() < 0


def test_mixed_sizes_and_counts():
    groups = W.workload_mixed(1000)
    assert [g.net.n_eq for g in groups] == list(W.MIXED_SIZES)
    assert [g.net.nsys for g in groups] == [400, 250, 200, 100, 50]
    for g in groups:
        assert g.net.n_react == 10 * g.net.n_eq
        assert g.net.species.max() < g.net.n_eq


def test_packed_constants_layout():
    rng = np.random.default_rng(1)
    net = W.random_mass_action(rng, 2, 3, 4, 1.0, 2.0)
    net.linear = W.dense_linear(rng, 2, 3, 1.0, 2.0)
    p = net.packed_constants()
    assert p.shape == (2, 5 * 4 + 9)
    assert np.array_equal(p[:, :4], net.rates)
    assert np.array_equal(p[:, 4:20].reshape(2, 4, 4), net.species.astype(np.float64))
    assert np.array_equal(p[:, 20:].reshape(2, 3, 3), net.linear.astype(np.float64))
