"""Shared helpers for the parity tests (test infrastructure)."""
import numpy as np

from wind_b200 import networks as W


def small_workloads():
    """Small seeded cases of every network, sized so the CPU oracle finishes
    in well under a second each."""
    nr = W.workload_nr(64)
    nr = W.Workload(nr.net, nr.y0, 0.0, 0.01, nr.atol, nr.rtol, 1, 1, "nr_test")
    k96 = W.workload_katz96(128)
    k96_tight = W.Workload(k96.net, k96.y0, 0.0, 1e11, 1e-8, 1e-6, 1, 1, "katz96_tight")
    trig = W.Workload(W.stifftrig(16), np.tile([0.0, 1.0], (16, 1)).astype(np.float64),
                      0.0, 0.5, 1e-6, 1e-6, 1, 1, "stifftrig")
    dense = W.workload_dense(4)
    dense = W.Workload(dense.net, dense.y0, 0.0, 2e-4, dense.atol, dense.rtol, 1, 1, "dense32")
    out = [nr, k96, k96_tight, trig, dense]
    for w in W.workload_mixed(40, sizes=(5, 16, 32), fractions=(0.5, 0.35, 0.15), dt=2e-5):
        out.append(w)
    return out


def rk2_variant(wl):
    """RK2 is explicit: keep the interval short enough for stiff networks."""
    if wl.net.kind == W.NET_KATZ96:
        return W.Workload(wl.net, wl.y0, 0.0, 1e6, wl.atol, wl.rtol, 1, 1, wl.label + "_rk2")
    if wl.net.kind == W.NET_MASS_ACTION:
        return W.Workload(wl.net, wl.y0, 0.0, (wl.tend - wl.tnow) * 0.1, wl.atol, wl.rtol, 1, 1,
                          wl.label + "_rk2")
    return wl


def max_rel_err(a, b, floor=1e-300):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.maximum(np.abs(b), floor)
    return float(np.max(np.abs(a - b) / den)) if a.size else 0.0


def mixed_err(a, b, atol):
    """max |a-b| / max(|b|, atol): relative where the value is resolved,
    absolute below the absolute tolerance."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), atol))) if a.size else 0.0


def cta_workloads():
    """Systems above 32 equations (the CTA-per-system kernels)."""
    out = []
    for n, dt in ((64, 1e-5), (157, 2e-6)):
        w = W.workload_mixed(60, seed=31, sizes=(n,), fractions=(1.0,), dt=dt, atol=1e-6,
                             rtol=1e-4)[0].subset(slice(0, 3))
        out.append(W.Workload(w.net, w.y0, w.tnow, w.tend, w.atol, w.rtol, 1, 1, f"cta_n{n}"))
    rng = np.random.default_rng(33)
    net = W.random_mass_action(rng, 3, 40, 80, 1e-3, 1e1)
    net.linear = W.dense_linear(rng, 3, 40, 1e-2, 1e4)
    y0 = rng.uniform(0.0, 1.0, (3, 40))
    out.append(W.Workload(net, y0, 0.0, 1e-4, 1e-6, 1e-4, 1, 1, "cta_n40_lin"))
    return out
