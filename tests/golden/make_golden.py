"""Generate the golden vectors: the reference's own CPU integrator
(cuda/c_baseline, compiled from the reference sources by oracle/build_ref.sh
in FP64 with -Dfloat=double) run on small seeded inputs of every network.

    WIND_REFERENCE=<reference checkout> python tests/golden/make_golden.py   # needs oracle/_ref built

Writes tests/golden/golden.npz.  Each case stores the inputs (network arrays,
y0, interval, tolerances) and the reference outputs (final state, total
substep count).  The tests compare the oracle restatement and the GPU path
against these arrays without needing the reference checkout.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402
from wind_b200 import networks as W  # noqa: E402


REFERENCE = os.environ.get("WIND_REFERENCE", "")
FIXTURE = os.path.join(REFERENCE, "cuda", "debug", "inputKatz96_1_1_1.h")


def reference_fixture(path=FIXTURE):
    """The reference's committed debug input (4 Katz96 cells), parsed from the
    header its dlopen driver includes (cuda/debug/debug.c:1); the driver runs
    it with tend = 10 and abs = rel = 5e-3 (debug.c:19,29-30)."""
    import re
    src = open(path).read()

    def arr(name):
        m = re.search(name + r"\[\d+\]\s*=\s*\{([^}]*)\}", src)
        return np.array([float(v) for v in m.group(1).split(",")], np.float32)

    eq = arr("equations").astype(np.float64).reshape(4, 5)
    c = arr("constants").astype(np.float64).reshape(4, 10)
    net = W.Network(W.NET_KATZ96, 5, 4, constants=c)
    return W.Workload(net, eq, 0.0, 10.0, float(np.float32(5e-3)), float(np.float32(5e-3)), 1, 1)


Y_HE = W.Y_HELIUM


def cases():
    out = []
    if REFERENCE and os.path.exists(FIXTURE):
        fx = reference_fixture()
        out.append(("fixture_katz96_debug_sie", "sie", fx))
        out.append(("fixture_katz96_debug_rk2", "rk2", fx))
    nr = W.workload_nr(16, seed=100)
    out.append(("nr_sie", "sie", W.Workload(nr.net, nr.y0, 0.0, 0.01, 1e-8, 1e-6, 1, 1)))
    out.append(("nr_rk2", "rk2", W.Workload(nr.net, nr.y0, 0.0, 0.01, 1e-8, 1e-6, 1, 1)))
    k = W.workload_katz96(32, seed=101)
    out.append(("katz96_sie", "sie", k))
    out.append(("katz96_sie_tight", "sie", W.Workload(k.net, k.y0, 0.0, 1e11, 1e-8, 1e-6, 1, 1)))
    out.append(("katz96_rk2", "rk2", W.Workload(k.net, k.y0, 0.0, 1e6, 5e-3, 5e-3, 1, 1)))
    # Ntile tiling (the reference's oracle build katz96_t<Ntile>): 3 tiles
    # starting in different states, so the tiles differ and the shared
    # electron density of tile 0 couples them; 8 identical tiles, as the
    # reference's tileEquations makes them
    kt = W.workload_katz96(8, seed=103)
    y3 = np.tile(kt.y0, (1, 3))
    y3[:, 5:10] = [0.3, 0.7, 0.02, Y_HE - 0.02, 0.0]
    y3[:, 10:15] = [0.9, 0.1, Y_HE, 0.0, 0.0]
    t3 = W.Workload(W.tile_network(kt.net, 3), y3, 0.0, 1e11, 1e-8, 1e-6, 1, 1)
    out.append(("katz96_t3_sie", "sie", t3))
    out.append(("katz96_t3_rk2", "rk2", W.Workload(t3.net, y3, 0.0, 1e6, 5e-3, 5e-3, 1, 1)))
    out.append(("katz96_t8_sie", "sie",
                W.tile_workload(W.Workload(kt.net, kt.y0, 0.0, 1e12, 1e-8, 1e-6, 1, 1), 8)))
    t = W.Workload(W.stifftrig(4), np.tile([0.0, 1.0], (4, 1)).astype(np.float64), 0.0, 0.5,
                   1e-6, 1e-6, 1, 1)
    out.append(("stifftrig_sie", "sie", t))
    out.append(("stifftrig_rk2", "rk2", t))
    rng = np.random.default_rng(102)
    for n, r, lin in ((3, 6, True), (8, 20, False), (12, 30, True)):
        net = W.random_mass_action(rng, 6, n, r, 1e-3, 1e1)
        if lin:
            net.linear = W.dense_linear(rng, 6, n, 1e-2, 1e3)
        y0 = rng.uniform(0.0, 1.0, (6, n))
        wl = W.Workload(net, y0, 0.0, 1e-2, 1e-6, 1e-4, 1, 1)
        out.append((f"{net.name}_sie", "sie", wl))
        out.append((f"{net.name}_rk2", "rk2", W.Workload(net, y0, 0.0, 1e-3, 1e-6, 1e-4, 1, 1)))
    return out


def main():
    blob = {}
    for name, method, wl in cases():
        y = wl.y0.copy()
        tot = O.reference(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, method,
                          wl.n_integration_steps)
        net = wl.net
        blob[f"{name}/meta"] = np.array([net.kind, net.n_eq, wl.tnow, wl.tend, wl.atol, wl.rtol,
                                         wl.n_integration_steps, tot], np.float64)
        blob[f"{name}/method"] = np.array(method)
        blob[f"{name}/y0"] = wl.y0
        blob[f"{name}/y"] = y
        for k in ("constants", "rates", "species", "linear"):
            a = getattr(net, k)
            if a is not None:
                blob[f"{name}/{k}"] = a
        print(f"{name:24s} {method} substeps={tot}")
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **blob)


if __name__ == "__main__":
    main()
