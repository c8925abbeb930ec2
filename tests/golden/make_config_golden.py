"""Golden outputs of the FP64 oracle (oracle/wind_oracle.c, pinned bit for bit
to the reference's c_baseline) on systems of the benchmark configurations
that are too slow to integrate on the CPU inside a test: the first systems
of each size class of the mixed-size batch (N = 5, 16, 32, 64, 157; 10N
reactions, seed 3) over dt = 1 at atol 1e-8 / rtol 1e-6, SIE, c_baseline
controller.  Writes tests/golden/config4.npz.

Some of these random networks are multistable: the FP64 trajectory of the
reference algorithm reaches one steady state, and any perturbation of the
linear solves at the 1e-14 level -- another elimination order, fused
multiply-adds -- makes it settle on another.  For each system the script
also integrates with partial-pivoting FP64 solves perturbed by 1e-14
relative noise; a system whose result then differs from the oracle's by
more than 1e-6 is marked sensitive (n<N>_sensitive): its reference result
is not a property of the equations, only of that exact arithmetic.

    python tests/golden/make_config_golden.py      (about 20 minutes, 8 cores)
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as O  # noqa: E402
from wind_b200 import networks as W  # noqa: E402

COUNTS = {5: 16, 16: 16, 32: 8, 64: 4, 157: 2}


def _perturbed_pivoted(net, s, y, t0, t1, atol, rtol, seed):
    """SIE with the c_baseline step-doubling controller (common_gold.c:48-153)
    and partial-pivoting FP64 solves perturbed by 1e-14 relative noise."""
    n = net.n_eq
    sp = net.species[s].astype(np.int64)
    k = net.rates[s]
    a, b = sp[:, 0], sp[:, 1]
    rng = np.random.default_rng(seed)
    eye = np.eye(n)
    sign = np.stack([-np.ones_like(k), -np.ones_like(k), np.ones_like(k), np.ones_like(k)], 1)

    def step(v, h):
        w = k * v[a] * v[b]
        f = np.zeros(n)
        np.add.at(f, sp.ravel(), (sign * w[:, None]).ravel())
        J = np.zeros((n, n))
        rows = sp.ravel()
        np.add.at(J, (rows, np.repeat(a, 4)), (sign * (k * v[b])[:, None]).ravel())
        np.add.at(J, (rows, np.repeat(b, 4)), (sign * (k * v[a])[:, None]).ravel())
        x = np.linalg.solve(eye - h * J, f)
        return v + h * x * (1.0 + 1e-14 * rng.standard_normal(n))

    t, h, unsolved = t0, t1 - t0, 0
    while t < t1:
        y1 = step(y, h)
        y2 = step(step(y, h * 0.5), h * 0.5)
        big = (np.abs(y1) > atol) & (np.abs(y2) > atol)
        err = np.any(np.abs(y2 - y1) >= atol) or np.any((np.abs((y2 - y1) / (y2 + 1e-12)) >= rtol) & big)
        if err and unsolved < 10:
            unsolved += 1
            h /= 2
        else:
            unsolved = 0
            y, t, h = y2, t + h, t1 - (t + h)
    return y


def main():
    out = {}
    for n, cnt in COUNTS.items():
        wl = W.workload_mixed_class(n, cnt, seed=3, dt=1.0, atol=1e-8, rtol=1e-6)
        y = wl.y0.copy()
        t0 = time.time()
        tot, st, steps = O.restated(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", "gold",
                                    threads=min(cnt, os.cpu_count() or 1))
        print(f"N={n}: {cnt} systems, {time.time() - t0:.0f} s, substeps {steps.tolist()}", flush=True)
        out[f"n{n}_y0"] = wl.y0
        out[f"n{n}_y"] = y
        out[f"n{n}_status"] = st
        out[f"n{n}_steps"] = steps
        import concurrent.futures as cf
        with cf.ProcessPoolExecutor(min(cnt, os.cpu_count() or 1)) as ex:
            yp = list(ex.map(_perturbed_pivoted, [wl.net] * cnt, range(cnt), list(wl.y0),
                             [wl.tnow] * cnt, [wl.tend] * cnt, [wl.atol] * cnt, [wl.rtol] * cnt,
                             range(cnt)))
        dev = np.max(np.abs(np.array(yp) - y) / np.maximum(np.abs(y), wl.atol), axis=1)
        out[f"n{n}_sensitive"] = dev > 1e-6
        print(f"  perturbed-solve deviation per system {np.array2string(dev, precision=1)}", flush=True)
    np.savez_compressed(os.path.join(HERE, "config4.npz"), **out)


if __name__ == "__main__":
    main()
