"""Golden outputs of the FP64 oracle (oracle/wind_oracle.c, pinned bit for bit
to the reference's c_baseline) on systems of the benchmark configurations
that are too slow to integrate on the CPU inside a test: the first systems
of each size class of the mixed-size batch (N = 5, 16, 32, 64, 157; 10N
reactions, seed 3) over dt = 1 at atol 1e-8 / rtol 1e-6, SIE, c_baseline
controller.  Writes tests/golden/config4.npz.

    python tests/golden/make_config_golden.py      (about 15 minutes, 8 cores)
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
    np.savez_compressed(os.path.join(HERE, "config4.npz"), **out)


if __name__ == "__main__":
    main()
