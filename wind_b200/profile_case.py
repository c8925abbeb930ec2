"""Run one workload's integration a few times on cuda:0 (profiling helper).

    python -m wind_b200.profile_case --workload ma32 --systems 256 --dt 1e-4 \\
        --solver lu_f64 --launches 3

Workloads are the ones bench.py defines (katz96, dense, ma<N>, nr).  Each
launch integrates every system from the same initial state with the arrays
already on the device; the last launch's time is printed.  Used as the
command under ncu, so captures run committed code only.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="katz96")
    ap.add_argument("--systems", type=int, default=0)
    ap.add_argument("--dt", type=float, default=0.0)
    ap.add_argument("--solver", default="lu_f64")
    ap.add_argument("--method", default="sie")
    ap.add_argument("--launches", type=int, default=3)
    a = ap.parse_args()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch
    import bench
    from wind_b200 import lib
    wl, desc = bench.make_workload(a.workload, a.systems, a.dt)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    arr = {k: torch.from_numpy(np.ascontiguousarray(getattr(wl.net, k))).to(dev)
           for k in ("constants", "rates", "species", "linear") if getattr(wl.net, k) is not None}
    y0 = torch.from_numpy(wl.y0).to(dev)
    for i in range(a.launches):
        y = y0.clone()
        torch.cuda.synchronize()
        t = time.perf_counter()
        tot, _, _ = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, a.method,
                                  a.solver, device_arrays=arr)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
    print(f"{desc}: {a.solver} {tot} substeps, last launch {dt:.4f} s")


if __name__ == "__main__":
    main()
