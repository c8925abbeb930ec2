"""Per-shape launch configuration tuner.

For a workload shape (network kind, N, reactions, dense term, method,
controller, batch size) it times the candidate configurations -- solver
(LU_F64 / MIXED / MIXED_TC above 32 species, plus the reference GJE_F64 as
the accuracy anchor) and,
for the thread-per-system kernel, the initial lanes per system
(`spec_width` 1, 2, 4, 8; helpers still join at the tail) -- on the GPU,
keeps the fastest one whose result stays within `tol` of the FP64
Gauss-Jordan result, and caches the choice in a JSON file keyed by GPU name
and shape.  ``choose()`` returns the cached entry (tuning on a miss).
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import lib, networks as W

CACHE = os.environ.get("WIND_TUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "wind_b200", "tuned.json"))


def _key(wl, method, controller, gpu):
    n = wl.net
    bucket = 1 << max(0, int(np.ceil(np.log2(max(1, n.nsys)))))
    return "|".join(map(str, [gpu, n.kind, n.n_eq, n.n_react, int(n.linear is not None), method,
                              controller, bucket]))


def _load():
    try:
        with open(CACHE) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _save(db):
    os.makedirs(os.path.dirname(CACHE), exist_ok=True)
    tmp = CACHE + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(db, fh, indent=1, sort_keys=True)
    os.replace(tmp, CACHE)


def tune(wl, method="sie", controller="device", tol=1e-5, sample=0, reps=2, widths=(1, 2, 4, 8),
         solvers=None):
    """Time every candidate on `wl` (or a strided sample of `sample` systems)
    and return (best, table).  Runs on the current CUDA device.  The default
    candidates are LU_F64 and MIXED, plus MIXED_TC (the tensor-core rank
    updates) for SIE on mass-action networks above 32 species."""
    import torch
    if solvers is None:
        solvers = ("lu_f64", "mixed")
        if wl.net.kind == W.NET_MASS_ACTION and wl.net.n_eq > 32 and method == "sie":
            solvers += ("mixed_tc",)
    dev = torch.device("cuda", torch.cuda.current_device())
    if sample and wl.net.nsys > sample:
        wl = wl.subset(slice(0, wl.net.nsys, max(1, wl.net.nsys // sample)))
    arr = {k: torch.from_numpy(np.ascontiguousarray(getattr(wl.net, k))).to(dev)
           for k in ("constants", "rates", "species", "linear") if getattr(wl.net, k) is not None}
    y0 = torch.from_numpy(wl.y0).to(dev)

    def run(solver, width):
        best = 1e30
        for _ in range(reps):
            y = y0.clone()
            torch.cuda.synchronize(dev)
            t = time.perf_counter()
            lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, method, solver,
                          controller, wl.n_integration_steps, spec_width=width,
                          device_arrays=arr, want_status=False)
            torch.cuda.synchronize(dev)
            best = min(best, time.perf_counter() - t)
        return best, y.cpu().numpy()

    _, y_ref = run("gje_f64", 0)
    builtin = wl.net.kind != W.NET_MASS_ACTION
    table = []
    for solver in solvers:
        for width in (widths if builtin else (0,)):
            t, y = run(solver, width)
            err = float(np.max(np.abs(y - y_ref) / np.maximum(np.abs(y_ref), wl.atol)))
            table.append({"solver": solver, "spec_width": width, "seconds": t, "err": err})
    ok = [r for r in table if r["err"] <= tol] or [{"solver": "gje_f64", "spec_width": 0,
                                                    "seconds": None, "err": 0.0}]
    best = min(ok, key=lambda r: r["seconds"] if r["seconds"] is not None else 1e30)
    return best, table


def choose(wl, method="sie", controller="device", **kw):
    """Cached best configuration for this shape (tunes and stores on a miss)."""
    import torch
    gpu = torch.cuda.get_device_name()
    key = _key(wl, method, controller, gpu)
    db = _load()
    if key in db:
        return db[key]
    best, table = tune(wl, method, controller, **kw)
    db[key] = {"solver": best["solver"], "spec_width": best["spec_width"], "table": table}
    _save(db)
    return db[key]
