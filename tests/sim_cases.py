"""The semi-implicit midpoint golden cases (tests/golden/sim_golden.npz,
made by tests/golden/make_sim_golden.py from the reference's
python/pysolvers/sim.py)."""
import os

import numpy as np

from wind_b200 import networks as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sim_golden.npz")
# relative error bar of the FP64 path against the reference and the oracle
TOL = 1e-10


def load():
    z = np.load(GOLDEN)
    out = []
    for name in z["cases"]:
        name = str(name)
        y0 = z[f"{name}/y0"]
        kw = {k: z[f"{name}/{k}"] for k in ("constants", "rates", "species", "linear")
              if f"{name}/{k}" in z}
        net = W.Network(int(z[f"{name}/kind"]), int(z[f"{name}/n_eq"]), y0.shape[0], **kw)
        out.append((name, net, y0, float(z[f"{name}/dt"]), int(z[f"{name}/m"]), z[f"{name}/y_ref"]))
    return out


def rel_err(y, ref, floor=1e-8):
    return float(np.max(np.abs(y - ref) / np.maximum(np.abs(ref), floor)))


def rel_err_systemwise(y, ref):
    """max over systems of max_i |y_i - ref_i| / max_i |ref_i|: the error
    relative to each system's own scale (the midpoint iteration does not
    damp its stiff modes, so the rounding of a system's large components
    stays in its small ones)."""
    scale = np.maximum(np.abs(ref).max(axis=1), 1e-300)
    return float((np.abs(y - ref).max(axis=1) / scale).max())
