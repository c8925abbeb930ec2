"""Generate the golden vectors of the semi-implicit midpoint method: the
reference's own python/pysolvers/sim.py (integrate_sie, :36-90) run on small
seeded inputs, imported from the reference checkout.

    WIND_REFERENCE=<reference checkout> python tests/golden/make_sim_golden.py

Writes tests/golden/sim_golden.npz.  sim.py takes f and J as Python callables
of one tuple argument (y, constants) with J[i, j] = df_i/dy_j (sim.py:11-20,
:45); they are supplied here from the oracle's plug-in restatements (pinned
to the reference's c_baseline plug-ins by tests/test_oracle.py), transposed
back from the plug-in layout.  sim.py uses ``np.float``, which NumPy 2 no
longer has; it is set to the builtin float before the call, nothing else of
the module is changed.

Each case stores the inputs, dt, the step count m the reference takes
(its t_arr = arange(0, tend + dt, dt) has M + 1 points, and it does the first
step, M interior steps and the smoothing step, so m = M + 1 steps over
m * dt) and its final row y_arr[-1].
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402
from wind_b200 import networks as W  # noqa: E402

REFERENCE = os.environ.get("WIND_REFERENCE", "")


def load_sim():
    path = os.path.join(REFERENCE, "python", "pysolvers", "sim.py")
    if not REFERENCE or not os.path.exists(path):
        raise SystemExit("set WIND_REFERENCE to the reference checkout")
    if not hasattr(np, "float"):
        np.float = float  # NumPy 1 alias used by sim.py:41
    spec = importlib.util.spec_from_file_location("wind_ref_sim", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def callables(net, s):
    def f(arg):
        y, _ = arg
        return O.rhs_jac(net, s, y)[0]

    def J(arg):
        y, _ = arg
        return O.rhs_jac(net, s, y)[1].T.copy()
    return f, J


def cases():
    out = []
    nr = W.workload_nr(6, seed=300)
    out.append(("nr", nr.net, nr.y0, 0.01, 0.5))
    k = W.workload_katz96(4, seed=301)
    out.append(("katz96", k.net, k.y0, 1e8, 2e9))
    # rates up to 1e4: steps of 1e-5 keep the explicit part of the method
    # stable (at 1e-3 the iteration grows and amplifies rounding)
    ma = W.workload_mixed_class(16, 3, seed=302, dt=1.0)
    out.append(("ma16", ma.net, ma.y0, 1e-5, 5e-4))
    ma5 = W.workload_mixed_class(5, 4, seed=304, dt=1.0)
    out.append(("ma5", ma5.net, ma5.y0, 1e-5, 3e-4))
    de = W.workload_dense(2, first=0)
    out.append(("dense32", de.net, de.y0, 1e-4, 2e-3))
    return out


def main():
    sim = load_sim()
    arrays = {}
    names = []
    for name, net, y0, dt, tend in cases():
        outs, ms = [], []
        for s in range(net.nsys):
            f, J = callables(net, s)
            t_arr, y_arr = sim.integrate_sie(np.array(y0[s], np.float64), None, dt, tend, f, J)
            outs.append(y_arr[-1])
            ms.append(len(t_arr))      # m = M + 1 = len(t_arr)
        assert len(set(ms)) == 1
        names.append(name)
        arrays[f"{name}/y0"] = np.asarray(y0, np.float64)
        arrays[f"{name}/y_ref"] = np.array(outs)
        arrays[f"{name}/dt"] = np.float64(dt)
        arrays[f"{name}/m"] = np.int64(ms[0])
        arrays[f"{name}/kind"] = np.int64(net.kind)
        arrays[f"{name}/n_eq"] = np.int64(net.n_eq)
        for key in ("constants", "rates", "species", "linear"):
            v = getattr(net, key)
            if v is not None:
                arrays[f"{name}/{key}"] = v
        print(f"{name}: {net.nsys} systems, m = {ms[0]}, |y| max {np.abs(outs).max():.3e}")
    arrays["cases"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "sim_golden.npz"), **arrays)


if __name__ == "__main__":
    main()
