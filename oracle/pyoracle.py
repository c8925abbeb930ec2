"""Python access to the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Two checkers live here, and only tests/, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may use them:

* :func:`restated` -- the FP64 C restatement (oracle/wind_oracle.c, built into
  oracle/_build/libwind_oracle.so by ``make -C oracle``);
* :func:`reference` -- the reference's own CPU integrator (cuda/c_baseline)
  compiled from its sources by oracle/build_ref.sh into oracle/_ref/, called
  through its ``goldIntegrateSystem`` entry (cuda/c_baseline/sie/sie_gold.c:81).

Both accept a :class:`wind_b200.networks.Workload`-style set of arrays and
update ``y`` in place.  Threads call disjoint system ranges (ctypes releases
the GIL during the foreign call; the reference function keeps no globals and
mallocs its own scratch, sie_gold.c:99-100).
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import os

import numpy as np

from wind_b200 import _capi
from wind_b200.networks import Network

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

_oracle_lib = None


def _load_oracle():
    global _oracle_lib
    if _oracle_lib is None:
        path = os.path.join(BUILD, "libwind_oracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        lib = C.CDLL(path)
        P = C.c_void_p
        lib.wind_oracle_integrate.argtypes = [
            C.c_int, C.c_int, C.POINTER(_capi.WindNetwork), C.c_double, C.c_double,
            C.c_int, P, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int64, P, P]
        lib.wind_oracle_integrate.restype = C.c_int64
        lib.wind_oracle_integrate_global.argtypes = [
            C.POINTER(_capi.WindNetwork), C.c_double, C.c_double, C.c_int, P, C.c_int64,
            C.c_double, C.c_double, C.POINTER(C.c_double)]
        lib.wind_oracle_integrate_global.restype = C.c_int64
        lib.wind_oracle_integrate_sim.argtypes = [
            C.POINTER(_capi.WindNetwork), C.c_double, C.c_double, C.c_int, P, C.c_int64,
            C.c_int64, P, P]
        lib.wind_oracle_integrate_sim.restype = C.c_int64
        lib.wind_oracle_rhs_jac.argtypes = [C.POINTER(_capi.WindNetwork), C.c_int64,
                                            P, P, P]
        lib.wind_oracle_rhs_jac.restype = C.c_int
        lib.wind_oracle_sie_substep.argtypes = [C.POINTER(_capi.WindNetwork), C.c_int64,
                                                C.c_int, C.c_double, P]
        lib.wind_oracle_sie_substep.restype = C.c_int
        _oracle_lib = lib
    return _oracle_lib


def _ranges(nsys, threads):
    if nsys <= 0:
        return [(0, 0)]
    threads = max(1, min(threads, nsys))
    edges = np.linspace(0, nsys, threads + 1).astype(np.int64)
    return [(int(edges[i]), int(edges[i + 1])) for i in range(threads) if edges[i + 1] > edges[i]]


def restated(net: Network, y: np.ndarray, tnow: float, tend: float, atol: float,
             rtol: float, method: str = "sie", controller: str = "gold",
             n_integration_steps: int = 1, max_attempts: int = 0, threads: int = 1):
    """Run the FP64 restatement on all systems; returns (total, status, nsteps)."""
    lib = _load_oracle()
    assert y.dtype == np.float64 and y.flags["C_CONTIGUOUS"]
    ns = _capi.network_struct(net)
    status = np.zeros(net.nsys, np.int32)
    steps = np.zeros(net.nsys, np.int64)
    m = _capi.METHODS[method]
    c = _capi.CONTROLLERS[controller]

    def run(r):
        return lib.wind_oracle_integrate(m, c, C.byref(ns), tnow, tend, n_integration_steps,
                                         y.ctypes.data, r[0], r[1], atol, rtol, max_attempts,
                                         status.ctypes.data, steps.ctypes.data)

    rr = _ranges(net.nsys, threads)
    if len(rr) == 1:
        tot = [run(rr[0])]
    else:
        with cf.ThreadPoolExecutor(len(rr)) as ex:
            tot = list(ex.map(run, rr))
    if any(t < 0 for t in tot):
        raise ValueError("oracle rejected the arguments")
    return int(sum(tot)), status, steps


def restated_global(net: Network, y: np.ndarray, tnow: float, tend: float, atol: float,
                    rtol: float, n_integration_steps: int = 1):
    """The SIE_host controller restated (one step shared by all systems);
    updates ``y`` in place, returns (total substeps, time reached)."""
    lib = _load_oracle()
    assert y.dtype == np.float64 and y.flags["C_CONTIGUOUS"]
    ns = _capi.network_struct(net)
    t = C.c_double(0.0)
    tot = lib.wind_oracle_integrate_global(C.byref(ns), tnow, tend, n_integration_steps,
                                           y.ctypes.data, net.nsys, atol, rtol, C.byref(t))
    if tot < 0:
        raise ValueError("oracle rejected the arguments")
    return int(tot), float(t.value)


def restated_sim(net: Network, y: np.ndarray, tnow: float, tend: float, m: int):
    """The semi-implicit midpoint rule restated (m steps of (tend - tnow)/m
    and the smoothing step); updates ``y`` in place, returns
    (total solves, status, nsteps)."""
    lib = _load_oracle()
    assert y.dtype == np.float64 and y.flags["C_CONTIGUOUS"]
    ns = _capi.network_struct(net)
    status = np.zeros(net.nsys, np.int32)
    steps = np.zeros(net.nsys, np.int64)
    tot = lib.wind_oracle_integrate_sim(C.byref(ns), tnow, tend, m, y.ctypes.data, 0, net.nsys,
                                        status.ctypes.data, steps.ctypes.data)
    if tot < 0:
        raise ValueError("oracle rejected the arguments")
    return int(tot), status, steps


def rhs_jac(net: Network, s: int, y: np.ndarray):
    lib = _load_oracle()
    ns = _capi.network_struct(net)
    f = np.zeros(net.n_eq)
    J = np.zeros(net.n_eq * net.n_eq)
    y = np.ascontiguousarray(y, np.float64)
    lib.wind_oracle_rhs_jac(C.byref(ns), s, y.ctypes.data, f.ctypes.data, J.ctypes.data)
    return f, J.reshape(net.n_eq, net.n_eq)


def sie_substep(net: Network, s: int, y: np.ndarray, h: float, controller="gold"):
    lib = _load_oracle()
    ns = _capi.network_struct(net)
    y = np.array(y, np.float64)
    lib.wind_oracle_sie_substep(C.byref(ns), s, _capi.CONTROLLERS[controller], h,
                                y.ctypes.data)
    return y


# ----------------------------------------------------------------------------
# the reference's own c_baseline
# ----------------------------------------------------------------------------
_ref_cache = {}


def reference_available(net: Network, method="sie", prec="f64") -> bool:
    return os.path.exists(os.path.join(REF, f"{method}_gold_{net.name}_{prec}.so"))


def _load_ref(name: str):
    if name not in _ref_cache:
        path = os.path.join(REF, name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run oracle/build_ref.sh")
        lib = C.CDLL(path)
        _ref_cache[name] = lib
    return _ref_cache[name]


def reference(net: Network, y: np.ndarray, tnow: float, tend: float, atol: float,
              rtol: float, method: str = "sie", n_integration_steps: int = 1,
              prec: str = "f64", threads: int = 1) -> int:
    """Run the reference c_baseline build for this network on all systems.
    ``y`` (float64 [S,N]) is updated in place; returns the total substeps."""
    lib = _load_ref(f"{method}_gold_{net.name}_{prec}.so")
    fn = lib.goldIntegrateSystem
    T = C.c_double if prec == "f64" else C.c_float
    dt = np.float64 if prec == "f64" else np.float32
    fn.argtypes = [T, T, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, T, T]
    fn.restype = C.c_int
    cst = np.ascontiguousarray(net.packed_constants(), dtype=dt)
    ywork = np.ascontiguousarray(y, dtype=dt)
    N = net.n_eq
    nc = cst.shape[1]

    def run(r):
        s0, s1 = r
        return fn(tnow, tend, n_integration_steps,
                  cst.ctypes.data + s0 * nc * cst.itemsize,
                  ywork.ctypes.data + s0 * N * ywork.itemsize,
                  s1 - s0, N, atol, rtol)

    rr = _ranges(net.nsys, threads)
    if len(rr) == 1:
        tot = [run(rr[0])]
    else:
        with cf.ThreadPoolExecutor(len(rr)) as ex:
            tot = list(ex.map(run, rr))
    y[...] = ywork
    return int(sum(tot))
