"""Serving: a request loop with continuous batching over the C ABI.

:class:`Server` wraps ``wind_server_*`` (include/wind.h): requests (a set of
cells of one network, an interval, tolerances) are admitted by device
footprint and merged, whatever their network size, into batch launches that
overlap on the device with the ones already running.  :func:`poisson_load`
drives a server with a seeded Poisson arrival stream and reports p50/p99
latency and systems/s.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import threading
import time

import numpy as np

from . import _capi, lib
from .networks import Network, Workload, random_mass_action, MIXED_SIZES, MIXED_FRACTIONS


class WindServerConfig(C.Structure):
    _fields_ = [("method", C.c_int32), ("solver", C.c_int32), ("controller", C.c_int32),
                ("max_inflight", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("max_waiting", C.c_int64), ("poll_us", C.c_int32), ("pad_", C.c_int32)]


class WindRequest(C.Structure):
    _fields_ = [("net", _capi.WindNetwork), ("y0", C.c_void_p), ("nsys", C.c_int64),
                ("tnow", C.c_double), ("tend", C.c_double), ("atol", C.c_double),
                ("rtol", C.c_double), ("n_integration_steps", C.c_int32), ("pad_", C.c_int32)]


def _declare(w):
    if getattr(w, "_serve_declared", False):
        return w
    P = C.c_void_p
    w.wind_server_default_config.argtypes = [C.POINTER(WindServerConfig)]
    w.wind_server_default_config.restype = None
    w.wind_server_create.argtypes = [C.POINTER(WindServerConfig), C.POINTER(P)]
    w.wind_server_create.restype = C.c_int
    w.wind_server_submit.argtypes = [P, C.POINTER(WindRequest), C.POINTER(C.c_int64)]
    w.wind_server_submit.restype = C.c_int
    w.wind_server_poll.argtypes = [P, C.c_int64, C.c_double, P, P, P, C.POINTER(C.c_double)]
    w.wind_server_poll.restype = C.c_int
    w.wind_server_stats.argtypes = [P, P]
    w.wind_server_stats.restype = C.c_int
    w.wind_server_destroy.argtypes = [P]
    w.wind_server_destroy.restype = C.c_int
    w._serve_declared = True
    return w


@dataclasses.dataclass
class Result:
    y: np.ndarray
    status: np.ndarray
    nsteps: np.ndarray
    latency_s: float


class Server:
    def __init__(self, method="sie", solver="lu_f64", controller="device", max_inflight=4,
                 hbm_budget_bytes=16 << 30, max_waiting=1 << 16, poll_us=100):
        self.w = _declare(lib.load())
        cfg = WindServerConfig()
        self.w.wind_server_default_config(C.byref(cfg))
        cfg.method = _capi.METHODS[method]
        cfg.solver = _capi.SOLVERS[solver]
        cfg.controller = _capi.CONTROLLERS[controller]
        cfg.max_inflight = max_inflight
        cfg.hbm_budget_bytes = hbm_budget_bytes
        cfg.max_waiting = max_waiting
        cfg.poll_us = poll_us
        h = C.c_void_p()
        code = self.w.wind_server_create(C.byref(cfg), C.byref(h))
        lib._check(code, "wind_server_create")
        self.h = h
        self._shapes = {}
        self._lock = threading.Lock()

    def submit(self, wl: Workload) -> int:
        net = wl.net
        q = WindRequest()
        q.net = _capi.network_struct(net)
        y0 = np.ascontiguousarray(wl.y0, np.float64)
        q.y0 = y0.ctypes.data
        q.nsys = net.nsys
        q.tnow, q.tend, q.atol, q.rtol = wl.tnow, wl.tend, wl.atol, wl.rtol
        q.n_integration_steps = wl.n_integration_steps
        rid = C.c_int64()
        code = self.w.wind_server_submit(self.h, C.byref(q), C.byref(rid))
        lib._check(code, "wind_server_submit")
        with self._lock:
            self._shapes[rid.value] = (net.nsys, net.n_eq)
        return rid.value

    def poll(self, rid: int, timeout_s: float = 60.0):
        """The request's Result, or None if not done within timeout_s."""
        nsys, n = self._shapes[rid]
        y = np.empty((nsys, n))
        st = np.empty(nsys, np.int32)
        ns = np.empty(nsys, np.int64)
        lat = C.c_double()
        code = self.w.wind_server_poll(self.h, rid, timeout_s, y.ctypes.data, st.ctypes.data,
                                       ns.ctypes.data, C.byref(lat))
        if code == _capi.WIND_ERR_TIMEOUT:
            return None
        with self._lock:
            self._shapes.pop(rid, None)
        lib._check(code, "wind_server_poll")
        return Result(y, st, ns, lat.value)

    def stats(self):
        out = np.zeros(6, np.int64)
        self.w.wind_server_stats(self.h, out.ctypes.data)
        return dict(zip(["waiting", "admitted", "running", "completed", "launches",
                         "resident_bytes"], out.tolist()))

    def close(self):
        if self.h:
            self.w.wind_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ---------------------------------------------------------------------------
def request_stream(n_requests: int, seed: int = 4, max_cells: int = 100_000,
                   sizes=MIXED_SIZES, fractions=MIXED_FRACTIONS, dt_range=(1e-2, 1e2),
                   atol=1e-6, rtol=1e-4, reactions_per_species: int = 10):
    """Seeded requests: cells per request log-uniform in [1, max_cells]
    (integer), the network size drawn from the mixed-size proportions, a random
    two-body network with 10N reactions (rates log-U[1e-4,1e4]) per cell,
    dt log-uniform in dt_range, y0 U[0,1]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_requests):
        cells = int(np.floor(np.exp(rng.uniform(0.0, np.log(max_cells + 1)))))
        cells = max(1, min(max_cells, cells))
        n = int(rng.choice(sizes, p=np.asarray(fractions) / np.sum(fractions)))
        net = random_mass_action(rng, cells, n, reactions_per_species * n, 1e-4, 1e4)
        dt = float(np.exp(rng.uniform(np.log(dt_range[0]), np.log(dt_range[1]))))
        y0 = rng.uniform(0.0, 1.0, (cells, n))
        out.append(Workload(net, y0, 0.0, dt, atol, rtol, 1, 1, f"req_n{n}_c{cells}"))
    return out


def poisson_load(server: Server, requests, rate_hz: float, seed: int = 4, timeout_s: float = 600):
    """Submit `requests` with exponential inter-arrival times at `rate_hz`
    (seeded), collect every result, and return the latency/throughput summary
    (latency = submit to completion, measured by the server)."""
    rng = np.random.default_rng(seed + 1)
    gaps = rng.exponential(1.0 / rate_hz, len(requests))
    ids = []
    t0 = time.perf_counter()
    t_next = t0
    for wl, gap in zip(requests, gaps):
        t_next += gap
        while True:
            now = time.perf_counter()
            if now >= t_next:
                break
            time.sleep(min(t_next - now, 0.001))
        ids.append(server.submit(wl))
    results = []
    for rid in ids:
        r = server.poll(rid, timeout_s)
        if r is None:
            raise TimeoutError(f"request {rid} not done in {timeout_s} s")
        results.append(r)
    wall = time.perf_counter() - t0
    lat = np.array([r.latency_s for r in results])
    cells = sum(wl.net.nsys for wl in requests)
    return {"requests": len(requests), "rate_hz": rate_hz, "p50_ms": 1e3 * float(np.percentile(lat, 50)),
            "p99_ms": 1e3 * float(np.percentile(lat, 99)), "mean_ms": 1e3 * float(lat.mean()),
            "systems_per_s": cells / wall, "wall_s": wall, "cells": int(cells),
            "flagged": int(sum(int(r.status.max() != 0) for r in results))}, results
