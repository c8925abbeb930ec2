#!/usr/bin/env python
"""Benchmark of the batched stiff-ODE integrators (one JSON line on stdout).

Default workload -- the metric's own configuration: the synthetic dense stiff
network, N = 32 species, 262,144 systems (seed 2): J = Q diag(-lambda) Q^T with
lambda log-U[1e-2,1e6] plus 64 two-body reactions with k log-U[1e-3,1e1],
y0 U[0,1], integrated over dt = 1 at atol 1e-8 / rtol 1e-6, FP64 state, SIE,
the c_baseline controller (cuda/c_baseline/common/common_gold.c:48-153, the
reference arm's own semantics).

The whole job -- all 262,144 systems over the full interval -- is timed once:
the K timed steps are K launches over disjoint contiguous slices that
together cover every system exactly once, each on its own stream.  W warm-up
launches on the first systems precede the timed region (untimed).

* ``value``        systems/s of the MIXED solver (FP32 factors + FP64
                   refinement) with inputs resident in HBM, CUDA events around
                   each launch, L2 flushed (256 MB write) between steps;
* ``solvers``      LU_F64 (plain FP64 LU, slice 0 timed) and GJE_F64 (the
                   reference's Gauss-Jordan in FP64, rate under a device
                   deadline) beside it; ``mixed_over_fp64`` = MIXED / LU_F64;
* ``max_rel_err_vs_reference`` every solver's result on the systems the CPU
                   baseline integrated, against that run of the reference's
                   own FP64 c_baseline;
* ``e2e``          the same metric through the C ABI with pinned host buffers
                   (host<->device copies inside the timed region);
* ``roofline``     the integrate kernel against a peak measured in this run;
* ``cpu_baseline`` the reference's c_baseline (built from its sources into
                   oracle/_ref) on the first systems, every host core.

``--workload katz96`` (config 2), ``nr`` (config 1), ``ma<N>`` (one class of
the mixed-size batch), ``mixed`` (the mixed-size batch in one launch) and
``serve`` (Poisson request streams) select the other workloads.
``--impl reference`` times only the reference's CPU integrator.
``--gpus N`` (under torchrun) splits the same job into N contiguous shards,
one per GPU (strong scaling; systems are independent, there is no exchange
step), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# One hardware work queue per stream for the K slice streams and the K
# concurrent end-to-end calls (the default of 8 queues makes a 9th stream's
# copies wait behind another stream's kernel); read when the CUDA context is
# created, so it is set before torch touches the GPU.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from wind_b200 import networks as W  # noqa: E402

METRIC = "systems/s at 1e-5 rel err vs FP64 (mixed vs plain FP64 GPU); serve p50/p99"


# ---------------------------------------------------------------------------
def make_workload(name: str, systems: int = 0, dt: float = 0.0, rank: int = 0, world: int = 1):
    """The workload and its description; with world > 1 this rank's
    contiguous shard of it (the job's size is fixed: strong scaling)."""
    from wind_b200.replicas import shard_range
    if name == "dense":
        n = systems or 262144
        b, e = shard_range(n, rank, world)
        wl = W.workload_dense(e - b, first=b)
        t = dt or 1.0
        wl = W.Workload(wl.net, wl.y0, 0.0, t, wl.atol, wl.rtol, 1, 1, "dense32")
        return wl, (f"dense N=32 + 64 reactions, {n:,} systems (seed 2), dt={t:g}, "
                    "atol=1e-8 rtol=1e-6")
    wl, desc = _make_other(name, systems, dt)
    b, e = shard_range(wl.net.nsys, rank, world)
    return (wl if world == 1 else wl.subset(slice(b, e))), desc


def _make_other(name: str, systems: int, dt: float):
    if name == "katz96":
        n = systems or 65536
        wl = W.workload_katz96(n, atol=1e-8, rtol=1e-6)
        return wl, f"Katz96 5-species, {n:,} cells (seed 1), dt=1e13 s, atol=1e-8 rtol=1e-6"
    if name == "nr":
        wl = W.workload_nr(1024)
        wl = W.Workload(wl.net, wl.y0, 0.0, 0.01, wl.atol, wl.rtol, 1, 1, "nr_test")
        return wl, "NR stiff linear test, 1024 systems, one output interval t=0..0.01"
    if name.startswith("ma"):
        N = int(name[2:])
        n = systems or dict(zip(W.MIXED_SIZES, W.mixed_counts(200000)))[N]
        t = dt or 1.0
        wl = W.workload_mixed_class(N, n, seed=3, dt=t)
        return wl, (f"mass action N={N}, {10 * N} reactions, {n:,} systems (seed 3), dt={t:g}, "
                    "atol=1e-8 rtol=1e-6")
    raise SystemExit(f"unknown workload {name}")


def sie_flops(n: int, f_f: float, f_j: float) -> float:
    """LU-equivalent FLOPs of one SIE substep: (2/3)N^3 + 4N^2 + F_f + F_J."""
    return (2.0 / 3.0) * n ** 3 + 4.0 * n * n + f_f + f_j


def flops_per_substep(wl, method: str) -> float:
    n = wl.net.n_eq
    if wl.net.kind == W.NET_KATZ96:
        f_f, f_j = 40.0, 20.0
    elif wl.net.kind in (W.NET_NR_TEST, W.NET_STIFFTRIG):
        f_f, f_j = 6.0, 0.0
    else:
        r = wl.net.n_react
        f_f = 5.0 * r + (2.0 * n * n if wl.net.linear is not None else 0.0)
        f_j = 8.0 * r
    if method == "rk2":
        return f_f + 2.0 * n
    return sie_flops(n, f_f, f_j)


def slice_bounds(nsys: int, k: int):
    """K contiguous slices covering [0, nsys) exactly once."""
    e = np.linspace(0, nsys, max(1, k) + 1).round().astype(np.int64)
    return [(int(e[i]), int(e[i + 1])) for i in range(len(e) - 1)]


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples (200 ms) while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_gemm_peak(torch, dev, dtype):
    """cuBLAS GEMM 8192^3 in `dtype` (TF32 off for float32), best of 5 (TFLOP/s)."""
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(8192, 8192, dtype=dtype, device=dev)
    b = torch.randn(8192, 8192, dtype=dtype, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    return 2.0 * 8192 ** 3 / best / 1e12


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


# ---------------------------------------------------------------------------
def reference_run(wl, first: int, count: int, method: str, threads: int):
    """The reference c_baseline (oracle/_ref) on systems [first, first+count):
    returns (seconds, final state) or (None, reason)."""
    from oracle import pyoracle as O
    if not O.reference_available(wl.net, method, "f64"):
        return None, "oracle/_ref not built for " + wl.net.name
    sub = wl.subset(slice(first, first + count))
    y = sub.y0.copy()
    t0 = time.perf_counter()
    O.reference(sub.net, y, sub.tnow, sub.tend, sub.atol, sub.rtol, method,
                sub.n_integration_steps, threads=threads)
    return time.perf_counter() - t0, y


def reference_sample_size(wl, method: str, target_s: float, cores: int) -> int:
    """Systems the reference integrates in about target_s on `cores` threads
    (calibrated on one system per core)."""
    n0 = min(wl.net.nsys, cores)
    dt, _ = reference_run(wl, 0, n0, method, cores)
    if dt is None:
        return 0
    per = dt / max(1, n0) * 1.0  # seconds per system per core-wave
    waves = max(1.0, target_s / max(dt, 1e-9))
    return int(min(wl.net.nsys, max(n0, round(waves * n0))))


def run_reference_arm(args, wl, desc):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    per_step = reference_sample_size(wl, args.method, args.ref_seconds, cores)
    if per_step == 0:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built for " + wl.net.name}))
        return
    vals, off, samples = [], 0, []
    for i in range(args.warmup + args.steps):
        if off + per_step > wl.net.nsys:
            off = 0
        dt, _ = reference_run(wl, off, per_step, args.method, cores)
        if i >= args.warmup:
            vals.append(per_step / dt)
            samples.append(f"{off}..{off + per_step - 1}")
        off += per_step
    value = statistics.median(vals)
    sample = (f"{per_step} systems per step ({args.steps} steps: systems {samples[0]} ... {samples[-1]}), "
              f"c_baseline FP64 (-Dfloat=double) built from the reference sources, "
              f"one contiguous shard per thread")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "systems/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict(args, wl, desc),
            "cpu_baseline": {"value": value, "unit": "systems/s", "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "systems/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(finite_json(line)), flush=True)


STATUS_BITS = {1: "nonfinite", 2: "max_attempts", 4: "stalled", 8: "refine_fallback",
               16: "timeout", 32: "bad_input"}


def status_counts(st) -> dict:
    """Systems carrying each per-system status bit (include/wind.h)."""
    st = np.asarray(st)
    return {name: int(((st & bit) != 0).sum()) for bit, name in STATUS_BITS.items()
            if ((st & bit) != 0).any()}


def error_stats(y, y_ref, atol: float) -> dict:
    """Max relative error of y against y_ref ([S, N]) over the systems finite
    in both, and how many systems diverge in both or in only one of them."""
    fa = np.isfinite(y).all(axis=1)
    fr = np.isfinite(y_ref).all(axis=1)
    both = fa & fr
    e = (np.abs(y[both] - y_ref[both]) / np.maximum(np.abs(y_ref[both]), atol)) if both.any() else None
    return {"max_rel_err": float(e.max()) if e is not None else None,
            "finite_systems": int(both.sum()), "nonfinite_both": int((~fa & ~fr).sum()),
            "finiteness_differs": int((fa != fr).sum())}


def finite_json(obj):
    """obj with every non-finite float replaced by None (strict JSON)."""
    if isinstance(obj, float):
        return obj if np.isfinite(obj) else None
    if isinstance(obj, dict):
        return {k: finite_json(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [finite_json(v) for v in obj]
    return obj


def config_dict(args, wl, desc):
    return {"workload": desc, "method": args.method, "controller": args.controller,
            "systems": wl.net.nsys, "equations": wl.net.n_eq,
            "l2": ("each step reads a slice of the inputs no earlier step of the timed region "
                   "read (the dense workload's 1.4 GB of inputs exceed L2); L2 flushed by a 256 MB "
                   "write before the timed region and before each solver-rate run"),
            "steps_cover": ("the K timed steps are K launches over disjoint slices covering every "
                            "system once, each on its own stream"),
            "parallelism": (f"{int(os.environ.get('WORLD_SIZE', '1'))} independent shards of the "
                            "job, one per GPU (no exchange step)")}


# ---------------------------------------------------------------------------
def run_main(args, wl, desc):
    import ctypes as C
    import torch
    from wind_b200 import _capi, lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    wlib = lib.load()
    stream = torch.cuda.current_stream(dev)
    net = wl.net
    N, S = net.n_eq, net.nsys
    keys = [k for k in ("constants", "rates", "species", "linear") if getattr(net, k) is not None]
    d_arr = {k: torch.from_numpy(np.ascontiguousarray(getattr(net, k))).to(dev) for k in keys}
    y0 = torch.from_numpy(wl.y0).to(dev)
    y = y0.clone()
    status = torch.zeros(S, dtype=torch.int32, device=dev)
    nsteps = torch.zeros(S, dtype=torch.int64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2
    bounds = slice_bounds(S, args.steps)

    def launch(solver, s0, s1, timeout_s=0.0):
        """One wind_integrate launch over systems [s0, s1) of the resident
        batch; returns the substeps counted on the device."""
        o = lib.options(args.method, solver, args.controller, args.spec_width, 0, timeout_s)
        ns = _capi.network_struct(net, {k: v[s0:s1] for k, v in d_arr.items()})
        total = C.c_int64(0)
        code = wlib.wind_integrate(C.byref(o), C.byref(ns), wl.tnow, wl.tend,
                                   wl.n_integration_steps, y[s0:s1].data_ptr(), s1 - s0, wl.atol,
                                   wl.rtol, status[s0:s1].data_ptr(), nsteps[s0:s1].data_ptr(),
                                   C.byref(total), _capi.MEM_DEVICE, stream.cuda_stream)
        if code != 0:
            raise RuntimeError(f"wind_integrate failed: {code} {wlib.wind_last_error().decode()}")
        return int(total.value)

    def timed(solver, s0, s1, timeout_s=0.0):
        y[s0:s1].copy_(y0[s0:s1])
        flush.zero_()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        n = launch(solver, s0, s1, timeout_s)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) * 1e-3, n

    # ---- warm-up (untimed): W launches of each fast solver on a few systems,
    # each cut by a 0.25 s device deadline (module load, occupancy and
    # allocator caches; a few slow systems would otherwise hold a warm-up
    # launch for tens of seconds)
    b0 = bounds[0]
    cand = ["mixed", "lu_f64"] if args.solver == "auto" else [args.solver]
    for s in cand:
        for i in range(args.warmup):
            timed(s, b0[0], min(b0[1], b0[0] + 1024), timeout_s=0.25)

    # ---- MIXED vs LU_F64 on the same first slice under the same device
    # deadline: substeps/s of each at full occupancy (the ratio), and
    # (solver "auto") the headline solver = the faster one
    # (mass action above 32 species: also MIXED_TC, the same solve with the
    # inverse's rank updates on the tensor cores -- the A/B of the two)
    results = {}
    compared = ["mixed", "lu_f64"]
    if net.kind == W.NET_MASS_ACTION and N > 32 and args.method == "sie":
        compared.append("mixed_tc")
    for s in compared:
        t, n = timed(s, *b0, timeout_s=args.compare_seconds)
        results[s] = {"substeps_per_s": n / t,
                      "timed": f"slice 0 under a {args.compare_seconds:g} s device deadline"}
    mixed_over_fp64 = results["mixed"]["substeps_per_s"] / results["lu_f64"]["substeps_per_s"]
    if "mixed_tc" in results:
        results["mixed_tc"]["over_mixed"] = (results["mixed_tc"]["substeps_per_s"] /
                                             results["mixed"]["substeps_per_s"])
    main_solver = args.solver if args.solver != "auto" else max(
        cand, key=lambda s: results[s]["substeps_per_s"])

    # ---- the timed job: every system once, K launches, each on its own
    # stream.  A persistent launch frees its SMs block by block as its queue
    # drains, so the next slice's blocks start beside the previous slice's
    # longest systems (the ones the refinement cap holds for ~10^6 substeps)
    # instead of waiting behind them, as in one launch over all systems; each
    # input byte is read once (the job's inputs are larger than L2), and the
    # region spans the first launch to the last completion.
    streams = [torch.cuda.Stream(dev) for _ in bounds]
    y.copy_(y0)
    flush.zero_()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = lib.launch_count()
    o_main = lib.options(args.method, main_solver, args.controller, args.spec_width)
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        done = []
        for i, (s0, s1) in enumerate(bounds):
            ss = streams[i]
            ss.wait_event(e0)
            ns = _capi.network_struct(net, {k: v[s0:s1] for k, v in d_arr.items()})
            code = wlib.wind_integrate(C.byref(o_main), C.byref(ns), wl.tnow, wl.tend,
                                       wl.n_integration_steps, y[s0:s1].data_ptr(), s1 - s0, wl.atol,
                                       wl.rtol, status[s0:s1].data_ptr(), nsteps[s0:s1].data_ptr(),
                                       None, _capi.MEM_DEVICE, ss.cuda_stream)
            if code != 0:
                raise RuntimeError(f"wind_integrate failed: {code} {wlib.wind_last_error().decode()}")
            ev = torch.cuda.Event()
            ev.record(ss)
            done.append(ev)
        for ev in done:
            stream.wait_event(ev)
        e1.record(stream)
        torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches = lib.launch_count() - launches0
    tot = e0.elapsed_time(e1) * 1e-3
    substeps = int(nsteps.sum())
    times = [tot]
    if dist is not None:
        tt = torch.tensor([tot], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot = float(tt.item())
    s_job = S
    if dist is not None:
        tt = torch.tensor([S], dtype=torch.int64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.SUM)
        s_job = int(tt.item())
    value = s_job / tot
    y_main = y.cpu().numpy()
    st_main = status.cpu().numpy()
    steps_main = nsteps.cpu().numpy()
    results[main_solver + "_full_job"] = {"systems_per_s": S / tot, "substeps": substeps,
                                          "systems": S, "timed": "all slices, one stream each",
                                          "status": status_counts(st_main)}
    outs = {main_solver: y_main}
    per_sys = float(steps_main[b0[0]:b0[1]].mean())
    for s in compared:
        results[s]["systems_per_s"] = results[s]["substeps_per_s"] / per_sys
        results[s]["systems_per_s_definition"] = "substeps/s / mean substeps per system of the main run"

    # ---- GJE_F64 (the reference's Gauss-Jordan in FP64): rate under a deadline
    t, n = timed("gje_f64", *b0, timeout_s=args.gje_seconds)
    results["gje_f64"] = {"substeps_per_s": n / t, "systems_per_s": n / t / per_sys,
                          "substeps": n, "timed": (f"slice 0 under a {args.gje_seconds:g} s device "
                                                   "deadline; systems/s = substeps/s / mean "
                                                   "substeps per system of the main run")}
    mixed_over_gje = results["mixed"]["substeps_per_s"] / results["gje_f64"]["substeps_per_s"]

    # ---- e2e through the C ABI with pinned host buffers: by default the
    # whole job again, as K concurrent wind_integrate calls over the same
    # slices as the resident run (host memory mode: each uploads its inputs,
    # integrates and downloads its state on its own stream, from its own
    # host thread -- ctypes releases the GIL), so one call's slowest systems
    # overlap the others' work as in the resident run; --e2e-systems /
    # --e2e-calls select a smaller sample.  Device time: an event before
    # every call's upload to an event after every call's download.
    e2e_lo, e2e_hi = 0, min(S, args.e2e_systems) if args.e2e_systems > 0 else S
    n_calls = args.e2e_calls if args.e2e_calls > 0 else len(bounds)
    e2e_calls = [(int(a0), int(a1)) for a0, a1 in zip(
        np.linspace(e2e_lo, e2e_hi, n_calls + 1).round()[:-1],
        np.linspace(e2e_lo, e2e_hi, n_calls + 1).round()[1:]) if a1 > a0]
    h_arr = {k: torch.from_numpy(np.ascontiguousarray(getattr(net, k)[e2e_lo:e2e_hi])).pin_memory()
             for k in keys}
    h_y0 = torch.from_numpy(np.ascontiguousarray(wl.y0[e2e_lo:e2e_hi])).pin_memory()
    h_y = h_y0.clone().pin_memory()
    o = lib.options(args.method, main_solver, args.controller, args.spec_width)
    e2e_streams = [torch.cuda.Stream(dev) for _ in e2e_calls]
    codes = [None] * len(e2e_calls)

    def e2e_call(i):
        a0, a1 = e2e_calls[i]
        torch.cuda.set_device(dev)
        hns = _capi.network_struct(net, {k: v[a0:a1] for k, v in h_arr.items()})
        codes[i] = wlib.wind_integrate(C.byref(o), C.byref(hns), wl.tnow, wl.tend,
                                       wl.n_integration_steps, h_y[a0:a1].data_ptr(), a1 - a0,
                                       wl.atol, wl.rtol, None, None, None, _capi.MEM_HOST,
                                       e2e_streams[i].cuda_stream)

    flush.zero_()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for ss in e2e_streams:
        ss.wait_event(e0)
    threads = [threading.Thread(target=e2e_call, args=(i,)) for i in range(len(e2e_calls))]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    for ss in e2e_streams:
        stream.wait_stream(ss)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if any(c != 0 for c in codes):
        raise RuntimeError(f"e2e wind_integrate failed: {codes}")
    e2e_times = [e0.elapsed_time(e1) * 1e-3]
    h2d = (e2e_hi - e2e_lo) * N * 8 + sum(v.numel() * v.element_size() for v in h_arr.values())
    d2h = (e2e_hi - e2e_lo) * N * 8 + 8 * len(e2e_calls)
    e2e_tot = sum(e2e_times)
    if dist is not None:
        tt = torch.tensor([e2e_tot], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_tot = float(tt.item())
    e2e_sys = e2e_hi - e2e_lo
    e2e_job = e2e_sys
    if dist is not None:
        tt = torch.tensor([e2e_sys], dtype=torch.int64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.SUM)
        e2e_job = int(tt.item())
    e2e_same = np.array_equal(h_y.numpy(), y_main[e2e_lo:e2e_hi], equal_nan=True)

    # ---- roofline of the integrate kernel
    fps = flops_per_substep(wl, args.method)
    flops = fps * substeps
    kernel_s = sum(times)
    achieved = flops / kernel_s / 1e12
    fp32_main = main_solver == "mixed"
    peak = measured_gemm_peak(torch, dev, torch.float32 if fp32_main else torch.float64)
    peak_fp64 = peak if not fp32_main else measured_gemm_peak(torch, dev, torch.float64)
    alg_bytes = S * (16 * N) + net.nbytes()
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    # DRAM bytes per launch from an ncu capture of the same kernel on a
    # smaller batch, scaled by systems (every system's network and state cross
    # HBM once per launch, so traffic grows in proportion to the systems):
    # k_warp LU_F64 on 4,096 dense systems read 22.2 MB (5,420 B per system
    # against 5,376 B of network and state; its state writes were still in L2
    # when the capture ended), k_lane LU_F64 on 16,384 Katz96 cells 136.7 B
    traffic_per_system = args.traffic_per_system or {
        ("dense", "lu_f64"): 5420.0, ("katz96", "lu_f64"): 136.7}.get((args.workload, main_solver), 0.0)
    traffic = traffic_per_system * S / len(bounds) if traffic_per_system else None
    roof = {"bound": "fp32" if fp32_main else "fp64", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, "
                               "smaller-batch capture scaled by systems" if traffic else None),
            "peak_source": ("cuBLAS SGEMM 8192^3 (TF32 off) measured in this run" if fp32_main
                            else "cuBLAS DGEMM 8192^3 measured in this run"),
            "frac_of_fp64_peak": achieved / peak_fp64, "fp64_peak": peak_fp64,
            "flops_per_substep": fps, "substeps": substeps,
            "hbm": {"alg_bytes_per_launch": alg_bytes / len(bounds),
                    "achieved_gbs": alg_bytes / kernel_s / 1e9, "peak_gbs": hbm_peak,
                    "frac": alg_bytes / kernel_s / 1e9 / hbm_peak,
                    "peak_source": "MEASURED_PEAKS.json" if "hbm_gbs" in peaks else "fallback"}}

    # ---- reference CPU baseline on the first systems, and every solver's
    # error against its FP64 result on those systems
    cpu, errs = None, {}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        n_cpu = reference_sample_size(wl, args.method, args.ref_seconds, cores)
        n_cpu = min(n_cpu, b0[1] - b0[0])
        if n_cpu > 0:
            dt, y_ref = reference_run(wl, 0, n_cpu, args.method, cores)
            for s in ("mixed", "lu_f64"):
                if s not in outs:
                    timed(s, 0, n_cpu)
                    outs[s] = y.cpu().numpy()[:n_cpu]
            cpu = {"value": n_cpu / dt, "unit": "systems/s", "cores": cores, "kind": "reference",
                   "sample": (f"systems 0..{n_cpu - 1} of {S:,}, {dt:.1f} s; c_baseline FP64 "
                              "(-Dfloat=double) built from the reference sources")}
            for s, yy in outs.items():
                errs[s] = error_stats(yy[:n_cpu], y_ref, wl.atol)
            errs["systems"] = n_cpu
            errs["metric"] = ("max |y - y_ref| / max(|y_ref|, atol) over the systems finite in "
                              "both; systems that diverge (non-finite) are counted")

    # ---- config 2 (Katz96) beside the headline, cheap
    extra = None
    if args.workload == "dense" and not args.no_extra:
        extra = katz96_extra(args, torch, dev, lib, _capi, C)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": "systems/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(bounds),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 factors + f64 refinement, f64 state" if fp32_main else "f64",
            "data": "synthetic",
            "config": dict(config_dict(args, wl, desc), solver=main_solver),
            "solvers": results, "mixed_over_fp64": mixed_over_fp64,
            "mixed_over_fp64_definition": ("MIXED / LU_F64 substeps/s on slice 0 under the same "
                                           "device deadline (same systems, full occupancy)"),
            "mixed_over_gje_f64": mixed_over_gje,
            "max_rel_err_vs_reference": errs or None,
            "e2e": {"value": e2e_job / e2e_tot, "unit": "systems/s",
                    "h2d_bytes_per_step": int(h2d / len(e2e_calls)),
                    "d2h_bytes_per_step": int(d2h / len(e2e_calls)),
                    "h2d_bytes_total": int(h2d), "d2h_bytes_total": int(d2h),
                    "systems": e2e_sys, "calls": len(e2e_calls),
                    "step": (f"systems 0..{e2e_sys - 1} as {len(e2e_calls)} concurrent "
                             "wind_integrate calls on host buffers, one stream each"),
                    "state_equals_resident_run": bool(e2e_same)},
            "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu,
            "clocks": clk.summary(), "config2_katz96": extra}
    print(json.dumps(finite_json(line)), flush=True)


def katz96_extra(args, torch, dev, lib, _capi, C):
    """Config 2 (Katz96, 65,536 cells, dt = 1e13 s) systems/s per solver."""
    wl = W.workload_katz96(65536, atol=1e-8, rtol=1e-6)
    net = wl.net
    d = {"constants": torch.from_numpy(net.constants).to(dev)}
    y0 = torch.from_numpy(wl.y0).to(dev)
    y = y0.clone()
    stream = torch.cuda.current_stream(dev)
    wlib = lib.load()
    out = {}
    for solver in ("lu_f64", "mixed", "gje_f64"):
        ts = []
        for i in range(4):
            y.copy_(y0)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            o = lib.options("sie", solver, args.controller)
            ns = _capi.network_struct(net, d)
            tot = C.c_int64(0)
            e0.record(stream)
            code = wlib.wind_integrate(C.byref(o), C.byref(ns), wl.tnow, wl.tend, 1, y.data_ptr(),
                                       net.nsys, wl.atol, wl.rtol, None, None, C.byref(tot),
                                       _capi.MEM_DEVICE, stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if code != 0:
                raise RuntimeError(f"katz96 {solver}: {code}")
            if i:
                ts.append(e0.elapsed_time(e1) * 1e-3)
        out[solver] = {"systems_per_s": net.nsys / statistics.median(ts), "substeps": int(tot.value)}
    # the reference caller's own path: the mangled cudaIntegrateSystem of
    # lib/katz96/sie.so on pageable float32 NumPy arrays (python/wind_harness.py:32-40,
    # python/ode_systems/ode_base.py:441-469), wall clock around the call
    try:
        fn = lib.legacy("katz96", "sie")
        c32 = np.ascontiguousarray(net.constants, dtype=np.float32)
        drop = {}
        for solver in ("gje_f64", "lu_f64"):
            os.environ["WIND_LEGACY_SOLVER"] = solver
            ts = []
            for i in range(3):
                y32 = np.ascontiguousarray(wl.y0, dtype=np.float32)
                t0 = time.perf_counter()
                n = fn(0.0, 1e13, 1, c32.ctypes.data, y32.ctypes.data, net.nsys, 5, 1e-8, 1e-6)
                if i:
                    ts.append(time.perf_counter() - t0)
                if n < 0:
                    raise RuntimeError(f"cudaIntegrateSystem returned {n}")
            drop[solver] = {"systems_per_s": net.nsys / statistics.median(ts)}
        os.environ.pop("WIND_LEGACY_SOLVER", None)
        drop["call"] = ("_Z19cudaIntegrateSystemffiPfS_iiff from lib/katz96/sie.so, pageable "
                        "float32 host arrays, wall clock per call (host conversions, copies and "
                        "the integration)")
        out["e2e_dropin"] = drop
    except Exception as exc:  # the headline line must still print
        os.environ.pop("WIND_LEGACY_SOLVER", None)
        out["e2e_dropin"] = {"error": str(exc)}
    out["workload"] = "Katz96 5-species, 65,536 cells (seed 1), dt=1e13 s, atol=1e-8 rtol=1e-6"
    return out


# ---------------------------------------------------------------------------
def run_mixed(args):
    """The mixed-size batch (N in {5,16,32,64,157} at 40/25/20/10/5 %, 10N
    reactions) through wind_integrate_batch -- one persistent launch for all
    sizes -- timed with CUDA events.  Beside it, per size class, MIXED and
    LU_F64 substeps/s under the same device deadline (the solver ratio per
    class, and over the batch weighted by each class's share of the work)."""
    import torch
    from wind_b200 import lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    nsys = args.systems or 200000
    dt = args.dt or 1.0
    groups = W.workload_mixed(nsys, seed=3, dt=dt, atol=1e-8, rtol=1e-6)
    solver = args.solver
    times = []
    for i in range(args.warmup + args.steps):
        dg = [lib.DeviceGroup(wl if i >= args.warmup else wl.subset(slice(0, min(wl.net.nsys, 512))), dev)
              for wl in groups]
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream(dev)
        arr = (lib._capi.WindGroup * len(dg))(*[g.struct() for g in dg])
        o = lib.options("sie", solver, args.controller)
        e0.record(stream)
        code = lib.load().wind_integrate_batch(lib.C.byref(o), arr, len(dg), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if code != 0:
            raise RuntimeError(f"wind_integrate_batch failed: {code}")
        if i >= args.warmup:
            times.append(e0.elapsed_time(e1) * 1e-3)
    work = {wl.net.n_eq: int(g.nsteps.sum()) for wl, g in zip(groups, dg)}
    status = status_counts(np.concatenate([g.status.cpu().numpy() for g in dg]))
    # per-class solver rates under a device deadline
    per_class = {}
    for wl in groups:
        d_arr = {k: torch.from_numpy(np.ascontiguousarray(getattr(wl.net, k))).to(dev)
                 for k in ("rates", "species", "linear") if getattr(wl.net, k) is not None}
        row = {}
        for s in ("lu_f64", "mixed"):
            y = torch.from_numpy(wl.y0).to(dev)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            tot, _, _ = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, "sie", s,
                                      args.controller, timeout_s=args.compare_seconds,
                                      device_arrays=d_arr)
            e1.record()
            torch.cuda.synchronize(dev)
            row[s] = tot / (e0.elapsed_time(e1) * 1e-3)
        row["mixed_over_lu_f64"] = row["mixed"] / row["lu_f64"]
        per_class[str(wl.net.n_eq)] = row
    t_lu = sum(work[int(n)] / r["lu_f64"] for n, r in per_class.items())
    t_mx = sum(work[int(n)] / r["mixed"] for n, r in per_class.items())
    line = {"metric": METRIC, "workload": "mixed", "unit": "systems/s",
            "value": nsys / statistics.median(times), "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median(times),
            "config": {"workload": (f"{nsys:,} systems, N in {{5,16,32,64,157}} at 40/25/20/10/5 %, "
                                    f"10N reactions (seed 3), dt={dt:g}, atol 1e-8 rtol 1e-6, one "
                                    "persistent launch (wind_integrate_batch)"),
                       "controller": args.controller, "solver": solver},
            "substeps_per_class": work, "status": status,
            "per_class_substeps_per_s": per_class,
            "mixed_over_fp64": t_lu / t_mx,
            "mixed_over_fp64_definition": ("batch time with LU_F64 / with MIXED, each class's "
                                           "substeps at that solver's per-class rate under a "
                                           f"{args.compare_seconds:g} s device deadline")}
    print(json.dumps(finite_json(line)), flush=True)


def run_ntile(args):
    """Katz96 tiled Ntile times (the Precompiler's tiling; the reference's
    NtileScaling sweep, python/ntbks/NtileScaling.ipynb, varies Ntile 1-50):
    device time of one wind_integrate call per (Ntile, method, solver), on
    resident inputs, median of --steps calls after --warmup."""
    import torch
    from wind_b200 import lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    cells = args.systems or 65536
    base = W.workload_katz96(cells, atol=args.ntile_tol, rtol=args.ntile_tol)
    rows = []
    for nt in [int(x) for x in args.ntiles.split(",")]:
        wl = W.tile_workload(base, nt)
        d = {"constants": torch.from_numpy(wl.net.constants).to(dev)}
        y0 = torch.from_numpy(wl.y0).to(dev)
        for method, tend, solvers in (("sie", 1e13, ("gje_f64", "lu_f64")), ("rk2", 1e9, ("gje_f64",))):
            for solver in solvers:
                ts = []
                for i in range(args.warmup + args.steps):
                    y = y0.clone()
                    torch.cuda.synchronize(dev)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    tot, st, _ = lib.integrate(wl.net, y, 0.0, tend, wl.atol, wl.rtol, method, solver,
                                               args.controller, device_arrays=d)
                    e1.record()
                    torch.cuda.synchronize(dev)
                    if i >= args.warmup:
                        ts.append(e0.elapsed_time(e1))
                rows.append({"ntile": nt, "neqn": 5 * nt, "method": method, "solver": solver,
                             "interval_s": tend, "ms": statistics.median(ts), "substeps": tot,
                             "flagged": int((st.cpu().numpy() != 0).sum())})
    line = {"metric": "time per call vs equations per system (tiled Katz96)", "workload": "ntile",
            "unit": "ms", "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": (f"Katz96 (seed 1), {cells:,} cells, each tiled Ntile times "
                                    f"(identical tiles, shared constants), atol=rtol={args.ntile_tol:g}, "
                                    "SIE over 1e13 s, RK2 over 1e9 s, one call"),
                       "controller": args.controller},
            "rows": rows}
    print(json.dumps(finite_json(line)), flush=True)


def run_serve(args):
    """Serving: seeded Poisson request streams at several rates; one JSON line
    with p50/p99 latency and systems/s per rate."""
    import torch
    from wind_b200 import serve
    torch.cuda.set_device(0)
    rates = [float(r) for r in args.rates.split(",")]
    out = []
    for i, rate in enumerate(rates):
        reqs = serve.request_stream(args.requests, seed=4 + i, max_cells=args.max_cells,
                                    dt_range=(args.dt_lo, args.dt_hi), atol=1e-6, rtol=1e-4)
        with serve.Server(solver=args.solver,
                          max_inflight=4) as srv:
            serve.poisson_load(srv, reqs[:8], rate)  # warm-up
            summary, _ = serve.poisson_load(srv, reqs, rate)
            summary["launches"] = srv.stats()["launches"]
        out.append(summary)
    line = {"metric": METRIC, "workload": "serve", "unit": "ms",
            "config": {"workload": (f"Poisson arrivals, {args.requests} requests per rate, cells "
                                    f"log-U[1,{args.max_cells}], N from {{5,16,32,64,157}} at "
                                    f"40/25/20/10/5 %, 10N reactions, dt log-U[{args.dt_lo},{args.dt_hi}], "
                                    "atol 1e-6 rtol 1e-4, seed 4+i"),
                       "max_inflight": 4},
            "rates": out}
    print(json.dumps(finite_json(line)), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="wind", choices=["wind", "reference"])
    ap.add_argument("--workload", default="dense")
    ap.add_argument("--systems", type=int, default=0, help="override the system count "
                    "(profiling runs on a small case; the headline uses the default)")
    ap.add_argument("--dt", type=float, default=0.0, help="interval override (profiling cases)")
    ap.add_argument("--method", default="sie", choices=["sie", "rk2"])
    ap.add_argument("--solver", default="auto", choices=["auto", "gje_f64", "lu_f64", "mixed", "mixed_tc"])
    ap.add_argument("--controller", default="gold", choices=["gold", "device"])
    ap.add_argument("--spec-width", type=int, default=0)
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--gje-seconds", type=float, default=3.0)
    ap.add_argument("--e2e-systems", type=int, default=0,
                    help="systems of the end-to-end (host buffer) measurement")
    ap.add_argument("--e2e-calls", type=int, default=0,
                    help="concurrent wind_integrate calls the end-to-end systems are split "
                         "into (0: one per timed step, as the resident run)")
    ap.add_argument("--compare-seconds", type=float, default=4.0,
                    help="device deadline of the MIXED and LU_F64 rate runs on slice 0")
    ap.add_argument("--traffic-per-system", type=float, default=0.0,
                    help="DRAM bytes per system per launch from an ncu capture (roofline.traffic)")
    ap.add_argument("--profile", action="store_true",
                    help="launch only the chosen solver's integrate kernel (warm-up + steps launches "
                         "on the first --systems systems) -- the small case an ncu capture runs")
    ap.add_argument("--deadline", type=float, default=0.0,
                    help="device deadline per launch in seconds (bounds a profiled launch)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--ntiles", default="1,2,5,10,20,50", help="Ntile values of --workload ntile")
    ap.add_argument("--ntile-tol", type=float, default=5e-3,
                    help="atol = rtol of --workload ntile (the reference sweep's 5e-3)")
    ap.add_argument("--rates", default="10,30,100,300,1000,2000", help="serving request rates (Hz)")
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--max-cells", type=int, default=2000)
    ap.add_argument("--dt-lo", type=float, default=1e-4)
    ap.add_argument("--dt-hi", type=float, default=1e-3)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "mixed":
        return run_mixed(args)
    if args.workload == "ntile":
        return run_ntile(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return None
        wl, desc = make_workload(args.workload, args.systems, args.dt)
        return run_reference_arm(args, wl, desc)
    wl, desc = make_workload(args.workload, args.systems, args.dt, rank, world)
    if args.profile:
        return run_profile(args, wl, desc)
    return run_main(args, wl, desc)


def run_profile(args, wl, desc):
    """Warm-up + K launches of one solver on the resident batch, nothing
    else on the GPU: the command an ncu capture of the integrate kernel runs."""
    import torch
    from wind_b200 import lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    solver = args.solver if args.solver != "auto" else (
        "mixed" if wl.net.kind == W.NET_MASS_ACTION else "lu_f64")
    d_arr = {k: torch.from_numpy(np.ascontiguousarray(getattr(wl.net, k))).to(dev)
             for k in ("constants", "rates", "species", "linear") if getattr(wl.net, k) is not None}
    y0 = torch.from_numpy(wl.y0).to(dev)
    out = []
    for i in range(args.warmup + args.steps):
        y = y0.clone()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        tot, st, _ = lib.integrate(wl.net, y, wl.tnow, wl.tend, wl.atol, wl.rtol, args.method, solver,
                                   args.controller, timeout_s=args.deadline, device_arrays=d_arr)
        e1.record()
        torch.cuda.synchronize(dev)
        if i >= args.warmup:
            out.append({"ms": e0.elapsed_time(e1), "substeps": tot,
                        "flagged": int((st.cpu().numpy() != 0).sum())})
    print(json.dumps({"profile": desc, "solver": solver, "controller": args.controller,
                      "deadline_s": args.deadline, "launches": out}), flush=True)


if __name__ == "__main__":
    main()
