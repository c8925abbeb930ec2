#!/usr/bin/env python
"""Benchmark of the batched stiff-ODE integrators (one JSON line on stdout).

Default workload: the Katz96 primordial H/He network, 65,536 cells with
T log-U[1e2,1e8] K, nH log-U[1e-4,1e4] cm^-3, UV log-U[1e-15,1e-11] 1/s
(seed 1), one integration over dt = 1e13 s, FP64 state, SIE, atol 1e-8 /
rtol 1e-6.  One "step" integrates every cell over the whole interval.

* ``value``   systems/s with inputs resident in HBM (CUDA events around each
              integrate launch; L2 flushed between steps);
* ``e2e``     the same through the C ABI with pinned host buffers, host<->device
              copies inside the timed region;
* ``roofline`` the integrate kernel against the measured FP64 peak (cuBLAS
              DGEMM timed in this run), algorithmic FLOPs = LU-equivalent count
              per substep x substeps counted on the device;
* ``cpu_baseline`` the reference's own CPU integrator (c_baseline, built from
              the reference sources into oracle/_ref) on a strided sample of the
              same cells with every host core.

``--impl reference`` times only the reference's CPU integrator on this config.
``--gpus N`` (under torchrun) runs N independent replicas ("replicas only":
systems are independent, there is no exchange step).
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

from wind_b200 import networks as W  # noqa: E402

METRIC = "systems/s at 1e-5 rel err vs FP64 (mixed vs plain FP64 GPU); serve p50/p99"


# ---------------------------------------------------------------------------
def make_workload(name: str, systems: int = 0, dt: float = 0.0):
    if name == "katz96":
        n = systems or 65536
        wl = W.workload_katz96(n, atol=1e-8, rtol=1e-6)
        return wl, f"Katz96 5-species, {n:,} cells, dt=1e13 s, atol=1e-8 rtol=1e-6"
    if name == "katz96_loose":
        n = systems or 65536
        wl = W.workload_katz96(n)
        return wl, f"Katz96 5-species, {n:,} cells, dt=1e13 s, atol=rtol=5e-3"
    if name == "nr":
        wl = W.workload_nr(1024)
        wl = W.Workload(wl.net, wl.y0, 0.0, 0.01, wl.atol, wl.rtol, 1, 1, "nr_test")
        return wl, "NR stiff linear test, 1024 systems, one output interval t=0..0.01"
    if name == "dense":
        n = systems or 16384
        wl = W.workload_dense(n)
        t = dt or 1.0
        wl = W.Workload(wl.net, wl.y0, 0.0, t, wl.atol, wl.rtol, 1, 1, "dense32")
        return wl, f"dense N=32 + 64 reactions, {n:,} systems, dt={t:g}, atol=1e-8 rtol=1e-6"
    if name.startswith("ma"):
        # one size class of the mixed-size batch: N = int(name[2:]), 10N reactions
        N = int(name[2:])
        n = systems or 2048
        t = dt or 1e-3
        wl = W.workload_mixed(n * 20, seed=3, sizes=(N,), fractions=(1.0,), dt=t)[0].subset(slice(0, n))
        return wl, (f"mass action N={N}, {10 * N} reactions, {n:,} systems, dt={t:g}, "
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


def measured_fp64_peak(torch, dev):
    """cuBLAS DGEMM 8192^3, best of 5 (TFLOP/s)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
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
def reference_sample(wl, method: str, target_s: float):
    """Time the reference c_baseline (oracle/_ref) on a strided sample with
    every host core.  Returns (systems/s, cores, sample description)."""
    from oracle import pyoracle as O
    cores = os.cpu_count() or 1
    if not O.reference_available(wl.net, method, "f64"):
        return None, cores, "oracle/_ref not built"
    nsys = wl.net.nsys
    # calibrate on a small strided sample, then size for ~target_s
    k = max(cores, 64)
    stride = max(1, nsys // k)
    sub = wl.subset(slice(0, nsys, stride))
    y = sub.y0.copy()
    t0 = time.perf_counter()
    O.reference(sub.net, y, sub.tnow, sub.tend, sub.atol, sub.rtol, method,
                sub.n_integration_steps, threads=cores)
    dt = time.perf_counter() - t0
    per = dt / sub.net.nsys
    want = int(min(nsys, max(sub.net.nsys, target_s / max(per, 1e-9))))
    stride = max(1, nsys // want)
    sub = wl.subset(slice(0, nsys, stride))
    y = sub.y0.copy()
    t0 = time.perf_counter()
    O.reference(sub.net, y, sub.tnow, sub.tend, sub.atol, sub.rtol, method,
                sub.n_integration_steps, threads=cores)
    dt = time.perf_counter() - t0
    return sub.net.nsys / dt, cores, f"{sub.net.nsys} of {nsys} cells (every {stride}th), {dt:.1f} s"


def run_reference_arm(args, wl, desc):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    vals = []
    cores = os.cpu_count() or 1
    sample = ""
    for i in range(args.warmup + args.steps):
        v, cores, sample = reference_sample(wl, args.method, args.ref_seconds)
        if v is None:
            print(json.dumps({"impl": "reference", "unavailable": sample}))
            return
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "systems/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": desc, "method": args.method},
            "cpu_baseline": {"value": value, "unit": "systems/s", "cores": cores,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "systems/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_mixed(args):
    """The mixed-size batch (N in {5,16,32,64,157} at 40/25/20/10/5 %, 10N
    reactions) through wind_integrate_batch -- one persistent launch for all
    sizes -- timed with CUDA events per solver; one JSON line with systems/s
    per solver, the MIXED/LU_F64 ratio and MIXED's error vs LU_F64."""
    import torch
    from wind_b200 import lib
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    nsys = args.systems or 200000
    dt = args.dt or 1e-4
    groups = W.workload_mixed(nsys, seed=3, dt=dt, atol=1e-8, rtol=1e-6)
    res, ys = {}, {}
    for solver in ("lu_f64", "mixed"):
        times = []
        for i in range(args.warmup + args.steps):
            dg = [lib.DeviceGroup(wl, dev) for wl in groups]
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            stream = torch.cuda.current_stream(dev)
            arr = (lib._capi.WindGroup * len(dg))(*[g.struct() for g in dg])
            o = lib.options("sie", solver, "device")
            e0.record(stream)
            code = lib.load().wind_integrate_batch(lib.C.byref(o), arr, len(dg), stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if code != 0:
                raise RuntimeError(f"wind_integrate_batch failed: {code}")
            if i >= args.warmup:
                times.append(e0.elapsed_time(e1) * 1e-3)
        ys[solver] = np.concatenate([g.y.cpu().numpy().ravel() for g in dg])
        res[solver] = {"systems_per_s": nsys / statistics.median(times),
                       "ms_per_step": 1e3 * statistics.median(times)}
    a, b = ys["mixed"], ys["lu_f64"]
    err = float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-8)))
    line = {"metric": METRIC, "workload": "mixed", "unit": "systems/s",
            "value": res["mixed"]["systems_per_s"], "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": (f"{nsys:,} systems, N in {{5,16,32,64,157}} at 40/25/20/10/5 %, "
                                    f"10N reactions, dt={dt:g}, atol 1e-8 rtol 1e-6, one persistent "
                                    "launch (wind_integrate_batch)")},
            "solvers": res, "mixed_over_fp64": res["mixed"]["systems_per_s"] / res["lu_f64"]["systems_per_s"],
            "max_rel_err_mixed_vs_fp64": err}
    print(json.dumps(line), flush=True)


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
        with serve.Server(solver=args.solver if args.solver != "auto" else "lu_f64",
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
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="wind", choices=["wind", "reference"])
    ap.add_argument("--workload", default="katz96")
    ap.add_argument("--systems", type=int, default=0, help="override the system count "
                    "(profiling runs on a small case; the headline uses the default)")
    ap.add_argument("--dt", type=float, default=0.0, help="interval override (profiling cases)")
    ap.add_argument("--method", default="sie", choices=["sie", "rk2"])
    ap.add_argument("--solver", default="auto", choices=["auto", "gje_f64", "lu_f64", "mixed"])
    ap.add_argument("--spec-width", type=int, default=0)
    ap.add_argument("--ref-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    wl, desc = make_workload(args.workload, args.systems, args.dt)
    if args.impl == "reference":
        return run_reference_arm(args, wl, desc)

    import torch
    import ctypes as C
    from wind_b200 import lib, _capi

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
    N = net.n_eq
    d_arrays = {}
    for k in ("constants", "rates", "species", "linear"):
        a = getattr(net, k)
        if a is not None:
            d_arrays[k] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    ns = _capi.network_struct(net, d_arrays)
    y0 = torch.from_numpy(wl.y0).to(dev)
    y = torch.empty_like(y0)
    status = torch.zeros(net.nsys, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2

    def run_once(solver, width, ybuf):
        o = lib.options(args.method, solver, "device", width)
        total = C.c_int64(0)
        code = wlib.wind_integrate(C.byref(o), C.byref(ns), wl.tnow, wl.tend,
                                   wl.n_integration_steps, ybuf.data_ptr(), net.nsys, wl.atol,
                                   wl.rtol, status.data_ptr(), None, C.byref(total),
                                   _capi.MEM_DEVICE, stream.cuda_stream)
        if code != 0:
            raise RuntimeError(f"wind_integrate failed: {code}")
        return int(total.value)

    def timed(solver, width, steps, warmup):
        times, substeps = [], 0
        for i in range(warmup + steps):
            y.copy_(y0)
            flush.zero_()
            if dist is not None:
                dist.barrier()
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            n = run_once(solver, width, y)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if i >= warmup:
                times.append(e0.elapsed_time(e1) * 1e-3)
                substeps = n
        return times, substeps

    # FP64 reference result on the device (the reference algorithm, GJE_F64)
    run_once("gje_f64", args.spec_width, y.copy_(y0))
    torch.cuda.synchronize(dev)
    y_ref = y.clone()

    solvers = ["gje_f64", "lu_f64", "mixed"] if args.solver == "auto" else [args.solver]
    results = {}
    for s in solvers:
        t, nsub = timed(s, args.spec_width, max(2, args.steps // 3), 1)
        run_once(s, args.spec_width, y.copy_(y0))
        torch.cuda.synchronize(dev)
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        err = float(np.max(np.abs(a - b) / np.maximum(np.abs(b), wl.atol)))
        results[s] = {"systems_per_s": net.nsys / statistics.median(t), "substeps": nsub,
                      "max_rel_err_vs_fp64": err}
    ok = [s for s in solvers if results[s]["max_rel_err_vs_fp64"] <= 1e-5]
    best = max(ok, key=lambda s: results[s]["systems_per_s"]) if ok else "gje_f64"
    width = args.spec_width
    tuning = None
    if args.solver == "auto" and args.spec_width == 0 and net.kind != W.NET_MASS_ACTION:
        # initial lanes per system (autotuner): widths 1..8 for the chosen solver
        from wind_b200 import autotune
        tbest, table = autotune.tune(wl, args.method, "device", widths=(1, 2, 4, 8),
                                     solvers=(best,))
        tuning = table
        if tbest["solver"] == best:
            width = tbest["spec_width"]

    # the timed run of the chosen path
    launches0 = lib.launch_count()
    with ClockSampler(local) as clk:
        times, nsub = timed(best, width, args.steps, args.warmup)
    launches = lib.launch_count() - launches0
    launches = launches * args.steps // (args.steps + args.warmup)
    tot = sum(times)
    if dist is not None:
        tt = torch.tensor([tot], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        tot = float(tt.item())
    value = world * net.nsys * args.steps / tot
    ms_per_step = 1e3 * tot / args.steps

    # e2e through the C ABI with pinned host buffers
    h_y0 = torch.from_numpy(wl.y0).pin_memory()
    h_y = torch.empty_like(h_y0).pin_memory()
    h_arr = {k: torch.from_numpy(np.ascontiguousarray(getattr(net, k))).pin_memory()
             for k in ("constants", "rates", "species", "linear") if getattr(net, k) is not None}
    hns = _capi.network_struct(net, h_arr)
    o = lib.options(args.method, best, "device", width)
    e2e_times = []
    for i in range(args.warmup + args.steps):
        h_y.copy_(h_y0)
        flush.zero_()
        torch.cuda.synchronize(dev)
        total = C.c_int64(0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        code = wlib.wind_integrate(C.byref(o), C.byref(hns), wl.tnow, wl.tend,
                                   wl.n_integration_steps, h_y.data_ptr(), net.nsys, wl.atol,
                                   wl.rtol, None, None, C.byref(total), _capi.MEM_HOST,
                                   stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if code != 0:
            raise RuntimeError(f"e2e wind_integrate failed: {code}")
        if i >= args.warmup:
            e2e_times.append(e0.elapsed_time(e1) * 1e-3)
    e2e_tot = sum(e2e_times)
    if dist is not None:
        tt = torch.tensor([e2e_tot], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_tot = float(tt.item())
    h2d = int(wl.y0.nbytes + sum(v.numel() * v.element_size() for v in h_arr.values()))
    d2h = int(wl.y0.nbytes + 8)

    # roofline of the integrate kernel (FP64 pipe)
    flops = flops_per_substep(wl, args.method) * nsub
    kernel_s = statistics.median(times)
    achieved = flops / kernel_s / 1e12
    peak = measured_fp64_peak(torch, dev)
    alg_bytes = net.nsys * (16 * N) + net.nbytes()
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    # DRAM bytes per launch from the committed ncu capture of the Katz96
    # kernel (profiles/k_lane_katz96_lu_16384cells.md: 2.000 MB read + 0.239
    # MB written for 16,384 cells, i.e. 136.7 B per cell; every cell's state
    # and constants cross HBM once, so it scales with the cell count)
    traffic = 136.7 * net.nsys if net.kind == W.NET_KATZ96 else None
    roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": traffic,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum, 16,384-cell "
                               "capture scaled by cells" if traffic is not None else None),
            "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
            "flops_per_substep": flops_per_substep(wl, args.method), "substeps_per_launch": nsub,
            "hbm": {"alg_bytes_per_launch": alg_bytes,
                    "achieved_gbs": alg_bytes / kernel_s / 1e9, "peak_gbs": hbm_peak,
                    "frac": alg_bytes / kernel_s / 1e9 / hbm_peak,
                    "peak_source": "MEASURED_PEAKS.json" if "hbm_gbs" in peaks else "fallback"}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, sample = reference_sample(wl, args.method, args.ref_seconds)
        if v is not None:
            cpu = {"value": v, "unit": "systems/s", "cores": cores, "kind": "reference",
                   "sample": sample + "; c_baseline FP64 (-Dfloat=double) built from the reference sources"}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": "systems/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": desc, "method": args.method, "solver": best,
                       "controller": "device (cuda/common/kernel.cu semantics)",
                       "systems": net.nsys, "equations": N, "l2": "flushed (256 MB write) between steps",
                       "parallelism": f"replicas x{world}"},
            "solvers": results, "spec_width": width, "tuning": tuning,
            "max_rel_err_vs_fp64": results[best]["max_rel_err_vs_fp64"],
            "e2e": {"value": world * net.nsys * args.steps / e2e_tot, "unit": "systems/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches), "roofline": roof, "cpu_baseline": cpu,
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
