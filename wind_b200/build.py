"""Build the native libraries in-tree (sm_100a), and the oracle checkers.

    python -m wind_b200.build            # libwind.so + legacy libraries
    python -m wind_b200.build --oracle   # also oracle/_build and oracle/_ref

Outputs (git-ignored, shipped with the tree):
    wind_b200/lib/libwind.so                     extern "C" API (include/wind.h)
    wind_b200/lib/<network>/{sie,rk2}.so         drop-in cudaIntegrateSystem
Compilation is incremental on file modification times.
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                "--expt-relaxed-constexpr", "-Xptxas", "-v"]

# translation units of libwind.so
UNITS = ["api", "batch", "noalloc", "dispatch_lane", "dispatch_team", "dispatch_team8",
         "dispatch_team16", "dispatch_team32", "dispatch_warp", "dispatch_cta", "dispatch_mixed", "server", "global",
         "dispatch_tile", "plugin", "dispatch_sim"]

# Kernel sources the runtime plug-ins compile with NVRTC (csrc/plugin.cu),
# embedded in the library under the names their #include lines use.
EMBEDDED = [("plugin_kernel.cuh", "csrc/plugin_kernel.cuh"), ("common.cuh", "csrc/common.cuh"),
            ("../../include/wind.h", "../include/wind.h")]

LEGACY_NETS = {"nr_test": "WIND_NET_NR_TEST", "katz96": "WIND_NET_KATZ96",
               "stifftrig": "WIND_NET_STIFFTRIG"}
LEGACY_METHODS = {"sie": "WIND_METHOD_SIE", "rk2": "WIND_METHOD_RK2"}


def _deps():
    return (glob.glob(os.path.join(CSRC, "*")) +
            [os.path.join(ROOT, "include", "wind.h"), os.path.join(ROOT, "include", "wind_legacy.h")])


def _unit_deps(path, seen=None):
    """The file and every local header it includes, recursively."""
    import re
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as fh:
        for inc in re.findall(r'^\s*#include\s+"([^"]+)"', fh.read(), re.M):
            _unit_deps(os.path.join(os.path.dirname(path), inc), seen)
    return seen


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd, log=None):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log:
        with open(log, "w") as fh:
            fh.write(r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:6]) + " ...")
    return r


def _write_embedded():
    """OBJ/embedded_sources.h: the EMBEDDED files as raw string literals."""
    out = os.path.join(OBJ, "embedded_sources.h")
    srcs = [os.path.join(HERE, rel) for _, rel in EMBEDDED]
    if not _stale(out, srcs + [__file__]):
        return out, srcs
    lines = ["// generated by wind_b200/build.py: kernel sources for NVRTC", "#pragma once",
             "struct EmbeddedSource { const char* name; const char* text; };",
             "static const EmbeddedSource kEmbedded[] = {"]
    for (name, _), path in zip(EMBEDDED, srcs):
        with open(path) as fh:
            text = fh.read()
        assert ")WINDSRC\"" not in text
        lines.append(f'    {{"{name}", R"WINDSRC({text})WINDSRC"}},')
    lines += ["};", f"static const int kEmbeddedCount = {len(EMBEDDED)};", ""]
    with open(out, "w") as fh:
        fh.write("\n".join(lines))
    return out, srcs


def build_native(verbose=False):
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    deps = _deps()
    emb, emb_srcs = _write_embedded()
    objs, jobs = [], []
    for unit in UNITS:
        obj = os.path.join(OBJ, unit + ".o")
        objs.append(obj)
        udeps = sorted(_unit_deps(os.path.join(CSRC, unit + ".cu")))
        if unit == "plugin":
            udeps += [emb] + emb_srcs
        if _stale(obj, udeps):
            if verbose:
                print(f"nvcc {unit}.cu", flush=True)
            jobs.append(([NVCC] + FLAGS + ["-I" + OBJ, "-c", os.path.join(CSRC, unit + ".cu"), "-o", obj],
                         os.path.join(OBJ, unit + ".ptxas.log")))
    if jobs:
        import concurrent.futures as cf
        with cf.ThreadPoolExecutor(max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            for f in [ex.submit(_run, cmd, log) for cmd, log in jobs]:
                f.result()
    libwind = os.path.join(LIB, "libwind.so")
    if _stale(libwind, objs):
        _run([NVCC] + ARCH + ["-shared"] + objs + ["-o", libwind, "-lcudart", "-ldl"])
    for net, netdef in LEGACY_NETS.items():
        os.makedirs(os.path.join(LIB, net), exist_ok=True)
        # sie.so / rk2.so export cudaIntegrateSystem; sie_host.so exports
        # cudaIntegrateSIE (the reference's lib/sie_host.so)
        for meth, mdef in list(LEGACY_METHODS.items()) + [("sie_host", "WIND_METHOD_SIE")]:
            out = os.path.join(LIB, net, f"{meth}.so")
            if _stale(out, deps + [libwind]):
                extra = ["-DWIND_LEGACY_HOST"] if meth == "sie_host" else []
                _run([NVCC] + ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                      f"-DWIND_LEGACY_NET={netdef}", f"-DWIND_LEGACY_METHOD={mdef}"] + extra +
                     [os.path.join(CSRC, "legacy.cu"), "-o", out,
                      "-L" + LIB, "-lwind", "-Xlinker", "-rpath=$ORIGIN/.."])
    return libwind


def build_oracle():
    """The CPU checkers: the restatement always; the reference's own
    c_baseline through oracle/build_ref.sh, which locates the reference
    checkout (WIND_REFERENCE) and exits 3 when its sources are absent -- then
    only the restatement is built."""
    oracle = os.path.join(ROOT, "oracle")
    _run(["make", "-s", "-C", oracle])
    stamp = os.path.join(oracle, "_ref", "sie_gold_katz96_f64.so")
    srcs = glob.glob(os.path.join(oracle, "plugins", "*.c")) + [os.path.join(oracle, "build_ref.sh")]
    if _stale(stamp, srcs):
        r = subprocess.run(["bash", os.path.join(oracle, "build_ref.sh")], capture_output=True, text=True)
        if r.returncode not in (0, 3):
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("oracle/build_ref.sh failed")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    build_native(verbose=a.v)
    if a.oracle:
        build_oracle()
    print("built", os.path.join(LIB, "libwind.so"))


if __name__ == "__main__":
    main()
