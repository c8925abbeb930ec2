"""CPU test of the tensor-core (MIXED_TC) staging in the CTA kernel's
shared-memory layout and of the tcgen05 instruction descriptor, compiled
host-side with nvcc: the staging is aligned for the MMA's shared-memory
descriptors (16 B), does not overlap the regions after it, and fits beside
the FP32 matrix up to the size the kernel accepts."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
#include <cstdio>
#include "cta_kernel.cuh"
using namespace wind;
int main() {
    const int cap = 232448 - 1024;
    for (int N = 33; N <= CTA_MAXN; N++) {
        const CtaLayout L(N, 10 * N, false, WIND_SOLVER_MIXED, cap, true);
        const CtaLayout P(N, 10 * N, false, WIND_SOLVER_MIXED, cap, false);
        printf("%d %d %d %d %d %d %d %d\n", N, L.tcs, CtaLayout::tc_stage_bytes(N), L.lt, L.mat,
               L.bytes, L.mat_in_smem ? 1 : 0, P.tcs == P.lt ? 1 : 0);
    }
    printf("idesc %u %u\n", tc::idesc_tf32(128, 160), tc::idesc_tf32(128, 48));
    return 0;
}
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("tclayout")
    src = d / "probe.cu"
    src.write_text(PROBE)
    exe = d / "probe"
    subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                    "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "wind_b200", "csrc"),
                    "-o", str(exe), str(src)], check=True, capture_output=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True,
                           text=True).stdout.strip().splitlines()
    rows = [[int(v) for v in ln.split()] for ln in lines[:-1]]
    idesc = [int(v) for v in lines[-1].split()[1:]]
    return rows, idesc


def test_staging_aligned_and_disjoint(probe):
    rows, _ = probe
    for N, tcs, stage, lt, mat, _, _, plain_empty in rows:
        assert tcs % 16 == 0
        # operand slabs start 64 B in, every slab a multiple of 256 B
        cols16 = (N + 15) & ~15
        assert stage == 64 + 4 * 4096 + 4 * cols16 * 32
        assert tcs + stage <= lt <= mat
        assert plain_empty == 1   # the MIXED layout without tensor cores stages nothing


def test_tensor_core_sizes_fit_up_to_the_accepted_limit(probe):
    rows, _ = probe
    fits = {r[0]: r[6] for r in rows}   # N -> matrix (and staging) in shared memory
    for N in (40, 64, 100, 130, 157, 176):
        assert fits[N] == 1, N
    assert fits[220] == 0


def test_instruction_descriptor_fields(probe):
    _, idesc = probe
    for val, n in zip(idesc, (160, 48)):
        assert (val >> 4) & 0x3 == 1          # F32 accumulator
        assert (val >> 7) & 0x7 == 2          # A: TF32
        assert (val >> 10) & 0x7 == 2         # B: TF32
        assert (val >> 15) & 0x3 == 0         # both K-major
        assert (val >> 17) & 0x3F == n // 8   # N / 8
        assert (val >> 24) & 0x1F == 128 // 16
