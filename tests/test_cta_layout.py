"""CPU test of the CTA kernel's shared-memory / scratch layout (CtaLayout in
wind_b200/csrc/cta_kernel.cuh), compiled host-side with nvcc: every offset
the kernel dereferences is aligned and inside its region, for every N the
kernel accepts, both matrix precisions and both shared-memory budgets."""
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
    const int caps[2] = {232448 - 1024, ((233472 / 2 - 1024 - 16) & ~127)};
    const int rs[4] = {0, 1, 10, 655};
    for (int solver = 0; solver < 3; solver++)
        for (int lin = 0; lin < 2; lin++)
            for (int N = 33; N <= CTA_MAXN; N++)
                for (int ri = 0; ri < 5; ri++)
                    for (int ci = 0; ci < 2; ci++) {
                        const int R = ri < 4 ? rs[ri] * (ri == 2 ? N : 1) : 4 * N + 3;
                        const CtaLayout L(N, R, lin != 0, solver, caps[ci]);
                        printf("%d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %zu %zu %zu\n",
                               solver, lin, N, R, caps[ci], L.ld, L.cols, L.esz, L.nvec, L.vec, L.piv,
                               L.act, L.misc, L.cand, L.lt, L.mat, L.inc_off, L.inc, L.rt, L.spc,
                               L.bytes, (L.mat_in_smem ? 1 : 0) | (L.inc_in_smem ? 2 : 0) | (L.data_in_smem ? 4 : 0),
                               L.g_mat, L.g_inc, L.g_doubles);
                    }
    printf("cand %zu %zu\n", sizeof(CtaCand<float>), sizeof(CtaCand<double>));
    return 0;
}
"""


@pytest.fixture(scope="module")
def layouts(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("ctalayout")
    src = d / "probe.cu"
    src.write_text(PROBE)
    exe = d / "probe"
    subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a", "-I",
                    os.path.join(ROOT, "wind_b200", "csrc"), "-o", str(exe), str(src)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    lines = out.strip().splitlines()
    cand = [int(v) for v in lines[-1].split()[1:]]
    rows = [[int(v) for v in ln.split()] for ln in lines[:-1]]
    return rows, cand


def test_candidate_slots(layouts):
    _, cand = layouts
    assert cand == [16 + 16 * 4, 16 + 16 * 8]


def test_layout_invariants(layouts):
    rows, _ = layouts
    assert len(rows) == 3 * 2 * 224 * 5 * 2
    for (solver, lin, N, R, cap, ld, cols, esz, nvec, vec, piv, act, misc, cand, lt, mat,
         inc_off, inc, rt, spc, nbytes, flags, g_mat, g_inc, g_doubles) in rows:
        mis, iis, dis = bool(flags & 1), bool(flags & 2), bool(flags & 4)
        assert esz == (4 if solver == 2 else 8)
        # columns: the right-hand side, whole 16-wide panels, whole 4-wide tiles
        assert cols >= N + 1 and cols % 4 == 0 and cols <= ld
        assert ((N - 1) // 16) * 16 + 15 < cols
        k0 = 0
        while k0 + 16 <= N:
            c0 = k0 + 16
            assert c0 + 4 * ((N + 1 - c0 + 3) // 4) - 1 < cols
            k0 += 16
        # rows 16 bytes apart modulo the 128-byte bank space, 16-byte aligned
        assert (ld * esz) % 128 == 16
        for off in (vec, piv, act, misc, cand, lt, mat, inc_off):
            assert off % 16 == 0
        # region order and sizes
        assert piv >= vec + nvec * N * 8 and act >= piv + 4 * N and misc >= act + 4 * N
        assert cand >= misc + 64  # warp counts, vote slots, convergence flag
        assert lt >= cand + (0 if solver == 0 else 2 * 8 * (16 + 16 * esz))
        assert mat >= lt + (N * N * 4 if lin else 0)
        if solver != 0 and mis:
            assert mat + N * ld * esz <= nbytes
        if iis:
            assert inc % 16 == 0 and inc >= inc_off + 4 * (N + 1)
            assert inc + 8 * R <= nbytes
        if dis:
            assert rt % 16 == 0 and spc % 16 == 0
            assert spc >= rt + 8 * R and spc + 8 * R <= nbytes
        if mis and iis:
            assert nbytes <= cap
        # global slot: 16-byte aligned pieces, even stride in doubles
        assert g_mat % 2 == 0 and g_inc % 2 == 0 and g_doubles % 2 == 0
        assert g_mat == (2 * N * N if solver == 0 else 0)
        if solver != 0 and not mis:
            assert g_inc >= g_mat + N * ld * esz // 8
        if not iis:
            assert g_doubles >= g_inc + (4 * (N + 1) + 8 * R) // 8
        if solver == 0:
            assert g_doubles >= 2 * N * N
