// cta_kernel.cuh -- persistent CTA-per-system integrator for mass-action
// networks with 32 < N <= 256 (the 64- and 157-species classes).
//
// One CTA (256 threads) integrates one system at a time and pulls the next
// ticket from the device work queue when it finishes.  Thread l owns
// equation l (N <= 256): its y, y1, y2 live in registers.  Per system the CTA
// builds per-species incidence lists of the reactions (CSR, reaction ids
// ascending), so thread j evaluates f_j and row j of the Jacobian from the
// ~4R/N reactions that touch species j instead of all R.
//
// Solvers (selected at compile time):
//  GJE_F64  the reference's unpivoted Gauss-Jordan inverse, reference
//           operation order, on M and Inv in a per-CTA global scratch slot
//           (2 N^2 doubles; L2-resident) -- bit-exact parity path;
//  LU_F64   blocked right-looking LU with partial pivoting, FP64, on the
//           matrix [A | b] in shared memory (global scratch when it does not
//           fit), followed by blocked triangular solves;
//  MIXED    FP32 factors without pivoting, FP64 residual r = f - (x - h J x)
//           evaluated from the reactions (no FP64 matrix), FP64 refinement
//           until the correction is below 1e-6 of |x| (per 32-row slice; at
//           most two steps), else the substep is redone with partial
//           pivoting.  Its footprint lets two CTAs share an SM at N = 157.
//
// Blocked LU (panel width CTA_NB = 16).  Rows never move: logical row i is
// physical row piv[i].  For each panel (cta_lu, partial pivoting):
//  1. panel factorisation: thread p holds the 16 panel entries of physical
//     row p in registers.  Per column one CTA barrier: each warp's best
//     candidate (max |a| by a __reduce_max_sync key) publishes its row's
//     panel entries and reciprocal pivot in a per-warp slot (double-
//     buffered) and its packed (key, row) in a 64-bit atomicMax vote (lowest
//     row on ties); after the barrier every thread reads the winner and
//     eliminates its own row in registers;
//  2. the still-active rows are compacted into act[] (warp ballots);
//  3. U12 = L11^-1 A12 for the 16 pivot rows, one thread per column;
//  4. trailing update A22 -= L21 U12 over act[] x columns, 4x4 register
//     tiles with 16-byte shared-memory vectors.
// The MIXED solver factors without pivoting (cta_lu_nopiv): warp 0 factors
// the 16x16 diagonal block with shuffles, the rows below form their own
// multipliers, then steps 3 and 4 -- three barriers per panel.
// The right-hand side is column N, so the forward elimination comes with the
// factorisation; the row stride is padded so that rows start 16 bytes apart
// in the bank space (no conflicts when 32 rows are read at one column).
#pragma once

#include <type_traits>

#include "common.cuh"
#include "tc_sm100.cuh"
#include "networks.cuh"

namespace wind {

constexpr int CTA_THREADS = 256;
constexpr int CTA_WARPS = CTA_THREADS / 32;
constexpr int CTA_MAXN = 256;
constexpr int CTA_NB = 16;  // LU panel width
constexpr int CTA_CONV = 14; // misc[] slot: refinement converged (0/1)
constexpr int CTA_TCPAR = 15; // misc[] slot: phase parity of the tensor-core mbarrier

// A warp's pivot candidate for one panel column: its best row's panel
// entries and the reciprocal of the entry in the column.
template <typename T>
struct CtaCand {
    T rcp;                      // 1 / vals[column] (computed before the vote)
    alignas(16) T vals[CTA_NB];
};
static_assert(sizeof(CtaCand<float>) == 16 + CTA_NB * 4, "candidate slot size");
static_assert(sizeof(CtaCand<double>) == 16 + CTA_NB * 8, "candidate slot size");

// Shared-memory and global-scratch layout of one CTA, computed on the host
// and the device alike.  Shared memory holds, in order of priority, the
// vectors, the pivot bookkeeping, the dense linear term, the matrix and the
// incidence lists; whatever does not fit under `smem_cap` goes to the CTA's
// global scratch slot.
struct CtaLayout {
    int ld;            // matrix row stride (elements)
    int cols;          // columns that hold data (<= ld, a multiple of 4)
    int esz;           // matrix element size (bytes)
    int nvec;          // FP64 vectors of length N
    int vec, piv, act, misc, cand, tcs, lt, mat, inc_off, inc, rt, spc, bytes;
    bool mat_in_smem, inc_in_smem, data_in_smem;
    size_t g_mat, g_inc, g_doubles;  // global slot: offsets and size in doubles
    __host__ __device__ static int a16(int x) { return (x + 15) & ~15; }
    // columns read or written: >= N+1, whole panels, whole 4-wide tiles
    __host__ __device__ static int data_cols(int N) {
        const int a = (N + 15) & ~15, b = (N + 1 + 3) & ~3;
        return a > b ? a : b;
    }
    // rows 16 bytes apart modulo the 128-byte bank space
    __host__ __device__ static int row_stride(int N, int esz) {
        const int base = data_cols(N);
        const int per = 128 / esz, want = 16 / esz;  // elements per bank sweep / per 16 B
        return base + ((want - base % per) + per) % per;
    }
    // Tensor-core staging of the MIXED inverse's rank-16 updates (tc): the
    // mbarrier and tensor-memory address (64 B), the update's left operand
    // (128 rows x 16, TF32 high and low parts, 16 KB) and right operand
    // (columns rounded up to 16 x 16, high and low parts).
    __host__ __device__ static int tc_stage_bytes(int N) {
        return 64 + 4 * 4096 + 4 * ((N + 15) & ~15) * 32;
    }
    __host__ __device__ CtaLayout(int N, int R, bool lin, int solver, int smem_cap, bool tc = false) {
        esz = (solver == WIND_SOLVER_MIXED) ? 4 : 8;
        ld = row_stride(N, esz);
        cols = data_cols(N);
        nvec = (solver == WIND_SOLVER_GJE_F64) ? 3 : (solver == WIND_SOLVER_LU_F64 ? 4 : 5);
        int off = 0;
        vec = off; off = a16(off + nvec * N * 8);
        piv = off; off = a16(off + N * 4);
        act = off; off = a16(off + N * 4);
        misc = off; off = a16(off + 2 * CTA_WARPS * 4);
        cand = off; off = a16(off + (solver == WIND_SOLVER_GJE_F64 ? 0 : 2 * CTA_WARPS * (16 + CTA_NB * esz)));
        tcs = off; off = a16(off + (tc ? tc_stage_bytes(N) : 0));
        lt = off; off = a16(off + (lin ? N * N * 4 : 0));
        const int mbytes = (solver == WIND_SOLVER_GJE_F64) ? 0 : a16(N * ld * esz);
        mat = off;
        mat_in_smem = (off + mbytes) <= smem_cap;
        if (mat_in_smem) off += mbytes;
        const int ibytes = a16((N + 1) * 4) + a16(4 * R * 2);
        inc_off = off;
        inc_in_smem = (off + ibytes) <= smem_cap;
        if (inc_in_smem) {
            inc = off + a16((N + 1) * 4);
            off += ibytes;
        } else {
            inc = 0;
        }
        // the system's rates and species, staged once per system
        rt = off;
        spc = a16(off + R * 8);
        data_in_smem = (spc + a16(R * 8)) <= smem_cap;
        if (data_in_smem) off = spc + a16(R * 8);
        bytes = off;
        // global slot: [GJE M, Inv][matrix][incidence lists]
        size_t g = (solver == WIND_SOLVER_GJE_F64) ? (size_t)2 * N * N : 0;
        g_mat = g;
        if (!mat_in_smem) g += ((size_t)N * ld * esz + 15) / 16 * 2;
        g_inc = g;
        if (!inc_in_smem) g += ((size_t)ibytes + 15) / 16 * 2;
        g_doubles = g;
    }
};

struct CtaCtx {
    int N, R, tid, ld, cols;
    const double* rates;     // global [R]
    const uint16_t* sp;      // global [R*4]
    const float* LT;         // smem [N*N] or null
    const int* inc_off;      // [N+1] (shared or global)
    const uint16_t* inc;
    double *v, *f, *x, *r, *rinv, *scr;
    int* piv;    // logical row -> physical row
    int* act;    // active rows of the trailing update
    int* misc;   // warp counts [CTA_WARPS]
    unsigned long long* best;  // pivot vote, three rotating slots
    void* cand;  // CtaCand<T>[2][CTA_WARPS]
    // tensor-core rank updates (MIXED_TC): accumulator base in tensor
    // memory, completion mbarrier, operand staging, columns rounded to 16
    uint32_t tmem;
    uint64_t* mbar;
    unsigned char* tcs;
    int tc_cols16;
};

// 4 consecutive elements through 16-byte shared/global vectors.
__device__ __forceinline__ void ld4(const float* p, float (&a)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    a[0] = t.x; a[1] = t.y; a[2] = t.z; a[3] = t.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&a)[4]) {
    const double2 t0 = reinterpret_cast<const double2*>(p)[0];
    const double2 t1 = reinterpret_cast<const double2*>(p)[1];
    a[0] = t0.x; a[1] = t0.y; a[2] = t1.x; a[3] = t1.y;
}
__device__ __forceinline__ void st4(float* p, const float (&a)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(a[0], a[1], a[2], a[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&a)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(a[0], a[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(a[2], a[3]);
}

template <typename T>
__device__ __forceinline__ void ld4at(const T* p, T* a) {
    T t[4];
    ld4(p, t);
    a[0] = t[0]; a[1] = t[1]; a[2] = t[2]; a[3] = t[3];
}
template <typename T>
__device__ __forceinline__ void st4at(T* p, const T* a) {
    const T t[4] = {a[0], a[1], a[2], a[3]};
    st4(p, t);
}

// Pivot ordering key: |a| as an unsigned integer (FP64: the high word, so
// magnitudes within 2^-20 of each other tie and the lower row wins).
__device__ __forceinline__ uint32_t mag_key(float a) { return __float_as_uint(fabsf(a)); }
__device__ __forceinline__ uint32_t mag_key(double a) {
    return (uint32_t)((unsigned long long)__double_as_longlong(fabs(a)) >> 32);
}

// f_j for j = tid (FP64, the sequential per-element order of the
// mass-action contract) into c.f.
__device__ __forceinline__ void cta_rhs(const CtaCtx& c) {
    const int N = c.N, j = c.tid;
    if (j < N) {
        xd acc = 0.0;
        if (c.LT)
            for (int k = 0; k < N; k++) acc += xd((double)c.LT[k * N + j]) * xd(c.v[k]);
        const int e0 = c.inc_off[j], e1 = c.inc_off[j + 1];
        for (int e = e0; e < e1; e++) {
            const int rr = c.inc[e];
            const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
            const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
            const xd w = xd(c.rates[rr]) * xd(c.v[a]) * xd(c.v[b]);
            if (a == j) acc -= w;
            if (b == j) acc -= w;
            if (cc == j) acc += w;
            if (d == j) acc += w;
        }
        c.f[j] = acc.v;
    }
    __syncthreads();
}

// Visit the reactions that touch species j (ascending ids) with up to B
// of them in flight: fn(k, a, b, s) with the reactants a, b and the net
// stoichiometry s = [C == j] + [D == j] - [A == j] - [B == j] (s = 0 skipped).
// The per-system rates and species sit in L2 when shared memory is full, so
// the loads are issued in batches before they are used.
template <int B = 8, typename F>
__device__ __forceinline__ void cta_incidences(const CtaCtx& c, int j, F&& fn) {
    const int e0 = c.inc_off[j], e1 = c.inc_off[j + 1];
    for (int e = e0; e < e1; e += B) {
        uint2 q[B];
        double k[B];
#pragma unroll
        for (int u = 0; u < B; u++) {
            if (e + u < e1) {
                const int rr = c.inc[e + u];
                q[u] = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
                k[u] = c.rates[rr];
            }
        }
#pragma unroll
        for (int u = 0; u < B; u++) {
            if (e + u < e1) {
                const int a = q[u].x & 0xffff, b = q[u].x >> 16, cc = q[u].y & 0xffff, d = q[u].y >> 16;
                const int sg = (cc == j) + (d == j) - (a == j) - (b == j);
                if (sg) fn(k[u], a, b, (double)sg);
            }
        }
    }
}

// [A | b] = [I - h J | f] in standard orientation (J[j][c] = Jt[c][j]), and
// f into c.f.  Thread j owns row j: it starts the row from L (or zero),
// accumulates f_j and the row's Jacobian entries from its reactions, then
// scales the row and writes f_j as column N.  (The LU and mixed solvers are
// not bit-exact by design; the reference-order evaluation is cta_rhs /
// cta_gje_exact.)
template <typename T>
__device__ __noinline__ void cta_build(const CtaCtx& c, double h, T* A) {
    const int N = c.N, j = c.tid, ld = c.ld;
    const int q4 = c.cols >> 2;  // 4-wide chunks per row that hold data
    if (j < N) {
        T* row = A + (size_t)j * ld;
        double acc = 0.0;
        if (c.LT) {
            for (int k = 0; k < c.cols; k++) row[k] = k < N ? (T)c.LT[k * N + j] : (T)0;
            for (int k = 0; k < N; k++) acc = fma((double)c.LT[k * N + j], c.v[k], acc);
        } else {
            const T z4[4] = {(T)0, (T)0, (T)0, (T)0};
            for (int q = 0; q < q4; q++) st4(row + 4 * q, z4);
        }
        cta_incidences<sizeof(T) == 4 ? 2 : 8>(c, j, [&](double k, int a, int b, double sg) {
            const double ya = c.v[a], yb = c.v[b];
            acc = fma(sg * k * ya, yb, acc);
            row[a] = (T)((double)row[a] + sg * k * yb);
            row[b] = (T)((double)row[b] + sg * k * ya);
        });
        c.f[j] = acc;
        if (j < 3) c.best[j] = 0ull;  // pivot-vote slots of the next LU
        for (int q = 0; q < q4; q++) {
            T a[4];
            ld4(row + 4 * q, a);
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const int cc = 4 * q + t;
                if (cc < N) a[t] = (T)((cc == j ? 1.0 : 0.0) - h * (double)a[t]);
                else if (cc == N) a[t] = (T)acc;
            }
            st4(row + 4 * q, a);
        }
    }
    __syncthreads();
}

// f_j for j = tid at the state in c.v, FP64 with fused multiply-adds (the
// mixed solver's right-hand side; the bit-exact evaluation is cta_rhs).
__device__ __forceinline__ void cta_rhs_fast(const CtaCtx& c) {
    const int N = c.N, j = c.tid;
    if (j < N) {
        double acc = 0.0;
        if (c.LT)
            for (int k = 0; k < N; k++) acc = fma((double)c.LT[k * N + j], c.v[k], acc);
        cta_incidences<4>(c, j, [&](double k, int a, int b, double sg) {
            acc = fma(sg * k * c.v[a], c.v[b], acc);
        });
        c.f[j] = acc;
    }
    __syncthreads();
}

// (J x)_j from the reactions (and L), FP64, for the refinement residual.
__device__ __forceinline__ double cta_jx(const CtaCtx& c, int j, const double* xv) {
    const int N = c.N;
    double acc = 0.0;
    if (c.LT)
        for (int k = 0; k < N; k++) acc = fma((double)c.LT[k * N + j], xv[k], acc);
    cta_incidences<4>(c, j, [&](double k, int a, int b, double sg) {
        acc = fma(sg * k, fma(c.v[b], xv[a], c.v[a] * xv[b]), acc);
    });
    return acc;
}

// U12 = L11^-1 A12 for the 16 pivot rows of the panel at k0 (row offsets
// prow[]), one thread per column c0..N.
template <typename T>
__device__ __forceinline__ void cta_u12(const CtaCtx& c, T* A, int k0, const int (&prow)[CTA_NB]) {
    const int N = c.N;
    for (int col = k0 + CTA_NB + c.tid; col <= N; col += CTA_THREADS) {
        T u[CTA_NB];
#pragma unroll
        for (int j = 0; j < CTA_NB; j++) u[j] = A[prow[j] + col];
#pragma unroll
        for (int i = 0; i < CTA_NB; i++) {
#pragma unroll
            for (int j = i + 1; j < CTA_NB; j++) u[j] = fma(-A[prow[j] + k0 + i], u[i], u[j]);
        }
#pragma unroll
        for (int j = 1; j < CTA_NB; j++) A[prow[j] + col] = u[j];
    }
}

// Trailing update A22 -= L21 U12 of the panel at k0: the active rows
// (act[0..m) with pivoting, rows c0..N-1 in order without) times columns
// c0..N, 4x4 register tiles with 16-byte vectors.
template <typename T, bool NATURAL>
__device__ __forceinline__ void cta_trailing(const CtaCtx& c, T* A, int k0, const int (&prow)[CTA_NB]) {
    constexpr int TR = 4;
    const int N = c.N, ld = c.ld, c0 = k0 + CTA_NB;
    const int m = N - c0, n = N + 1 - c0;
    const int tr = (m + TR - 1) / TR, tc = (n + 3) >> 2;
    for (int t = c.tid; t < tr * tc; t += CTA_THREADS) {
        const int ti = t / tc, col = c0 + 4 * (t - ti * tc);
        int rows[TR];
#pragma unroll
        for (int r = 0; r < TR; r++) {
            const int rr = TR * ti + r;
            rows[r] = rr < m ? (NATURAL ? c0 + rr : c.act[rr]) * ld : -1;
        }
        T acc[TR][4];
#pragma unroll
        for (int r = 0; r < TR; r++) {
            if (rows[r] >= 0) ld4(A + rows[r] + col, acc[r]);
            else {
#pragma unroll
                for (int q = 0; q < 4; q++) acc[r][q] = (T)0;
            }
        }
#pragma unroll 1  // (full unrolling hoists every load and spills)
        for (int jc = 0; jc < CTA_NB / 4; jc++) {
            T u[4][4];
#pragma unroll
            for (int q = 0; q < 4; q++) ld4(A + prow[4 * jc + q] + col, u[q]);
#pragma unroll
            for (int r = 0; r < TR; r++) {
                T l[4] = {(T)0, (T)0, (T)0, (T)0};
                if (rows[r] >= 0) ld4(A + rows[r] + k0 + 4 * jc, l);
#pragma unroll
                for (int q = 0; q < 4; q++)
#pragma unroll
                    for (int cc = 0; cc < 4; cc++) acc[r][cc] = fma(-l[q], u[q][cc], acc[r][cc]);
            }
        }
#pragma unroll
        for (int r = 0; r < TR; r++)
            if (rows[r] >= 0) st4(A + rows[r] + col, acc[r]);
    }
}

// Blocked right-looking LU with partial pivoting of [A | b] in place (see
// the file comment).  On return: c.piv[i] = physical row of logical row i,
// c.rinv[i] = 1/U_ii, the multipliers below the pivots, U above, and
// column N holds the forward-eliminated right-hand side.
template <typename T>
__device__ void cta_lu(const CtaCtx& c, T* A) {
    const int N = c.N, tid = c.tid, ld = c.ld;
    const int warp = tid >> 5, lane = tid & 31;
    CtaCand<T>* cand = static_cast<CtaCand<T>*>(c.cand);
    T* myrow = A + (size_t)(tid < N ? tid : 0) * ld;
    bool done = tid >= N;  // row is a pivot row already (or no row)
    for (int k0 = 0; k0 < N; k0 += CTA_NB) {
        const int kb = min(CTA_NB, N - k0);
        const bool act0 = !done;
        T a[CTA_NB];
        if (act0) {
#pragma unroll
            for (int q = 0; q < CTA_NB / 4; q++) ld4at(myrow + k0 + 4 * q, a + 4 * q);
        } else {
#pragma unroll
            for (int q = 0; q < CTA_NB; q++) a[q] = (T)0;
        }
        // 1. panel factorisation, one barrier per column
#pragma unroll
        for (int j = 0; j < CTA_NB; j++) {
            if (j < kb) {
                // vote: each warp's best row publishes its panel entries and
                // its packed (key, row) into the step's 64-bit max slot
                const int g = k0 + j;  // global step: slots rotate mod 3
                const uint32_t key = done ? 0u : mag_key(a[j]) + 1u;
                const T myr = nr_rcp(a[j]);  // off the post-vote path
                const uint32_t wmax = __reduce_max_sync(0xffffffffu, key);
                const int wl = __ffs(__ballot_sync(0xffffffffu, key == wmax)) - 1;
                CtaCand<T>* slot = cand + (j & 1) * CTA_WARPS;
                if (lane == wl && wmax) {
                    slot[warp].rcp = myr;
#pragma unroll
                    for (int q = 0; q < CTA_NB / 4; q++)
                        st4at(slot[warp].vals + 4 * q, a + 4 * q);
                    atomicMax(c.best + g % 3, ((unsigned long long)wmax << 32) | (unsigned)(0xffff - tid));
                }
                __syncthreads();
                // the slot read two steps from now is cleared here: its last
                // readers passed this barrier, its writers have not started
                if (tid == 0) c.best[(g + 2) % 3] = 0ull;
                const int pr = 0xffff - (int)(c.best[g % 3] & 0xffffu);
                const CtaCand<T>& win = slot[pr >> 5];
                const T ri = win.rcp;
                if (tid == pr) {
                    done = true;
                    c.piv[k0 + j] = pr;
                    c.rinv[k0 + j] = (double)ri;
                } else if (!done) {
                    const T l = a[j] * ri;
                    a[j] = l;
#pragma unroll
                    for (int jj = j + 1; jj < CTA_NB; jj++) a[jj] = fma(-l, win.vals[jj], a[jj]);
                }
            }
        }
        if (act0) {
#pragma unroll
            for (int q = 0; q < CTA_NB / 4; q++) st4at(myrow + k0 + 4 * q, a + 4 * q);
        }
        // 2. compaction of the active rows (physical order)
        const unsigned am = __ballot_sync(0xffffffffu, !done);
        if (lane == 0) c.misc[warp] = __popc(am);
        __syncthreads();
        const int c0 = k0 + CTA_NB;  // first trailing column
        if (c0 > N) break;           // last panel: b was eliminated in registers
        if (!done) {
            int rank = __popc(am & ((1u << lane) - 1u));
            for (int w = 0; w < warp; w++) rank += c.misc[w];
            c.act[rank] = tid;
        }
        // 3. U12 = L11^-1 A12, one thread per column c0..N
        int prow[CTA_NB];
#pragma unroll
        for (int j = 0; j < CTA_NB; j++) prow[j] = c.piv[k0 + j] * ld;
        cta_u12<T>(c, A, k0, prow);
        __syncthreads();
        // 4. trailing update over act[0..m) x [c0, N]
        cta_trailing<T, false>(c, A, k0, prow);
        __syncthreads();
    }
}

// LU without pivoting (the elimination order of the reference's
// Gauss-Jordan inverse), for the FP32 factors of MIXED, whose refinement
// checks convergence and falls back to cta_lu.  Per panel at k0: warp 0
// factors the 16 x 16 diagonal block with shuffles; every row below then
// computes its own multipliers in registers from U11 while the U12 columns
// are formed; then the trailing update -- three barriers per panel against
// nineteen with the pivot vote.
template <typename T>
__device__ void cta_lu_nopiv(const CtaCtx& c, T* A) {
    const int N = c.N, tid = c.tid, ld = c.ld;
    if (tid < N) c.piv[tid] = tid;
    for (int k0 = 0; k0 < N; k0 += CTA_NB) {
        const int kb = min(CTA_NB, N - k0);
        if (tid < 32) {
            const int lane = tid;
            const bool mine = lane < kb;
            T* row = A + (size_t)(k0 + (mine ? lane : 0)) * ld + k0;
            T a[CTA_NB];
#pragma unroll
            for (int q = 0; q < CTA_NB / 4; q++) {
                if (mine) ld4at(row + 4 * q, a + 4 * q);
                else a[4 * q] = a[4 * q + 1] = a[4 * q + 2] = a[4 * q + 3] = (T)0;
            }
#pragma unroll
            for (int j = 0; j < CTA_NB; j++) {
                if (j < kb) {
                    const T ri = __shfl_sync(0xffffffffu, nr_rcp(a[j]), j);
                    if (lane == j) c.rinv[k0 + j] = (double)ri;
                    const bool upd = mine && lane > j;
                    const T l = a[j] * ri;
                    if (upd) a[j] = l;
#pragma unroll
                    for (int jj = j + 1; jj < CTA_NB; jj++) {
                        const T pv = __shfl_sync(0xffffffffu, a[jj], j);
                        if (upd) a[jj] = fma(-l, pv, a[jj]);
                    }
                }
            }
            if (mine) {
#pragma unroll
                for (int q = 0; q < CTA_NB / 4; q++) st4at(row + 4 * q, a + 4 * q);
            }
        }
        __syncthreads();
        const int c0 = k0 + CTA_NB;
        if (c0 > N) break;  // last panel: b was eliminated with the block
        int prow[CTA_NB];
#pragma unroll
        for (int j = 0; j < CTA_NB; j++) prow[j] = (k0 + j) * ld;
        if (tid >= c0 && tid < N) {
            T* row = A + (size_t)tid * ld + k0;
            T a[CTA_NB];
#pragma unroll
            for (int q = 0; q < CTA_NB / 4; q++) ld4at(row + 4 * q, a + 4 * q);
#pragma unroll
            for (int j = 0; j < CTA_NB; j++) {
                const T l = a[j] * (T)c.rinv[k0 + j];
                a[j] = l;
#pragma unroll
                for (int jj = j + 1; jj < CTA_NB; jj++) a[jj] = fma(-l, A[prow[j] + k0 + jj], a[jj]);
            }
#pragma unroll
            for (int q = 0; q < CTA_NB / 4; q++) st4at(row + 4 * q, a + 4 * q);
        }
        cta_u12<T>(c, A, k0, prow);
        __syncthreads();
        cta_trailing<T, true>(c, A, k0, prow);
        __syncthreads();
    }
}

// Triangular solves with the factors of cta_lu, on warp 0 alone: lane l
// owns logical rows l, l+32, ... (z in registers), column sweeps broadcast
// each finished value by shuffle -- no CTA barrier inside, one at the end.
//  REFINE = false: z_i = A[piv[i]][N] (already forward-eliminated), solve
//                  U x = z, write c.x;
//  REFINE = true:  z_i = c.r[piv[i]], solve L U dx = z, c.x += dx.
template <typename T, bool REFINE>
__device__ void cta_solve(const CtaCtx& c, const T* A) {
    if (c.tid < 32) {
        const int N = c.N, lane = c.tid, ld = c.ld;
        constexpr int M = CTA_MAXN / 32;
        double z[M], xr[M];
        int rp[M];  // row offsets
#pragma unroll
        for (int m = 0; m < M; m++) {
            const int i = lane + 32 * m;
            const bool in = i < N;
            const int pr = c.piv[in ? i : 0];
            rp[m] = pr * ld;
            z[m] = in ? (REFINE ? c.r[pr] : (double)A[rp[m] + N]) : 0.0;
            xr[m] = 0.0;
        }
        if (REFINE) {
            // L z = z, unit lower: k = 0 .. N-2
#pragma unroll
            for (int b = 0; b < M; b++) {
                if (32 * b < N) {
                    const int kend = min(N - 1, 32 * b + 32);
                    T u[M];  // column k of my rows, loaded one step ahead
#pragma unroll
                    for (int m = b; m < M; m++) u[m] = A[rp[m] + 32 * b];
                    for (int k = 32 * b; k < kend; k++) {
                        T un[M];
                        const int kn = k + 1 < kend ? k + 1 : k;
#pragma unroll
                        for (int m = b; m < M; m++) un[m] = A[rp[m] + kn];
                        const double zk = __shfl_sync(0xffffffffu, z[b], k - 32 * b);
#pragma unroll
                        for (int m = b; m < M; m++) {
                            const int i = lane + 32 * m;
                            if (i > k && i < N) z[m] = fma(-(double)u[m], zk, z[m]);
                            u[m] = un[m];
                        }
                    }
                }
            }
        }
        // U x = z: k = N-1 .. 0
#pragma unroll
        for (int b = M - 1; b >= 0; b--) {
            if (32 * b < N) {
                const int ktop = min(N, 32 * b + 32) - 1;
                T u[M];  // column k of my rows, loaded one step ahead
#pragma unroll
                for (int m = 0; m <= b; m++) u[m] = A[rp[m] + ktop];
                for (int k = ktop; k >= 32 * b; k--) {
                    T un[M];
                    const int kn = k > 32 * b ? k - 1 : k;
#pragma unroll
                    for (int m = 0; m <= b; m++) un[m] = A[rp[m] + kn];
                    const double xk = __shfl_sync(0xffffffffu, z[b] * c.rinv[k], k - 32 * b);
                    xr[b] = (lane == k - 32 * b) ? xk : xr[b];  // kept by its owner, no branch
#pragma unroll
                    for (int m = 0; m <= b; m++) {
                        const int i = lane + 32 * m;
                        if (i < k) z[m] = fma(-(double)u[m], xk, z[m]);
                        u[m] = un[m];
                    }
                }
            }
        }
        double dxm = 0.0, xm = 0.0;
        bool finite = true;
#pragma unroll
        for (int m = 0; m < M; m++) {
            const int i = lane + 32 * m;
            if (i < N) {
                const double xn = REFINE ? c.x[i] + xr[m] : xr[m];
                c.x[i] = xn;
                dxm = fmax(dxm, fabs(xr[m]));
                xm = fmax(xm, fabs(xn));
                finite = finite && isfinite(xr[m]) && isfinite(xn);  // (fmax drops NaN)
            }
        }
        if (REFINE) {
            // converged: on every lane the last correction is finite and below
            // 1e-6 of the largest |x| among the lane's rows (l, l+32, ...) --
            // at least as strict as the same test over all rows
            int ok = finite && dxm <= 1e-6 * xm;
            ok = __all_sync(0xffffffffu, ok);
            if (lane == 0) c.misc[CTA_CONV] = ok;
        }
    }
    __syncthreads();
}

// ---- MIXED: FP32 Gauss-Jordan inverse reused across an attempt ----------
// misc[] slots 8..10: rotating CTA-wide maxima (unsigned float bits).
constexpr int CTA_MAXSLOT = 8;

// CTA-wide max of |v| (one barrier).  `phase` rotates over three slots; the
// slot of the next call is cleared here -- its last readers read it two
// calls ago, before the barrier of the previous call.
__device__ __forceinline__ double cta_max_abs(const CtaCtx& c, double v, int& phase) {
    unsigned* slot = reinterpret_cast<unsigned*>(c.misc + CTA_MAXSLOT);
    const unsigned w = __reduce_max_sync(0xffffffffu, fmax_bits(v));
    if ((c.tid & 31) == 0) atomicMax(slot + phase, w);
    if (c.tid == 0) slot[(phase + 1) % 3] = 0u;
    __syncthreads();
    const unsigned m = slot[phase];
    phase = (phase + 1) % 3;
    return (double)__uint_as_float(m);
}

// A[R][R] -= A[R][P] A[P][R] (P = panel [k0, k0+kb), R the other indices)
// over 4x4 register tiles of the 4-aligned row and column chunks that miss P,
// for the row chunks from `rc0` on (0: every row; 32: the rows below the
// 128 the tensor cores update).
static __device__ __forceinline__ void cta_rank_update(const CtaCtx& c, float* A, int k0, int kb, int rc0) {
    const int N = c.N, tid = c.tid, ld = c.ld;
    const int nch = (N + 3) >> 2;
    const int pc0 = k0 >> 2, pc1 = (k0 + kb + 3) >> 2;  // chunks touching P
    const int r_lo = pc0 > rc0 ? pc0 : rc0, r_hi = pc1 > rc0 ? pc1 : rc0;  // P's chunks at or above rc0
    const int mr = (nch - rc0) - (r_hi - r_lo);  // row chunks to update
    const int m4 = nch - (pc1 - pc0);            // column chunks outside P
    for (int t = tid; t < mr * m4; t += CTA_THREADS) {
        const int ti = t / m4, tj = t - ti * m4;
        const int ri = rc0 + ti < r_lo ? rc0 + ti : rc0 + ti + (r_hi - r_lo);
        const int cj = tj < pc0 ? tj : tj + (pc1 - pc0);
        const int col = 4 * cj;
        float acc[4][4];
        int rows[4];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            const int i = 4 * ri + r;
            rows[r] = i < N ? i * ld : -1;
            if (rows[r] >= 0) ld4(A + rows[r] + col, acc[r]);
            else acc[r][0] = acc[r][1] = acc[r][2] = acc[r][3] = 0.0f;
        }
#pragma unroll 1
        for (int q0 = 0; q0 < CTA_NB; q0 += 4) {
            float u[4][4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (q0 + q < kb) ld4(A + (size_t)(k0 + q0 + q) * ld + col, u[q]);
                else u[q][0] = u[q][1] = u[q][2] = u[q][3] = 0.0f;
            }
#pragma unroll
            for (int r = 0; r < 4; r++) {
                float l[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (rows[r] >= 0) ld4(A + rows[r] + k0 + q0, l);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float lq = (q0 + q < kb) ? l[q] : 0.0f;
#pragma unroll
                    for (int cc = 0; cc < 4; cc++) acc[r][cc] = fmaf(-lq, u[q][cc], acc[r][cc]);
                }
            }
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
            if (rows[r] >= 0) st4(A + rows[r] + col, acc[r]);
    }
}

// Step 3 of the blocked inverse on the tensor cores.  The rows [0, M) of
// A, M = min(N, 128), go into the tensor-memory accumulator (row i = lane i),
// one kind::tf32 MMA chain adds (-A[R][P]) (A[P][R]) with both operands split
// into TF32 high and low parts (hi*hi + hi*lo + lo*hi: FP32-level products,
// the 3xTF32 scheme), and the accumulator is copied back.  Rows of P and
// columns of P are zero in the operands, so they come back unchanged.  Rows
// [128, N) are updated on the CUDA cores while the MMAs run.  `par` is the
// mbarrier's phase parity, flipped once per panel.  A wait that runs out
// (it never should) leaves those rows un-updated: the inverse is then wrong,
// the refinement that uses it does not converge, and the substep goes to the
// pivoted recovery path (flagged WIND_SYS_REFINE_FALLBACK).
static __device__ __forceinline__ void cta_rank_update_tc(const CtaCtx& c, float* A, int k0, int kb,
                                                           uint32_t& par) {
    const int N = c.N, tid = c.tid, ld = c.ld;
    const int M = N < 128 ? N : 128;
    const int cols16 = c.tc_cols16;
    const int w = tid >> 5, lane = tid & 31;
    const int sub = w & 3, half = w >> 2;          // two warps per lane quarter
    const int row = sub * 32 + lane;
    const uint32_t trow = c.tmem + ((uint32_t)(sub * 32) << 16);
    unsigned char* xs = c.tcs;                     // [hi s0 | hi s1 | lo s0 | lo s1], 4 KB each
    unsigned char* gs = c.tcs + 4 * 4096;          // same, cols16 * 32 B each
    const int gsl = cols16 * 32;
    // (a) rows [0, M) into the accumulator, 16 columns per store
    for (int c0 = half * 16; c0 < cols16; c0 += 32) {
        float v[16];
        const float* src = A + (size_t)(row < M ? row : 0) * ld + c0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float a4[4];
            ld4(src + 4 * q, a4);
#pragma unroll
            for (int e = 0; e < 4; e++) v[4 * q + e] = row < M ? a4[e] : 0.0f;
        }
        tc::tmem_st16(trow + c0, v);
    }
    // (b) operands: X = -A[R][P] (rows < M), G = A[P][R] stored by output column
    for (int t = tid; t < 128 * CTA_NB; t += CTA_THREADS) {
        const int i = t >> 4, q = t & 15;
        float x = 0.0f;
        if (i < M && (i < k0 || i >= k0 + kb) && q < kb) x = -A[(size_t)i * ld + k0 + q];
        const float hi = tc::to_tf32(x), lo = tc::to_tf32(x - hi);
        const int off = (q >> 3) * 4096 + tc::slab_off(i, q & 7);
        *reinterpret_cast<float*>(xs + off) = hi;
        *reinterpret_cast<float*>(xs + 2 * 4096 + off) = lo;
    }
    for (int t = tid; t < cols16 * CTA_NB; t += CTA_THREADS) {
        const int j = t >> 4, q = t & 15;
        float g = 0.0f;
        if (j < N && (j < k0 || j >= k0 + kb) && q < kb) g = A[(size_t)(k0 + q) * ld + j];
        const float hi = tc::to_tf32(g), lo = tc::to_tf32(g - hi);
        const int off = (q >> 3) * gsl + tc::slab_off(j, q & 7);
        *reinterpret_cast<float*>(gs + off) = hi;
        *reinterpret_cast<float*>(gs + 2 * gsl + off) = lo;
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        tc::fence_after_sync();
        const uint32_t id = tc::idesc_tf32(128, cols16);
        for (int sl = 0; sl < 2 && 8 * sl < kb; sl++) {
            const uint64_t xh = tc::smem_desc(tc::smem_u32(xs + sl * 4096));
            const uint64_t xl = tc::smem_desc(tc::smem_u32(xs + (2 + sl) * 4096));
            const uint64_t gh = tc::smem_desc(tc::smem_u32(gs + sl * gsl));
            const uint64_t gl = tc::smem_desc(tc::smem_u32(gs + (2 + sl) * gsl));
            tc::mma_tf32(c.tmem, xh, gh, id, true);
            tc::mma_tf32(c.tmem, xh, gl, id, true);
            tc::mma_tf32(c.tmem, xl, gh, id, true);
        }
        tc::mma_commit(c.mbar);
    }
    // (c) rows [128, N) on the CUDA cores meanwhile
    if (N > 128) cta_rank_update(c, A, k0, kb, 32);
    // (d) the accumulator back into rows [0, M)
    bool ok = tc::mbar_wait(c.mbar, par, 1u << 24);
    ok = __all_sync(0xffffffffu, ok);
    par ^= 1u;
    tc::fence_after_sync();
    if (ok) {
        for (int c0 = half * 16; c0 < cols16; c0 += 32) {
            float v[16];
            tc::tmem_ld16(trow + c0, v);
            if (row < M) {
                float* dst = A + (size_t)row * ld + c0;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    float a4[4] = {v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]};
                    st4(dst + 4 * q, a4);
                }
            }
        }
    }
    tc::fence_before_sync();
}

// Unpivoted blocked Gauss-Jordan inversion of A (N x N, FP32, row stride
// c.ld, shared memory) in place.  Per panel P = [k0, k0+kb) with the other
// indices R = [0, N) \ P:
//  1. warp 0 inverts D = A[P][P] in registers (element Gauss-Jordan with
//     shuffles; lane i holds row i of D);
//  2. A[P][R] <- D^-1 A[P][R]          one thread per column of R;
//  3. A[R][R] <- A[R][R] - A[R][P] A[P][R]   4x4 register tiles over the
//     4-aligned row and column chunks that miss P (the rank-kb update);
//  4. A[R][P] <- -A[R][P] D^-1         one thread per row of R.
// Four CTA barriers per panel.  Without pivoting the diagonal blocks must be
// invertible; a bad inverse shows up as a refinement that does not converge.
//
// TC = true (the MIXED_TC solver) runs step 3 for the first 128 rows on the
// tensor cores (cta_rank_update_tc) and for the rows below them on the CUDA
// cores at the same time.
template <bool TC>
static __device__ __noinline__ void cta_gj_invert(const CtaCtx& c, float* A) {
    const int N = c.N, tid = c.tid, ld = c.ld;
    if (tid < N) c.act[tid] = tid;   // row i expresses unknown i (no pivoting)
    uint32_t tc_par = TC ? (uint32_t)c.misc[CTA_TCPAR] : 0u;  // mbarrier phase parity
    for (int k0 = 0; k0 < N; k0 += CTA_NB) {
        const int kb = min(CTA_NB, N - k0);
        // 1. D^-1 on warp 0
        if (tid < 32) {
            const int lane = tid;
            const bool mine = lane < kb;
            float d[CTA_NB];
            const float* row = A + (size_t)(k0 + (mine ? lane : 0)) * ld + k0;
#pragma unroll
            for (int q = 0; q < CTA_NB / 4; q++) ld4at(row + 4 * q, d + 4 * q);
#pragma unroll
            for (int q = 0; q < CTA_NB; q++)
                if (!mine || q >= kb) d[q] = 0.0f;
#pragma unroll
            for (int k = 0; k < CTA_NB; k++) {
                if (k < kb) {
                    const float r = nr_rcp(__shfl_sync(0xffffffffu, d[k], k));
                    const float f = (lane == k) ? 0.0f : d[k] * r;
#pragma unroll
                    for (int q = 0; q < CTA_NB; q++) {
                        const float pq = __shfl_sync(0xffffffffu, d[q], k);
                        if (q != k) d[q] = (lane == k) ? d[q] * r : fmaf(-f, pq, d[q]);
                    }
                    d[k] = (lane == k) ? r : -f;
                }
            }
            if (mine) {
                float* wrow = A + (size_t)(k0 + lane) * ld + k0;
#pragma unroll
                for (int q = 0; q < CTA_NB; q++)
                    if (q < kb) wrow[q] = d[q];
            }
        }
        __syncthreads();
        // 2. row panel: one thread per column of R
        for (int t = tid; t < N - kb; t += CTA_THREADS) {
            const int j = t < k0 ? t : t + kb;
            float u[CTA_NB];
#pragma unroll
            for (int q = 0; q < CTA_NB; q++) u[q] = q < kb ? A[(size_t)(k0 + q) * ld + j] : 0.0f;
            // the column is in registers: each result is stored as it is formed
#pragma unroll
            for (int q = 0; q < CTA_NB; q++) {
                if (q < kb) {
                    const float* drow = A + (size_t)(k0 + q) * ld + k0;
                    float acc = 0.0f;
#pragma unroll
                    for (int pp = 0; pp < CTA_NB; pp++)
                        if (pp < kb) acc = fmaf(drow[pp], u[pp], acc);
                    A[(size_t)(k0 + q) * ld + j] = acc;
                }
            }
        }
        __syncthreads();
        // 3. rank-kb update of R x R: on the tensor cores for the first 128
        //    rows (TC), on the CUDA cores for the rest
        if constexpr (TC) {
            cta_rank_update_tc(c, A, k0, kb, tc_par);
        } else {
            cta_rank_update(c, A, k0, kb, 0);
        }
        __syncthreads();
        // 4. column panel: one thread per row of R
        for (int t = tid; t < N - kb; t += CTA_THREADS) {
            const int i = t < k0 ? t : t + kb;
            float* row = A + (size_t)i * ld + k0;
            float l[CTA_NB];
#pragma unroll
            for (int q = 0; q < CTA_NB; q++) l[q] = q < kb ? row[q] : 0.0f;
            // the row segment is in registers: each result is stored as it is formed
#pragma unroll
            for (int pp = 0; pp < CTA_NB; pp++) {
                if (pp < kb) {
                    float acc = 0.0f;
#pragma unroll
                    for (int q = 0; q < CTA_NB; q++)
                        if (q < kb) acc = fmaf(l[q], A[(size_t)(k0 + q) * ld + k0 + pp], acc);
                    row[pp] = -acc;
                }
            }
        }
        __syncthreads();
    }
    if (TC && tid == 0) c.misc[CTA_TCPAR] = (int)tc_par;
}

// Gauss-Jordan inversion of A in place with partial pivoting and no row
// exchanges, for systems whose matrices the unpivoted elimination cannot
// handle (mass-action Jacobians are not diagonally dominant: a reaction
// A + B -> C + D puts +h k y_B in row B of column A).  Column k's pivot is
// the largest |a_ik| over the rows not yet chosen, voted CTA-wide as in
// cta_lu (warp reduce, packed 64-bit atomicMax, rotating slots); the chosen
// row is copied to a broadcast buffer and every thread updates its own row
// over all N columns.  Two barriers per column.  On return row i expresses
// unknown c.act[i]: x_{act[i]} = sum_j M[i][j] b_{p_j} with p_j the row
// chosen at step j.
static __device__ __noinline__ void cta_gj_invert_pivoted(const CtaCtx& c, float* A) {
    const int N = c.N, tid = c.tid, ld = c.ld;
    float* bc = static_cast<float*>(c.cand);  // >= 1280 bytes: one row of up to 256 + 4 floats
    float* myrow = A + (size_t)(tid < N ? tid : 0) * ld;
    bool done = tid >= N;
    if (tid < 3) c.best[tid] = 0ull;
    __syncthreads();
    for (int k = 0; k < N; k++) {
        const uint32_t key = done ? 0u : mag_key(myrow[k]) + 1u;
        const uint32_t wmax = __reduce_max_sync(0xffffffffu, key);
        const int wl = __ffs(__ballot_sync(0xffffffffu, key == wmax)) - 1;
        if ((tid & 31) == wl && wmax)
            atomicMax(c.best + k % 3, ((unsigned long long)wmax << 32) | (unsigned)(0xffff - tid));
        __syncthreads();
        if (tid == 0) c.best[(k + 2) % 3] = 0ull;
        const int pr = 0xffff - (int)(c.best[k % 3] & 0xffffu);
        if (tid == pr) {
            for (int t = 0; t < N; t += 4) st4(bc + t, *reinterpret_cast<const float(*)[4]>(myrow + t));
            c.act[tid] = k;
            done = true;
        }
        __syncthreads();
        if (tid < N) {
            const float r = nr_rcp(bc[k]);
            const float alpha = (tid == pr) ? r - 1.0f : -myrow[k] * r;
            for (int t = 0; t < N; t += 4) {
                float a[4], w[4];
                ld4(myrow + t, a);
                ld4(bc + t, w);
#pragma unroll
                for (int q = 0; q < 4; q++)
                    if (t + q != k) a[q] = fmaf(alpha, w[q], a[q]);
                st4(myrow + t, a);
            }
            myrow[k] = (tid == pr) ? r : alpha;
        }
    }
    __syncthreads();
}

// Row j of M times the FP32 vector qb (shared memory), four accumulators.
__device__ __forceinline__ double cta_apply_row(const float* mrow, const float* qb, int N) {
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    const int n4 = N & ~3;
    for (int k = 0; k < n4; k += 4) {
        float a[4];
        ld4(mrow + k, a);
        const float4 b = *reinterpret_cast<const float4*>(qb + k);
        s0 = fmaf(a[0], b.x, s0);
        s1 = fmaf(a[1], b.y, s1);
        s2 = fmaf(a[2], b.z, s2);
        s3 = fmaf(a[3], b.w, s3);
    }
    for (int k = n4; k < N; k++) s0 = fmaf(mrow[k], qb[k], s0);
    return (double)((s0 + s1) + (s2 + s3));
}

enum { CTA_REFINE_OK = 0, CTA_REFINE_GAVE_UP = 1 };

// FP64 iterative refinement of (I - h J(v)) x = f (v in c.v, f in c.f)
// around the approximate inverse A: x = M f, then r = f - (x - h J x),
// x += M r.  Stop and give-up rules as the team kernel's (predicted error
// below 2^-33 max|x|; contraction worse than `abort0` on the first sweep or
// 1/2 later).  The result is left in c.x (natural order).  Uniform across
// the CTA.
static __device__ __noinline__ int cta_refine(const CtaCtx& c, const float* A, double h, int maxit, double abort0,
                          int& phase) {
    const int N = c.N, j = c.tid, ld = c.ld;
    const bool own = j < N;
    // FP32 broadcast vector in the residual slot (c.r starts 32N bytes into
    // the 16-byte aligned vector block, so float4 reads of it are aligned).
    // Row j of the inverse gives unknown act[j]: right-hand sides are
    // scattered to qb[act[j]], results gathered through c.x[act[j]].
    float* qb = reinterpret_cast<float*>(c.r);
    const int sj = own ? c.act[j] : 0;
    if (own) qb[sj] = (float)c.f[j];
    __syncthreads();
    double xt = own ? cta_apply_row(A + (size_t)j * ld, qb, N) : 0.0;  // x_{act[j]}
    const double xmax = cta_max_abs(c, xt, phase);
    double dprev = 0.0;
    int outcome = CTA_REFINE_GAVE_UP;
    for (int it = 0; it < maxit; it++) {
        if (own) c.x[sj] = xt;
        __syncthreads();
        const double r = own ? c.f[j] - fma(-h, cta_jx(c, j, c.x), c.x[j]) : 0.0;
        if (own) qb[sj] = (float)r;
        __syncthreads();
        const double d = own ? cta_apply_row(A + (size_t)j * ld, qb, N) : 0.0;
        xt += d;
        const double dmax = cta_max_abs(c, d, phase);
        const double rho = (it == 0) ? dmax / fmax(xmax, 1e-300) : dmax / fmax(dprev, 1e-300);
        if (dmax * rho <= 0x1p-33 * xmax || dmax == 0.0) { outcome = CTA_REFINE_OK; break; }
        if (rho > (it == 0 ? abort0 : 0.5)) break;
        dprev = dmax;
    }
    if (own) c.x[sj] = xt;
    __syncthreads();
    return outcome;
}

// The substep solve with pivoting (FP32 LU with partial pivoting and up to
// two FP64 refinement sweeps): the recovery path when the Gauss-Jordan
// inverse does not refine.  Builds [I - hJ(v) | f] itself; result in c.x.
static __device__ __noinline__ void cta_mixed_pivoted_solve(const CtaCtx& c, double h, float* A) {
    const int tid = c.tid;
    const bool own = tid < c.N;
    cta_build<float>(c, h, A);
    cta_lu<float>(c, A);
    cta_solve<float, false>(c, A);
    for (int it = 0; it < 2; it++) {
        if (own) c.r[tid] = c.f[tid] - (c.x[tid] - h * cta_jx(c, tid, c.x));
        __syncthreads();
        cta_solve<float, true>(c, A);
        if (c.misc[CTA_CONV]) break;
    }
}

// The reference Gauss-Jordan inverse, CTA-parallel, on global scratch.
// M = I - hJt in the reference orientation (rows of Jt), Inv starts as I.
template <int CTRL>
__device__ void cta_gje_exact(const CtaCtx& c, double h, double* M, double* Inv) {
    const int N = c.N, tid = c.tid;
    // build M; thread j owns column j (Jt[.][j] = d f_j / d y_.)
    for (int j = tid; j < N; j += CTA_THREADS) {
        for (int i = 0; i < N; i++) M[(size_t)i * N + j] = c.LT ? (double)c.LT[i * N + j] : 0.0;
        const int e0 = c.inc_off[j], e1 = c.inc_off[j + 1];
        for (int e = e0; e < e1; e++) {
            const int rr = c.inc[e];
            const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
            const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
            const xd k = c.rates[rr];
            const xd da = k * xd(c.v[b]), db = k * xd(c.v[a]);
            double* ra = M + (size_t)a * N + j;
            double* rb = M + (size_t)b * N + j;
            if (a == j) *ra = xd(*ra) - da;
            if (b == j) *ra = xd(*ra) - da;
            if (cc == j) *ra = xd(*ra) + da;
            if (d == j) *ra = xd(*ra) + da;
            if (a == j) *rb = xd(*rb) - db;
            if (b == j) *rb = xd(*rb) - db;
            if (cc == j) *rb = xd(*rb) + db;
            if (d == j) *rb = xd(*rb) + db;
        }
        for (int i = 0; i < N; i++) {
            double* m = M + (size_t)i * N + j;
            if (CTRL == WIND_CTRL_GOLD) {
                xd v = -xd(h) * xd(*m);
                if (i == j) v += 1.0;
                *m = v.v;
            } else {
                *m = (xd(i == j ? 1.0 : 0.0) - xd(*m) * xd(h)).v;
            }
            Inv[(size_t)i * N + j] = (i == j) ? 1.0 : 0.0;
        }
    }
    __syncthreads();
    // U phase (gje_gold.c:56-100)
    for (int i = 0; i < N; i++) {
        for (int k = i + 1 + tid; k < N; k += CTA_THREADS) c.scr[k] = M[(size_t)k * N + i];
        if (tid == 0) c.scr[i] = M[(size_t)i * N + i];
        __syncthreads();
        const xd s = c.scr[i];
        for (int t = tid; t < N; t += CTA_THREADS) {
            M[(size_t)i * N + t] = (xd(M[(size_t)i * N + t]) / s).v;
            Inv[(size_t)i * N + t] = (xd(Inv[(size_t)i * N + t]) / s).v;
        }
        __syncthreads();
        const int rows = N - 1 - i;
        for (int idx = tid; idx < rows * N; idx += CTA_THREADS) {
            const int k = i + 1 + idx / N, t = idx % N;
            const xd fct = c.scr[k];
            M[(size_t)k * N + t] = (xd(M[(size_t)k * N + t]) - fct * xd(M[(size_t)i * N + t])).v;
            Inv[(size_t)k * N + t] = (xd(Inv[(size_t)k * N + t]) - fct * xd(Inv[(size_t)i * N + t])).v;
        }
        __syncthreads();
    }
    // L phase, pivot rows bottom-up (gje_gold.c:102-134)
    for (int b = N - 1; b >= 0; b--) {
        for (int k = tid; k < b; k += CTA_THREADS) c.scr[k] = M[(size_t)k * N + b];
        __syncthreads();
        for (int idx = tid; idx < b * N; idx += CTA_THREADS) {
            const int k = idx / N, t = idx % N;
            const xd fct = c.scr[k];
            M[(size_t)k * N + t] = (xd(M[(size_t)k * N + t]) - fct * xd(M[(size_t)b * N + t])).v;
            Inv[(size_t)k * N + t] = (xd(Inv[(size_t)k * N + t]) - fct * xd(Inv[(size_t)b * N + t])).v;
        }
        __syncthreads();
    }
    for (int l = tid; l < N; l += CTA_THREADS) {
        if (CTRL == WIND_CTRL_GOLD) {
            // matrix_ops.c:6-27 then sie_gold.c:72-74
            xd out = 0.0;
            for (int k = 0; k < N; k++) out += xd(Inv[(size_t)k * N + l]) * xd(c.f[k]);
            c.v[l] = (xd(c.v[l]) + xd(h) * out).v;
        } else {
            // kernel.cu:121-125
            xd yl = c.v[l];
            for (int k = 0; k < N; k++) yl += xd(Inv[(size_t)k * N + l]) * xd(c.f[k]) * xd(h);
            c.v[l] = yl.v;
        }
    }
    __syncthreads();
}

// One substep of size h on c.v (in place).  Returns true when the MIXED
// solve had to be redone with pivoting (uniform across the CTA).
template <int METHOD, int CTRL, int SOLVER>
__device__ bool cta_substep(const CtaCtx& c, double h, void* mat, double* gM) {
    const int N = c.N, tid = c.tid;
    const bool own = tid < N;
    if (METHOD == WIND_METHOD_RK2) {
        cta_rhs(c);
        if (own) c.v[tid] = (xd(c.v[tid]) + xd(h) * xd(c.f[tid])).v;
        __syncthreads();
        return false;
    }
    if (SOLVER == WIND_SOLVER_GJE_F64) {
        cta_rhs(c);
        cta_gje_exact<CTRL>(c, h, gM, gM + (size_t)N * N);
        return false;
    }
    using T = typename std::conditional<SOLVER == WIND_SOLVER_MIXED, float, double>::type;
    T* A = static_cast<T*>(mat);
    bool fell = false;
    cta_build<T>(c, h, A);
    if (SOLVER == WIND_SOLVER_MIXED) {
        // unpivoted FP32 factors and up to two FP64 refinement steps (the
        // second only when the first correction is not yet small); if the
        // last correction is not small, redo the substep with pivoting
        for (int pass = 0; pass < 2; pass++) {
            if (pass == 0) cta_lu_nopiv<T>(c, A);
            else cta_lu<T>(c, A);
            cta_solve<T, false>(c, A);
            for (int it = 0; it < 2; it++) {
                if (own) c.r[tid] = c.f[tid] - (c.x[tid] - h * cta_jx(c, tid, c.x));
                __syncthreads();
                cta_solve<T, true>(c, A);
                if (c.misc[CTA_CONV]) break;
            }
            if (c.misc[CTA_CONV] || pass == 1) break;
            fell = true;
            cta_build<T>(c, h, A);
        }
    } else {
        cta_lu<T>(c, A);
        cta_solve<T, false>(c, A);
    }
    if (own) c.v[tid] = c.v[tid] + h * c.x[tid];
    __syncthreads();
    return fell;
}

// The persistent CTA loop over one group's systems (blockDim.x must be
// CTA_THREADS).  `gscratch` holds one slot of `gstride` >=
// CtaLayout::g_doubles doubles per block (null when the layout needs none).
template <int METHOD, int CTRL, int SOLVER, bool TC>
__device__ __forceinline__ void cta_run(const KParams& p, unsigned char* smem_raw, double* gscratch,
                                        size_t gstride, int smem_cap) {
    constexpr int CAP = Cap<METHOD, CTRL>::value;
    const int N = p.n_eq, R = p.n_react, tid = threadIdx.x;
    const bool own = tid < N;
    const bool lin = p.linear != nullptr;
    const CtaLayout lay(N, R, lin, SOLVER, smem_cap, TC);
    CtaCtx c;
    c.N = N;
    c.R = R;
    c.tid = tid;
    c.ld = lay.ld;
    c.cols = lay.cols;
    double* vec = reinterpret_cast<double*>(smem_raw + lay.vec);
    c.v = vec;
    c.f = vec + N;
    c.x = c.r = c.rinv = c.scr = nullptr;
    if (SOLVER == WIND_SOLVER_GJE_F64) {
        c.scr = vec + 2 * N;
    } else {
        c.x = vec + 2 * N;
        c.rinv = vec + 3 * N;
        if (SOLVER == WIND_SOLVER_MIXED) c.r = vec + 4 * N;
    }
    c.piv = reinterpret_cast<int*>(smem_raw + lay.piv);
    c.act = reinterpret_cast<int*>(smem_raw + lay.act);
    c.misc = reinterpret_cast<int*>(smem_raw + lay.misc);
    c.best = reinterpret_cast<unsigned long long*>(smem_raw + lay.misc + 4 * CTA_WARPS);
    c.cand = smem_raw + lay.cand;
    double* gslot = gscratch ? gscratch + (size_t)blockIdx.x * gstride : nullptr;
    unsigned char* incbase = lay.inc_in_smem ? smem_raw + lay.inc_off
                                             : reinterpret_cast<unsigned char*>(gslot + lay.g_inc);
    int* inc_off = reinterpret_cast<int*>(incbase);
    uint16_t* inc = reinterpret_cast<uint16_t*>(incbase + CtaLayout::a16((N + 1) * 4));
    c.inc_off = inc_off;
    c.inc = inc;
    float* LT = lin ? reinterpret_cast<float*>(smem_raw + lay.lt) : nullptr;
    c.LT = LT;
    double* gM = gslot;
    void* mat = lay.mat_in_smem ? (void*)(smem_raw + lay.mat) : (void*)(gslot + lay.g_mat);
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;
    __shared__ unsigned long long s_ticket;
    __shared__ int s_flag;
    // MIXED_TC: the accumulator's tensor-memory columns (a power of two
    // >= 32 covering the columns rounded to 16), held for the whole launch
    uint32_t tc_ncols = 32;
    if constexpr (TC) {
        c.tc_cols16 = (N + 15) & ~15;
        while ((int)tc_ncols < c.tc_cols16) tc_ncols <<= 1;
        c.mbar = reinterpret_cast<uint64_t*>(smem_raw + lay.tcs);
        uint32_t* taddr = reinterpret_cast<uint32_t*>(smem_raw + lay.tcs + 8);
        c.tcs = smem_raw + lay.tcs + 64;
        if (tid < 32) tc::tmem_alloc(taddr, tc_ncols);
        if (tid == 0) {
            tc::mbar_init(c.mbar, 1);
            c.misc[CTA_TCPAR] = 0;
        }
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        c.tmem = *taddr;
    } else {
        c.tmem = 0;
        c.mbar = nullptr;
        c.tcs = nullptr;
        c.tc_cols16 = 0;
    }

    while (true) {
        if (tid == 0) s_ticket = atomicAdd(&p.counters[CNT_QUEUE], 1ull);
        __syncthreads();
        const int64_t s = (int64_t)s_ticket;
        if (s >= p.nsys) break;
        c.rates = p.rates + s * R;
        c.sp = p.species + (s * R) * 4;
        if (lay.data_in_smem) {
            double* srt = reinterpret_cast<double*>(smem_raw + lay.rt);
            uint2* ssp = reinterpret_cast<uint2*>(smem_raw + lay.spc);
            for (int r = tid; r < R; r += CTA_THREADS) {
                srt[r] = c.rates[r];
                ssp[r] = *reinterpret_cast<const uint2*>(c.sp + 4 * r);
            }
            c.rates = srt;
            c.sp = reinterpret_cast<const uint16_t*>(ssp);
        }
        // validate species indices, then build the per-species incidence lists
        if (tid == 0) s_flag = 0;
        __syncthreads();
        for (int r = tid; r < R; r += CTA_THREADS) {
            const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * r);
            const unsigned nn = (unsigned)N;
            if ((q.x & 0xffffu) >= nn || (q.x >> 16) >= nn || (q.y & 0xffffu) >= nn || (q.y >> 16) >= nn)
                s_flag = 1;
        }
        __syncthreads();
        const bool bad = s_flag != 0;
        if (!bad) {
            if (own) {
                int cnt = 0;
                for (int r = 0; r < R; r++) {
                    const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * r);
                    const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
                    cnt += (a == tid || b == tid || cc == tid || d == tid);
                }
                inc_off[tid + 1] = cnt;
            }
            __syncthreads();
            if (tid == 0) {
                inc_off[0] = 0;
                for (int j = 0; j < N; j++) inc_off[j + 1] += inc_off[j];
            }
            __syncthreads();
            if (own) {
                int o = inc_off[tid];
                for (int r = 0; r < R; r++) {
                    const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * r);
                    const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
                    if (a == tid || b == tid || cc == tid || d == tid) inc[o++] = (uint16_t)r;
                }
            }
            if (lin) {
                const float* Lg = p.linear + s * (int64_t)N * N;
                for (int idx = tid; idx < N * N; idx += CTA_THREADS) {
                    const int j = idx / N, k = idx % N;
                    LT[k * N + j] = Lg[idx];
                }
            }
        }
        double yl = own ? p.y[s * N + tid] : 0.0, y1l = 0.0, y2l = 0.0;
        if (tid < 3) reinterpret_cast<unsigned*>(c.misc + CTA_MAXSLOT)[tid] = 0u;
        __syncthreads();

        double tnow = p.tnow;
        const double tend = p.tend;
        double h = p.h0;
        int unsolved = 0;
        int64_t attempts = 0;
        int32_t st = bad ? WIND_SYS_BAD_INPUT : WIND_SYS_OK;
        // MIXED: f(y) cached while y is unchanged; the matrix area holds the
        // inverse for the next full step; rotating max-slot phase
        bool fy_ok = false, inv_ok = false;
        double h_pivot = INFINITY;  // MIXED: fresh inverses at this step size and above pivot
        double fyl = 0.0;
        int phase = 0;
        while (!bad && tnow < tend) {
            if (attempts >= p.max_attempts) { st |= WIND_SYS_MAX_ATTEMPTS; break; }
            if (p.timeout_ns) {
                // thread 0's clock decides for the whole CTA
                if (__syncthreads_or(tid == 0 && global_ns() - t_start > p.timeout_ns)) {
                    st |= WIND_SYS_TIMEOUT;
                    break;
                }
            }
            attempts++;
            h = fmin(tend - tnow, h);
            const double t1 = tnow + h;
            if constexpr (METHOD == WIND_METHOD_SIE && SOLVER == WIND_SOLVER_MIXED) {
                // One FP32 Gauss-Jordan inverse serves the attempt: the
                // previous attempt's half-step inverse (same y, same size)
                // for the full step, a fresh one for the first half step,
                // reused for the second half step while it still contracts.
                // Fresh inverses are unpivoted (blocked, fast) below the
                // smallest step size at which an unpivoted one failed to
                // refine for this system, pivoted (column vote) at and above
                // it: the growth of the unpivoted elimination rises with h.
                // A fresh pivoted inverse that does not refine either (I - hJ
                // too ill-conditioned for FP32) leaves the substep to the FP32
                // LU recovery.  Any recovery flags the system
                // WIND_SYS_REFINE_FALLBACK.
                const double hf = t1 - tnow, h1 = (t1 - tnow) * 0.5;
                const double h2 = (CTRL == WIND_CTRL_DEVICE) ? fmin(t1 - (tnow + h1), h1) : h1;
                float* A = static_cast<float*>(mat);
                // a fresh inverse of this substep's own matrix, and its solve
                auto fresh_solve = [&](double hh) {
                    cta_build<float>(c, hh, A);
                    if (hh < h_pivot) {
                        cta_gj_invert<TC>(c, A);
                        if (cta_refine(c, A, hh, 24, 1.0, phase) == CTA_REFINE_OK) return true;
                        h_pivot = hh;
                        cta_build<float>(c, hh, A);
                    }
                    st |= WIND_SYS_REFINE_FALLBACK;
                    cta_gj_invert_pivoted(c, A);
                    if (cta_refine(c, A, hh, 24, 1.0, phase) == CTA_REFINE_OK) return true;
                    cta_mixed_pivoted_solve(c, hh, A);
                    return false;
                };
                if (own) c.v[tid] = yl;
                __syncthreads();
                if (!fy_ok) {
                    cta_rhs_fast(c);
                    fyl = own ? c.f[tid] : 0.0;
                    fy_ok = true;
                } else {
                    if (own) c.f[tid] = fyl;
                    __syncthreads();
                }
                if (!inv_ok || cta_refine(c, A, hf, 8, 0.5, phase) != CTA_REFINE_OK) fresh_solve(hf);
                y1l = own ? yl + hf * c.x[tid] : 0.0;
                inv_ok = fresh_solve(h1);  // the inverse stays for the next full step
                const double vhl = own ? yl + h1 * c.x[tid] : 0.0;
                if (own) c.v[tid] = vhl;
                __syncthreads();
                cta_rhs_fast(c);
                if (!inv_ok || cta_refine(c, A, h2, 8, 0.0625, phase) != CTA_REFINE_OK) {
                    fresh_solve(h2);
                    inv_ok = false;
                }
                y2l = own ? vhl + h2 * c.x[tid] : 0.0;
            } else
            for (int pass = 0; pass < 2; pass++) {
                const int nsub = pass + 1;
                if (own) c.v[tid] = yl;
                __syncthreads();
                // (t1-t0)/nsub, nsub in {1,2}: exact as a multiplication
                double hs = (t1 - tnow) * (nsub == 1 ? 1.0 : 0.5);
                double t = tnow;
                for (int k = 0; k < nsub; k++) {
                    if (CTRL == WIND_CTRL_DEVICE) hs = fmin(t1 - t, hs);
                    if (cta_substep<METHOD, CTRL, SOLVER>(c, hs, mat, gM)) st |= WIND_SYS_REFINE_FALLBACK;
                    t += hs;
                }
                if (own) {
                    if (pass == 0) y1l = c.v[tid];
                    else y2l = c.v[tid];
                }
            }
            const int e = own && elem_error<METHOD, CTRL>(xd(y1l), xd(y2l), p.atol, p.rtol) ? 1 : 0;
            const bool err = __syncthreads_or(e) != 0;
            if (err && unsolved < CAP) {
                unsolved++;
                h /= 2.0;
            } else {
                unsolved = 0;
                fy_ok = inv_ok = false;
                if (own) yl = (METHOD == WIND_METHOD_RK2) ? (xd(2.0) * xd(y2l) - xd(y1l)).v : y2l;
                if (tnow + h == tnow) { st |= WIND_SYS_STALLED; break; }
                tnow += h;
                h = (METHOD == WIND_METHOD_RK2) ? h * 2 : tend - tnow;
            }
        }
        int nonfinite = 0;
        if (own) {
            if (!finite64(yl)) nonfinite = 1;
            p.y[s * N + tid] = yl;
        }
        if (__syncthreads_or(nonfinite)) st |= WIND_SYS_NONFINITE;
        if (tid == 0) {
            if (p.sys_status) p.sys_status[s] = st;
            if (p.sys_nsteps) p.sys_nsteps[s] = 3 * attempts;
            atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)(3 * attempts));
        }
        __syncthreads();
    }
    if constexpr (TC) {
        // every MMA was waited for; the columns go back before the CTA exits
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (tid < 32) tc::tmem_dealloc(c.tmem, tc_ncols);
    }
}

// Two CTAs per SM for the FP32 factors (the 157-species matrix is ~100 KB).
#ifndef WIND_CTA_MIXED_BLOCKS
#define WIND_CTA_MIXED_BLOCKS 2
#endif
template <int SOLVER>
struct CtaMinBlocks {
    static constexpr int value = SOLVER == WIND_SOLVER_MIXED ? WIND_CTA_MIXED_BLOCKS : 1;
};

// TC = true: MIXED with the inverse's rank updates on the tensor cores
// (the MIXED_TC solver).
template <int METHOD, int CTRL, int SOLVER, bool TC = false>
__global__ void __launch_bounds__(CTA_THREADS, CtaMinBlocks<SOLVER>::value)
    k_cta(const KParams p, double* gscratch, size_t gstride, int smem_cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cta_run<METHOD, CTRL, SOLVER, TC>(p, smem_raw, gscratch, gstride, smem_cap);
}

}  // namespace wind
