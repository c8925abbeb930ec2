// cta_kernel.cuh -- persistent CTA-per-system integrator for mass-action
// networks with 32 < N <= 256 (the 64- and 157-species classes).
//
// One CTA (256 threads) integrates one system at a time and pulls the next
// ticket from the device work queue when it finishes.  Per system it stages
// in shared memory: the state vectors, the dense linear term (transposed,
// FP32) if any, and per-species incidence lists of the reactions (CSR,
// reaction ids ascending), so thread j evaluates f_j and row j of the
// Jacobian from the ~4R/N reactions that touch species j instead of all R.
//
// Solvers (selected at compile time):
//  GJE_F64  the reference's unpivoted Gauss-Jordan inverse, reference
//           operation order, on M and Inv in a per-CTA global scratch slot
//           (2 N^2 doubles; L2-resident) -- bit-exact parity path;
//  LU_F64   right-looking LU with partial pivoting on the matrix in shared
//           memory (global scratch when N^2 doubles do not fit), rows
//           permuted implicitly (no row moves), the right-hand side carried as
//           column N, two CTA barriers per pivot;
//  MIXED    the same LU with FP32 factors in shared memory, FP64 residual
//           r = f - (x - h J x) evaluated from the reactions (no FP64
//           matrix), two FP64 refinement steps.
#pragma once

#include "common.cuh"
#include "networks.cuh"

namespace wind {

constexpr int CTA_THREADS = 256;
constexpr int CTA_MAXN = 256;

// Shared-memory layout of one CTA (byte offsets), computed on the host and
// the device alike.
struct CtaLayout {
    int vec, piv, inc_off, inc, lt, mat, bytes;
    bool mat_in_smem;
    __host__ __device__ static int a16(int x) { return (x + 15) & ~15; }
    __host__ __device__ CtaLayout(int N, int R, bool lin, int solver, int smem_cap) {
        int off = 0;
        vec = off; off = a16(off + 10 * N * 8);            // v f y y1 y2 x r z rinv scratch
        piv = off; off = a16(off + (2 * N + 8) * 4);       // permutation, pivot step per row, misc
        inc_off = off; off = a16(off + (N + 1) * 4);       // CSR offsets
        inc = off; off = a16(off + 4 * R * 2);             // CSR reaction ids (uint16)
        lt = off; off = a16(off + (lin ? N * N * 4 : 0));  // L^T, FP32
        mat = off;
        const int esz = (solver == WIND_SOLVER_MIXED) ? 4 : 8;
        const int mbytes = (solver == WIND_SOLVER_GJE_F64) ? 0 : a16(N * (N + 1) * esz);
        mat_in_smem = (off + mbytes) <= smem_cap;
        if (mat_in_smem) off += mbytes;
        bytes = off;
    }
    // doubles of global scratch per CTA
    __host__ __device__ static size_t gscratch_doubles(int N, int solver) {
        if (solver == WIND_SOLVER_GJE_F64) return (size_t)2 * N * N;
        if (solver == WIND_SOLVER_LU_F64) return (size_t)N * (N + 1);
        return (size_t)(N * (N + 1) + 1) / 2;
    }
};

struct CtaCtx {
    int N, R, tid;
    const double* rates;     // global [R]
    const uint16_t* sp;      // global [R*4]
    const float* LT;         // smem [N*N] or null
    const int* inc_off;      // smem [N+1]
    const uint16_t* inc;     // smem
    double *v, *f, *y, *y1, *y2, *x, *r, *z, *rinv, *scr;
    int* piv;    // logical row -> physical row
    int* pstep;  // physical row -> step at which it became the pivot row (N = not yet)
    int* misc;
};

// f_j and, with JAC, row j of A = I - h J in standard orientation (J[j][c] =
// Jt[c][j]) with the right-hand side f_j as column N, for j = tid, tid+256...
// Per element the update sequence is the sequential one of the mass-action
// contract.
template <bool JAC, typename T>
__device__ __forceinline__ void cta_rhs_jac(const CtaCtx& c, double h, T* A, int ldA) {
    const int N = c.N;
    for (int j = c.tid; j < N; j += CTA_THREADS) {
        xd acc = 0.0;
        T* row = JAC ? A + (size_t)j * ldA : nullptr;
        if (c.LT) {
            for (int k = 0; k < N; k++) acc += xd((double)c.LT[k * N + j]) * xd(c.v[k]);
        }
        if (JAC) {
            // J[j][c] = Jt[c][j]; start from L[j][c] = LT[c][j] or 0
            for (int cc = 0; cc < N; cc++) row[cc] = c.LT ? (T)c.LT[cc * N + j] : (T)0;
        }
        const int e0 = c.inc_off[j], e1 = c.inc_off[j + 1];
        for (int e = e0; e < e1; e++) {
            const int rr = c.inc[e];
            const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
            const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
            const xd k = __ldg(c.rates + rr);
            const xd ya = c.v[a], yb = c.v[b];
            const xd w = k * ya * yb;
            if (a == j) acc -= w;
            if (b == j) acc -= w;
            if (cc == j) acc += w;
            if (d == j) acc += w;
            if (JAC) {
                // element (j, a) = Jt[a][j]: updates in the sequential order
                const xd da = k * yb, db = k * ya;
                if (a == j) row[a] = (T)(xd((double)row[a]) - da);
                if (b == j) row[a] = (T)(xd((double)row[a]) - da);
                if (cc == j) row[a] = (T)(xd((double)row[a]) + da);
                if (d == j) row[a] = (T)(xd((double)row[a]) + da);
                if (a == j) row[b] = (T)(xd((double)row[b]) - db);
                if (b == j) row[b] = (T)(xd((double)row[b]) - db);
                if (cc == j) row[b] = (T)(xd((double)row[b]) + db);
                if (d == j) row[b] = (T)(xd((double)row[b]) + db);
            }
        }
        c.f[j] = acc.v;
        if (JAC) {
            for (int cc = 0; cc < N; cc++) row[cc] = (T)((cc == j ? 1.0 : 0.0) - h * (double)row[cc]);
            row[N] = (T)acc.v;  // right-hand side as column N
        }
    }
    __syncthreads();
}

// (J x)_j from the reactions (and L), FP64, for the refinement residual.
__device__ __forceinline__ double cta_jx(const CtaCtx& c, int j, const double* xv) {
    const int N = c.N;
    double acc = 0.0;
    if (c.LT)
        for (int k = 0; k < N; k++) acc = fma((double)c.LT[k * N + j], xv[k], acc);
    const int e0 = c.inc_off[j], e1 = c.inc_off[j + 1];
    for (int e = e0; e < e1; e++) {
        const int rr = c.inc[e];
        const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
        const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
        const double k = __ldg(c.rates + rr);
        const double dw = k * (c.v[b] * xv[a] + c.v[a] * xv[b]);
        if (a == j) acc -= dw;
        if (b == j) acc -= dw;
        if (cc == j) acc += dw;
        if (d == j) acc += dw;
    }
    return acc;
}

// Right-looking LU with partial pivoting on A (N rows, N+1 columns: the last
// is the right-hand side).  Implicit row permutation piv[] (logical row i is
// physical row piv[i]).  On return c.x holds the solution and c.rinv[i]
// holds 1/U_ii; with STORE_L the multipliers are kept in A's column i of the
// rows below (for later re-solves).  The multipliers of step i-1 are scaled
// during step i's pivot search, on the rows whose pivot step is >= i (a set
// the concurrent swap cannot change).
template <typename T, bool STORE_L>
__device__ void cta_lu_solve(const CtaCtx& c, T* A, int ldA) {
    const int N = c.N, tid = c.tid;
    const int warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < N; i += CTA_THREADS) {
        c.piv[i] = i;
        c.pstep[i] = N;
    }
    __syncthreads();
    // 2-D thread grid for the trailing update
    const int ty = tid >> 4, tx = tid & 15;
    for (int i = 0; i < N; i++) {
        if (warp == 0) {
            // pivot search over logical rows i..N-1 of column i
            double best = -1.0;
            int bk = N;
            for (int k = i + lane; k < N; k += 32) {
                const double v = fabs((double)A[(size_t)c.piv[k] * ldA + i]);
                if (v > best || (v == best && k < bk)) { best = v; bk = k; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int ok = __shfl_xor_sync(0xffffffffu, bk, o);
                if (ob > best || (ob == best && ok < bk)) { best = ob; bk = ok; }
            }
            if (lane == 0) {
                if (bk >= N) bk = i;  // all-NaN column: keep the diagonal
                const int pi = c.piv[i];
                c.piv[i] = c.piv[bk];
                c.piv[bk] = pi;
                c.pstep[c.piv[i]] = i;
                c.rinv[i] = (double)nr_rcp(A[(size_t)c.piv[i] * ldA + i]);
            }
        } else if (STORE_L && i > 0) {
            // the previous step's multipliers, on physical rows not yet pivot
            // before step i (pivot step >= i, whatever the swap does)
            const T ri = (T)c.rinv[i - 1];
            for (int pr = tid - 32; pr < N; pr += CTA_THREADS - 32)
                if (c.pstep[pr] >= i) A[(size_t)pr * ldA + (i - 1)] *= ri;
        }
        __syncthreads();
        const T ri = (T)c.rinv[i];
        const T* prow = A + (size_t)c.piv[i] * ldA;
        for (int k = i + 1 + ty; k < N; k += 16) {
            T* row = A + (size_t)c.piv[k] * ldA;
            const T l = row[i] * ri;
            for (int t = i + 1 + tx; t <= N; t += 16) row[t] = fma(-l, prow[t], row[t]);
        }
        __syncthreads();
    }
    // back substitution on warp 0, column-oriented: z[k] = A[piv[k]][N]
    if (warp == 0) {
        for (int k = lane; k < N; k += 32) c.z[k] = (double)A[(size_t)c.piv[k] * ldA + N];
        __syncwarp();
        for (int i = N - 1; i >= 0; i--) {
            const double xi = c.z[i] * c.rinv[i];
            for (int k = lane; k < i; k += 32) c.z[k] = fma(-(double)A[(size_t)c.piv[k] * ldA + i], xi, c.z[k]);
            if (lane == 0) c.x[i] = xi;
            __syncwarp();
        }
    }
    __syncthreads();
}

// Re-solve with stored factors for right-hand side c.r (original order);
// result in c.x.  Warp 0 only, then a CTA barrier.
template <typename T>
__device__ void cta_lu_resolve(const CtaCtx& c, const T* A, int ldA) {
    const int N = c.N, tid = c.tid;
    if ((tid >> 5) == 0) {
        const int lane = tid & 31;
        for (int k = lane; k < N; k += 32) c.z[k] = c.r[c.piv[k]];
        __syncwarp();
        for (int i = 0; i < N; i++) {
            const double zi = c.z[i];
            for (int k = i + 1 + lane; k < N; k += 32)
                c.z[k] = fma(-(double)A[(size_t)c.piv[k] * ldA + i], zi, c.z[k]);
            __syncwarp();
        }
        for (int i = N - 1; i >= 0; i--) {
            const double xi = c.z[i] * c.rinv[i];
            for (int k = lane; k < i; k += 32) c.z[k] = fma(-(double)A[(size_t)c.piv[k] * ldA + i], xi, c.z[k]);
            if (lane == 0) c.x[i] = xi;
            __syncwarp();
        }
    }
    __syncthreads();
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
            const xd k = __ldg(c.rates + rr);
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

template <int METHOD, int CTRL, int SOLVER>
__device__ void cta_substep(const CtaCtx& c, double h, void* mat, int ldA, double* gM) {
    const int N = c.N, tid = c.tid;
    if (METHOD == WIND_METHOD_RK2) {
        cta_rhs_jac<false, double>(c, h, nullptr, 0);
        for (int l = tid; l < N; l += CTA_THREADS) c.v[l] = (xd(c.v[l]) + xd(h) * xd(c.f[l])).v;
        __syncthreads();
        return;
    }
    if (SOLVER == WIND_SOLVER_GJE_F64) {
        cta_rhs_jac<false, double>(c, h, nullptr, 0);
        cta_gje_exact<CTRL>(c, h, gM, gM + (size_t)N * N);
        return;
    }
    if (SOLVER == WIND_SOLVER_LU_F64) {
        double* A = static_cast<double*>(mat);
        cta_rhs_jac<true, double>(c, h, A, ldA);
        cta_lu_solve<double, false>(c, A, ldA);
        for (int l = tid; l < N; l += CTA_THREADS) c.v[l] = c.v[l] + h * c.x[l];
        __syncthreads();
        return;
    }
    float* A = static_cast<float*>(mat);
    cta_rhs_jac<true, float>(c, h, A, ldA);
    cta_lu_solve<float, true>(c, A, ldA);
    // two FP64 refinement steps with the FP32 factors
    for (int it = 0; it < 2; it++) {
        for (int l = tid; l < N; l += CTA_THREADS) c.r[l] = c.f[l] - (c.x[l] - h * cta_jx(c, l, c.x));
        for (int l = tid; l < N; l += CTA_THREADS) c.scr[l] = c.x[l];
        __syncthreads();
        cta_lu_resolve<float>(c, A, ldA);
        for (int l = tid; l < N; l += CTA_THREADS) c.x[l] = c.scr[l] + c.x[l];
        __syncthreads();
    }
    for (int l = tid; l < N; l += CTA_THREADS) c.v[l] = c.v[l] + h * c.x[l];
    __syncthreads();
}

// The persistent CTA loop over one group's systems (blockDim.x must be
// CTA_THREADS).  `gscratch` holds one matrix slot per block when the layout
// does not keep the matrix in shared memory (and always for GJE_F64).
template <int METHOD, int CTRL, int SOLVER>
__device__ __forceinline__ void cta_run(const KParams& p, unsigned char* smem_raw, double* gscratch, int smem_cap) {
    constexpr int CAP = Cap<METHOD, CTRL>::value;
    const int N = p.n_eq, R = p.n_react, tid = threadIdx.x;
    const bool lin = p.linear != nullptr;
    const CtaLayout lay(N, R, lin, SOLVER, smem_cap);
    CtaCtx c;
    c.N = N;
    c.R = R;
    c.tid = tid;
    double* vec = reinterpret_cast<double*>(smem_raw + lay.vec);
    c.v = vec;
    c.f = vec + N;
    c.y = vec + 2 * N;
    c.y1 = vec + 3 * N;
    c.y2 = vec + 4 * N;
    c.x = vec + 5 * N;
    c.r = vec + 6 * N;
    c.z = vec + 7 * N;
    c.rinv = vec + 8 * N;
    c.scr = vec + 9 * N;
    c.piv = reinterpret_cast<int*>(smem_raw + lay.piv);
    c.pstep = c.piv + N;
    c.misc = c.piv + 2 * N;
    int* inc_off = reinterpret_cast<int*>(smem_raw + lay.inc_off);
    uint16_t* inc = reinterpret_cast<uint16_t*>(smem_raw + lay.inc);
    c.inc_off = inc_off;
    c.inc = inc;
    float* LT = lin ? reinterpret_cast<float*>(smem_raw + lay.lt) : nullptr;
    c.LT = LT;
    const size_t gsz = CtaLayout::gscratch_doubles(N, SOLVER);
    double* gM = gscratch ? gscratch + (size_t)blockIdx.x * gsz : nullptr;
    void* mat = lay.mat_in_smem ? (void*)(smem_raw + lay.mat) : (void*)gM;
    const int ldA = N + 1;
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;
    __shared__ unsigned long long s_ticket;
    __shared__ int s_flag;

    while (true) {
        if (tid == 0) s_ticket = atomicAdd(&p.counters[CNT_QUEUE], 1ull);
        __syncthreads();
        const int64_t s = (int64_t)s_ticket;
        if (s >= p.nsys) break;
        c.rates = p.rates + s * R;
        c.sp = p.species + (s * R) * 4;
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
            for (int j = tid; j < N; j += CTA_THREADS) {
                int cnt = 0;
                for (int r = 0; r < R; r++) {
                    const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * r);
                    const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
                    cnt += (a == j || b == j || cc == j || d == j);
                }
                inc_off[j + 1] = cnt;
            }
            __syncthreads();
            if (tid == 0) {
                inc_off[0] = 0;
                for (int j = 0; j < N; j++) inc_off[j + 1] += inc_off[j];
            }
            __syncthreads();
            for (int j = tid; j < N; j += CTA_THREADS) {
                int o = inc_off[j];
                for (int r = 0; r < R; r++) {
                    const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * r);
                    const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
                    if (a == j || b == j || cc == j || d == j) inc[o++] = (uint16_t)r;
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
        for (int l = tid; l < N; l += CTA_THREADS) c.y[l] = p.y[s * N + l];
        __syncthreads();

        double tnow = p.tnow;
        const double tend = p.tend;
        double h = p.h0;
        int unsolved = 0;
        int64_t attempts = 0;
        int32_t st = bad ? WIND_SYS_BAD_INPUT : WIND_SYS_OK;
        while (!bad && tnow < tend) {
            if (attempts >= p.max_attempts) { st |= WIND_SYS_MAX_ATTEMPTS; break; }
            if (p.timeout_ns && global_ns() - t_start > p.timeout_ns) { st |= WIND_SYS_TIMEOUT; break; }
            attempts++;
            h = fmin(tend - tnow, h);
            const double t1 = tnow + h;
            for (int pass = 0; pass < 2; pass++) {
                const int nsub = pass + 1;
                for (int l = tid; l < N; l += CTA_THREADS) c.v[l] = c.y[l];
                __syncthreads();
                // (t1-t0)/nsub, nsub in {1,2}: exact as a multiplication
                double hs = (t1 - tnow) * (nsub == 1 ? 1.0 : 0.5);
                double t = tnow;
                for (int k = 0; k < nsub; k++) {
                    if (CTRL == WIND_CTRL_DEVICE) hs = fmin(t1 - t, hs);
                    cta_substep<METHOD, CTRL, SOLVER>(c, hs, mat, ldA, gM);
                    t += hs;
                }
                double* dst = pass == 0 ? c.y1 : c.y2;
                for (int l = tid; l < N; l += CTA_THREADS) dst[l] = c.v[l];
                __syncthreads();
            }
            int e = 0;
            for (int l = tid; l < N; l += CTA_THREADS)
                e |= elem_error<METHOD, CTRL>(xd(c.y1[l]), xd(c.y2[l]), p.atol, p.rtol) ? 1 : 0;
            const bool err = __syncthreads_or(e) != 0;
            if (err && unsolved < CAP) {
                unsolved++;
                h /= 2.0;
            } else {
                unsolved = 0;
                for (int l = tid; l < N; l += CTA_THREADS)
                    c.y[l] = (METHOD == WIND_METHOD_RK2) ? (xd(2.0) * xd(c.y2[l]) - xd(c.y1[l])).v : c.y2[l];
                if (tnow + h == tnow) { st |= WIND_SYS_STALLED; __syncthreads(); break; }
                tnow += h;
                h = (METHOD == WIND_METHOD_RK2) ? h * 2 : tend - tnow;
            }
            __syncthreads();
        }
        int nonfinite = 0;
        for (int l = tid; l < N; l += CTA_THREADS) {
            if (!finite64(c.y[l])) nonfinite = 1;
            p.y[s * N + l] = c.y[l];
        }
        if (__syncthreads_or(nonfinite)) st |= WIND_SYS_NONFINITE;
        if (tid == 0) {
            if (p.sys_status) p.sys_status[s] = st;
            if (p.sys_nsteps) p.sys_nsteps[s] = 3 * attempts;
            atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)(3 * attempts));
        }
        __syncthreads();
    }
}

template <int METHOD, int CTRL, int SOLVER>
__global__ void __launch_bounds__(CTA_THREADS) k_cta(const KParams p, double* gscratch, int smem_cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cta_run<METHOD, CTRL, SOLVER>(p, smem_raw, gscratch, smem_cap);
}

}  // namespace wind
