// warp_kernel.cuh -- register-resident team-per-system SIE for runtime
// mass-action networks with N <= 32 (optionally with a dense linear term).
//
// A team is NMAX lanes of one warp (NMAX = 8, 16 or 32); a 128-thread block
// holds 128/NMAX teams, each with its own shared-memory slice.  Lane l owns
// equation l: its row of the matrix lives in registers (NMAX elements,
// indexed only by compile-time constants), the state components y_l, v_l,
// f_l, x_l are scalars in registers, and whatever another lane must read --
// the state, a solution vector, the pivot row of an elimination step -- goes
// through a small broadcast buffer in shared memory.  Loops over columns and
// elimination steps are unrolled, so a step costs one reduction for the
// pivot, one row broadcast and NMAX fused multiply-adds per lane.
//
// Solvers (SIE only; RK2 and the reference Gauss-Jordan stay in the team
// kernel):
//  LU_F64  the plain FP64 path: I - hJ built at every substep, LU with
//          partial pivoting (pivot = one warp reduction over a packed
//          |a|/lane key, rows never move), right-hand side eliminated with the
//          factorisation, column-oriented back substitution;
//  MIXED   FP32 Gauss-Jordan inverse of I - hJ with partial pivoting, computed
//          ONCE per step-doubling attempt at the half-step size and the
//          attempt's state, and used as the approximate inverse of every solve
//          of the attempt (both half steps, and the next attempt's full step
//          after a rejection, whose size is that half-step size) inside an
//          FP64 iterative refinement: r = f - (x - h J x) in FP64 from the
//          network itself at the substep's own state, x += M r, until the
//          predicted error is below 2^-33 |x|.  A refinement that stalls is
//          restarted with a fresh inverse of the substep's own matrix; if that
//          one does not refine either (I - hJ too ill-conditioned for FP32),
//          the substep is solved by the plain FP64 LU, the system is flagged
//          WIND_SYS_REFINE_FALLBACK, and its substeps of that size and larger
//          go straight to the FP64 LU from then on.
// The step sizes, substep sequence, error test and accept/reject decisions
// are the reference controller's (cuda/common/kernel.cu:191-296 DEVICE,
// cuda/c_baseline/common/common_gold.c:48-153 GOLD); only the linear solve
// differs.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "team_kernel.cuh"

namespace wind {

constexpr int WARP_THREADS = 128;
constexpr int WARP_MIX_MAXIT = 8;     // refinement sweeps with a reused inverse
constexpr int WARP_MIX_MAXIT2 = 24;   // ... and with a fresh one

// Row pitch (elements) of the per-lane scatter rows: a multiple of 16 bytes,
// 16 bytes off a multiple of 128 so a quarter warp's 16-byte accesses to
// their own rows fall in distinct bank groups.
template <int NMAX, typename T>
__host__ __device__ constexpr int warp_ldr() {
    return sizeof(T) == 8 ? NMAX + 2 : NMAX + 4;
}

struct WarpLayout {
    // byte offsets inside one team's slice
    int rates, species, inc_off, inc, lt, vb, xb, qf, piv, rows, pb, sv, bytes;
    __host__ __device__ static int align16(int x) { return (x + 15) & ~15; }
    __host__ __device__ WarpLayout(int nmax, int R, bool lin, int solver) {
        const int esz = (solver == WIND_SOLVER_MIXED) ? 4 : 8;
        const int ldr = (esz == 8) ? nmax + 2 : nmax + 4;
        int off = 0;
        rates = off; off = align16(off + R * 8);
        species = off; off = align16(off + R * 8);
        inc_off = off; off = align16(off + (nmax + 1) * 4);
        inc = off; off = align16(off + 4 * R * 2);
        lt = off; off = align16(off + (lin ? nmax * nmax * 4 : 0));
        vb = off; off = align16(off + nmax * 8);   // broadcast state (FP64)
        xb = off; off = align16(off + nmax * 8);   // broadcast solution (FP64)
        qf = off; off = align16(off + nmax * 8);   // permuted right-hand side
        piv = off; off = align16(off + nmax * 4);  // lane of each pivot step
        rows = off; off = align16(off + nmax * ldr * esz);   // Jacobian scatter rows
        pb = off; off = align16(off + 2 * (nmax + 4) * 8);  // pivot-row buffers (FP64-sized:
                                                             // MIXED's FP64 fallback uses them)
        // MIXED: the attempt's half-step inverse, kept for the next full step
        sv = off; off = align16(off + (esz == 4 ? nmax * ldr * 4 : 0));
        bytes = off;
    }
};

template <int NMAX, typename T>
struct WarpCtx {
    unsigned mask;
    int l, leader, N, R;
    const double* rates;
    const uint16_t* sp;
    const int* inc_off;
    const uint16_t* inc;
    const float* LT;   // LT[k*NMAX + l] = L[l][k], or null
    double* vb;
    double* xb;
    T* qf;
    int* piv;
    T* rows;
    T* pb;
    float* sv;
};

template <int NMAX, typename T>
__device__ __forceinline__ double team_max_abs(const WarpCtx<NMAX, T>& c, double a) {
    const unsigned m = __reduce_max_sync(c.mask, fmax_bits(a));
    return (double)__uint_as_float(m);
}

// Species multiplicity of equation l in reaction (a, b -> cc, d).
__device__ __forceinline__ int stoich(int l, int a, int b, int cc, int d) {
    return (cc == l) + (d == l) - (a == l) - (b == l);
}

// sum_k L[l][k] w[k] for the dense term (w in shared memory, FP64), four
// independent accumulators over a compile-time column loop.
template <int NMAX>
__device__ __forceinline__ double warp_dense_dot(const float* LT, const double* w, int l, int N) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
    for (int k = 0; k < NMAX; k += 4) {
        if (k < N) {
            const double2 w01 = *reinterpret_cast<const double2*>(w + k);
            const double2 w23 = *reinterpret_cast<const double2*>(w + k + 2);
            s0 = fma((double)LT[k * NMAX + l], w01.x, s0);
            if (k + 1 < N) s1 = fma((double)LT[(k + 1) * NMAX + l], w01.y, s1);
            if (k + 2 < N) s2 = fma((double)LT[(k + 2) * NMAX + l], w23.x, s2);
            if (k + 3 < N) s3 = fma((double)LT[(k + 3) * NMAX + l], w23.y, s3);
        }
    }
    return (s0 + s1) + (s2 + s3);
}

// f_l at the state in vb: dense term L v plus the incident reactions.
template <int NMAX, typename T>
__device__ __forceinline__ double warp_rhs(const WarpCtx<NMAX, T>& c) {
    const int l = c.l;
    double acc = 0.0, acc2 = 0.0;
    if (l < c.N) {
        if (c.LT) acc = warp_dense_dot<NMAX>(c.LT, c.vb, l, c.N);
        const int e0 = c.inc_off[l], e1 = c.inc_off[l + 1];
        for (int e = e0; e < e1; e++) {
            const int rr = c.inc[e];
            const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
            const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
            const int s = stoich(l, a, b, cc, d);
            const double w = (double)s * c.rates[rr] * c.vb[a] * c.vb[b];
            if ((e - e0) & 1) acc2 += w; else acc += w;
        }
    }
    return acc + acc2;
}

// (J x)_l at the state in vb for the vector in xb, in FP64.
template <int NMAX, typename T>
__device__ __forceinline__ double warp_jx(const WarpCtx<NMAX, T>& c) {
    const int l = c.l;
    double acc = 0.0, acc2 = 0.0;
    if (l < c.N) {
        if (c.LT) acc = warp_dense_dot<NMAX>(c.LT, c.xb, l, c.N);
        const int e0 = c.inc_off[l], e1 = c.inc_off[l + 1];
        for (int e = e0; e < e1; e++) {
            const int rr = c.inc[e];
            const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
            const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
            const int s = stoich(l, a, b, cc, d);
            const double w = (double)s * c.rates[rr] * fma(c.vb[b], c.xb[a], c.vb[a] * c.xb[b]);
            if ((e - e0) & 1) acc2 += w; else acc += w;
        }
    }
    return acc + acc2;
}

// Mass-action Jacobian row l at the state in vb, scattered into this lane's
// scatter row (only the lane itself touches its row, so no team barrier).
template <int NMAX, typename T>
__device__ __forceinline__ void warp_jma_row(const WarpCtx<NMAX, T>& c) {
    constexpr int ldr = warp_ldr<NMAX, T>();
    constexpr int V = 16 / sizeof(T);
    using Vt = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
    const int l = c.l;
    if (l >= c.N) return;
    T* row = c.rows + l * ldr;
    const Vt z = {};
#pragma unroll
    for (int t = 0; t < NMAX; t += V) *reinterpret_cast<Vt*>(row + t) = z;
    const int e1 = c.inc_off[l + 1];
    for (int e = c.inc_off[l]; e < e1; e++) {
        const int rr = c.inc[e];
        const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
        const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
        const int s = stoich(l, a, b, cc, d);
        if (s == 0) continue;
        const double ks = (double)s * c.rates[rr];
        row[a] = (T)((double)row[a] + ks * c.vb[b]);
        row[b] = (T)((double)row[b] + ks * c.vb[a]);
    }
}

// a[] = row l of I - h J, from the dense term and the scatter row.
template <int NMAX, typename T>
__device__ __forceinline__ void warp_load_matrix(const WarpCtx<NMAX, T>& c, double h, T (&a)[NMAX]) {
    constexpr int ldr = warp_ldr<NMAX, T>();
    constexpr int V = 16 / sizeof(T);
    using Vt = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
    const int l = c.l;
    if (l >= c.N) {
#pragma unroll
        for (int t = 0; t < NMAX; t++) a[t] = (T)0;
        return;
    }
    const T* row = c.rows + l * ldr;
    const T mh = (T)(-h);
#pragma unroll
    for (int t0 = 0; t0 < NMAX; t0 += V) {
        const Vt w = *reinterpret_cast<const Vt*>(row + t0);
        const T* wv = reinterpret_cast<const T*>(&w);
#pragma unroll
        for (int q = 0; q < V; q++) {
            const int t = t0 + q;
            T j = wv[q];
            if (c.LT && t < c.N) j += (T)c.LT[t * NMAX + l];
            a[t] = (t == l) ? (T)fma(-h, (double)j, 1.0) : mh * j;
        }
    }
}

// ---- plain FP64 LU --------------------------------------------------------
// Factor a[] (row l of A, in registers) with partial pivoting and solve for
// the right-hand side b (this lane's component).  Returns x_l.
template <int NMAX>
__device__ __forceinline__ double warp_lu_solve(const WarpCtx<NMAX, double>& c, double (&a)[NMAX],
                                                double b) {
    const int l = c.l, N = c.N;
    int mystep = (l < N) ? NMAX : -1;
    double myrcp = 0.0;  // 1 / U_kk of this lane's pivot step
#pragma unroll
    for (int k = 0; k < NMAX; k++) {
        if (k < N) {
            const unsigned key = pivot_key(a[k], l, mystep == NMAX);
            const int p = 31 - (int)(__reduce_max_sync(c.mask, key) & 31u);
            double* buf = c.pb + (k & 1) * (NMAX + 4);
            if (l == p) {
                // the reciprocal of the pivot (off the other lanes' path),
                // columns k..NMAX-1 of the pivot row, its right-hand side
                myrcp = nr_rcp(a[k]);
                buf[NMAX + 1] = myrcp;
#pragma unroll
                for (int t = k & ~1; t < NMAX; t += 2)
                    *reinterpret_cast<double2*>(buf + t) = make_double2(a[t], a[t + 1]);
                buf[NMAX] = b;
                c.piv[k] = l;
                mystep = k;
            }
            __syncwarp(c.mask);
            if (mystep == NMAX) {
                const double m = a[k] * buf[NMAX + 1];
#pragma unroll
                for (int t = (k + 1) & ~1; t < NMAX; t += 2) {
                    const double2 w = *reinterpret_cast<const double2*>(buf + t);
                    if (t > k) a[t] = fma(-m, w.x, a[t]);
                    a[t + 1] = fma(-m, w.y, a[t + 1]);
                }
                b = fma(-m, buf[NMAX], b);
            }
        }
    }
    __syncwarp(c.mask);
    // back substitution by columns: x_i from the lane that pivoted at step i
    double z = b, xl = 0.0;
#pragma unroll
    for (int i = NMAX - 1; i >= 0; i--) {
        if (i < N) {
            const int p = c.piv[i];
            double xi = (l == p) ? z * myrcp : 0.0;
            xi = __shfl_sync(c.mask, xi, c.leader + p);
            if (mystep >= 0 && mystep < i) z = fma(-a[i], xi, z);
            if (l == i) xl = xi;
        }
    }
    return xl;
}

// I - hJ from the scatter rows, solved by the FP64 LU, as one out-of-line
// body: the three solves of an attempt share its instructions (inlined, each
// was its own copy of the unrolled elimination, and the kernel stalled on
// instruction fetch).
// The context's fields travel as scalars, so the call passes them in
// registers instead of through a stack copy of the whole context.
template <int NMAX>
__device__ __noinline__ double warp_lu_solve_at(unsigned mask, int l, int leader, int N,
                                                const float* LT, double* rows, double* pb, int* piv,
                                                double h, double b) {
    WarpCtx<NMAX, double> c;
    c.mask = mask;
    c.l = l;
    c.leader = leader;
    c.N = N;
    c.LT = LT;
    c.rows = rows;
    c.pb = pb;
    c.piv = piv;
    double a[NMAX];
    warp_load_matrix(c, h, a);
    return warp_lu_solve(c, a, b);
}
template <int NMAX>
__device__ __forceinline__ double warp_lu_solve_at(const WarpCtx<NMAX, double>& c, double h, double b) {
    return warp_lu_solve_at<NMAX>(c.mask, c.l, c.leader, c.N, c.LT, c.rows, c.pb, c.piv, h, b);
}

// ---- FP32 Gauss-Jordan inverse --------------------------------------------
// In-place inversion of A (row l in a[]) with partial pivoting and no row
// exchanges: after step k the pivot lane's row expresses unknown k.  The
// result M satisfies x_k = sum_j M[p_k][j] b_{p_j}, where p_j is the lane
// that pivoted at step j; returns this lane's step (-1 for l >= N).
template <int NMAX>
__device__ __forceinline__ int warp_gj_invert(const WarpCtx<NMAX, float>& c, float (&a)[NMAX]) {
    const int l = c.l, N = c.N;
    int mystep = (l < N) ? NMAX : -1;
#pragma unroll
    for (int k = 0; k < NMAX; k++) {
        if (k < N) {
            const unsigned key = pivot_key((double)a[k], l, mystep == NMAX);
            const int p = 31 - (int)(__reduce_max_sync(c.mask, key) & 31u);
            float* buf = c.pb + (k & 1) * (NMAX + 4);
            if (l == p) {
                buf[NMAX] = nr_rcp(a[k]);  // the pivot's reciprocal, off the others' path
#pragma unroll
                for (int t = 0; t < NMAX; t += 4)
                    *reinterpret_cast<float4*>(buf + t) = make_float4(a[t], a[t + 1], a[t + 2], a[t + 3]);
                mystep = k;
            }
            __syncwarp(c.mask);
            if (l < N) {
                const float r = buf[NMAX];
                // pivot row: a <- r a (as (r-1) a + a); others: a <- a - (a_k r) pivot
                const float alpha = (l == p) ? r - 1.0f : -a[k] * r;
#pragma unroll
                for (int t0 = 0; t0 < NMAX; t0 += 4) {
                    const float4 w = *reinterpret_cast<const float4*>(buf + t0);
                    const float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        if (t0 + q != k) a[t0 + q] = fmaf(alpha, wv[q], a[t0 + q]);
                }
                a[k] = (l == p) ? r : alpha;
            }
        }
    }
    __syncwarp(c.mask);
    return mystep;
}

// Permuted product with the inverse rows in a[] (owner convention of
// warp_gj_invert): b is this lane's component in natural order; the result
// is component mystep of M b.  One team barrier.
template <int NMAX>
__device__ __forceinline__ double warp_inv_apply(const WarpCtx<NMAX, float>& c, const float (&a)[NMAX],
                                                 int mystep, double b) {
    if (mystep >= 0) c.qf[mystep] = (float)b;
    __syncwarp(c.mask);
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
    for (int t = 0; t < NMAX; t += 4) {
        const float4 w = *reinterpret_cast<const float4*>(c.qf + t);
        s0 = fmaf(a[t], w.x, s0);
        s1 = fmaf(a[t + 1], w.y, s1);
        s2 = fmaf(a[t + 2], w.z, s2);
        s3 = fmaf(a[t + 3], w.w, s3);
    }
    return (mystep >= 0) ? (double)((s0 + s1) + (s2 + s3)) : 0.0;
}

// Outcome of a refinement.
enum { REFINE_OK = 0, REFINE_GAVE_UP = 1 };

// Solve (I - h J(v)) x = f (v in vb) by FP64 iterative refinement around the
// approximate inverse in a[]: x = M f, then r = f - (x - h J x), x += M r.
// Lane l carries the component x_{mystep(l)} of the iterate; the full x is
// broadcast in xb (natural order) for the product J x.  Stops when the
// predicted error -- the last correction times the observed contraction
// (|d|/|x| for the first sweep) -- is below 2^-33 max|x|; gives up when a
// sweep contracts by less than `abort0` (first sweep) or 1/2 (later ones),
// or after `maxit` sweeps.  On return x_l (natural order) is in `x`.
template <int NMAX>
__device__ __forceinline__ int warp_refine(const WarpCtx<NMAX, float>& c, const float (&a)[NMAX],
                                           int mystep, double h, double f, double& x, int maxit,
                                           double abort0) {
    const int l = c.l;
    double xt = warp_inv_apply(c, a, mystep, f);
    const double xmax = team_max_abs(c, xt);
    double dprev = 0.0;
    int outcome = REFINE_GAVE_UP;
    for (int it = 0; it < maxit; it++) {
        if (mystep >= 0) c.xb[mystep] = xt;
        __syncwarp(c.mask);
        const double jx = warp_jx(c);
        const double r = (l < c.N) ? f - fma(-h, jx, c.xb[l]) : 0.0;
        const double d = warp_inv_apply(c, a, mystep, r);
        xt += d;
        const double dmax = team_max_abs(c, d);
        const double rho = (it == 0) ? dmax / fmax(xmax, 1e-300) : dmax / fmax(dprev, 1e-300);
        if (dmax * rho <= 0x1p-33 * xmax || dmax == 0.0) { outcome = REFINE_OK; break; }
        if (rho > (it == 0 ? abort0 : 0.5)) break;
        dprev = dmax;
    }
    if (mystep >= 0) c.xb[mystep] = xt;
    __syncwarp(c.mask);
    x = (l < c.N) ? c.xb[l] : 0.0;
    return outcome;
}

// Copy the inverse rows and their step order to / from the save area.
template <int NMAX>
__device__ __forceinline__ void warp_save_inverse(const WarpCtx<NMAX, float>& c, const float (&a)[NMAX]) {
    float* row = c.sv + c.l * warp_ldr<NMAX, float>();
#pragma unroll
    for (int t = 0; t < NMAX; t += 4)
        *reinterpret_cast<float4*>(row + t) = make_float4(a[t], a[t + 1], a[t + 2], a[t + 3]);
}
template <int NMAX>
__device__ __forceinline__ void warp_load_inverse(const WarpCtx<NMAX, float>& c, float (&a)[NMAX]) {
    const float* row = c.sv + c.l * warp_ldr<NMAX, float>();
#pragma unroll
    for (int t = 0; t < NMAX; t += 4) {
        const float4 w = *reinterpret_cast<const float4*>(row + t);
        a[t] = w.x; a[t + 1] = w.y; a[t + 2] = w.z; a[t + 3] = w.w;
    }
}

// MIXED's last resort: the substep solved by the plain FP64 LU, the row of
// I - h J(v) (v in vb) built exactly in FP64 -- the dense term by a
// compile-time column loop, the reactions by compare-and-add over the
// columns (no scatter row).  Slow, and only reached when a fresh FP32
// inverse did not refine (I - hJ too ill-conditioned for FP32).
template <int NMAX>
__device__ __noinline__ double warp_fp64_fallback(const WarpCtx<NMAX, float>& cf, double h, double f) {
    WarpCtx<NMAX, double> c;
    c.mask = cf.mask; c.l = cf.l; c.leader = cf.leader; c.N = cf.N; c.R = cf.R;
    c.rates = cf.rates; c.sp = cf.sp; c.inc_off = cf.inc_off; c.inc = cf.inc; c.LT = cf.LT;
    c.vb = cf.vb; c.xb = cf.xb; c.qf = reinterpret_cast<double*>(cf.qf); c.piv = cf.piv;
    c.rows = nullptr; c.pb = reinterpret_cast<double*>(cf.pb); c.sv = cf.sv;
    const int l = c.l, N = c.N;
    double a[NMAX];
#pragma unroll
    for (int t = 0; t < NMAX; t++) {
        const double lt = (c.LT && t < N && l < N) ? (double)c.LT[t * NMAX + l] : 0.0;
        a[t] = (l < N && t < N) ? ((t == l ? 1.0 : 0.0) - h * lt) : 0.0;
    }
    if (l < N) {
        const int e1 = c.inc_off[l + 1];
        for (int e = c.inc_off[l]; e < e1; e++) {
            const int rr = c.inc[e];
            const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
            const int ra = q.x & 0xffff, rb = q.x >> 16, rc = q.y & 0xffff, rd = q.y >> 16;
            const int s = stoich(l, ra, rb, rc, rd);
            if (s == 0) continue;
            const double ks = -h * (double)s * c.rates[rr];
            const double ca = ks * c.vb[rb], cb = ks * c.vb[ra];
#pragma unroll
            for (int t = 0; t < NMAX; t++) {
                if (t == ra) a[t] += ca;
                if (t == rb) a[t] += cb;
            }
        }
    }
    __syncwarp(c.mask);
    const double x = warp_lu_solve(c, a, f);
    __syncwarp(c.mask);
    return x;
}

// ---------------------------------------------------------------------------
// The persistent team loop over one group's systems.
// Stage system s's network in the team's shared-memory slice: rates and
// species (a species index >= N marks the system BAD_INPUT and is replaced by
// 0 so every later access stays in bounds), the per-species incidence lists,
// and the dense term transposed.  Returns true for BAD_INPUT.
template <int NMAX, typename T>
__device__ __forceinline__ bool warp_stage_system(const WarpCtx<NMAX, T>& c, const KParams& p,
                                                  int64_t s, double* rates_s, uint16_t* sp_s,
                                                  int* inc_off, uint16_t* inc, float* LT) {
    const int N = c.N, R = c.R, l = c.l;
    const bool lin = LT != nullptr;
    // stage the system's network; a species index >= N marks the system
    // BAD_INPUT and is replaced by 0 so every later access stays in bounds
    bool bad_idx = false;
    for (int r = l; r < R; r += NMAX) {
        rates_s[r] = p.rates[s * R + r];
        uint2 q = *reinterpret_cast<const uint2*>(p.species + (s * R + r) * 4);
        const unsigned nn = (unsigned)N;
        if ((q.x & 0xffffu) >= nn || (q.x >> 16) >= nn || (q.y & 0xffffu) >= nn || (q.y >> 16) >= nn) {
            bad_idx = true;
            q = make_uint2(0u, 0u);
        }
        *reinterpret_cast<uint2*>(sp_s + 4 * r) = q;
    }
    bad_idx = __any_sync(c.mask, bad_idx);
    __syncwarp(c.mask);
    // per-species incidence lists (reaction ids ascending)
    if (l < N) {
        int cnt = 0;
        for (int r = 0; r < R; r++) {
            const uint2 q = *reinterpret_cast<const uint2*>(sp_s + 4 * r);
            cnt += ((q.x & 0xffff) == (unsigned)l) | ((q.x >> 16) == (unsigned)l) |
                   ((q.y & 0xffff) == (unsigned)l) | ((q.y >> 16) == (unsigned)l);
        }
        inc_off[l + 1] = cnt;
    }
    __syncwarp(c.mask);
    if (l == 0) {
        inc_off[0] = 0;
        for (int j = 0; j < N; j++) inc_off[j + 1] += inc_off[j];
    }
    __syncwarp(c.mask);
    if (l < N) {
        int o = inc_off[l];
        for (int r = 0; r < R; r++) {
            const uint2 q = *reinterpret_cast<const uint2*>(sp_s + 4 * r);
            if ((q.x & 0xffff) == (unsigned)l || (q.x >> 16) == (unsigned)l ||
                (q.y & 0xffff) == (unsigned)l || (q.y >> 16) == (unsigned)l)
                inc[o++] = (uint16_t)r;
        }
    }
    if (lin && l < N) {
        const float* Lg = p.linear + s * (int64_t)N * N;
        for (int k = 0; k < N; k++) LT[k * NMAX + l] = Lg[l * N + k];
    }
    return bad_idx;
}

template <int NMAX, int CTRL, int SOLVER>
__device__ __forceinline__ void warp_run(const KParams& p, unsigned char* smem_raw) {
    using T = typename std::conditional<SOLVER == WIND_SOLVER_MIXED, float, double>::type;
    constexpr int CAP = Cap<WIND_METHOD_SIE, CTRL>::value;
    const bool lin = p.linear != nullptr;
    const WarpLayout lay(NMAX, p.n_react, lin, SOLVER);
    const int team = threadIdx.x / NMAX;
    const int lane = threadIdx.x & 31;
    WarpCtx<NMAX, T> c;
    c.l = threadIdx.x % NMAX;
    c.leader = lane - c.l;
    c.mask = (NMAX >= 32) ? 0xffffffffu : (((1u << NMAX) - 1u) << c.leader);
    c.N = p.n_eq;
    c.R = p.n_react;
    unsigned char* base = smem_raw + team * lay.bytes;
    double* rates_s = reinterpret_cast<double*>(base + lay.rates);
    uint16_t* sp_s = reinterpret_cast<uint16_t*>(base + lay.species);
    int* inc_off = reinterpret_cast<int*>(base + lay.inc_off);
    uint16_t* inc = reinterpret_cast<uint16_t*>(base + lay.inc);
    float* LT = lin ? reinterpret_cast<float*>(base + lay.lt) : nullptr;
    c.rates = rates_s;
    c.sp = sp_s;
    c.inc_off = inc_off;
    c.inc = inc;
    c.LT = LT;
    c.vb = reinterpret_cast<double*>(base + lay.vb);
    c.xb = reinterpret_cast<double*>(base + lay.xb);
    c.qf = reinterpret_cast<T*>(base + lay.qf);
    c.piv = reinterpret_cast<int*>(base + lay.piv);
    c.rows = reinterpret_cast<T*>(base + lay.rows);
    c.pb = reinterpret_cast<T*>(base + lay.pb);
    c.sv = reinterpret_cast<float*>(base + lay.sv);
    const int N = c.N, R = c.R, l = c.l;
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;

    while (true) {
        unsigned long long ticket = 0;
        if (l == 0) ticket = atomicAdd(&p.counters[CNT_QUEUE], 1ull);
        ticket = __shfl_sync(c.mask, ticket, c.leader);
        const int64_t s = (int64_t)ticket;
        if (s >= p.nsys) break;

        const bool bad_idx = warp_stage_system(c, p, s, rates_s, sp_s, inc_off, inc, LT);
        // padding of the permuted right-hand side stays zero
        c.qf[l] = (T)0;
        double y = (l < N) ? p.y[s * N + l] : 0.0;
        __syncwarp(c.mask);

        double tnow = p.tnow;
        const double tend = p.tend;
        double h = p.h0;
        int unsolved = 0;
        int64_t attempts = 0;
        int32_t st = bad_idx ? WIND_SYS_BAD_INPUT : WIND_SYS_OK;
        double fy = 0.0;          // f(y), valid while y is unchanged
        bool fy_ok = false, jy_ok = false;  // scatter rows hold J_ma(y)
        T a[NMAX];
        int mystep = -1, svstep = -1;
        bool inv_ok = false;      // MIXED: the save area inverts I - h' J(y), h' the next full step
        // MIXED: substeps of this size and larger go straight to the FP64 LU
        // (a fresh FP32 inverse failed to refine at this size: I - hJ is too
        // ill-conditioned for FP32 factors, and grows more so with h)
        double h_fp64 = INFINITY;
        // A fresh solve of the substep's own matrix (scatter rows of the
        // state in vb): FP32 inverse and FP64 refinement, or the FP64 LU.
        auto mixed_fresh = [&](double hh, double ff, bool save) -> double {
            double xx = 0.0;
            if constexpr (SOLVER == WIND_SOLVER_MIXED) {
                if (hh < h_fp64) {
                    warp_load_matrix(c, hh, a);
                    mystep = warp_gj_invert(c, a);
                    if (warp_refine(c, a, mystep, hh, ff, xx, WARP_MIX_MAXIT2, 0.25) == REFINE_OK) {
                        if (save) {
                            warp_save_inverse(c, a);
                            svstep = mystep;
                            inv_ok = true;
                        }
                        return xx;
                    }
                    h_fp64 = hh;
                }
                st |= WIND_SYS_REFINE_FALLBACK;
                xx = warp_fp64_fallback(c, hh, ff);
            }
            return xx;
        };
        while (!bad_idx && tnow < tend) {
            if (attempts >= p.max_attempts) { st |= WIND_SYS_MAX_ATTEMPTS; break; }
            if (p.timeout_ns) {
                const int late = global_ns() - t_start > p.timeout_ns;
                if (__shfl_sync(c.mask, late, c.leader)) { st |= WIND_SYS_TIMEOUT; break; }
            }
            attempts++;
            h = fmin(tend - tnow, h);
            const double t1 = tnow + h;
            const double hf = t1 - tnow;            // the full substep
            const double h1 = (t1 - tnow) * 0.5;    // the first half substep
            const double h2 = (CTRL == WIND_CTRL_DEVICE) ? fmin(t1 - (tnow + h1), h1) : h1;

            // ---- full step and first half step, both from y
            __syncwarp(c.mask);
            if (l < N) c.vb[l] = y;
            __syncwarp(c.mask);
            if (!fy_ok) { fy = warp_rhs(c); fy_ok = true; }
            if (!jy_ok) { warp_jma_row(c); jy_ok = true; }
            double y1, vh;
            if constexpr (SOLVER == WIND_SOLVER_MIXED) {
                double x;
                // full step: the previous attempt's half-step inverse is
                // the inverse of this matrix (same state, same size) when y
                // is unchanged; else a fresh one
                if (hf < h_fp64 && inv_ok) {
                    warp_load_inverse(c, a);
                    mystep = svstep;
                    if (warp_refine(c, a, mystep, hf, fy, x, WARP_MIX_MAXIT, 0.5) != REFINE_OK)
                        x = mixed_fresh(hf, fy, false);
                } else {
                    x = mixed_fresh(hf, fy, false);
                }
                y1 = y + hf * x;
                // first half step: a fresh inverse, saved for the next attempt
                inv_ok = false;
                x = mixed_fresh(h1, fy, true);
                vh = y + h1 * x;
            } else {
                y1 = y + hf * warp_lu_solve_at(c, hf, fy);
                __syncwarp(c.mask);
                vh = y + h1 * warp_lu_solve_at(c, h1, fy);
            }
            // ---- second half step from vh
            __syncwarp(c.mask);
            if (l < N) c.vb[l] = vh;
            __syncwarp(c.mask);
            const double f2 = warp_rhs(c);
            double y2;
            if constexpr (SOLVER == WIND_SOLVER_MIXED) {
                double x;
                // the half-step inverse again, if it still contracts well at
                // vh (small steps); else an inverse of this substep's own
                // matrix (the scatter rows then hold J(vh), not J(y))
                if (!inv_ok || h2 >= h_fp64 ||
                    warp_refine(c, a, mystep, h2, f2, x, WARP_MIX_MAXIT, 0.0625) != REFINE_OK) {
                    warp_jma_row(c);
                    jy_ok = false;
                    x = mixed_fresh(h2, f2, false);
                }
                y2 = vh + h2 * x;
            } else {
                warp_jma_row(c);
                jy_ok = false;
                __syncwarp(c.mask);
                y2 = vh + h2 * warp_lu_solve_at(c, h2, f2);
            }
            bool err = false;
            if (l < N) err = elem_error<WIND_METHOD_SIE, CTRL>(xd(y1), xd(y2), p.atol, p.rtol);
            err = __any_sync(c.mask, err);
            if (err && unsolved < CAP) {
                unsolved++;
                h /= 2.0;
                // y unchanged: f(y) stays valid; the scatter rows hold J_ma(y)
                // unless the second half step rebuilt them
            } else {
                unsolved = 0;
                y = y2;
                fy_ok = jy_ok = inv_ok = false;
                if (tnow + h == tnow) { st |= WIND_SYS_STALLED; break; }
                tnow += h;
                h = tend - tnow;
            }
        }
        __syncwarp(c.mask);
        const bool bad = (l < N) && !finite64(y);
        if (__any_sync(c.mask, bad)) st |= WIND_SYS_NONFINITE;
        if (l < N) p.y[s * N + l] = y;
        if (l == 0) {
            if (p.sys_status) p.sys_status[s] = st;
            if (p.sys_nsteps) p.sys_nsteps[s] = 3 * attempts;
            atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)(3 * attempts));
        }
        __syncwarp(c.mask);
    }
}

template <int NMAX, int CTRL, int SOLVER>
__global__ void __launch_bounds__(WARP_THREADS, 4) k_warp(const KParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    warp_run<NMAX, CTRL, SOLVER>(p, smem_raw);
}

}  // namespace wind
