// team_kernel.cuh -- persistent team-per-system integrator for runtime
// mass-action networks with N <= 32 (optionally with a dense linear term).
//
// A team is NMAX lanes of one warp (NMAX = 8, 16 or 32); a CTA of 128 threads
// holds 128/NMAX teams, each with its own shared-memory slice.  Lane l:
//  * evaluates RHS component f_l and Jacobian column l (d f_l / d y_*) by
//    scanning the system's reactions, scattering into the shared Jacobian;
//  * owns row l of the matrix being eliminated, in registers, so the
//    elimination reads only its own registers plus one broadcast pivot row
//    from shared memory per step;
//  * for pivoted LU, the pivot search over the team is one warp reduction
//    (__reduce_max_sync on a packed |a_kl|/lane key); rows are not moved --
//    a lane retires when its row becomes the pivot row.
// Solvers:
//  GJE_F64  the reference's unpivoted Gauss-Jordan inverse (row scaling by
//           division, full-width row updates, U then L phase) and its
//           transposed matvec -- bit-exact with the reference's FP64 build;
//  LU_F64   partial-pivot LU in FP64 (fma);
//  MIXED    partial-pivot LU with FP32 factors, FP64 residual from the FP64
//           Jacobian kept in shared memory, one refinement step.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "networks.cuh"

namespace wind {

constexpr int TEAM_THREADS = 128;
constexpr int TEAM_MAXN = 32;

struct TeamLayout {
    // byte offsets inside one team's shared slice.  GJE_F64 keeps the FP64
    // Jacobian Js (reference orientation) and the broadcast rows; LU_F64 and
    // MIXED keep the matrix A = I - hJ row-major with the right-hand side as
    // column N (leading dimension NMAX+1: odd, so the lanes' rows fall in
    // distinct banks), the per-species reaction incidence lists and the pivot
    // order.
    int js, bc, vec, lt, rates, species, mat, inc_off, inc, piv, bytes;
    __host__ __device__ static int align16(int x) { return (x + 15) & ~15; }
    __host__ __device__ TeamLayout(int nmax, int R, bool lin, int solver = WIND_SOLVER_GJE_F64) {
        const bool gje = (solver == WIND_SOLVER_GJE_F64);
        const int esz = (solver == WIND_SOLVER_MIXED) ? 4 : 8;
        int off = 0;
        js = off; off = align16(off + (gje ? nmax * nmax * 8 : 0));
        bc = off; off = align16(off + (gje ? 2 * (2 * nmax + 4) * 8 : 0));
        vec = off; off = align16(off + 10 * nmax * 8);
        lt = off; off = align16(off + (lin ? nmax * nmax * 4 : 0));
        rates = off; off = align16(off + R * 8);
        species = off; off = align16(off + R * 4 * 2);
        mat = off; off = align16(off + (gje ? 0 : nmax * (nmax + (esz == 8 ? 2 : 4)) * esz));
        inc_off = off; off = align16(off + (gje ? 0 : (nmax + 1) * 4));
        inc = off; off = align16(off + (gje ? 0 : 4 * R * 2));
        piv = off; off = align16(off + (gje ? 0 : nmax * 4));
        bytes = off;
    }
};

// Team-local synchronisation: teams never span warps here.
__device__ __forceinline__ void team_sync(unsigned mask) { __syncwarp(mask); }

template <int NMAX>
struct TeamCtx {
    unsigned mask;
    int l;          // lane within team
    int leader;     // warp lane of the team's lane 0
    int N, R;
    double* Js;     // [NMAX*NMAX] row-major, Js[i*NMAX + j] = d f_j / d y_i
    double* bc;     // [2][2*NMAX+4] pivot-row broadcast buffers
    double* v;      // [NMAX] state being stepped
    double* f;      // [NMAX] RHS
    double* y;      // [NMAX] accepted state
    double* y1;     // [NMAX]
    double* y2;     // [NMAX]
    double* x;      // [NMAX] solve workspace
    float* LT;      // [NMAX*NMAX] LT[i*NMAX+j] = L[j][i], or null
    double* rates;  // [R]
    const uint16_t* sp;  // [R*4]
    void* A;        // [NMAX*(NMAX+1)] LU/MIXED matrix (double or float)
    int* inc_off;   // [NMAX+1] CSR offsets
    uint16_t* inc;  // CSR reaction ids
    int* piv;       // [NMAX] lane chosen at pivot step i
    double* r;      // [NMAX] refinement residual
};

// f_l and column l of Jt for the current v (mass action + optional L).
template <int NMAX, bool JAC>
__device__ __forceinline__ void team_rhs_jac(const TeamCtx<NMAX>& c) {
    const int l = c.l;
    if (l < c.N) {
        xd acc = 0.0;
        if (c.LT) {
            for (int k = 0; k < c.N; k++) acc += xd((double)c.LT[k * NMAX + l]) * xd(c.v[k]);
            if (JAC)
                for (int i = 0; i < c.N; i++) c.Js[i * NMAX + l] = (double)c.LT[i * NMAX + l];
        } else if (JAC) {
            for (int i = 0; i < c.N; i++) c.Js[i * NMAX + l] = 0.0;
        }
        for (int r = 0; r < c.R; r++) {
            const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * r);
            const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
            if (a != l && b != l && cc != l && d != l) continue;
            const xd k = c.rates[r];
            const xd ya = c.v[a], yb = c.v[b];
            const xd w = k * ya * yb;
            if (a == l) acc -= w;
            if (b == l) acc -= w;
            if (cc == l) acc += w;
            if (d == l) acc += w;
            if (JAC) {
                const xd da = k * yb, db = k * ya;
                double* ra = c.Js + a * NMAX + l;
                double* rb = c.Js + b * NMAX + l;
                if (a == l) *ra = xd(*ra) - da;
                if (b == l) *ra = xd(*ra) - da;
                if (cc == l) *ra = xd(*ra) + da;
                if (d == l) *ra = xd(*ra) + da;
                if (a == l) *rb = xd(*rb) - db;
                if (b == l) *rb = xd(*rb) - db;
                if (cc == l) *rb = xd(*rb) + db;
                if (d == l) *rb = xd(*rb) + db;
            }
        }
        c.f[l] = acc.v;
    }
    team_sync(c.mask);
}

// Exact Gauss-Jordan (reference order) on rows held one per lane.
template <int NMAX, int CTRL>
__device__ __forceinline__ void team_gje_exact(const TeamCtx<NMAX>& c, double h) {
    const int l = c.l, N = c.N;
    xd Mr[NMAX], Ir[NMAX];
#pragma unroll
    for (int t = 0; t < NMAX; t++) {
        const double j = (l < N && t < N) ? c.Js[l * NMAX + t] : 0.0;
        if (CTRL == WIND_CTRL_GOLD) {
            xd m = -xd(h) * xd(j);
            if (t == l) m += 1.0;
            Mr[t] = m;
        } else {
            Mr[t] = xd(t == l ? 1.0 : 0.0) - xd(j) * xd(h);
        }
        Ir[t] = (t == l) ? 1.0 : 0.0;
    }
    // gjeUFactor (gje_gold.c:56-100)
#pragma unroll
    for (int i = 0; i < NMAX; i++) {
        if (i < N) {
            double* buf = c.bc + (i & 1) * (2 * NMAX + 4);
            if (l == i) {
                const xd s = Mr[i];
#pragma unroll
                for (int t = 0; t < NMAX; t++) { Mr[t] /= s; Ir[t] /= s; }
#pragma unroll
                for (int t = 0; t < NMAX; t++) { buf[t] = Mr[t].v; buf[NMAX + t] = Ir[t].v; }
            }
            team_sync(c.mask);
            if (l > i && l < N) {
                const xd fct = Mr[i];
#pragma unroll
                for (int t = 0; t < NMAX; t++) {
                    Mr[t] -= fct * xd(buf[t]);
                    Ir[t] -= fct * xd(buf[NMAX + t]);
                }
            }
        }
    }
    // gjeLFactor (gje_gold.c:102-134): pivot rows bottom-up
#pragma unroll
    for (int b = NMAX - 1; b >= 0; b--) {
        if (b < N) {
            // parity (b+1)&1 alternates with the U phase's last buffer
            double* buf = c.bc + ((b + 1) & 1) * (2 * NMAX + 4);
            if (l == b) {
#pragma unroll
                for (int t = 0; t < NMAX; t++) { buf[t] = Mr[t].v; buf[NMAX + t] = Ir[t].v; }
            }
            team_sync(c.mask);
            if (l < b) {
                const xd fct = Mr[b];
#pragma unroll
                for (int t = 0; t < NMAX; t++) {
                    Mr[t] -= fct * xd(buf[t]);
                    Ir[t] -= fct * xd(buf[NMAX + t]);
                }
            }
        }
    }
    team_sync(c.mask);
    // Inverse rows to shared memory (Js is free now), then the matvec by
    // columns: lane r owns output r.
    if (l < N) {
#pragma unroll
        for (int t = 0; t < NMAX; t++) c.Js[l * NMAX + t] = Ir[t].v;
    }
    team_sync(c.mask);
    if (l < N) {
        if (CTRL == WIND_CTRL_GOLD) {
            // matrix_ops.c:6-27 then sie_gold.c:72-74
            xd out = 0.0;
            for (int k = 0; k < N; k++) out += xd(c.Js[k * NMAX + l]) * xd(c.f[k]);
            c.v[l] = (xd(c.v[l]) + xd(h) * out).v;
        } else {
            // kernel.cu:121-125
            xd yl = c.v[l];
            for (int k = 0; k < N; k++) yl += xd(c.Js[k * NMAX + l]) * xd(c.f[k]) * xd(h);
            c.v[l] = yl.v;
        }
    }
    team_sync(c.mask);
}

// Packed pivot key: |a| as float bits (low 5 mantissa bits replaced by the
// inverted lane index, so ties go to the lowest lane), 0 for retired lanes.
__device__ __forceinline__ unsigned pivot_key(double a, int lane_in_team, bool active) {
    if (!active) return 0u;
    const float m = fabsf((float)a);
    return (__float_as_uint(m) & ~31u) | (31u - (unsigned)lane_in_team);
}

// Row pitch of the shared LU matrix, in elements: a multiple of 16 bytes so
// rows can be read as 16-byte vectors (2 doubles / 4 floats), and 16 bytes
// more than a multiple of 128 so the 8 lanes of a quarter warp hit distinct
// bank groups.
template <int NMAX, typename T>
__host__ __device__ constexpr int team_ld() {
    return sizeof(T) == 8 ? NMAX + 2 : NMAX + 4;
}

// f_l and, with JAC, row l of A = I - hJ (standard orientation, J[l][c] =
// d f_l / d y_c) with f_l as column N, from the CSR incidence list of species
// l: the per-element update sequence is the sequential one of the
// mass-action contract (reactions ascending).
template <int NMAX, typename T, bool JAC>
__device__ __forceinline__ void team_rhs_row(const TeamCtx<NMAX>& c, double h) {
    constexpr int ld = team_ld<NMAX, T>();
    const int l = c.l, N = c.N;
    if (l < N) {
        T* row = static_cast<T*>(c.A) + l * ld;
        xd acc = 0.0;
        if (c.LT)
            for (int k = 0; k < N; k++) acc += xd((double)c.LT[k * NMAX + l]) * xd(c.v[k]);
        if (JAC)
            for (int cc = 0; cc < N; cc++) row[cc] = c.LT ? (T)c.LT[cc * NMAX + l] : (T)0;
        const int e1 = c.inc_off[l + 1];
        for (int e = c.inc_off[l]; e < e1; e++) {
            const int rr = c.inc[e];
            const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
            const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
            const xd k = c.rates[rr];
            const xd ya = c.v[a], yb = c.v[b];
            const xd w = k * ya * yb;
            if (a == l) acc -= w;
            if (b == l) acc -= w;
            if (cc == l) acc += w;
            if (d == l) acc += w;
            if (JAC) {
                const xd da = k * yb, db = k * ya;
                if (a == l) row[a] = (T)(xd((double)row[a]) - da);
                if (b == l) row[a] = (T)(xd((double)row[a]) - da);
                if (cc == l) row[a] = (T)(xd((double)row[a]) + da);
                if (d == l) row[a] = (T)(xd((double)row[a]) + da);
                if (a == l) row[b] = (T)(xd((double)row[b]) - db);
                if (b == l) row[b] = (T)(xd((double)row[b]) - db);
                if (cc == l) row[b] = (T)(xd((double)row[b]) + db);
                if (d == l) row[b] = (T)(xd((double)row[b]) + db);
            }
        }
        c.f[l] = acc.v;
        if (JAC) {
            for (int cc = 0; cc < N; cc++) row[cc] = (T)((cc == l ? 1.0 : 0.0) - h * (double)row[cc]);
            row[N] = (T)acc.v;
        }
    }
    team_sync(c.mask);
}

// (J x)_l in FP64 from the reactions and L (refinement residual).
template <int NMAX>
__device__ __forceinline__ double team_jx(const TeamCtx<NMAX>& c, const double* xv) {
    const int l = c.l, N = c.N;
    double acc = 0.0;
    if (c.LT)
        for (int k = 0; k < N; k++) acc = fma((double)c.LT[k * NMAX + l], xv[k], acc);
    const int e1 = c.inc_off[l + 1];
    for (int e = c.inc_off[l]; e < e1; e++) {
        const int rr = c.inc[e];
        const uint2 q = *reinterpret_cast<const uint2*>(c.sp + 4 * rr);
        const int a = q.x & 0xffff, b = q.x >> 16, cc = q.y & 0xffff, d = q.y >> 16;
        const double dw = c.rates[rr] * (c.v[b] * xv[a] + c.v[a] * xv[b]);
        if (a == l) acc -= dw;
        if (b == l) acc -= dw;
        if (cc == l) acc += dw;
        if (d == l) acc += dw;
    }
    return acc;
}

// Partial-pivot LU of A (shared memory, lane l owns row l, rows never move)
// and the solve of its right-hand side column N.  Step i: one warp reduction
// picks the pivot lane p, every active lane reads the pivot row straight from
// shared memory and updates its own row.  Loops stay rolled, so the code is
// small for every N.  Returns this lane's pivot step (-1 for l >= N); x in c.x.
template <int NMAX, typename T, bool STORE_L>
__device__ __forceinline__ int team_lu_smem(const TeamCtx<NMAX>& c) {
    constexpr int ld = team_ld<NMAX, T>();
    constexpr int V = 16 / sizeof(T);  // elements per 16-byte vector
    const int l = c.l, N = c.N;
    T* A = static_cast<T*>(c.A);
    T* my = A + l * ld;
    int mystep = (l < N) ? NMAX : -1;
    for (int i = 0; i < N; i++) {
        const unsigned key = pivot_key((double)my[i], l, mystep == NMAX);
        const int p = 31 - (int)(__reduce_max_sync(c.mask, key) & 31u);
        const T* prow = A + p * ld;
        if (l == p) {
            mystep = i;
            c.piv[i] = p;
        } else if (mystep == NMAX) {
            const T lk = my[i] * nr_rcp(prow[i]);
            if (STORE_L) my[i] = lk;
            // columns i+1..N in 16-byte vectors; the first vector starts at the
            // aligned column at or below i+1 and leaves columns <= i as they are
            using Vt = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
            for (int t0 = (i + 1) & ~(V - 1); t0 <= N; t0 += V) {
                Vt a = *reinterpret_cast<const Vt*>(my + t0);
                const Vt b = *reinterpret_cast<const Vt*>(prow + t0);
                T* av = reinterpret_cast<T*>(&a);
                const T* bv = reinterpret_cast<const T*>(&b);
#pragma unroll
                for (int q = 0; q < V; q++)
                    if (t0 + q > i) av[q] = fma(-lk, bv[q], av[q]);
                *reinterpret_cast<Vt*>(my + t0) = a;
            }
        }
        team_sync(c.mask);
    }
    // back substitution, column-oriented: x_i from the pivot lane of step i
    double z = (l < N) ? (double)my[N] : 0.0, xl = 0.0;
    for (int i = N - 1; i >= 0; i--) {
        const int p = c.piv[i];
        double xi = (l == p) ? z * (double)nr_rcp(my[i]) : 0.0;
        xi = __shfl_sync(c.mask, xi, c.leader + p);
        if (mystep >= 0 && mystep < i) z = fma(-(double)my[i], xi, z);
        if (l == i) xl = xi;
    }
    if (l < N) c.x[l] = xl;
    team_sync(c.mask);
    return mystep;
}

// Re-solve with the stored factors (STORE_L) for right-hand side r (this
// lane's row, original order); result in c.x.
template <int NMAX, typename T>
__device__ __forceinline__ void team_lu_resolve(const TeamCtx<NMAX>& c, int mystep, double r) {
    constexpr int ld = team_ld<NMAX, T>();
    const int l = c.l, N = c.N;
    const T* my = static_cast<const T*>(c.A) + l * ld;
    for (int i = 0; i < N; i++) {
        const double rp = __shfl_sync(c.mask, r, c.leader + c.piv[i]);
        if (mystep > i) r = fma(-(double)my[i], rp, r);
    }
    double xl = 0.0;
    for (int i = N - 1; i >= 0; i--) {
        const int p = c.piv[i];
        double xi = (l == p) ? r * (double)nr_rcp(my[i]) : 0.0;
        xi = __shfl_sync(c.mask, xi, c.leader + p);
        if (mystep >= 0 && mystep < i) r = fma(-(double)my[i], xi, r);
        if (l == i) xl = xi;
    }
    if (l < N) c.x[l] = xl;
    team_sync(c.mask);
}

template <int NMAX, int METHOD, int CTRL, int SOLVER>
__device__ __forceinline__ void team_substep(const TeamCtx<NMAX>& c, double h) {
    if (METHOD == WIND_METHOD_RK2) {
        team_rhs_jac<NMAX, false>(c);
        if (c.l < c.N) c.v[c.l] = (xd(c.v[c.l]) + xd(h) * xd(c.f[c.l])).v;
        team_sync(c.mask);
        return;
    }
    if (SOLVER == WIND_SOLVER_GJE_F64) {
        team_rhs_jac<NMAX, true>(c);
        team_gje_exact<NMAX, CTRL>(c, h);
        return;
    }
    if (SOLVER == WIND_SOLVER_LU_F64) {
        team_rhs_row<NMAX, double, true>(c, h);
        team_lu_smem<NMAX, double, false>(c);
        if (c.l < c.N) c.v[c.l] = c.v[c.l] + h * c.x[c.l];
        team_sync(c.mask);
        return;
    }
    // MIXED: FP32 factors, one FP64 refinement step with r = f - (x - h J x)
    team_rhs_row<NMAX, float, true>(c, h);
    const int mystep = team_lu_smem<NMAX, float, true>(c);
    double r = 0.0, x0 = 0.0;
    if (c.l < c.N) {
        x0 = c.x[c.l];
        r = c.f[c.l] - (x0 - h * team_jx(c, c.x));
    }
    team_sync(c.mask);
    team_lu_resolve<NMAX, float>(c, mystep, r);
    if (c.l < c.N) c.v[c.l] = c.v[c.l] + h * (x0 + c.x[c.l]);
    team_sync(c.mask);
}

template <int NMAX, int METHOD, int CTRL, int SOLVER>
__device__ __forceinline__ void team_take_step(const TeamCtx<NMAX>& c, double t0, double H,
                                               int nsub) {
    const double t1 = t0 + H;
    // (t1-t0)/nsub for nsub in {1,2}: multiplying by 1 or 0.5 rounds the
    // same real number, so it equals the division bit for bit
    double h = (t1 - t0) * (nsub == 1 ? 1.0 : 0.5);
    double t = t0;
    for (int i = 0; i < nsub; i++) {
        if (CTRL == WIND_CTRL_DEVICE) h = fmin(t1 - t, h);
        team_substep<NMAX, METHOD, CTRL, SOLVER>(c, h);
        t += h;
    }
}

// The persistent team loop over one group's systems: every team of NMAX
// lanes of the block takes tickets from the group's queue until it is empty.
// `smem_raw` holds blockDim.x / NMAX team slices.
template <int NMAX, int METHOD, int CTRL, int SOLVER>
__device__ __forceinline__ void team_run(const KParams& p, unsigned char* smem_raw) {
    constexpr int CAP = Cap<METHOD, CTRL>::value;
    const bool lin = p.linear != nullptr;
    const TeamLayout lay(NMAX, p.n_react, lin, SOLVER);
    const int team = threadIdx.x / NMAX;
    const int lane = threadIdx.x & 31;
    TeamCtx<NMAX> c;
    c.l = threadIdx.x % NMAX;
    c.leader = lane - c.l;
    c.mask = (NMAX >= 32) ? 0xffffffffu : (((1u << NMAX) - 1u) << c.leader);
    c.N = p.n_eq;
    c.R = p.n_react;
    unsigned char* base = smem_raw + team * lay.bytes;
    c.Js = reinterpret_cast<double*>(base + lay.js);
    c.bc = reinterpret_cast<double*>(base + lay.bc);
    double* vec = reinterpret_cast<double*>(base + lay.vec);
    c.v = vec;
    c.f = vec + NMAX;
    c.y = vec + 2 * NMAX;
    c.y1 = vec + 3 * NMAX;
    c.y2 = vec + 4 * NMAX;
    c.x = vec + 5 * NMAX;
    c.LT = lin ? reinterpret_cast<float*>(base + lay.lt) : nullptr;
    c.rates = reinterpret_cast<double*>(base + lay.rates);
    uint16_t* sp_s = reinterpret_cast<uint16_t*>(base + lay.species);
    c.sp = sp_s;
    c.A = base + lay.mat;
    c.inc_off = reinterpret_cast<int*>(base + lay.inc_off);
    c.inc = reinterpret_cast<uint16_t*>(base + lay.inc);
    c.piv = reinterpret_cast<int*>(base + lay.piv);
    c.r = vec + 6 * NMAX;
    const int N = c.N, R = c.R, l = c.l;
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;

    while (true) {
        unsigned long long ticket = 0;
        if (l == 0) ticket = atomicAdd(&p.counters[CNT_QUEUE], 1ull);
        ticket = __shfl_sync(c.mask, ticket, c.leader);
        const int64_t s = (int64_t)ticket;
        if (s >= p.nsys) break;

        // stage this system's network into shared memory
        bool bad_idx = false;
        for (int r = l; r < R; r += NMAX) {
            c.rates[r] = p.rates[s * R + r];
            uint2 q = *reinterpret_cast<const uint2*>(p.species + (s * R + r) * 4);
            const unsigned nn = (unsigned)N;
            if ((q.x & 0xffffu) >= nn || (q.x >> 16) >= nn || (q.y & 0xffffu) >= nn || (q.y >> 16) >= nn) {
                bad_idx = true;
                q = make_uint2(0u, 0u);  // keep every later access in bounds
            }
            *reinterpret_cast<uint2*>(sp_s + 4 * r) = q;
        }
        bad_idx = __any_sync(c.mask, bad_idx);
        if (SOLVER != WIND_SOLVER_GJE_F64 && !bad_idx) {
            // per-species incidence lists (reaction ids ascending)
            team_sync(c.mask);
            if (l < N) {
                int cnt = 0;
                for (int r = 0; r < R; r++) {
                    const uint2 q = *reinterpret_cast<const uint2*>(sp_s + 4 * r);
                    cnt += ((q.x & 0xffff) == (unsigned)l) | ((q.x >> 16) == (unsigned)l) |
                           ((q.y & 0xffff) == (unsigned)l) | ((q.y >> 16) == (unsigned)l);
                }
                c.inc_off[l + 1] = cnt;
            }
            team_sync(c.mask);
            if (l == 0) {
                c.inc_off[0] = 0;
                for (int j = 0; j < N; j++) c.inc_off[j + 1] += c.inc_off[j];
            }
            team_sync(c.mask);
            if (l < N) {
                int o = c.inc_off[l];
                for (int r = 0; r < R; r++) {
                    const uint2 q = *reinterpret_cast<const uint2*>(sp_s + 4 * r);
                    if ((q.x & 0xffff) == (unsigned)l || (q.x >> 16) == (unsigned)l ||
                        (q.y & 0xffff) == (unsigned)l || (q.y >> 16) == (unsigned)l)
                        c.inc[o++] = (uint16_t)r;
                }
            }
        }
        if (lin && l < N) {
            const float* Lg = p.linear + s * (int64_t)N * N;
            for (int k = 0; k < N; k++) c.LT[k * NMAX + l] = Lg[l * N + k];
        }
        if (l < N) c.y[l] = p.y[s * N + l];
        team_sync(c.mask);

        double tnow = p.tnow;
        const double tend = p.tend;
        double h = p.h0;
        int unsolved = 0;
        int64_t attempts = 0;
        int32_t st = bad_idx ? WIND_SYS_BAD_INPUT : WIND_SYS_OK;
        while (!bad_idx && tnow < tend) {
            if (attempts >= p.max_attempts) { st |= WIND_SYS_MAX_ATTEMPTS; break; }
            if (p.timeout_ns) {
                // the leader's clock decides for the whole team
                const int late = global_ns() - t_start > p.timeout_ns;
                if (__shfl_sync(c.mask, late, c.leader)) { st |= WIND_SYS_TIMEOUT; break; }
            }
            attempts++;
            h = fmin(tend - tnow, h);
            // full step into y1
            if (l < N) c.v[l] = c.y[l];
            team_sync(c.mask);
            team_take_step<NMAX, METHOD, CTRL, SOLVER>(c, tnow, h, 1);
            if (l < N) c.y1[l] = c.v[l];
            // two half steps into y2
            if (l < N) c.v[l] = c.y[l];
            team_sync(c.mask);
            team_take_step<NMAX, METHOD, CTRL, SOLVER>(c, tnow, h, 2);
            bool err = false;
            if (l < N) {
                c.y2[l] = c.v[l];
                err = elem_error<METHOD, CTRL>(xd(c.y1[l]), xd(c.v[l]), p.atol, p.rtol);
            }
            err = __any_sync(c.mask, err);
            if (err && unsolved < CAP) {
                unsolved++;
                h /= 2.0;
            } else {
                unsolved = 0;
                if (l < N)
                    c.y[l] = (METHOD == WIND_METHOD_RK2) ? (xd(2.0) * xd(c.y2[l]) - xd(c.y1[l])).v
                                                         : c.y2[l];
                if (tnow + h == tnow) { st |= WIND_SYS_STALLED; break; }
                tnow += h;
                h = (METHOD == WIND_METHOD_RK2) ? h * 2 : tend - tnow;
            }
            team_sync(c.mask);
        }
        team_sync(c.mask);
        bool bad = (l < N) && !finite64(c.y[l]);
        if (__any_sync(c.mask, bad)) st |= WIND_SYS_NONFINITE;
        if (l < N) p.y[s * N + l] = c.y[l];
        if (l == 0) {
            if (p.sys_status) p.sys_status[s] = st;
            if (p.sys_nsteps) p.sys_nsteps[s] = 3 * attempts;
            atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)(3 * attempts));
        }
        team_sync(c.mask);
    }
}

template <int NMAX, int METHOD, int CTRL, int SOLVER>
__global__ void __launch_bounds__(TEAM_THREADS) k_team(const KParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    team_run<NMAX, METHOD, CTRL, SOLVER>(p, smem_raw);
}

}  // namespace wind
