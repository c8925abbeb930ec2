// sim_kernel.cuh -- the semi-implicit midpoint rule with smoothing step
// (Bader-Deuflhard; Numerical Recipes 16.6) of python/pysolvers/sim.py:36-90,
// as a batched fixed-step integrator (WIND_METHOD_SIM).
//
// Per system, m = n_integration_steps steps of h = (tend - tnow)/m:
//   D_0 = (I - hJ(y_0))^-1 h f(y_0),                         y_1 = y_0 + D_0
//   D_k = D_{k-1} + 2 (I - hJ(y_k))^-1 (h f(y_k) - D_{k-1}),  y_{k+1} = y_k + D_k
//   ybar = y_m + (I - hJ(y_m))^-1 (h f(y_m) - D_{m-1})         (the result)
// with the Jacobian re-evaluated at every y_k as the reference does
// (sim.py:59).  The reference inverts I - hJ with numpy.linalg.inv and
// multiplies (sim.py:61-64); here every solve is the FP64 partial-pivot LU,
// the same solve up to rounding.  There is no error control, so every system
// does the same m + 1 solves and the work needs no queue: thread-per-system
// kernels stride over the batch, team kernels take tickets only to spread
// systems over the resident teams.
//
//  k_sim_lane  builtin networks (compile-time N <= 5): one thread per
//              system, state, Jacobian and factors in registers;
//  k_sim_warp  mass-action networks, N <= 32: a team of NMAX lanes per
//              system, lane l owning row l of I - hJ (the register-resident
//              team layout and LU of warp_kernel.cuh).
#pragma once

#include "common.cuh"
#include "networks.cuh"
#include "solvers_reg.cuh"
#include "warp_kernel.cuh"

namespace wind {

constexpr int SIM_THREADS = 128;

template <class Net>
__global__ void __launch_bounds__(SIM_THREADS) k_sim_lane(const KParams p) {
    constexpr int N = Net::N;
    constexpr int NC = Net::NC;
    const int m = p.n_steps;
    const double h = p.h0;
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < p.nsys;
         s += (int64_t)gridDim.x * blockDim.x) {
        double c[NC];
#pragma unroll
        for (int k = 0; k < NC; k++) c[k] = __ldg(p.constants + s * p.n_const + k);
        xd y[N];
        double d[N];
#pragma unroll
        for (int i = 0; i < N; i++) { y[i] = p.y[s * N + i]; d[i] = 0.0; }
        int32_t st = WIND_SYS_OK;
        int64_t solves = 0;
        for (int k = 0; k <= m; k++) {
            if (p.timeout_ns && global_ns() - t_start > p.timeout_ns) {
                st |= WIND_SYS_TIMEOUT;
                break;
            }
            xd f[N];
            Net::rhs(c, y, f);
            xd Jt[N * N];
#pragma unroll
            for (int e = 0; e < N * N; e++) Jt[e] = 0.0;
            Net::jac(c, y, Jt);
            // A[r][c] = delta_rc - h J_rc, J_rc = Jt[c][r]
            double A[N * N], rinv[N];
            int perm[N];
#pragma unroll
            for (int r = 0; r < N; r++)
#pragma unroll
                for (int cc = 0; cc < N; cc++)
                    A[r * N + cc] = (r == cc ? 1.0 : 0.0) - h * Jt[cc * N + r].v;
            lu_factor_reg<N, double>(A, rinv, perm);
            double x[N];
#pragma unroll
            for (int e = 0; e < N; e++) x[e] = h * f[e].v - (k ? d[e] : 0.0);
            lu_solve_reg<N, double, double>(A, rinv, perm, x);
#pragma unroll
            for (int e = 0; e < N; e++) {
                d[e] = (k == 0 || k == m) ? x[e] : d[e] + 2.0 * x[e];
                y[e] = y[e].v + d[e];
            }
            solves++;
        }
#pragma unroll
        for (int i = 0; i < N; i++) {
            if (!finite64(y[i].v)) st |= WIND_SYS_NONFINITE;
            p.y[s * N + i] = y[i].v;
        }
        if (p.sys_status) p.sys_status[s] = st;
        if (p.sys_nsteps) p.sys_nsteps[s] = solves;
        atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)solves);
    }
}

template <int NMAX>
__global__ void __launch_bounds__(WARP_THREADS) k_sim_warp(const KParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const bool lin = p.linear != nullptr;
    const WarpLayout lay(NMAX, p.n_react, lin, WIND_SOLVER_LU_F64);
    const int team = threadIdx.x / NMAX;
    const int lane = threadIdx.x & 31;
    WarpCtx<NMAX, double> c;
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
    c.qf = reinterpret_cast<double*>(base + lay.qf);
    c.piv = reinterpret_cast<int*>(base + lay.piv);
    c.rows = reinterpret_cast<double*>(base + lay.rows);
    c.pb = reinterpret_cast<double*>(base + lay.pb);
    c.sv = nullptr;
    const int N = c.N, l = c.l;
    const int m = p.n_steps;
    const double h = p.h0;
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;

    while (true) {
        unsigned long long ticket = 0;
        if (l == 0) ticket = atomicAdd(&p.counters[CNT_QUEUE], 1ull);
        ticket = __shfl_sync(c.mask, ticket, c.leader);
        const int64_t s = (int64_t)ticket;
        if (s >= p.nsys) break;

        const bool bad_idx = warp_stage_system(c, p, s, rates_s, sp_s, inc_off, inc, LT);
        double y = (l < N) ? p.y[s * N + l] : 0.0;
        double d = 0.0;
        int32_t st = bad_idx ? WIND_SYS_BAD_INPUT : WIND_SYS_OK;
        int64_t solves = 0;
        for (int k = 0; k <= m && !bad_idx; k++) {
            // the deadline, decided by the team's first lane for the team
            int late = 0;
            if (l == 0 && p.timeout_ns && global_ns() - t_start > p.timeout_ns) late = 1;
            if (__shfl_sync(c.mask, late, c.leader)) {
                st |= WIND_SYS_TIMEOUT;
                break;
            }
            __syncwarp(c.mask);  // the previous step's readers of vb are done
            c.vb[l] = y;
            __syncwarp(c.mask);
            const double f = warp_rhs(c);
            warp_jma_row(c);
            double a[NMAX];
            warp_load_matrix(c, h, a);
            const double b = (l < N) ? h * f - (k ? d : 0.0) : 0.0;
            const double x = warp_lu_solve(c, a, b);
            if (l < N) {
                d = (k == 0 || k == m) ? x : d + 2.0 * x;
                y = y + d;
            }
            solves++;
        }
        const bool nonfinite = __any_sync(c.mask, (l < N) && !finite64(y));
        if (nonfinite) st |= WIND_SYS_NONFINITE;
        if (l < N && !bad_idx) p.y[s * N + l] = y;
        if (l == 0) {
            if (p.sys_status) p.sys_status[s] = st;
            if (p.sys_nsteps) p.sys_nsteps[s] = solves;
            atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)solves);
        }
        __syncwarp(c.mask);  // the slice is free for the next system
    }
}

}  // namespace wind
