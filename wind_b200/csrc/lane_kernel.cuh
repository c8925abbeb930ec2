// lane_kernel.cuh -- persistent thread-per-system integrator for the builtin
// networks (compile-time N <= 5): NR_test, StiffTrig, Katz96.
//
// Design (replaces cuda/common/kernel.cu:140-311, which ran one CTA of N
// threads per system with the matrices in global memory):
//  * the whole system -- state, Jacobian, inverse/factors -- lives in the
//    registers of one thread; no shared or global scratch besides the work
//    counter;
//  * persistent grid: a team of W lanes pulls the next system index from a
//    device work queue (atomic ticket) the moment it finishes one, so systems
//    with very different step counts do not idle a warp;
//  * speculative refinement: the W lanes of a team evaluate the next W
//    refinement levels h, h/2, ..., h/2^(W-1) of the same attempt at once and
//    keep the first that passes (or the one at the refinement cap).  Each
//    attempt is computed exactly as the serial controller would compute it,
//    so results and step counts are identical to the serial loop
//    (kernel.cu:191-296, common_gold.c:77-149); only latency changes.
#pragma once

#include "common.cuh"
#include "networks.cuh"
#include "solvers_reg.cuh"

namespace wind {

constexpr int LANE_THREADS = 128;

// One SIE or explicit-Euler substep of length h, in place on y.
template <class Net, int METHOD, int CTRL, int SOLVER>
__device__ __forceinline__ void lane_substep(const double (&c)[Net::NC], xd h, xd (&y)[Net::N]) {
    constexpr int N = Net::N;
    xd f[N];
    Net::rhs(c, y, f);
    if (METHOD == WIND_METHOD_RK2) {
        // rk2_gold.c:31-34, kernel.cu:128-130: y += h*f
#pragma unroll
        for (int e = 0; e < N; e++) y[e] += h * f[e];
        return;
    }
    xd M[N * N];
#pragma unroll
    for (int e = 0; e < N * N; e++) M[e] = 0.0;
    Net::jac(c, y, M);
    if (SOLVER == WIND_SOLVER_GJE_F64) {
        if (CTRL == WIND_CTRL_GOLD) {
            // sie_gold.c:17-36: J = -h*J; diag += 1
#pragma unroll
            for (int e = 0; e < N * N; e++) M[e] = -h * M[e];
#pragma unroll
            for (int i = 0; i < N; i++) M[i * (N + 1)] += 1.0;
        } else {
            // kernel.cu:49-52: J[i][j] = (i==j) - J[i][j]*h
#pragma unroll
            for (int i = 0; i < N; i++)
#pragma unroll
                for (int j = 0; j < N; j++) M[i * N + j] = xd(i == j ? 1.0 : 0.0) - M[i * N + j] * h;
        }
        xd Inv[N * N];
        gje_invert_reg<N>(M, Inv);
        if (CTRL == WIND_CTRL_GOLD) {
            // matrix_ops.c:6-27 (transposed matvec), then sie_gold.c:72-74
            xd out[N];
#pragma unroll
            for (int r = 0; r < N; r++) out[r] = 0.0;
#pragma unroll
            for (int cc = 0; cc < N; cc++)
#pragma unroll
                for (int r = 0; r < N; r++) out[r] += Inv[cc * N + r] * f[cc];
#pragma unroll
            for (int e = 0; e < N; e++) y[e] += h * out[e];
        } else {
            // kernel.cu:116-125: y_j += (Inv[k][j]*f_k)*h, k ascending
#pragma unroll
            for (int k = 0; k < N; k++)
#pragma unroll
                for (int j = 0; j < N; j++) y[j] += Inv[k * N + j] * f[k] * h;
        }
        return;
    }
    // Standard orientation A[r][c] = delta_rc - h * J_rc, J_rc = Jt[c][r].
    if (SOLVER == WIND_SOLVER_LU_F64) {
        double A[N * N], rinv[N];
        int perm[N];
#pragma unroll
        for (int r = 0; r < N; r++)
#pragma unroll
            for (int cc = 0; cc < N; cc++)
                A[r * N + cc] = (r == cc ? 1.0 : 0.0) - h.v * M[cc * N + r].v;
        lu_factor_reg<N, double>(A, rinv, perm);
        double x[N];
#pragma unroll
        for (int e = 0; e < N; e++) x[e] = f[e].v;
        lu_solve_reg<N, double, double>(A, rinv, perm, x);
#pragma unroll
        for (int e = 0; e < N; e++) y[e] = y[e].v + h.v * x[e];
        return;
    }
    // MIXED: FP32 factor, FP64 residual, one refinement step.
    float Af[N * N], rinvf[N];
    int perm[N];
#pragma unroll
    for (int r = 0; r < N; r++)
#pragma unroll
        for (int cc = 0; cc < N; cc++)
            Af[r * N + cc] = (float)((r == cc ? 1.0 : 0.0) - h.v * M[cc * N + r].v);
    lu_factor_reg<N, float>(Af, rinvf, perm);
    double x[N];
#pragma unroll
    for (int e = 0; e < N; e++) x[e] = f[e].v;
    lu_solve_reg<N, float, double>(Af, rinvf, perm, x);
    // r = f - A x with A = I - h J (FP64, from Jt)
    double res[N];
#pragma unroll
    for (int r = 0; r < N; r++) {
        double acc = 0.0;
#pragma unroll
        for (int cc = 0; cc < N; cc++) acc = fma(M[cc * N + r].v, x[cc], acc);
        res[r] = f[r].v - (x[r] - h.v * acc);
    }
    lu_solve_reg<N, float, double>(Af, rinvf, perm, res);
#pragma unroll
    for (int e = 0; e < N; e++) y[e] = y[e].v + h.v * (x[e] + res[e]);
}

// take_step (sie_gold.c:38-51) / innerstep (kernel.cu:69-91): nsub substeps
// over [t0, t0+H]; DEVICE clamps each substep with fmin.
template <class Net, int METHOD, int CTRL, int SOLVER>
__device__ __forceinline__ void lane_take_step(const double (&c)[Net::NC], double t0, double H,
                                               int nsub, xd (&y)[Net::N]) {
    const double t1 = t0 + H;
    double h = (t1 - t0) / nsub;
    double t = t0;
    for (int i = 0; i < nsub; i++) {
        if (CTRL == WIND_CTRL_DEVICE) h = fmin(t1 - t, h);
        lane_substep<Net, METHOD, CTRL, SOLVER>(c, xd(h), y);
        t += h;
    }
}

template <class Net, int METHOD, int CTRL, int SOLVER>
__global__ void __launch_bounds__(LANE_THREADS) k_lane(const KParams p, const int W) {
    constexpr int N = Net::N;
    constexpr int NC = Net::NC;
    constexpr int CAP = Cap<METHOD, CTRL>::value;
    const int lane = threadIdx.x & 31;
    const int level = lane % W;
    const int leader = lane - level;
    const unsigned team_mask = (W >= 32) ? 0xffffffffu : (((1u << W) - 1u) << leader);
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;

    while (true) {
        unsigned long long ticket = 0;
        if (level == 0) ticket = atomicAdd(&p.counters[CNT_QUEUE], 1ull);
        ticket = __shfl_sync(team_mask, ticket, leader);
        const int64_t s = (int64_t)ticket;
        if (s >= p.nsys) break;

        double c[NC];
#pragma unroll
        for (int k = 0; k < NC; k++) c[k] = __ldg(p.constants + s * p.n_const + k);
        xd y[N];
#pragma unroll
        for (int i = 0; i < N; i++) y[i] = p.y[s * N + i];

        double tnow = p.tnow;
        const double tend = p.tend;
        double h = p.h0;
        int unsolved = 0;
        int64_t attempts = 0;
        int32_t st = WIND_SYS_OK;
        while (tnow < tend) {
            if (attempts >= p.max_attempts) { st |= WIND_SYS_MAX_ATTEMPTS; break; }
            if (p.timeout_ns && global_ns() - t_start > p.timeout_ns) { st |= WIND_SYS_TIMEOUT; break; }
            // kernel.cu:195 / common_gold.c:79
            const double hw = fmin(tend - tnow, h);
            double hl = hw;
            for (int q = 0; q < level; q++) hl /= 2.0;
            const int lvl = unsolved + level;
            const bool valid = (lvl <= CAP) && (attempts + level < p.max_attempts);
            xd y1[N], y2[N];
#pragma unroll
            for (int i = 0; i < N; i++) { y1[i] = y[i]; y2[i] = y[i]; }
            bool err = true;
            if (valid) {
                lane_take_step<Net, METHOD, CTRL, SOLVER>(c, tnow, hl, 1, y1);
                lane_take_step<Net, METHOD, CTRL, SOLVER>(c, tnow, hl, 2, y2);
                err = false;
#pragma unroll
                for (int i = 0; i < N; i++) err |= elem_error<METHOD, CTRL>(y1[i], y2[i], p.atol, p.rtol);
            }
            const bool acc = valid && (!err || lvl == CAP);
            const unsigned bal = __ballot_sync(team_mask, acc);
            if (bal == 0) {
                // every evaluated level refines: kernel.cu:259-270
                int done = W;
                if (attempts + W > p.max_attempts) done = (int)(p.max_attempts - attempts);
                attempts += done;
                unsolved += done;
                h = hw;
                for (int q = 0; q < done; q++) h /= 2.0;
                continue;
            }
            const int a_lane = __ffs(bal) - 1;
            attempts += (a_lane - leader) + 1;
            double ynew[N];
#pragma unroll
            for (int i = 0; i < N; i++)
                ynew[i] = (METHOD == WIND_METHOD_RK2) ? (xd(2.0) * y2[i] - y1[i]).v : y2[i].v;
            const double ha = __shfl_sync(team_mask, hl, a_lane);
#pragma unroll
            for (int i = 0; i < N; i++) y[i] = __shfl_sync(team_mask, ynew[i], a_lane);
            unsolved = 0;
            if (tnow + ha == tnow) { st |= WIND_SYS_STALLED; break; }
            tnow += ha;
            // kernel.cu:271-294: RK2 doubles h, SIE goes for gold
            h = (METHOD == WIND_METHOD_RK2) ? ha * 2 : tend - tnow;
        }
#pragma unroll
        for (int i = 0; i < N; i++)
            if (!finite64(y[i].v)) st |= WIND_SYS_NONFINITE;
        if (level == 0) {
#pragma unroll
            for (int i = 0; i < N; i++) p.y[s * N + i] = y[i].v;
            if (p.sys_status) p.sys_status[s] = st;
            if (p.sys_nsteps) p.sys_nsteps[s] = 3 * attempts;
            atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)(3 * attempts));
        }
    }
}

}  // namespace wind
