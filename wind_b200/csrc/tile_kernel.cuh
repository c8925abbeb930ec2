// tile_kernel.cuh -- persistent integrator for tiled builtin networks: a
// system of Ntile copies of NR_test, StiffTrig or Katz96 (N = Ntile x base).
//
// The reference builds such a system with the Precompiler's Ntile tiling
// (python/ode_systems/ode_base.py:86-88, 219-281) and integrates it like any
// other: a dense N x N Jacobian, block diagonal, inverted by the full
// unpivoted Gauss-Jordan elimination (cuda/common/kernel.cu:42-66,
// cuda/linear_algebra/gauss_jordan_elimination.cu:15-212), so its cost grows
// as N^3.  Every off-block entry of that elimination is a zero multiplied
// into a row or added to a sum, which leaves every in-block value unchanged:
// the full elimination IS the per-block elimination, value for value (only
// the sign of a zero can differ).  Here each tile is solved on its own, so
// the cost grows as Ntile:
//  * a team of `ts` lanes of one warp owns a system (ts = the power of two
//    >= Ntile, at most 32); lane l owns tiles l, l + ts, ... (at most KT),
//    their state in registers, and runs each tile's substep with the
//    register solvers of the thread-per-system kernel;
//  * the controller (step doubling, refinement cap, go for gold / doubling)
//    is the reference's, shared by the team: the error test is one ballot
//    over the team, so a step is accepted only when every tile passes;
//  * Katz96 tiles read tile 0's electron density (the generated prefix
//    computes ne from equations 1, 3 and 4 only), broadcast from the team's
//    first lane before each right-hand side / Jacobian evaluation.
// Results are bit-identical to the reference algorithm on the full matrix
// with the Gauss-Jordan solver (GJE_F64); LU_F64 and MIXED solve the blocks
// with their own factorisations.
#pragma once

#include "api_internal.h"
#include "lane_kernel.cuh"

namespace wind {

constexpr int TILE_THREADS = 128;

template <class Net, int METHOD, int CTRL, int SOLVER, int KT>
__global__ void __launch_bounds__(TILE_THREADS) k_tile(const KParams p, const int ntile, const int ts) {
    using TT = TileOf<Net>;
    using TN = typename TT::Tile;
    constexpr int N = Net::N;
    constexpr int NC = Net::NC;
    constexpr int CAP = Cap<METHOD, CTRL>::value;
    const int lane = threadIdx.x & 31;
    const int leader = lane - lane % ts;
    const int tl = lane - leader;
    const unsigned tmask = ts == 32 ? 0xffffffffu : (((1u << ts) - 1u) << leader);
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;
    const int NE = p.n_eq;
    const double tend = p.tend;

    while (true) {
        unsigned long long ticket = 0;
        if (tl == 0) ticket = atomicAdd(&p.counters[CNT_QUEUE], 1ull);
        ticket = __shfl_sync(tmask, ticket, leader);
        if ((int64_t)ticket >= p.nsys) break;
        const int64_t s = (int64_t)ticket;
        double c[TN::NC];
#pragma unroll
        for (int k = 0; k < NC; k++) c[k] = __ldg(p.constants + s * p.n_const + k);
        bool own[KT];
        xd y[KT][N];
#pragma unroll
        for (int j = 0; j < KT; j++) {
            const int tile = tl + ts * j;
            own[j] = tile < ntile;
#pragma unroll
            for (int i = 0; i < N; i++) {
                y[j][i] = 0.0;
                if (own[j]) y[j][i] = p.y[s * NE + tile * N + i];
            }
        }
        double t = p.tnow, h = p.h0;
        int u = 0;
        int64_t a = 0;
        int32_t st = WIND_SYS_OK;
        // common_gold.c:77-149 / kernel.cu:191-296, every quantity uniform
        // over the team
        while (t < tend) {
            if (a >= p.max_attempts) { st |= WIND_SYS_MAX_ATTEMPTS; break; }
            if (p.timeout_ns) {
                const bool late = __shfl_sync(tmask, tl == 0 && global_ns() - t_start > p.timeout_ns, leader);
                if (late) { st |= WIND_SYS_TIMEOUT; break; }
            }
            a++;
            const double hw = fmin(tend - t, h);
            // lane_attempt's arithmetic, tile by tile: the full step into
            // y1 and the two half steps into y2
            const double t1 = t + hw;
            double hf = (t1 - t) * 1.0;
            double hh = (t1 - t) * 0.5;
            if (CTRL == WIND_CTRL_DEVICE) {
                hf = fmin(t1 - t, hf);
                hh = fmin(t1 - t, hh);
            }
            xd y1[KT][N], y2[KT][N];
#pragma unroll
            for (int j = 0; j < KT; j++)
#pragma unroll
                for (int i = 0; i < N; i++) { y1[j][i] = y[j][i]; y2[j][i] = y[j][i]; }
            if constexpr (TT::coupled) c[NC] = __shfl_sync(tmask, TT::shared(y[0]), leader);
#pragma unroll
            for (int j = 0; j < KT; j++) {
                if (own[j]) {
                    lane_substep<TN, METHOD, CTRL, SOLVER>(c, xd(hf), y1[j]);
                    lane_substep<TN, METHOD, CTRL, SOLVER>(c, xd(hh), y2[j]);
                }
            }
            const double tm = t + hh;
            double hh2 = hh;
            if (CTRL == WIND_CTRL_DEVICE) hh2 = fmin(t1 - tm, hh);
            if constexpr (TT::coupled) c[NC] = __shfl_sync(tmask, TT::shared(y2[0]), leader);
#pragma unroll
            for (int j = 0; j < KT; j++)
                if (own[j]) lane_substep<TN, METHOD, CTRL, SOLVER>(c, xd(hh2), y2[j]);
            bool err = false;
#pragma unroll
            for (int j = 0; j < KT; j++)
                if (own[j])
#pragma unroll
                    for (int i = 0; i < N; i++) err |= elem_error<METHOD, CTRL>(y1[j][i], y2[j][i], p.atol, p.rtol);
            err = __any_sync(tmask, err);
            if (err && u < CAP) {
                u++;
                h = hw / 2.0;
                continue;
            }
            u = 0;
#pragma unroll
            for (int j = 0; j < KT; j++)
#pragma unroll
                for (int i = 0; i < N; i++)
                    y[j][i] = (METHOD == WIND_METHOD_RK2) ? xd(2.0) * y2[j][i] - y1[j][i] : y2[j][i];
            if (t + hw == t) { st |= WIND_SYS_STALLED; break; }
            t += hw;
            // kernel.cu:285-294: RK2 doubles h, SIE goes for gold
            h = (METHOD == WIND_METHOD_RK2) ? hw * 2 : tend - t;
        }
        bool bad = false;
#pragma unroll
        for (int j = 0; j < KT; j++) {
            if (!own[j]) continue;
            const int tile = tl + ts * j;
#pragma unroll
            for (int i = 0; i < N; i++) {
                bad |= !finite64(y[j][i].v);
                p.y[s * NE + tile * N + i] = y[j][i].v;
            }
        }
        if (__any_sync(tmask, bad)) st |= WIND_SYS_NONFINITE;
        if (tl == 0) {
            if (p.sys_status) p.sys_status[s] = st;
            if (p.sys_nsteps) p.sys_nsteps[s] = 3 * a;
            atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)(3 * a));
        }
    }
}

}  // namespace wind
