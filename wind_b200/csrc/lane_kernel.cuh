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
// Minimum resident blocks per SM the compiler must plan registers for.  The
// LU solver runs faster capped at 128 registers (4 blocks of 128 threads per
// SM: 51-52 ms against 63-64 ms per 65,536-cell Katz96 call, measured back
// to back on one B200, despite ~230 bytes of spills); the Gauss-Jordan path
// loses under the same cap (600 -> 678 ms) and the mixed path was not
// measured capped, so both keep the uncapped allocation.
template <int SOLVER>
struct LaneMinBlocks {
    static constexpr int value = SOLVER == WIND_SOLVER_LU_F64 ? 4 : 1;
};

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
    // (t1-t0)/nsub for nsub in {1,2}: multiplying by 1 or 0.5 rounds the
    // same real number, so it equals the division bit for bit
    double h = (t1 - t0) * (nsub == 1 ? 1.0 : 0.5);
    double t = t0;
    for (int i = 0; i < nsub; i++) {
        if (CTRL == WIND_CTRL_DEVICE) h = fmin(t1 - t, h);
        lane_substep<Net, METHOD, CTRL, SOLVER>(c, xd(h), y);
        t += h;
    }
}

// One attempt: the full step into y1 and the two half steps into y2, written
// as straight-line code so the full step and the first half step -- which
// are independent -- can be interleaved by the scheduler; the attempt's
// critical path is then two substeps instead of three.  Each substep is the
// same arithmetic as lane_take_step's (take_step, sie_gold.c:38-51;
// innerstep, kernel.cu:69-91).
template <class Net, int METHOD, int CTRL, int SOLVER>
__device__ __forceinline__ void lane_attempt(const double (&c)[Net::NC], double t0, double H,
                                             xd (&y1)[Net::N], xd (&y2)[Net::N]) {
    const double t1 = t0 + H;
    double hf = (t1 - t0) * 1.0;
    double hh = (t1 - t0) * 0.5;
    if (CTRL == WIND_CTRL_DEVICE) {
        hf = fmin(t1 - t0, hf);
        hh = fmin(t1 - t0, hh);
    }
    lane_substep<Net, METHOD, CTRL, SOLVER>(c, xd(hf), y1);
    lane_substep<Net, METHOD, CTRL, SOLVER>(c, xd(hh), y2);
    const double tm = t0 + hh;
    double hh2 = hh;
    if (CTRL == WIND_CTRL_DEVICE) hh2 = fmin(t1 - tm, hh);
    lane_substep<Net, METHOD, CTRL, SOLVER>(c, xd(hh2), y2);
}

// Lanes of the warp that point at the same owner form a team.  With a
// systems in the warp (owners), lane i works on owner (i mod a) at
// refinement level (i div a): lanes are spread round-robin, so team sizes
// differ by at most one and the lowest lane of a team carries level 0.
__device__ __forceinline__ unsigned team_mask_of(int j, int nact, int wmax) {
    unsigned m = 0u;
    for (int k = j, r = 0; k < 32 && r < wmax; k += nact, r++) m |= 1u << k;
    return m;
}

// Persistent kernel.  Every lane owns at most one system (its state lives in
// the owner's registers).  Each round:
//  1. lanes without a system take the next ticket from the work queue;
//  2. the a owned systems of the warp are assigned all 32 lanes round-robin;
//     a lane fetches its assigned system's state from the owner by shuffle;
//  3. each lane evaluates one attempt (full step + two half steps + error
//     test) at its refinement level;
//  4. per team, the lowest level that passes (or the one at the cap) is the
//     accepted attempt; every level below it is exactly the serial
//     controller's rejected attempt, so the owner applies "levels refined,
//     then accept" with results identical to the serial loop.
// While the queue is full every lane owns a system and a round is one attempt
// per system (no speculation, no waste).  As the queue drains, idle lanes join
// the remaining systems, which cuts the tail of slow systems by up to the
// refinement cap.  Only lanes below `opw` (owners per warp) take tickets; the
// others start as helpers, which spreads a small batch over many warps
// (opw = 32 / initial lanes per system).
template <class Net, int METHOD, int CTRL, int SOLVER>
__global__ void __launch_bounds__(LANE_THREADS, LaneMinBlocks<SOLVER>::value) k_lane(const KParams p, const int opw) {
    constexpr int N = Net::N;
    constexpr int NC = Net::NC;
    constexpr int CAP = Cap<METHOD, CTRL>::value;
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int wmax = 32;
    const int lane = threadIdx.x & 31;
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;
    const double tend = p.tend;

    // owner state
    bool has = false, drained = (lane >= opw);
    int64_t s_own = -1;
    double y_own[N];
    double t_own = 0.0, h_own = 0.0;
    int u_own = 0;
    int64_t a_own = 0;
    int32_t st_own = WIND_SYS_OK;
    // worker cache
    int64_t s_work = -1;
    double c[NC];

    while (true) {
        // 1. refill: take new tickets while without a system
        while (!has && !drained) {
            const unsigned long long ticket = atomicAdd(&p.counters[CNT_QUEUE], 1ull);
            if ((int64_t)ticket >= p.nsys) { drained = true; break; }
            s_own = (int64_t)ticket;
#pragma unroll
            for (int i = 0; i < N; i++) y_own[i] = p.y[s_own * N + i];
            t_own = p.tnow;
            h_own = p.h0;
            u_own = 0;
            a_own = 0;
            st_own = WIND_SYS_OK;
            has = true;
        }
        // finish systems that are done
        if (has) {
            bool fin = !(t_own < tend);
            if (!fin && a_own >= p.max_attempts) { st_own |= WIND_SYS_MAX_ATTEMPTS; fin = true; }
            if (!fin && p.timeout_ns && global_ns() - t_start > p.timeout_ns) {
                st_own |= WIND_SYS_TIMEOUT;
                fin = true;
            }
            if (fin) {
#pragma unroll
                for (int i = 0; i < N; i++) {
                    if (!finite64(y_own[i])) st_own |= WIND_SYS_NONFINITE;
                    p.y[s_own * N + i] = y_own[i];
                }
                if (p.sys_status) p.sys_status[s_own] = st_own;
                if (p.sys_nsteps) p.sys_nsteps[s_own] = 3 * a_own;
                atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)(3 * a_own));
                has = false;
                continue;  // refill before the warp-wide round
            }
        }
        const unsigned owners = __ballot_sync(FULL, has);
        if (owners == 0u) {
            if (__all_sync(FULL, drained)) break;
            continue;
        }
        // 2. assignment and state fetch
        const int nact = __popc(owners);
        const int j = lane % nact;
        const int r = lane / nact;
        const int src = __fns(owners, 0, j + 1);
        const int64_t s_j = __shfl_sync(FULL, s_own, src);
        const double t_j = __shfl_sync(FULL, t_own, src);
        const double h_j = __shfl_sync(FULL, h_own, src);
        const int u_j = __shfl_sync(FULL, u_own, src);
        const int64_t a_j = __shfl_sync(FULL, a_own, src);
        xd y[N];
#pragma unroll
        for (int i = 0; i < N; i++) y[i] = __shfl_sync(FULL, y_own[i], src);
        if (s_j != s_work) {
            s_work = s_j;
#pragma unroll
            for (int k = 0; k < NC; k++) c[k] = __ldg(p.constants + s_j * p.n_const + k);
        }
        // 3. one attempt at level r: kernel.cu:195 / common_gold.c:79 clamp,
        //    then r halvings (kernel.cu:262 / common_gold.c:123)
        const double hw = fmin(tend - t_j, h_j);
        double hl = hw;
        for (int q = 0; q < r; q++) hl /= 2.0;
        const int lvl = u_j + r;
        const bool valid = (r < wmax) && (lvl <= CAP) && (a_j + r < p.max_attempts);
        xd y1[N], y2[N];
#pragma unroll
        for (int i = 0; i < N; i++) { y1[i] = y[i]; y2[i] = y[i]; }
        bool err = true;
        if (valid) {
            lane_attempt<Net, METHOD, CTRL, SOLVER>(c, t_j, hl, y1, y2);
            err = false;
#pragma unroll
            for (int i = 0; i < N; i++) err |= elem_error<METHOD, CTRL>(y1[i], y2[i], p.atol, p.rtol);
        }
        const bool acc = valid && (!err || lvl == CAP);
        const unsigned bal = __ballot_sync(FULL, acc);
        // 4. owners apply their team's outcome
        int take = lane;   // lane whose attempt this owner adopts (self = none)
        int done = 0;      // attempts consumed this round
        bool accepted = false;
        if (has) {
            const int jo = __popc(owners & ((1u << lane) - 1u));
            const unsigned tm = team_mask_of(jo, nact, wmax);
            const int tsz = __popc(tm);
            const unsigned mine = bal & tm;
            if (mine) {
                take = __ffs(mine) - 1;
                done = take / nact + 1;
                accepted = true;
            } else {
                // every level of the team refined (the cap level would accept)
                int lim = tsz;
                if (a_own + lim > p.max_attempts) lim = (int)(p.max_attempts - a_own);
                done = lim;
            }
        }
        double ytake[N];
#pragma unroll
        for (int i = 0; i < N; i++)
            ytake[i] = (METHOD == WIND_METHOD_RK2) ? (xd(2.0) * y2[i] - y1[i]).v : y2[i].v;
        const double htake = __shfl_sync(FULL, hl, take);
#pragma unroll
        for (int i = 0; i < N; i++) ytake[i] = __shfl_sync(FULL, ytake[i], take);
        if (has) {
            a_own += done;
            if (accepted) {
#pragma unroll
                for (int i = 0; i < N; i++) y_own[i] = ytake[i];
                u_own = 0;
                if (t_own + htake == t_own) {
                    st_own |= WIND_SYS_STALLED;
                    t_own = tend;  // finishes at the top of the next round
                } else {
                    t_own += htake;
                    // kernel.cu:285-294: RK2 doubles h, SIE goes for gold
                    h_own = (METHOD == WIND_METHOD_RK2) ? htake * 2 : tend - t_own;
                }
            } else {
                u_own += done;
                double hh = fmin(tend - t_own, h_own);
                for (int q = 0; q < done; q++) hh /= 2.0;
                h_own = hh;
            }
        }
    }
}

}  // namespace wind
