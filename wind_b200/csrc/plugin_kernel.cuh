// plugin_kernel.cuh -- persistent integrator for a runtime network plug-in:
// a network given as source text in the reference's host plug-in contract
// (cuda/include/ode_gold.h:1-12, the Precompiler's output,
// python/ode_systems/ode_base.py:16-123) and compiled at run time with
// NVRTC (csrc/plugin.cu), in FP64.
//
// The plug-in computes a whole system's RHS and (transposed) Jacobian in one
// call, as the reference's c_baseline calls it (sie_gold.c:38-79), so one
// lane of a team calls it; the team then does the reference's algorithm with
// the work spread over its lanes:
//  * a team of TS lanes (the power of two >= N, at most 32) per system, the
//    system's matrices and vectors in the team's slice of shared memory;
//  * A = I - hJ (GOLD: -hJ then diag += 1; DEVICE: (i==j) - J h), the
//    unpivoted Gauss-Jordan inverse with the rows of each elimination step
//    spread over the lanes (every element sees the reference's operation
//    sequence: cuda/c_baseline/linear_algebra/gje_gold.c:5-144), then the
//    update (GOLD matvec then y += h out, matrix_ops.c:6-27; DEVICE
//    y_j += (Inv_kj f_k) h term by term, kernel.cu:116-125);
//  * the step-doubling controller of the thread-per-system kernels, uniform
//    over the team, the error test one ballot.
// Results are bit-identical to the reference algorithm when the plug-in is
// compiled without contraction (NVRTC --fmad=false, as the c_baseline's
// x86-64 build rounds every product).  The header compiles under NVRTC.
#pragma once

#include "common.cuh"

namespace wind {

constexpr int PLUGIN_THREADS = 128;
constexpr int PLUGIN_MAX_EQ = 64;

__host__ __device__ constexpr int plugin_team(int n) {
    return n <= 1 ? 1 : n <= 2 ? 2 : n <= 4 ? 4 : n <= 8 ? 8 : n <= 16 ? 16 : 32;
}

// Shared-memory slice of one team, in doubles.
template <int N, int NC>
struct PluginLayout {
    static constexpr int M = 0;
    static constexpr int INV = N * N;
    static constexpr int F = 2 * N * N;
    static constexpr int Y = F + N;
    static constexpr int Y1 = Y + N;
    static constexpr int Y2 = Y1 + N;
    static constexpr int OUT = Y2 + N;
    static constexpr int C = OUT + N;
    static constexpr int SIZE = C + (NC > 0 ? NC : 1);
};

template <class P>
struct PluginTeam {
    static constexpr int N = P::N;
    static constexpr int NC = P::NC;
    static constexpr int TS = plugin_team(N);
    using L = PluginLayout<N, NC>;
    double* s;       // this team's slice
    int tl;          // lane within the team
    unsigned mask;   // the team's lanes
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
};

// One SIE substep of length h from the state at ys (in place), the plug-in
// evaluated at time t.
template <class P, int CTRL>
__device__ __forceinline__ void plugin_sie_substep(const PluginTeam<P>& T, double* ys, double t, xd h) {
    constexpr int N = P::N, TS = PluginTeam<P>::TS;
    using L = typename PluginTeam<P>::L;
    double* M = T.s + L::M;
    double* Inv = T.s + L::INV;
    double* f = T.s + L::F;
    double* out = T.s + L::OUT;
    const double* c = T.s + L::C;
    // the Jacobian is zero-filled before each evaluation (sie_gold.c:57-59)
    for (int e = T.tl; e < N * N; e += TS) M[e] = 0.0;
    T.sync();
    if (T.tl == 0) {
        P::rhs(t, c, ys, f);
        P::jac(c, ys, M);
    }
    T.sync();
    if (CTRL == WIND_CTRL_GOLD) {
        // sie_gold.c:17-36: J = -h*J, then diag += 1
        for (int e = T.tl; e < N * N; e += TS) M[e] = (-h * xd(M[e])).v;
        T.sync();
        for (int i = T.tl; i < N; i += TS) M[i * (N + 1)] = (xd(M[i * (N + 1)]) + 1.0).v;
    } else {
        // kernel.cu:49-52: (i==j) - J*h
        for (int e = T.tl; e < N * N; e += TS)
            M[e] = (xd((e / N) == (e % N) ? 1.0 : 0.0) - xd(M[e]) * h).v;
    }
    for (int e = T.tl; e < N * N; e += TS) Inv[e] = (e / N) == (e % N) ? 1.0 : 0.0;
    T.sync();
    // gjeUFactor (gje_gold.c:56-100): scale the pivot row, then eliminate
    // below; each lane owns rows of the elimination
    for (int i = 0; i < N; i++) {
        const xd piv = M[i * N + i];
        T.sync();
        for (int q = T.tl; q < N; q += TS) {
            M[i * N + q] = (xd(M[i * N + q]) / piv).v;
            Inv[i * N + q] = (xd(Inv[i * N + q]) / piv).v;
        }
        T.sync();
        for (int k = i + 1 + T.tl; k < N; k += TS) {
            const xd fk = M[k * N + i];
            for (int q = 0; q < N; q++) {
                M[k * N + q] = (xd(M[k * N + q]) - fk * xd(M[i * N + q])).v;
                Inv[k * N + q] = (xd(Inv[k * N + q]) - fk * xd(Inv[i * N + q])).v;
            }
        }
        T.sync();
    }
    // gjeLFactor (gje_gold.c:102-134): eliminate above, bottom-up
    for (int ri = 0; ri < N; ri++) {
        const int bri = N - 1 - ri;
        for (int bnri = bri - 1 - T.tl; bnri >= 0; bnri -= TS) {
            const xd fk = M[bnri * N + bri];
            for (int q = 0; q < N; q++) {
                M[bnri * N + q] = (xd(M[bnri * N + q]) - fk * xd(M[bri * N + q])).v;
                Inv[bnri * N + q] = (xd(Inv[bnri * N + q]) - fk * xd(Inv[bri * N + q])).v;
            }
        }
        T.sync();
    }
    if (CTRL == WIND_CTRL_GOLD) {
        // matrix_ops.c:6-27, then sie_gold.c:72-74
        for (int r = T.tl; r < N; r += TS) {
            xd acc = 0.0;
            for (int cc = 0; cc < N; cc++) acc += xd(Inv[cc * N + r]) * xd(f[cc]);
            out[r] = acc.v;
        }
        T.sync();
        for (int e = T.tl; e < N; e += TS) ys[e] = (xd(ys[e]) + h * xd(out[e])).v;
    } else {
        // kernel.cu:116-125: y_j += (Inv[k][j]*f_k)*h, k ascending
        for (int j = T.tl; j < N; j += TS) {
            xd yj = ys[j];
            for (int k = 0; k < N; k++) yj += xd(Inv[k * N + j]) * xd(f[k]) * h;
            ys[j] = yj.v;
        }
    }
    T.sync();
}

// One explicit Euler substep (rk2_gold.c:19-46, kernel.cu:128-130).
template <class P>
__device__ __forceinline__ void plugin_euler_substep(const PluginTeam<P>& T, double* ys, double t, xd h) {
    constexpr int N = P::N, TS = PluginTeam<P>::TS;
    using L = typename PluginTeam<P>::L;
    double* f = T.s + L::F;
    if (T.tl == 0) P::rhs(t, T.s + L::C, ys, f);
    T.sync();
    for (int e = T.tl; e < N; e += TS) ys[e] = (xd(ys[e]) + h * xd(f[e])).v;
    T.sync();
}

template <class P, int METHOD, int CTRL>
__device__ __forceinline__ void plugin_substep(const PluginTeam<P>& T, double* ys, double t, double h) {
    if (METHOD == WIND_METHOD_RK2) plugin_euler_substep<P>(T, ys, t, xd(h));
    else plugin_sie_substep<P, CTRL>(T, ys, t, xd(h));
}

template <class P, int METHOD, int CTRL>
__global__ void __launch_bounds__(PLUGIN_THREADS) k_plugin(const KParams p) {
    constexpr int N = P::N, NC = P::NC, TS = PluginTeam<P>::TS;
    constexpr int CAP = Cap<METHOD, CTRL>::value;
    using L = typename PluginTeam<P>::L;
    extern __shared__ double plugin_smem[];
    const int lane = threadIdx.x & 31;
    const int leader = lane - lane % TS;
    const int team = threadIdx.x / TS;
    PluginTeam<P> T;
    T.s = plugin_smem + team * L::SIZE;
    T.tl = lane - leader;
    T.mask = TS == 32 ? 0xffffffffu : (((1u << TS) - 1u) << leader);
    double* y = T.s + L::Y;
    double* y1 = T.s + L::Y1;
    double* y2 = T.s + L::Y2;
    const uint64_t t_start = p.timeout_ns ? global_ns() : 0;
    const double tend = p.tend;
    while (true) {
        unsigned long long ticket = 0;
        if (T.tl == 0) ticket = atomicAdd(&p.counters[CNT_QUEUE], 1ull);
        ticket = __shfl_sync(T.mask, ticket, leader);
        if ((int64_t)ticket >= p.nsys) break;
        const int64_t s = (int64_t)ticket;
        for (int k = T.tl; k < NC; k += TS) T.s[L::C + k] = p.constants[s * p.n_const + k];
        for (int e = T.tl; e < N; e += TS) y[e] = p.y[s * N + e];
        T.sync();
        double t = p.tnow, h = p.h0;
        int u = 0;
        int64_t a = 0;
        int32_t st = WIND_SYS_OK;
        // common_gold.c:77-149 / kernel.cu:191-296
        while (t < tend) {
            if (a >= p.max_attempts) { st |= WIND_SYS_MAX_ATTEMPTS; break; }
            if (p.timeout_ns) {
                const bool late = __shfl_sync(T.mask, T.tl == 0 && global_ns() - t_start > p.timeout_ns, leader);
                if (late) { st |= WIND_SYS_TIMEOUT; break; }
            }
            a++;
            const double hw = fmin(tend - t, h);
            const double t1 = t + hw;
            double hf = (t1 - t) * 1.0;
            double hh = (t1 - t) * 0.5;
            if (CTRL == WIND_CTRL_DEVICE) {
                hf = fmin(t1 - t, hf);
                hh = fmin(t1 - t, hh);
            }
            for (int e = T.tl; e < N; e += TS) { y1[e] = y[e]; y2[e] = y[e]; }
            T.sync();
            plugin_substep<P, METHOD, CTRL>(T, y1, t, hf);
            plugin_substep<P, METHOD, CTRL>(T, y2, t, hh);
            const double tm = t + hh;
            double hh2 = hh;
            if (CTRL == WIND_CTRL_DEVICE) hh2 = fmin(t1 - tm, hh);
            plugin_substep<P, METHOD, CTRL>(T, y2, tm, hh2);
            bool err = false;
            for (int e = T.tl; e < N; e += TS) err |= elem_error<METHOD, CTRL>(xd(y1[e]), xd(y2[e]), p.atol, p.rtol);
            err = __any_sync(T.mask, err);
            if (err && u < CAP) {
                u++;
                h = hw / 2.0;
                continue;
            }
            u = 0;
            for (int e = T.tl; e < N; e += TS)
                y[e] = (METHOD == WIND_METHOD_RK2) ? (xd(2.0) * xd(y2[e]) - xd(y1[e])).v : y2[e];
            T.sync();
            if (t + hw == t) { st |= WIND_SYS_STALLED; break; }
            t += hw;
            // kernel.cu:285-294: RK2 doubles h, SIE goes for gold
            h = (METHOD == WIND_METHOD_RK2) ? hw * 2 : tend - t;
        }
        bool bad = false;
        for (int e = T.tl; e < N; e += TS) {
            bad |= !finite64(y[e]);
            p.y[s * N + e] = y[e];
        }
        if (__any_sync(T.mask, bad)) st |= WIND_SYS_NONFINITE;
        if (T.tl == 0) {
            if (p.sys_status) p.sys_status[s] = st;
            if (p.sys_nsteps) p.sys_nsteps[s] = 3 * a;
            atomicAdd(&p.counters[CNT_STEPS], (unsigned long long)(3 * a));
        }
        T.sync();
    }
}

}  // namespace wind
