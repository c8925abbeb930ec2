// networks.cuh -- device ode_system plug-ins.
//
// Contract (the reference's, cuda/include/device.h:1-13 and
// cuda/include/ode_gold.h:1-12, restated for FP64 and whole systems):
//   rhs(c, y, f)   f[j] = dy_j/dt
//   jac(c, y, J)   J[i*N + j] = d f_j / d y_i  (transposed, reference layout),
//                  writing only the nonzeros into a zero-filled J.
// Builtin networks have a compile-time N so their state lives in registers.
// Expression order follows the reference bodies exactly (bit-exact parity).
#pragma once

#include "common.cuh"

namespace wind {

// NR 16.6.1 test, python/ode_systems/NR_test.py:575-603 (generated bodies).
struct NetNR {
    static constexpr int N = 2;
    static constexpr int NC = 4;
    template <class C, class Y, class F>
    __device__ __forceinline__ static void rhs(const C& c, const Y& y, F& f) {
        f[0] = xd(c[0]) * y[0] + xd(c[1]) * y[1];
        f[1] = xd(c[2]) * y[0] + xd(c[3]) * y[1];
    }
    template <class C, class Y, class J>
    __device__ __forceinline__ static void jac(const C& c, const Y& y, J& M) {
        M[0] = c[0];
        M[1] = c[2];
        M[2] = c[1];
        M[3] = c[3];
    }
};

// StiffTrig, python/ode_systems/stifftrig.py:625-661.
struct NetTrig {
    static constexpr int N = 2;
    static constexpr int NC = 2;
    template <class C, class Y, class F>
    __device__ __forceinline__ static void rhs(const C& c, const Y& y, F& f) {
        f[0] = -y[0] + xd(c[1]) * y[1];
        f[1] = -y[1] - xd(c[0]) * y[0];
    }
    template <class C, class Y, class J>
    __device__ __forceinline__ static void jac(const C& c, const Y& y, J& M) {
        M[0] = -1.0;
        M[2] = c[1];
        M[1] = -c[0];
        M[3] = -1.0;
    }
};

// Katz96 primordial H/He network, cuda/ode_system/ode_gold.c:3-93 and
// cuda/ode_system/device_dydt.cu:4-114.  J[13] = J[12] is the reference's
// sign (ode_gold.c:79); it is kept so results match the reference.
struct NetKatz96 {
    static constexpr int N = 5;
    static constexpr int NC = 10;
    template <class C, class Y, class F>
    __device__ __forceinline__ static void rhs(const C& cc, const Y& y, F& f) {
        xd c[10];
#pragma unroll
        for (int k = 0; k < 10; k++) c[k] = cc[k];
        xd ne = y[1] + y[3] + y[4] * 2.0;
        f[0] = c[2] * ne * y[1] - (c[0] * ne + c[1]) * y[0];
        f[1] = -c[2] * ne * y[1] + (c[0] * ne + c[1]) * y[0];
        f[2] = (c[7] + c[8]) * ne * y[3] - (c[3] * ne + c[4]) * y[2];
        f[3] = c[9] * ne * y[4] + (c[3] * ne + c[4]) * y[2] - (c[7] + c[8]) * ne * y[3] -
               (c[5] * ne + c[6]) * y[3];
        f[4] = (c[5] * ne + c[6]) * y[3] - c[9] * ne * y[4];
    }
    template <class C, class Y, class J>
    __device__ __forceinline__ static void jac(const C& cc, const Y& y, J& M) {
        xd c[10];
#pragma unroll
        for (int k = 0; k < 10; k++) c[k] = cc[k];
        xd ne = y[1] + y[3] + y[4] * 2.0;
        M[0] = -(c[0] * ne + c[1]);
        M[1] = -xd(M[0]);
        M[6] = -c[2] * ne;
        M[5] = -xd(M[6]);
        M[12] = -(c[3] * ne + c[4]);
        M[13] = M[12];
        M[19] = c[5] * ne + c[6];
        M[17] = (c[7] + c[8]) * ne;
        M[18] = -xd(M[17]) - xd(M[19]);
        M[24] = -c[9] * ne;
        M[23] = -xd(M[24]);
    }
};

// ---------------------------------------------------------------------------
// Mass action (runtime network).  Operation order, shared with the oracle:
//   f_j  = sum_k L_jk y_k  (k ascending from 0.0), then for r ascending with
//   w = (k_r*y_A)*y_B:  f_A -= w; f_B -= w; f_C += w; f_D += w.
//   Jt_ij = L_ji, then for r ascending, dA = k_r*y_B, dB = k_r*y_A:
//   Jt[A][A]-=dA; Jt[A][B]-=dA; Jt[A][C]+=dA; Jt[A][D]+=dA;
//   Jt[B][A]-=dB; Jt[B][B]-=dB; Jt[B][C]+=dB; Jt[B][D]+=dB.
// The team kernels evaluate one column j per lane: the per-element update
// sequence is the sequential one restricted to that element.
// ---------------------------------------------------------------------------
struct Reaction {
    double k;
    int a, b, c, d;
};

}  // namespace wind
