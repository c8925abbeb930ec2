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
// sign (ode_gold.c:79); it is kept so results match the reference.  The
// electron density ne is computed once per evaluation (the generated
// prefix, python/ode_systems/katz96.py:485-500) and passed to the bodies, so
// a tile of a tiled network can take tile 0's ne with the same arithmetic.
struct NetKatz96 {
    static constexpr int N = 5;
    static constexpr int NC = 10;
    template <class Y>
    __device__ __forceinline__ static xd ne_of(const Y& y) {
        return y[1] + y[3] + y[4] * 2.0;
    }
    template <class C, class Y, class F>
    __device__ __forceinline__ static void rhs_ne(const C& cc, xd ne, const Y& y, F& f) {
        xd c[10];
#pragma unroll
        for (int k = 0; k < 10; k++) c[k] = cc[k];
        f[0] = c[2] * ne * y[1] - (c[0] * ne + c[1]) * y[0];
        f[1] = -c[2] * ne * y[1] + (c[0] * ne + c[1]) * y[0];
        f[2] = (c[7] + c[8]) * ne * y[3] - (c[3] * ne + c[4]) * y[2];
        f[3] = c[9] * ne * y[4] + (c[3] * ne + c[4]) * y[2] - (c[7] + c[8]) * ne * y[3] -
               (c[5] * ne + c[6]) * y[3];
        f[4] = (c[5] * ne + c[6]) * y[3] - c[9] * ne * y[4];
    }
    template <class C, class J>
    __device__ __forceinline__ static void jac_ne(const C& cc, xd ne, J& M) {
        xd c[10];
#pragma unroll
        for (int k = 0; k < 10; k++) c[k] = cc[k];
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
    template <class C, class Y, class F>
    __device__ __forceinline__ static void rhs(const C& cc, const Y& y, F& f) {
        rhs_ne(cc, ne_of(y), y, f);
    }
    template <class C, class Y, class J>
    __device__ __forceinline__ static void jac(const C& cc, const Y& y, J& M) {
        jac_ne(cc, ne_of(y), M);
    }
};

// ---------------------------------------------------------------------------
// Tiled builtin networks (python/ode_systems/ode_base.py:86-88, 219-281, the
// Precompiler's Ntile): one system of Ntile x N equations made of Ntile
// copies of the network, tile t owning equations [tN, tN + N), every tile
// reading the system's one set of constants; the Jacobian is block diagonal
// (reindex, ode_base.py:86-88).  Katz96's generated prefix computes ne from
// equations 1, 3 and 4 -- tile 0 -- and every tile's body uses it
// (katz96.py:331-448 reindex only the bodies).  TileOf<Net>::Tile is the
// functor one tile integrates with; for Katz96 it reads ne from constant
// slot 10, which the kernel fills with tile 0's ne before each evaluation.
// ---------------------------------------------------------------------------
struct NetKatz96Tile {
    static constexpr int N = 5;
    static constexpr int NC = 11;
    template <class C, class Y, class F>
    __device__ __forceinline__ static void rhs(const C& cc, const Y& y, F& f) {
        NetKatz96::rhs_ne(cc, xd(cc[10]), y, f);
    }
    template <class C, class Y, class J>
    __device__ __forceinline__ static void jac(const C& cc, const Y& y, J& M) {
        NetKatz96::jac_ne(cc, xd(cc[10]), M);
    }
};

template <class Net>
struct TileOf {
    using Tile = Net;
    static constexpr bool coupled = false;
    template <class Y>
    __device__ __forceinline__ static double shared(const Y&) { return 0.0; }
};
template <>
struct TileOf<NetKatz96> {
    using Tile = NetKatz96Tile;
    static constexpr bool coupled = true;
    template <class Y>
    __device__ __forceinline__ static double shared(const Y& y) { return NetKatz96::ne_of(y).v; }
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
