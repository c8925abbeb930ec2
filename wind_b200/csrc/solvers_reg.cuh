// solvers_reg.cuh -- register-resident linear solves for small compile-time N
// (one thread owns a whole system).  All loops unroll, so the matrices stay in
// registers.
#pragma once

#include "common.cuh"

namespace wind {

// The reference's unpivoted Gauss-Jordan inverse of M (row-major), same
// operation order as cuda/c_baseline/linear_algebra/gje_gold.c:5-144 and
// cuda/linear_algebra/gauss_jordan_elimination.cu:15-212: per pivot row, every
// element of the row of M and of Inv is divided by the saved pivot; rows below
// (U phase) then rows above (L phase, bottom-up) subtract factor*pivot row
// over the full width.
template <int N>
__device__ __forceinline__ void gje_invert_reg(xd (&M)[N * N], xd (&Inv)[N * N]) {
#pragma unroll
    for (int e = 0; e < N * N; e++) Inv[e] = 0.0;
#pragma unroll
    for (int i = 0; i < N; i++) Inv[i * (N + 1)] = 1.0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        xd s = M[i * N + i];
#pragma unroll
        for (int t = 0; t < N; t++) M[i * N + t] /= s;
#pragma unroll
        for (int t = 0; t < N; t++) Inv[i * N + t] /= s;
#pragma unroll
        for (int k = i + 1; k < N; k++) {
            xd f = M[k * N + i];
#pragma unroll
            for (int t = 0; t < N; t++) M[k * N + t] -= f * M[i * N + t];
#pragma unroll
            for (int t = 0; t < N; t++) Inv[k * N + t] -= f * Inv[i * N + t];
        }
    }
#pragma unroll
    for (int ri = 0; ri < N; ri++) {
        const int bri = N - 1 - ri;
#pragma unroll
        for (int nri = ri + 1; nri < N; nri++) {
            const int bnri = N - 1 - nri;
            xd f = M[bnri * N + bri];
#pragma unroll
            for (int t = 0; t < N; t++) M[bnri * N + t] -= f * M[bri * N + t];
#pragma unroll
            for (int t = 0; t < N; t++) Inv[bnri * N + t] -= f * Inv[bri * N + t];
        }
    }
}

// Partial-pivot LU factorisation of A (row-major, standard orientation) in
// place, with the row swaps applied as predicated selects so indexing stays
// static.  Returns the reciprocal pivots in `rinv` and applies the same row
// permutation to the right-hand sides through `perm` (perm[i] = original row).
template <int N, typename T>
__device__ __forceinline__ void lu_factor_reg(T (&A)[N * N], T (&rinv)[N], int (&perm)[N]) {
#pragma unroll
    for (int i = 0; i < N; i++) perm[i] = i;
#pragma unroll
    for (int i = 0; i < N; i++) {
        int p = i;
        T best = fabs(A[i * N + i]);
#pragma unroll
        for (int k = i + 1; k < N; k++) {
            T v = fabs(A[k * N + i]);
            if (v > best) { best = v; p = k; }
        }
#pragma unroll
        for (int k = i + 1; k < N; k++) {
            const bool sw = (p == k);
#pragma unroll
            for (int t = 0; t < N; t++) {
                T a = A[i * N + t], b = A[k * N + t];
                A[i * N + t] = sw ? b : a;
                A[k * N + t] = sw ? a : b;
            }
            int pa = perm[i], pb = perm[k];
            perm[i] = sw ? pb : pa;
            perm[k] = sw ? pa : pb;
        }
        T r = nr_rcp(A[i * N + i]);
        rinv[i] = r;
#pragma unroll
        for (int k = i + 1; k < N; k++) {
            T l = A[k * N + i] * r;
            A[k * N + i] = l;
#pragma unroll
            for (int t = i + 1; t < N; t++) A[k * N + t] = fma(-l, A[i * N + t], A[k * N + t]);
        }
    }
}

// Solve with the factors from lu_factor_reg: x = A^-1 b (b in original row
// order, x in place of b).
template <int N, typename T, typename B>
__device__ __forceinline__ void lu_solve_reg(const T (&A)[N * N], const T (&rinv)[N],
                                             const int (&perm)[N], B (&b)[N]) {
    B z[N];
    // permute: z[i] = b[perm[i]] via selects
#pragma unroll
    for (int i = 0; i < N; i++) {
        B v = b[0];
#pragma unroll
        for (int q = 1; q < N; q++) v = (perm[i] == q) ? b[q] : v;
        z[i] = v;
    }
    // forward (unit lower)
#pragma unroll
    for (int i = 1; i < N; i++) {
        B acc = z[i];
#pragma unroll
        for (int t = 0; t < i; t++) acc = fma(-(B)A[i * N + t], z[t], acc);
        z[i] = acc;
    }
    // backward
#pragma unroll
    for (int i = N - 1; i >= 0; i--) {
        B acc = z[i];
#pragma unroll
        for (int t = i + 1; t < N; t++) acc = fma(-(B)A[i * N + t], z[t], acc);
        z[i] = acc * (B)rinv[i];
    }
#pragma unroll
    for (int i = 0; i < N; i++) b[i] = z[i];
}

}  // namespace wind
