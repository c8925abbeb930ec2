// common.cuh -- shared definitions of the B200 integrator kernels.
//
// Arithmetic: every operation that must reproduce the reference's FP64 result
// bit for bit goes through `xd`, whose operators map to the IEEE
// round-to-nearest intrinsics (__dadd_rn, __dmul_rn, ...).  The compiler never
// contracts those into FMA, so a product is rounded before it is added, which
// is what the reference's x86-64 build does.  Division is IEEE-correct in both.
#pragma once

#ifndef __CUDACC_RTC__
#include <cstdint>
#include <cuda_runtime.h>
#endif

#include "../../include/wind.h"

namespace wind {

struct xd {
    double v;
    __device__ __forceinline__ xd() {}
    __device__ __forceinline__ xd(double x) : v(x) {}
    __device__ __forceinline__ operator double() const { return v; }
};
__device__ __forceinline__ xd operator+(xd a, xd b) { return xd(__dadd_rn(a.v, b.v)); }
__device__ __forceinline__ xd operator-(xd a, xd b) { return xd(__dsub_rn(a.v, b.v)); }
__device__ __forceinline__ xd operator*(xd a, xd b) { return xd(__dmul_rn(a.v, b.v)); }
__device__ __forceinline__ xd operator/(xd a, xd b) { return xd(__ddiv_rn(a.v, b.v)); }
__device__ __forceinline__ xd operator-(xd a) { return xd(-a.v); }
__device__ __forceinline__ xd operator+(xd a, double b) { return a + xd(b); }
__device__ __forceinline__ xd operator-(xd a, double b) { return a - xd(b); }
__device__ __forceinline__ xd operator*(xd a, double b) { return a * xd(b); }
__device__ __forceinline__ xd operator/(xd a, double b) { return a / xd(b); }
__device__ __forceinline__ xd operator+(double a, xd b) { return xd(a) + b; }
__device__ __forceinline__ xd operator-(double a, xd b) { return xd(a) - b; }
__device__ __forceinline__ xd operator*(double a, xd b) { return xd(a) * b; }
__device__ __forceinline__ xd& operator+=(xd& a, xd b) { a = a + b; return a; }
__device__ __forceinline__ xd& operator-=(xd& a, xd b) { a = a - b; return a; }
__device__ __forceinline__ xd& operator*=(xd& a, xd b) { a = a * b; return a; }
__device__ __forceinline__ xd& operator/=(xd& a, xd b) { a = a / b; return a; }

// Kernel parameters shared by all kernel families (passed by value).
struct KParams {
    // network
    int32_t kind, n_eq, n_const, n_react;
    const double* constants;
    const double* rates;
    const uint16_t* species;
    const float* linear;
    // integration
    double tnow, tend, h0, atol, rtol;
    double* y;
    int64_t nsys;
    int32_t* sys_status;        // may be null
    int64_t* sys_nsteps;        // may be null
    unsigned long long* counters;  // [0] work queue, [1] substep total, [2] done
    int64_t max_attempts;
    uint64_t timeout_ns;        // 0 = none
    int32_t n_steps;            // n_integration_steps (the fixed-step method's m)
};

// Counter slots in the per-call scratch block.
enum { CNT_QUEUE = 0, CNT_STEPS = 1, CNT_DONE = 2, CNT_SLOTS = 4 };

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool finite64(double x) { return isfinite(x); }

// Reciprocals for the LU and mixed solvers (not bit-exact by design): the
// hardware approximation refined by Newton-Raphson, y <- y + y(1 - b y)
// (Muller et al., Handbook of Floating-Point Arithmetic, 2nd ed., sec. 4.7 /
// 5.3); each step doubles the correct bits.  Stays inline, so the solvers
// need no call frame.  b = 0 gives NaN (a singular pivot).
__device__ __forceinline__ double nr_rcp(double b) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    double e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    return y;
}
__device__ __forceinline__ float nr_rcp(float b) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
    const float e = fmaf(-b, y, 1.0f);
    return fmaf(y, e, y);
}

// |a| as a float bit pattern: monotone for non-negative values, and a NaN
// sorts above +inf, so a max-reduction over these keys never reads a NaN
// correction as small.
__device__ __forceinline__ unsigned fmax_bits(double a) { return __float_as_uint((float)fabs(a)); }

// Refinement cap before an attempt is accepted regardless of its error:
// kernel.cu:259 (RK2 20, SIE 10) for DEVICE, common_gold.c:121 (10) for GOLD.
template <int METHOD, int CTRL>
struct Cap {
    static constexpr int value = (CTRL == WIND_CTRL_DEVICE && METHOD == WIND_METHOD_RK2) ? 20 : 10;
};

// Per-element error test.  DEVICE: kernel.cu:12-39 (strict); GOLD:
// common_gold.c:8-46 ('>=').  Relative denominator y2+1e-12 (SIE) or
// 2*y2-y1+1e-12 (RK2).
template <int METHOD, int CTRL>
__device__ __forceinline__ bool elem_error(xd y1, xd y2, double atol, double rtol) {
    xd d = y2 - y1;
    double ae = fabs(d.v);
    xd den = (METHOD == WIND_METHOD_RK2) ? (xd(2.0) * y2 - y1 + 1e-12) : (y2 + 1e-12);
    double re = fabs((d / den).v);
    bool big = fabs(y1.v) > atol && fabs(y2.v) > atol;
    if (CTRL == WIND_CTRL_GOLD) return (ae >= atol) || (re >= rtol && big);
    return (ae > atol) || (re > rtol && big);
}

}  // namespace wind
