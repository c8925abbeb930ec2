// legacy.cu -- the reference solver libraries' drop-in entry point.
//
//   int cudaIntegrateSystem(float tnow, float tend, int n_integration_steps,
//                           float* constants, float* equations, int Nsystems,
//                           int Nequations_per_system, float ABSOLUTE,
//                           float RELATIVE);
//
// Same C++ linkage and therefore the same exported symbol as the reference
// (cuda/common/harness.cu:5-14, _Z19cudaIntegrateSystemffiPfS_iiff, bound by
// python/wind_harness.py:34,40 and cuda/debug/debug.c:14-17).  One library is
// built per (network, method), as the reference builds lib/sie.so and
// lib/rk2.so per network (cuda/Makefile:13-15, -DSIE / -DRK2).
//
// Semantics kept: host arrays in and out, `equations` updated in place,
// synchronous, returns the substep total (3 per attempt).  Differences, all
// deliberate: the state and the controller run in FP64 (results are rounded
// back to float on return; the reference's FP32 loop can stall when h falls
// below ulp(t)); the constants stride is the network's constant count (the
// reference uses the compile-time NUM_CONST=2 of cuda/include/ode.h:15 for
// every network); on a CUDA failure it returns -1 instead of garbage.
// Environment overrides: WIND_LEGACY_SOLVER = gje_f64 | lu_f64 | mixed,
// WIND_LEGACY_CONTROLLER = device | gold.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/wind.h"
#include "../../include/wind_legacy.h"

#ifndef WIND_LEGACY_NET
#error "WIND_LEGACY_NET must name the network (WIND_NET_*)"
#endif
#ifndef WIND_LEGACY_METHOD
#error "WIND_LEGACY_METHOD must be WIND_METHOD_SIE or WIND_METHOD_RK2"
#endif

static int legacy_n_const(int kind) {
    return kind == WIND_NET_KATZ96 ? 10 : (kind == WIND_NET_NR_TEST ? 4 : 2);
}

#ifdef WIND_LEGACY_HOST
// The SIE_host library: cudaIntegrateSIE with the shared-step controller.
int cudaIntegrateSIE(float tnow, float tend, int n_integration_steps, float* constants,
                     float* equations, int Nsystems, int Neqn_p_sys, float ABSOLUTE, float RELATIVE) {
    if (Nsystems <= 0) return 0;
    const int N = Neqn_p_sys;
    const int nc = legacy_n_const(WIND_LEGACY_NET);
    std::vector<double> c((size_t)Nsystems * nc), y((size_t)Nsystems * N);
    for (size_t i = 0; i < c.size(); i++) c[i] = constants[i];
    for (size_t i = 0; i < y.size(); i++) y[i] = equations[i];
    wind_network net;
    std::memset(&net, 0, sizeof(net));
    net.kind = WIND_LEGACY_NET;
    net.n_eq = N;
    net.n_const = nc;
    net.constants = c.data();
    wind_options o;
    wind_default_options(&o);
    if (const char* s = std::getenv("WIND_LEGACY_SOLVER")) {
        if (!std::strcmp(s, "lu_f64")) o.solver = WIND_SOLVER_LU_F64;
        else if (!std::strcmp(s, "mixed")) o.solver = WIND_SOLVER_MIXED;
        else if (!std::strcmp(s, "auto")) o.solver = WIND_SOLVER_AUTO;
    }
    int64_t total = 0;
    const int st = wind_integrate_global(&o, &net, (double)tnow, (double)tend, n_integration_steps,
                                         y.data(), Nsystems, (double)ABSOLUTE, (double)RELATIVE,
                                         &total, nullptr, WIND_MEM_HOST, nullptr);
    if (st != WIND_OK) return -1;
    for (size_t i = 0; i < y.size(); i++) equations[i] = (float)y[i];
    return (int)total;
}
#else
int cudaIntegrateSystem(float tnow, float tend, int n_integration_steps, float* constants,
                        float* equations, int Nsystems, int Nequations_per_system,
                        float ABSOLUTE, float RELATIVE) {
    if (Nsystems <= 0) return 0;
    const int N = Nequations_per_system;
    const int nc = legacy_n_const(WIND_LEGACY_NET);
    std::vector<double> c((size_t)Nsystems * nc), y((size_t)Nsystems * N);
    for (size_t i = 0; i < c.size(); i++) c[i] = constants[i];
    for (size_t i = 0; i < y.size(); i++) y[i] = equations[i];
    wind_network net;
    std::memset(&net, 0, sizeof(net));
    net.kind = WIND_LEGACY_NET;
    net.n_eq = N;
    net.n_const = nc;
    net.constants = c.data();
    wind_options o;
    wind_default_options(&o);
    o.method = WIND_LEGACY_METHOD;
    if (const char* s = std::getenv("WIND_LEGACY_SOLVER")) {
        if (!std::strcmp(s, "lu_f64")) o.solver = WIND_SOLVER_LU_F64;
        else if (!std::strcmp(s, "mixed")) o.solver = WIND_SOLVER_MIXED;
        else if (!std::strcmp(s, "auto")) o.solver = WIND_SOLVER_AUTO;
    }
    if (const char* s = std::getenv("WIND_LEGACY_CONTROLLER"))
        if (!std::strcmp(s, "gold")) o.controller = WIND_CTRL_GOLD;
    int64_t total = 0;
    const int st = wind_integrate(&o, &net, (double)tnow, (double)tend, n_integration_steps,
                                  y.data(), Nsystems, (double)ABSOLUTE, (double)RELATIVE, nullptr,
                                  nullptr, &total, WIND_MEM_HOST, nullptr);
    if (st != WIND_OK) return -1;
    for (size_t i = 0; i < y.size(); i++) equations[i] = (float)y[i];
    return (int)total;
}
#endif
