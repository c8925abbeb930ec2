/*
 * wind_legacy.h -- the reference solver libraries' entry point, unchanged.
 *
 * Declared with C++ linkage on purpose: the reference exports it mangled as
 * _Z19cudaIntegrateSystemffiPfS_iiff (cuda/common/harness.cu:5-14) and its
 * callers look it up by that name (python/wind_harness.py:34,40;
 * cuda/debug/debug.c:14,17).  Built once per (network, method) into
 * wind_b200/lib/<network>/{sie,rk2}.so, like the reference's lib/sie.so and
 * lib/rk2.so (cuda/Makefile:13-15).
 *
 * Replaces cudaIntegrateSystem of cuda/common/harness.cu:5-106: integrates
 * Nsystems systems of Nequations_per_system equations from tnow to tend
 * with initial step (tend-tnow)/n_integration_steps; constants[s*NC + k]
 * (NC = the network's constant count), equations[s*N + i] updated in place;
 * returns the total substep count (3 per attempt), or -1 on a CUDA failure.
 */
#ifndef WIND_LEGACY_H
#define WIND_LEGACY_H

#ifdef __cplusplus
int cudaIntegrateSystem(float tnow, float tend, int n_integration_steps,
                        float* constants, float* equations, int Nsystems,
                        int Nequations_per_system, float ABSOLUTE, float RELATIVE);

/* Replaces cudaIntegrateSIE of cuda/SIE_host/harness_kernel.cu:427-532
 * (exported mangled as _Z16cudaIntegrateSIEffiPfS_iiff, looked up by
 * python/wind_harness.py:27-28), built into wind_b200/lib/<network>/sie_host.so
 * like the reference's lib/sie_host.so: the same arguments as
 * cudaIntegrateSystem, one step shared by all systems (wind_integrate_global
 * in wind.h), returns the substep count per system times Nsystems, or -1 on
 * a CUDA failure. */
int cudaIntegrateSIE(float tnow, float tend, int n_integration_steps, float* constants,
                     float* equations, int Nsystems, int Neqn_p_sys, float ABSOLUTE,
                     float RELATIVE);
#endif

#endif /* WIND_LEGACY_H */
