/* Mass-action host plug-in for the reference CPU twin, against the host
 * contract of cuda/include/ode_gold.h:1-12.  The reference ships no such
 * network; this lets its own integrator (cuda/c_baseline) run the synthetic
 * dense and mixed-size networks.  Test infrastructure only (built by
 * oracle/build_ref.sh with -DMA_N, -DMA_R, -DMA_LINEAR).
 *
 * Per-system constants (NUM_CONST = 5*MA_R + MA_LINEAR*MA_N*MA_N):
 *   [0, R)          rate k_r
 *   [R, 5R)         species A,B,C,D of reaction r at R + 4r + q
 *   [5R, 5R+N*N)    dense linear term L (row-major, f_j += L_jk y_k)
 * Operation order is the one documented for WIND_NET_MASS_ACTION. */
#include "ode_gold.h"

#ifndef MA_LINEAR
#define MA_LINEAR 0
#endif

void calculate_dydt(float tnow, float *equations, float *constants,
                    float *dydt, int Neqn_p_sys) {
    const float *rates = constants;
    const float *sp = constants + MA_R;
    for (int j = 0; j < MA_N; j++) {
        float acc = 0.0;
#if MA_LINEAR
        const float *L = constants + 5 * MA_R;
        for (int q = 0; q < MA_N; q++) acc += L[j * MA_N + q] * equations[q];
#endif
        dydt[j] = acc;
    }
    for (int r = 0; r < MA_R; r++) {
        int a = (int)sp[4 * r], b = (int)sp[4 * r + 1];
        int c = (int)sp[4 * r + 2], d = (int)sp[4 * r + 3];
        float w = rates[r] * equations[a] * equations[b];
        dydt[a] -= w;
        dydt[b] -= w;
        dydt[c] += w;
        dydt[d] += w;
    }
}

void calculate_jacobian(float *equations, float *constants, float *Jacobian) {
    const float *rates = constants;
    const float *sp = constants + MA_R;
#if MA_LINEAR
    const float *L = constants + 5 * MA_R;
    for (int i = 0; i < MA_N; i++)
        for (int j = 0; j < MA_N; j++) Jacobian[i * MA_N + j] = L[j * MA_N + i];
#endif
    for (int r = 0; r < MA_R; r++) {
        int a = (int)sp[4 * r], b = (int)sp[4 * r + 1];
        int c = (int)sp[4 * r + 2], d = (int)sp[4 * r + 3];
        float da = rates[r] * equations[b];
        float db = rates[r] * equations[a];
        Jacobian[a * MA_N + a] -= da;
        Jacobian[a * MA_N + b] -= da;
        Jacobian[a * MA_N + c] += da;
        Jacobian[a * MA_N + d] += da;
        Jacobian[b * MA_N + a] -= db;
        Jacobian[b * MA_N + b] -= db;
        Jacobian[b * MA_N + c] += db;
        Jacobian[b * MA_N + d] += db;
    }
}
