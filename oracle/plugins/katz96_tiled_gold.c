/* Katz96 tiled NTILE times, host plug-in for the reference CPU twin
 * (cuda/c_baseline), written against the reference's host contract
 * (cuda/include/ode_gold.h:1-12).  It is what the reference's Precompiler
 * emits for Ntile = NTILE (python/ode_systems/ode_base.py:54-94,
 * katz96.py:331-400): the prefix computes ne once from equations 1, 3 and 4
 * (tile 0, katz96.py:485-500), then each tile's RHS lines
 * (make_derivative_block, ridx(x) = x + 5*tile) and Jacobian lines
 * (make_jacobian_block, reindex ode_base.py:86-88: base entry r*5+q lands at
 * (5*tile + r)*N + 5*tile + q) with the same expressions as the untiled body
 * (cuda/ode_system/ode_gold.c:3-93).  Test infrastructure only: compiled into
 * oracle/_ref by oracle/build_ref.sh. */
#include "ode_gold.h"

#ifndef NTILE
#error "NTILE must be defined"
#endif
#define NEQ (5 * NTILE)

void calculate_dydt(float tnow, float *equations, float *constants,
                    float *dydt, int Neqn_p_sys) {
    float ne = equations[1] + equations[3] + equations[4] * 2.0;
    for (int t = 0; t < NTILE; t++) {
        float *y = equations + 5 * t;
        float *f = dydt + 5 * t;
        f[0] = constants[2] * ne * y[1] - (constants[0] * ne + constants[1]) * y[0];
        f[1] = -constants[2] * ne * y[1] + (constants[0] * ne + constants[1]) * y[0];
        f[2] = (constants[7] + constants[8]) * ne * y[3] - (constants[3] * ne + constants[4]) * y[2];
        f[3] = constants[9] * ne * y[4] + (constants[3] * ne + constants[4]) * y[2]
             - (constants[7] + constants[8]) * ne * y[3] - (constants[5] * ne + constants[6]) * y[3];
        f[4] = (constants[5] * ne + constants[6]) * y[3] - constants[9] * ne * y[4];
    }
}

void calculate_jacobian(float *equations, float *constants, float *Jacobian) {
    float ne = equations[1] + equations[3] + equations[4] * 2.0;
    for (int t = 0; t < NTILE; t++) {
        float *J = Jacobian + 5 * t * NEQ + 5 * t;   /* the tile's diagonal block */
        J[0] = -(constants[0] * ne + constants[1]);
        J[1] = -J[0];
        J[NEQ + 1] = -constants[2] * ne;
        J[NEQ + 0] = -J[NEQ + 1];
        J[2 * NEQ + 2] = -(constants[3] * ne + constants[4]);
        J[2 * NEQ + 3] = J[2 * NEQ + 2];
        J[3 * NEQ + 4] = constants[5] * ne + constants[6];
        J[3 * NEQ + 2] = (constants[7] + constants[8]) * ne;
        J[3 * NEQ + 3] = -J[3 * NEQ + 2] - J[3 * NEQ + 4];
        J[4 * NEQ + 4] = -constants[9] * ne;
        J[4 * NEQ + 3] = -J[4 * NEQ + 4];
    }
}
