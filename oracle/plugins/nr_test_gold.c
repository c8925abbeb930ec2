/* NR_test host plug-in for the reference CPU twin (cuda/c_baseline), written
 * against the reference's host contract (cuda/include/ode_gold.h:1-12).  The
 * body is what the reference's generator emits for Ntile=1
 * (python/ode_systems/NR_test.py:575-590).  Test infrastructure only: it is
 * compiled into oracle/_ref by oracle/build_ref.sh. */
#include "ode_gold.h"

void calculate_dydt(float tnow, float *equations, float *constants,
                    float *dydt, int Neqn_p_sys) {
    dydt[0] = constants[0] * equations[0] + constants[1] * equations[1];
    dydt[1] = constants[2] * equations[0] + constants[3] * equations[1];
}

void calculate_jacobian(float *equations, float *constants, float *Jacobian) {
    Jacobian[0] = constants[0];
    Jacobian[1] = constants[2];
    Jacobian[2] = constants[1];
    Jacobian[3] = constants[3];
}
