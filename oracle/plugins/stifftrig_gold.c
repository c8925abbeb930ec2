/* StiffTrig host plug-in for the reference CPU twin, against the host
 * contract of cuda/include/ode_gold.h:1-12; body as generated by
 * python/ode_systems/stifftrig.py:625-647 for Ntile=1.  Test infrastructure
 * only (built by oracle/build_ref.sh). */
#include "ode_gold.h"

void calculate_dydt(float tnow, float *equations, float *constants,
                    float *dydt, int Neqn_p_sys) {
    dydt[0] = -equations[0] + constants[1] * equations[1];
    dydt[1] = -equations[1] - constants[0] * equations[0];
}

void calculate_jacobian(float *equations, float *constants, float *Jacobian) {
    Jacobian[0] = -1;
    Jacobian[2] = constants[1];
    Jacobian[1] = -constants[0];
    Jacobian[3] = -1;
}
