// dispatch_team16.cu -- team kernels with NMAX = 16 (one file per NMAX so
// the instantiations compile in parallel).
#include "api_internal.h"
#include "team_kernel.cuh"

namespace wind {

using TeamFn = void (*)(KParams);

template <int NMAX, int METHOD, int CTRL>
static TeamFn team_by_solver(int solver) {
    if constexpr (METHOD == WIND_METHOD_RK2) return k_team<NMAX, METHOD, CTRL, 0>;
    else {
        switch (solver) {
        case WIND_SOLVER_GJE_F64: return k_team<NMAX, METHOD, CTRL, WIND_SOLVER_GJE_F64>;
        case WIND_SOLVER_LU_F64: return k_team<NMAX, METHOD, CTRL, WIND_SOLVER_LU_F64>;
        default: return k_team<NMAX, METHOD, CTRL, WIND_SOLVER_MIXED>;
        }
    }
}

TeamFn team_fn_16(int method, int ctrl, int solver) {
    if (method == WIND_METHOD_SIE)
        return ctrl == WIND_CTRL_GOLD ? team_by_solver<16, WIND_METHOD_SIE, WIND_CTRL_GOLD>(solver)
                                      : team_by_solver<16, WIND_METHOD_SIE, WIND_CTRL_DEVICE>(solver);
    return ctrl == WIND_CTRL_GOLD ? team_by_solver<16, WIND_METHOD_RK2, WIND_CTRL_GOLD>(solver)
                                  : team_by_solver<16, WIND_METHOD_RK2, WIND_CTRL_DEVICE>(solver);
}

}  // namespace wind
