// mixed_kernel.cuh -- one persistent launch for a batch of mass-action
// groups of different sizes.
//
// The groups are visited in the order given (largest N first, so the longest
// systems start earliest and the short ones fill the tail).  For each group
// every block works on that group's device work queue -- one system per block
// for N > 32 (cta_run), one system per team of 8/16/32 lanes for N <= 32
// (warp_run for SIE with the LU or mixed solve, team_run otherwise) -- until
// the queue is empty, then moves on to the next group.
// A block that finishes a group early starts the next one while others are
// still on their last systems, so the groups overlap on the device.
#pragma once

#include "cta_kernel.cuh"
#include "team_kernel.cuh"
#include "warp_kernel.cuh"

namespace wind {

constexpr int MIXED_THREADS = CTA_THREADS;

// Two blocks per SM (128 registers) for the LU and mixed solvers, whose team
// and CTA paths fit that budget; the reference Gauss-Jordan keeps a row of M
// and of the inverse per lane in registers and gets the whole file.
// SMALL is the solver of the groups with N <= 32 (SOLVER for the others);
// the AUTO solver runs MIXED above 32 species and LU_F64 below in one launch.
template <int METHOD, int CTRL, int SOLVER, int SMALL = SOLVER>
__global__ void __launch_bounds__(MIXED_THREADS, SOLVER == WIND_SOLVER_GJE_F64 ? 1 : 2)
    k_mixed(const KParams* __restrict__ groups, const int* __restrict__ order, int ngroups,
            double* gscratch, size_t gstride, int smem_cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int gi = 0; gi < ngroups; gi++) {
        const KParams p = groups[order[gi]];
        if (p.nsys > 0) {
            constexpr bool REG = METHOD == WIND_METHOD_SIE && SMALL != WIND_SOLVER_GJE_F64;
            if (p.n_eq > 32) cta_run<METHOD, CTRL, SOLVER, false>(p, smem_raw, gscratch, gstride, smem_cap);
            else if constexpr (REG) {
                if (p.n_eq > 16) warp_run<32, CTRL, SMALL>(p, smem_raw);
                else if (p.n_eq > 8) warp_run<16, CTRL, SMALL>(p, smem_raw);
                else warp_run<8, CTRL, SMALL>(p, smem_raw);
            } else {
                if (p.n_eq > 16) team_run<32, METHOD, CTRL, SOLVER>(p, smem_raw);
                else if (p.n_eq > 8) team_run<16, METHOD, CTRL, SOLVER>(p, smem_raw);
                else team_run<8, METHOD, CTRL, SOLVER>(p, smem_raw);
            }
        }
        __syncthreads();
    }
}

}  // namespace wind
