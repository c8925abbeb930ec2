// dispatch_team.cu -- launch of the team-per-system kernels (mass action,
// N <= 32).
#include <mutex>
#include <vector>

#include "api_internal.h"
#include "team_kernel.cuh"

namespace wind {

using TeamFn = void (*)(KParams);
TeamFn team_fn_8(int method, int ctrl, int solver);
TeamFn team_fn_16(int method, int ctrl, int solver);
TeamFn team_fn_32(int method, int ctrl, int solver);

int team_nmax(int n) { return n <= 8 ? 8 : (n <= 16 ? 16 : 32); }

// The RK2 instantiations are compiled with the GJE_F64 layout (no matrix).
size_t team_smem_bytes(int n, int R, bool lin, int method, int solver) {
    const int nmax = team_nmax(n);
    const int eff = (method == WIND_METHOD_RK2) ? WIND_SOLVER_GJE_F64 : solver;
    return (size_t)(TEAM_THREADS / nmax) * TeamLayout(nmax, R, lin, eff).bytes;
}

static int team_blocks_per_sm(TeamFn fn, size_t smem) {
    static std::mutex mu;
    static std::vector<std::pair<std::pair<const void*, size_t>, int>> cache;
    std::lock_guard<std::mutex> g(mu);
    for (auto& e : cache)
        if (e.first.first == (const void*)fn && e.first.second == smem) return e.second;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, TEAM_THREADS, smem) != cudaSuccess || nb < 1)
        nb = 0;
    cache.push_back({{(const void*)fn, smem}, nb});
    return nb;
}

wind_status launch_warp(const wind_options& o, const KParams& p, cudaStream_t stream);

wind_status launch_team(const wind_options& o, const KParams& p, cudaStream_t stream) {
    // SIE with an LU or mixed solve: the register-resident kernel
    if (o.method == WIND_METHOD_SIE && o.solver != WIND_SOLVER_GJE_F64) return launch_warp(o, p, stream);
    const int nmax = team_nmax(p.n_eq);
    TeamFn fn = nmax == 8 ? team_fn_8(o.method, o.controller, o.solver)
              : nmax == 16 ? team_fn_16(o.method, o.controller, o.solver)
                           : team_fn_32(o.method, o.controller, o.solver);
    const size_t smem = team_smem_bytes(p.n_eq, p.n_react, p.linear != nullptr, o.method, o.solver);
    if (smem > 227 * 1024) return WIND_ERR_UNSUPPORTED;
    const int nb = team_blocks_per_sm(fn, smem);
    if (nb < 1) return WIND_ERR_UNSUPPORTED;
    const int teams = TEAM_THREADS / nmax;
    const int64_t need = (p.nsys + teams - 1) / teams;
    const int64_t cap = (int64_t)nb * device_sm_count();
    const int grid = (int)(need < cap ? need : cap);
    // the attribute is per function, and the cached occupancy above may come
    // from a launch with another size: set it for this launch every time
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return launch_status("k_team shared-memory attribute");
    fn<<<grid, TEAM_THREADS, smem, stream>>>(p);
    g_launches++;
    return launch_status("k_team launch");
}

}  // namespace wind

