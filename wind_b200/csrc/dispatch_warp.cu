// dispatch_warp.cu -- launch of the register-resident team kernels (mass
// action, N <= 32, SIE with the LU_F64 or MIXED solver).
#include <mutex>
#include <vector>

#include "api_internal.h"
#include "warp_kernel.cuh"

namespace wind {

using WarpFn = void (*)(KParams);

template <int NMAX, int CTRL>
static WarpFn warp_by_solver(int solver) {
    return solver == WIND_SOLVER_MIXED ? k_warp<NMAX, CTRL, WIND_SOLVER_MIXED>
                                       : k_warp<NMAX, CTRL, WIND_SOLVER_LU_F64>;
}

template <int NMAX>
static WarpFn warp_fn(int ctrl, int solver) {
    return ctrl == WIND_CTRL_GOLD ? warp_by_solver<NMAX, WIND_CTRL_GOLD>(solver)
                                  : warp_by_solver<NMAX, WIND_CTRL_DEVICE>(solver);
}

int warp_nmax(int n) { return n <= 8 ? 8 : (n <= 16 ? 16 : 32); }

// Shared memory of a block of `threads` threads running teams for N = n.
size_t warp_smem_bytes(int n, int R, bool lin, int solver, int threads) {
    const int nmax = warp_nmax(n);
    return (size_t)(threads / nmax) * WarpLayout(nmax, R, lin, solver).bytes;
}

// Resident blocks per SM of `fn` at `threads` threads and `smem` bytes.
static int warp_blocks_per_sm(WarpFn fn, int threads, size_t smem) {
    static std::mutex mu;
    static std::vector<std::pair<std::pair<const void*, size_t>, std::pair<int, int>>> cache;
    std::lock_guard<std::mutex> g(mu);
    for (auto& e : cache)
        if (e.first.first == (const void*)fn && e.first.second == smem && e.second.first == threads)
            return e.second.second;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess || nb < 1) {
        (void)cudaGetLastError();
        nb = 0;
    }
    cache.push_back({{(const void*)fn, smem}, {threads, nb}});
    return nb;
}

wind_status launch_warp(const wind_options& o, const KParams& p, cudaStream_t stream) {
    const int nmax = warp_nmax(p.n_eq);
    WarpFn fn = nmax == 8 ? warp_fn<8>(o.controller, o.solver)
              : nmax == 16 ? warp_fn<16>(o.controller, o.solver)
                           : warp_fn<32>(o.controller, o.solver);
    const int threads = WARP_THREADS;
    const size_t smem = warp_smem_bytes(p.n_eq, p.n_react, p.linear != nullptr, o.solver, threads);
    if (smem > 227 * 1024) return WIND_ERR_UNSUPPORTED;
    const int nb = warp_blocks_per_sm(fn, threads, smem);
    if (nb < 1) return WIND_ERR_UNSUPPORTED;
    const int teams = threads / nmax;
    const int64_t need = (p.nsys + teams - 1) / teams;
    const int64_t cap = (int64_t)nb * device_sm_count();
    const int grid = (int)(need < cap ? need : cap);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return launch_status("k_warp shared-memory attribute");
    fn<<<grid, threads, smem, stream>>>(p);
    g_launches++;
    return launch_status("k_warp launch");
}

}  // namespace wind
