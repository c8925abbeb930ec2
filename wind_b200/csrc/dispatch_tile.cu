// dispatch_tile.cu -- instantiations and launch of the tiled-network kernel.
#include <mutex>
#include <vector>

#include "api_internal.h"
#include "tile_kernel.cuh"

namespace wind {

using TileFn = void (*)(KParams, int, int);

template <class Net, int METHOD, int CTRL, int KT>
static TileFn tile_by_solver(int solver) {
    if constexpr (METHOD == WIND_METHOD_RK2) return k_tile<Net, METHOD, CTRL, 0, KT>;
    else {
        switch (solver) {
        case WIND_SOLVER_GJE_F64: return k_tile<Net, METHOD, CTRL, WIND_SOLVER_GJE_F64, KT>;
        case WIND_SOLVER_LU_F64: return k_tile<Net, METHOD, CTRL, WIND_SOLVER_LU_F64, KT>;
        default: return k_tile<Net, METHOD, CTRL, WIND_SOLVER_MIXED, KT>;
        }
    }
}
template <class Net, int KT>
static TileFn tile_for_net(int method, int ctrl, int solver) {
    if (method == WIND_METHOD_SIE)
        return ctrl == WIND_CTRL_GOLD ? tile_by_solver<Net, WIND_METHOD_SIE, WIND_CTRL_GOLD, KT>(solver)
                                      : tile_by_solver<Net, WIND_METHOD_SIE, WIND_CTRL_DEVICE, KT>(solver);
    return ctrl == WIND_CTRL_GOLD ? tile_by_solver<Net, WIND_METHOD_RK2, WIND_CTRL_GOLD, KT>(solver)
                                  : tile_by_solver<Net, WIND_METHOD_RK2, WIND_CTRL_DEVICE, KT>(solver);
}
template <int KT>
static TileFn tile_kernel_kt(int kind, int method, int ctrl, int solver) {
    switch (kind) {
    case WIND_NET_NR_TEST: return tile_for_net<NetNR, KT>(method, ctrl, solver);
    case WIND_NET_KATZ96: return tile_for_net<NetKatz96, KT>(method, ctrl, solver);
    case WIND_NET_STIFFTRIG: return tile_for_net<NetTrig, KT>(method, ctrl, solver);
    default: return nullptr;
    }
}

static int tile_blocks_per_sm(TileFn fn) {
    static std::mutex mu;
    static std::vector<std::pair<const void*, int>> cache;
    std::lock_guard<std::mutex> g(mu);
    for (auto& e : cache)
        if (e.first == (const void*)fn) return e.second;
    int nb = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, TILE_THREADS, 0) != cudaSuccess || nb < 1)
        nb = 1;
    cache.push_back({(const void*)fn, nb});
    return nb;
}

// Team size: the power of two >= Ntile, at most one warp; tiles per lane
// KT = ceil(Ntile / ts) (1 up to 32 tiles, 2 up to 64).
void tile_shape(int ntile, int* ts, int* kt) {
    int t = 1;
    while (t < ntile && t < 32) t *= 2;
    *ts = t;
    *kt = (ntile + t - 1) / t;
}

wind_status launch_tile(const wind_options& o, const KParams& p, int base_n, cudaStream_t stream) {
    const int ntile = p.n_eq / base_n;
    if (ntile < 1 || ntile > WIND_MAX_TILES || ntile * base_n != p.n_eq) return WIND_ERR_UNSUPPORTED;
    int ts = 1, kt = 1;
    tile_shape(ntile, &ts, &kt);
    TileFn fn = kt == 1 ? tile_kernel_kt<1>(p.kind, o.method, o.controller, o.solver)
                        : tile_kernel_kt<2>(p.kind, o.method, o.controller, o.solver);
    if (!fn) return WIND_ERR_UNSUPPORTED;
    const int nb = tile_blocks_per_sm(fn);
    const int64_t resident = (int64_t)nb * device_sm_count();
    const int64_t teams = TILE_THREADS / ts;
    const int64_t need = (p.nsys + teams - 1) / teams;
    const int grid = (int)(need < resident ? need : resident);
    fn<<<grid, TILE_THREADS, 0, stream>>>(p, ntile, ts);
    g_launches++;
    return launch_status("k_tile launch");
}

}  // namespace wind
