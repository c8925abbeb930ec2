// dispatch_lane.cu -- instantiations and launch of the thread-per-system
// kernels (builtin networks).
#include <mutex>
#include <vector>

#include "api_internal.h"
#include "lane_kernel.cuh"

namespace wind {

using LaneFn = void (*)(KParams, int);

template <class Net, int METHOD, int CTRL>
static LaneFn lane_by_solver(int solver) {
    if constexpr (METHOD == WIND_METHOD_RK2) return k_lane<Net, METHOD, CTRL, 0>;
    else {
        switch (solver) {
        case WIND_SOLVER_GJE_F64: return k_lane<Net, METHOD, CTRL, WIND_SOLVER_GJE_F64>;
        case WIND_SOLVER_LU_F64: return k_lane<Net, METHOD, CTRL, WIND_SOLVER_LU_F64>;
        default: return k_lane<Net, METHOD, CTRL, WIND_SOLVER_MIXED>;
        }
    }
}
template <class Net>
static LaneFn lane_for_net(int method, int ctrl, int solver) {
    if (method == WIND_METHOD_SIE)
        return ctrl == WIND_CTRL_GOLD ? lane_by_solver<Net, WIND_METHOD_SIE, WIND_CTRL_GOLD>(solver)
                                      : lane_by_solver<Net, WIND_METHOD_SIE, WIND_CTRL_DEVICE>(solver);
    return ctrl == WIND_CTRL_GOLD ? lane_by_solver<Net, WIND_METHOD_RK2, WIND_CTRL_GOLD>(solver)
                                  : lane_by_solver<Net, WIND_METHOD_RK2, WIND_CTRL_DEVICE>(solver);
}
static LaneFn lane_kernel(int kind, int method, int ctrl, int solver) {
    switch (kind) {
    case WIND_NET_NR_TEST: return lane_for_net<NetNR>(method, ctrl, solver);
    case WIND_NET_KATZ96: return lane_for_net<NetKatz96>(method, ctrl, solver);
    case WIND_NET_STIFFTRIG: return lane_for_net<NetTrig>(method, ctrl, solver);
    default: return nullptr;
    }
}


static int lane_blocks_per_sm(LaneFn fn) {
    static std::mutex mu;
    static std::vector<std::pair<const void*, int>> cache;
    std::lock_guard<std::mutex> g(mu);
    for (auto& e : cache)
        if (e.first == (const void*)fn) return e.second;
    int nb = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, LANE_THREADS, 0) != cudaSuccess || nb < 1)
        nb = 1;
    cache.push_back({(const void*)fn, nb});
    return nb;
}

// Initial lanes per system: 1 when the batch fills the resident lanes, more
// (a power of two up to the refinement depth) for small batches.  Helpers
// beyond it still join when the queue drains.
int choose_width(int64_t nsys, int slots, int method, int ctrl) {
    const int cap = (ctrl == WIND_CTRL_DEVICE && method == WIND_METHOD_RK2) ? 20 : 10;
    const int wmax = cap >= 16 ? 32 : 16;
    int w = 1;
    while (w < wmax && nsys * (int64_t)(2 * w) <= (int64_t)slots) w *= 2;
    return w;
}

wind_status launch_lane(const wind_options& o, const KParams& p, cudaStream_t stream) {
    LaneFn fn = lane_kernel(p.kind, o.method, o.controller, o.solver);
    if (!fn) return WIND_ERR_UNSUPPORTED;
    const int nb = lane_blocks_per_sm(fn);
    const int64_t resident = (int64_t)nb * device_sm_count();  // blocks
    const int slots = (int)(resident * LANE_THREADS);
    int w = o.spec_width;
    if (w <= 0) w = choose_width(p.nsys, slots, o.method, o.controller);
    if (w != 1 && w != 2 && w != 4 && w != 8 && w != 16 && w != 32) return WIND_ERR_ARGUMENT;
    const int opw = 32 / w;
    const int64_t warps = (p.nsys + opw - 1) / opw;
    const int64_t need = (warps + LANE_THREADS / 32 - 1) / (LANE_THREADS / 32);
    const int grid = (int)(need < resident ? need : resident);
    fn<<<grid, LANE_THREADS, 0, stream>>>(p, opw);
    g_launches++;
    return launch_status("k_lane launch");
}

}  // namespace wind
