// dispatch_mixed.cu -- the single persistent launch over mass-action groups.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "api_internal.h"
#include "mixed_kernel.cuh"

namespace wind {

using MixedFn = void (*)(const KParams*, const int*, int, double*, size_t, int);

template <int METHOD, int CTRL>
static MixedFn mixed_by_solver(int solver) {
    if constexpr (METHOD == WIND_METHOD_RK2) return k_mixed<METHOD, CTRL, WIND_SOLVER_LU_F64>;
    else {
        switch (solver) {
        case WIND_SOLVER_GJE_F64: return k_mixed<METHOD, CTRL, WIND_SOLVER_GJE_F64>;
        case WIND_SOLVER_LU_F64: return k_mixed<METHOD, CTRL, WIND_SOLVER_LU_F64>;
        case WIND_SOLVER_AUTO: return k_mixed<METHOD, CTRL, WIND_SOLVER_MIXED, WIND_SOLVER_LU_F64>;
        default: return k_mixed<METHOD, CTRL, WIND_SOLVER_MIXED>;
        }
    }
}

static MixedFn mixed_fn(int method, int ctrl, int solver) {
    if (method == WIND_METHOD_SIE)
        return ctrl == WIND_CTRL_GOLD ? mixed_by_solver<WIND_METHOD_SIE, WIND_CTRL_GOLD>(solver)
                                      : mixed_by_solver<WIND_METHOD_SIE, WIND_CTRL_DEVICE>(solver);
    return ctrl == WIND_CTRL_GOLD ? mixed_by_solver<WIND_METHOD_RK2, WIND_CTRL_GOLD>(solver)
                                  : mixed_by_solver<WIND_METHOD_RK2, WIND_CTRL_DEVICE>(solver);
}

static int nmax_of(int n) { return n <= 8 ? 8 : (n <= 16 ? 16 : 32); }

// Launch all mass-action groups `ps` (kernel parameters with their counters
// already set) in one kernel on `stream`.
wind_status launch_mixed(const wind_options& o, const std::vector<KParams>& ps, cudaStream_t stream) {
    if (ps.empty()) return WIND_OK;
    const int solver = (o.method == WIND_METHOD_RK2) ? WIND_SOLVER_LU_F64 : o.solver;
    int dev = 0, cap = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cap -= 1024;
    size_t smem = 0, gslot = 0;
    for (const KParams& p : ps) {
        // the solver each group runs (AUTO: MIXED above 32 species, LU_F64 below)
        const int gs = resolve_solver(solver, p.kind, p.n_eq);
        if (p.n_eq > 32) {
            const CtaLayout lay(p.n_eq, p.n_react, p.linear != nullptr, gs, cap);
            smem = std::max(smem, (size_t)lay.bytes);
            gslot = std::max(gslot, lay.g_doubles);
        } else {
            const int nm = nmax_of(p.n_eq);
            const bool reg = o.method == WIND_METHOD_SIE && gs != WIND_SOLVER_GJE_F64;
            const size_t team_bytes = reg ? (size_t)WarpLayout(nm, p.n_react, p.linear != nullptr, gs).bytes
                                          : (size_t)TeamLayout(nm, p.n_react, p.linear != nullptr, gs).bytes;
            smem = std::max(smem, (size_t)(MIXED_THREADS / nm) * team_bytes);
        }
    }
    if (smem > (size_t)cap) return WIND_ERR_UNSUPPORTED;
    MixedFn fn = mixed_fn(o.method, o.controller, o.solver);
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return launch_status("k_mixed shared-memory attribute");
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, MIXED_THREADS, smem) != cudaSuccess || nb < 1)
        return WIND_ERR_UNSUPPORTED;
    const int grid = nb * device_sm_count();
    // largest N first, then the larger group
    std::vector<int> order(ps.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        if (ps[a].n_eq != ps[b].n_eq) return ps[a].n_eq > ps[b].n_eq;
        return ps[a].nsys > ps[b].nsys;
    });
    const size_t pbytes = ps.size() * sizeof(KParams), obytes = order.size() * sizeof(int);
    unsigned char* dparams = nullptr;
    if (cudaMallocAsync((void**)&dparams, pbytes + obytes + 16, stream) != cudaSuccess) return WIND_ERR_NOMEM;
    double* gscratch = nullptr;
    if (gslot && cudaMallocAsync((void**)&gscratch, gslot * grid * sizeof(double), stream) != cudaSuccess) {
        cudaFreeAsync(dparams, stream);
        return WIND_ERR_NOMEM;
    }
    // one pageable host-to-device copy: it returns once the source has been
    // staged, so the host blob may go out of scope right after
    std::vector<unsigned char> blob(pbytes + obytes);
    std::memcpy(blob.data(), ps.data(), pbytes);
    std::memcpy(blob.data() + pbytes, order.data(), obytes);
    wind_status st = WIND_OK;
    st = cuda_status(cudaMemcpyAsync(dparams, blob.data(), blob.size(), cudaMemcpyHostToDevice, stream),
                     "group table upload");
    if (st == WIND_OK) {
        fn<<<grid, MIXED_THREADS, smem, stream>>>(reinterpret_cast<const KParams*>(dparams),
                                                  reinterpret_cast<const int*>(dparams + pbytes),
                                                  (int)ps.size(), gscratch, gslot, cap);
        g_launches++;
        st = launch_status("k_mixed launch");
    }
    cudaFreeAsync(dparams, stream);
    if (gscratch) cudaFreeAsync(gscratch, stream);
    return st;
}

}  // namespace wind
