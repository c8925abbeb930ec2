// dispatch_cta.cu -- instantiations and launch of the CTA-per-system kernels
// (mass action, 32 < N <= 256).
#include <mutex>
#include <vector>

#include "api_internal.h"
#include "cta_kernel.cuh"

namespace wind {

using CtaFn = void (*)(KParams, double*, int);

template <int METHOD, int CTRL>
static CtaFn cta_by_solver(int solver) {
    if constexpr (METHOD == WIND_METHOD_RK2) return k_cta<METHOD, CTRL, WIND_SOLVER_LU_F64>;
    else {
        switch (solver) {
        case WIND_SOLVER_GJE_F64: return k_cta<METHOD, CTRL, WIND_SOLVER_GJE_F64>;
        case WIND_SOLVER_LU_F64: return k_cta<METHOD, CTRL, WIND_SOLVER_LU_F64>;
        default: return k_cta<METHOD, CTRL, WIND_SOLVER_MIXED>;
        }
    }
}

static CtaFn cta_fn(int method, int ctrl, int solver) {
    if (method == WIND_METHOD_SIE)
        return ctrl == WIND_CTRL_GOLD ? cta_by_solver<WIND_METHOD_SIE, WIND_CTRL_GOLD>(solver)
                                      : cta_by_solver<WIND_METHOD_SIE, WIND_CTRL_DEVICE>(solver);
    return ctrl == WIND_CTRL_GOLD ? cta_by_solver<WIND_METHOD_RK2, WIND_CTRL_GOLD>(solver)
                                  : cta_by_solver<WIND_METHOD_RK2, WIND_CTRL_DEVICE>(solver);
}

static int smem_optin() {
    int dev = 0, v = 227 * 1024;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v - 1024;  // room for the kernel's static shared variables
}

static int cta_blocks_per_sm(CtaFn fn, size_t smem) {
    static std::mutex mu;
    static std::vector<std::pair<std::pair<const void*, size_t>, int>> cache;
    std::lock_guard<std::mutex> g(mu);
    for (auto& e : cache)
        if (e.first.first == (const void*)fn && e.first.second == smem) return e.second;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, CTA_THREADS, smem) != cudaSuccess) nb = 0;
    cache.push_back({{(const void*)fn, smem}, nb});
    return nb;
}

static int method_solver(const wind_options& o) {
    return (o.method == WIND_METHOD_RK2) ? WIND_SOLVER_LU_F64 : o.solver;
}

// Global scratch bytes a CTA launch needs (0 = none) and its grid.
size_t cta_scratch_bytes(const wind_options& o, const KParams& p, int* grid_out) {
    const int solver = method_solver(o);
    const int cap = smem_optin();
    const CtaLayout lay(p.n_eq, p.n_react, p.linear != nullptr, solver, cap);
    CtaFn fn = cta_fn(o.method, o.controller, o.solver);
    const int nb = lay.bytes <= cap ? cta_blocks_per_sm(fn, lay.bytes) : 0;
    const int64_t resident = (int64_t)(nb > 0 ? nb : 1) * device_sm_count();
    const int grid = (int)(p.nsys < resident ? p.nsys : resident);
    if (grid_out) *grid_out = grid;
    const bool need = (solver == WIND_SOLVER_GJE_F64) || !lay.mat_in_smem;
    return need ? (size_t)grid * CtaLayout::gscratch_doubles(p.n_eq, solver) * sizeof(double) : 0;
}

wind_status launch_cta(const wind_options& o, const KParams& p, cudaStream_t stream, double* scratch,
                       size_t scratch_bytes) {
    if (p.n_eq > CTA_MAXN || p.n_react > 65535) return WIND_ERR_UNSUPPORTED;
    const int solver = method_solver(o);
    const int cap = smem_optin();
    const CtaLayout lay(p.n_eq, p.n_react, p.linear != nullptr, solver, cap);
    if (lay.bytes > cap) return WIND_ERR_UNSUPPORTED;
    CtaFn fn = cta_fn(o.method, o.controller, o.solver);
    const int nb = cta_blocks_per_sm(fn, lay.bytes);
    if (nb < 1) return WIND_ERR_UNSUPPORTED;
    int grid = 0;
    const size_t need = cta_scratch_bytes(o, p, &grid);
    if (need > scratch_bytes) return WIND_ERR_NOMEM;
    // set for this launch every time (the occupancy cache may come from a
    // launch of the same kernel with another size)
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, lay.bytes) != cudaSuccess)
        return launch_status("k_cta shared-memory attribute");
    fn<<<grid, CTA_THREADS, lay.bytes, stream>>>(p, need ? scratch : nullptr, cap);
    g_launches++;
    return launch_status("k_cta launch");
}

}  // namespace wind
