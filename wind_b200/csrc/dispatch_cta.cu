// dispatch_cta.cu -- instantiations and launch of the CTA-per-system kernels
// (mass action, 32 < N <= 256).
#include <mutex>
#include <vector>

#include "api_internal.h"
#include "cta_kernel.cuh"

namespace wind {

using CtaFn = void (*)(KParams, double*, size_t, int);

template <int METHOD, int CTRL>
static CtaFn cta_by_solver(int solver) {
    if constexpr (METHOD == WIND_METHOD_RK2) return k_cta<METHOD, CTRL, WIND_SOLVER_LU_F64>;
    else {
        switch (solver) {
        case WIND_SOLVER_GJE_F64: return k_cta<METHOD, CTRL, WIND_SOLVER_GJE_F64>;
        case WIND_SOLVER_LU_F64: return k_cta<METHOD, CTRL, WIND_SOLVER_LU_F64>;
        case WIND_SOLVER_MIXED_TC: return k_cta<METHOD, CTRL, WIND_SOLVER_MIXED, true>;
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

// Dynamic shared memory per block that leaves room for two blocks per SM.
static int smem_half(CtaFn fn) {
    int dev = 0, per_sm = 228 * 1024;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaFuncAttributes fa{};
    size_t stat = 64;
    if (cudaFuncGetAttributes(&fa, fn) == cudaSuccess) stat = fa.sharedSizeBytes;
    return (int)((per_sm / 2 - 1024 - (int)stat) & ~127);
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

// The solver whose layout a launch uses (MIXED_TC is MIXED with the
// tensor-core staging added).
static int method_solver(const wind_options& o) {
    if (o.method == WIND_METHOD_RK2) return WIND_SOLVER_LU_F64;
    return o.solver == WIND_SOLVER_MIXED_TC ? WIND_SOLVER_MIXED : o.solver;
}

// Choose the shared-memory budget (full, or half an SM for the FP32
// factors), the grid and the per-block global scratch of a CTA launch.
// With allow_global = false only layouts without global scratch qualify.
wind_status plan_cta(const wind_options& o, const KParams& p, bool allow_global, CtaPlan* out) {
    if (p.n_eq > CTA_MAXN || p.n_react > 65535) return WIND_ERR_UNSUPPORTED;
    const int solver = method_solver(o);
    const bool tc = o.method == WIND_METHOD_SIE && o.solver == WIND_SOLVER_MIXED_TC;
    CtaFn fn = cta_fn(o.method, o.controller, o.solver);
    int caps[2] = {smem_optin(), 0};
    int ncap = 1;
    if (solver == WIND_SOLVER_MIXED && CtaMinBlocks<WIND_SOLVER_MIXED>::value >= 2) caps[ncap++] = smem_half(fn);
    // ranking: the matrix in shared memory first (a matrix in global memory
    // is read and written on every trailing update), then blocks per SM;
    // ties keep the larger budget
    bool found = false;
    CtaPlan best{};
    int best_score = 0;
    for (int i = 0; i < ncap; i++) {
        const CtaLayout lay(p.n_eq, p.n_react, p.linear != nullptr, solver, caps[i], tc);
        if (lay.bytes > caps[i]) continue;
        // the tensor-core staging must sit in shared memory, and the matrix
        // with it (the MMA operands are built from it every panel)
        if (tc && !lay.mat_in_smem) continue;
        if (!allow_global && lay.g_doubles > 0) continue;
        const int nb = cta_blocks_per_sm(fn, lay.bytes);
        const int score = nb + (lay.mat_in_smem ? 1000 : 0);
        if (nb < 1 || score <= best_score) continue;
        const int64_t resident = (int64_t)nb * device_sm_count();
        best.fn = (const void*)fn;
        best.smem_cap = caps[i];
        best.smem_bytes = lay.bytes;
        best.grid = (int)(p.nsys < resident ? p.nsys : resident);
        best.gstride = lay.g_doubles;
        best_score = score;
        found = true;
    }
    if (!found) return WIND_ERR_UNSUPPORTED;
    *out = best;
    return WIND_OK;
}

size_t cta_scratch_bytes_per_block(int n_eq, int n_react, bool lin, int solver) {
    const CtaLayout lay(n_eq, n_react, lin, solver, smem_optin());
    return lay.g_doubles * sizeof(double);
}

wind_status launch_cta(const CtaPlan& pl, const KParams& p, cudaStream_t stream, double* scratch) {
    if (pl.gstride && !scratch) return WIND_ERR_ARGUMENT;
    CtaFn fn = reinterpret_cast<CtaFn>(const_cast<void*>(pl.fn));
    // set for this launch every time (the occupancy cache may come from a
    // launch of the same kernel with another size)
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, pl.smem_bytes) != cudaSuccess)
        return launch_status("k_cta shared-memory attribute");
    fn<<<pl.grid, CTA_THREADS, pl.smem_bytes, stream>>>(p, pl.gstride ? scratch : nullptr, pl.gstride,
                                                        pl.smem_cap);
    g_launches++;
    return launch_status("k_cta launch");
}

}  // namespace wind
