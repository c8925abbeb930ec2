// api_internal.h -- host-side pieces shared by the entry points.
#pragma once

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/wind.h"
#include "common.cuh"

namespace wind {

int device_sm_count();
wind_status check_network(const wind_network* net, int64_t nsys);

// Range checks of the options every entry point applies: an unknown method,
// controller or solver is an argument error, never read as a default.
// `sim_ok`: the entry point runs the fixed-step WIND_METHOD_SIM (only
// wind_integrate and wind_integrate_output_steps do).
inline wind_status check_options(const wind_options& o, bool sim_ok = false) {
    if (o.method != WIND_METHOD_SIE && o.method != WIND_METHOD_RK2 &&
        !(sim_ok && o.method == WIND_METHOD_SIM))
        return WIND_ERR_ARGUMENT;
    if (o.controller != WIND_CTRL_DEVICE && o.controller != WIND_CTRL_GOLD) return WIND_ERR_ARGUMENT;
    if (o.solver < WIND_SOLVER_GJE_F64 || o.solver > WIND_SOLVER_MIXED_TC) return WIND_ERR_ARGUMENT;
    if (o.spec_width < 0 || o.max_attempts < 0 || !(o.timeout_s >= 0.0)) return WIND_ERR_ARGUMENT;
    return WIND_OK;
}

// The solver WIND_SOLVER_AUTO stands for on one network shape: the FP64 LU
// for the compiled networks and up to 32 species, the mixed solve above.
inline int resolve_solver(int solver, int kind, int n_eq) {
    if (solver != WIND_SOLVER_AUTO) return solver;
    return (kind == WIND_NET_MASS_ACTION && n_eq > 32) ? WIND_SOLVER_MIXED : WIND_SOLVER_LU_F64;
}
// Launch the kernel family for one homogeneous batch.  `allow_alloc` = false
// makes configurations that need global scratch return WIND_ERR_UNSUPPORTED
// instead of taking it from the stream-ordered allocator.
wind_status launch_integrate(const wind_options& o, const KParams& p, cudaStream_t stream,
                             bool allow_alloc = true);
wind_status launch_team(const wind_options& o, const KParams& p, cudaStream_t stream);
// The fixed-step semi-implicit midpoint rule (WIND_METHOD_SIM): untiled
// builtin networks and mass action with N <= 32, FP64 LU solves.
wind_status launch_sim(const wind_options& o, const KParams& p, cudaStream_t stream);
wind_status launch_lane(const wind_options& o, const KParams& p, cudaStream_t stream);
// Tiled builtin network (n_eq = Ntile x base_n, 1 < Ntile <= WIND_MAX_TILES).
wind_status launch_tile(const wind_options& o, const KParams& p, int base_n, cudaStream_t stream);
// A CTA-kernel launch: kernel, shared-memory budget and size, grid, and
// the per-block global scratch (doubles; 0 = none).
struct CtaPlan {
    const void* fn;
    int smem_cap, smem_bytes, grid;
    size_t gstride;
};
wind_status plan_cta(const wind_options& o, const KParams& p, bool allow_global, CtaPlan* out);
wind_status launch_cta(const CtaPlan& pl, const KParams& p, cudaStream_t stream, double* scratch);
// Global scratch (bytes) one resident CTA-kernel block needs for an N > 32
// mass-action system with the full shared-memory budget (0 when everything
// fits in shared memory).
size_t cta_scratch_bytes_per_block(int n_eq, int n_react, bool lin, int solver);
extern std::atomic<int64_t> g_launches;
// Largest N any kernel family accepts (lane/team kernels up to 32, CTA
// kernels up to 256).
constexpr int WIND_MAX_EQ = 256;
constexpr int WIND_TEAM_MAX_EQ = 32;
// Most copies of a builtin network one tiled system may hold.
constexpr int WIND_MAX_TILES = 64;

// The name of the last CUDA error this thread mapped to WIND_ERR_CUDA, with
// the place it was seen (read back through wind_last_error()).
void record_cuda_error(cudaError_t e, const char* where);
const char* last_error_text();
inline wind_status cuda_status(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return WIND_OK;
    record_cuda_error(e, where);
    return WIND_ERR_CUDA;
}
// Status of the launch just issued.
inline wind_status launch_status(const char* where) { return cuda_status(cudaGetLastError(), where); }

// True for null or for memory a kernel may dereference (device or managed).
inline bool device_ptr(const void* ptr) {
    if (!ptr) return true;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();  // clear the error of an unknown pointer
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// One wind_integrate call: device copies of host inputs (when memory is
// HOST), the counters block, and the kernel parameters.  Allocations are
// stream-ordered (cudaMallocAsync / cudaFreeAsync) and released in release().
struct IntegrateCall {
    KParams params{};
    cudaStream_t stream = nullptr;
    int memory = WIND_MEM_HOST;
    double* h_y = nullptr;
    int32_t* h_status = nullptr;
    int64_t* h_nsteps = nullptr;
    size_t ybytes = 0;
    void* allocs[10] = {};
    int nalloc = 0;
    bool failed = false;

    void* alloc(size_t bytes) {
        void* p = nullptr;
        if (bytes == 0) bytes = 16;
        if (cudaMallocAsync(&p, bytes, stream) != cudaSuccess) { failed = true; return nullptr; }
        allocs[nalloc++] = p;
        return p;
    }
    template <typename T>
    const T* upload(const T* host, size_t count) {
        if (!host || count == 0) return nullptr;
        T* d = static_cast<T*>(alloc(count * sizeof(T)));
        if (!d) return nullptr;
        if (cudaMemcpyAsync(d, host, count * sizeof(T), cudaMemcpyHostToDevice, stream) != cudaSuccess)
            failed = true;
        return d;
    }

    wind_status prepare(const wind_options& o, const wind_network& net, double tnow, double tend,
                        int32_t n_integration_steps, double* y, int64_t nsys, double atol,
                        double rtol, int32_t* sys_status, int64_t* sys_nsteps, int32_t mem,
                        cudaStream_t s) {
        stream = s;
        memory = mem;
        const int N = net.n_eq;
        KParams& p = params;
        p.kind = net.kind;
        p.n_eq = N;
        p.n_const = net.n_const;
        p.n_react = net.n_react;
        p.tnow = tnow;
        p.tend = tend;
        // cuda/common/harness.cu:80, cuda/c_baseline/sie/sie_gold.c:105
        p.h0 = (tend - tnow) / n_integration_steps;
        p.n_steps = n_integration_steps;
        p.atol = atol;
        p.rtol = rtol;
        p.nsys = nsys;
        p.max_attempts = o.max_attempts > 0 ? o.max_attempts : ((int64_t)1 << 40);
        p.timeout_ns = o.timeout_s > 0 ? (uint64_t)(o.timeout_s * 1e9) : 0;
        p.counters = static_cast<unsigned long long*>(alloc(CNT_SLOTS * sizeof(unsigned long long)));
        if (failed) return WIND_ERR_NOMEM;
        if (cudaMemsetAsync(p.counters, 0, CNT_SLOTS * sizeof(unsigned long long), stream) != cudaSuccess)
            return launch_status("counters memset");
        if (mem == WIND_MEM_DEVICE) {
            // every array must be device (or managed) memory of a device:
            // a host pointer handed to a kernel would fault
            if (!device_ptr(net.constants) || !device_ptr(net.rates) || !device_ptr(net.species) ||
                !device_ptr(net.linear) || !device_ptr(y) || !device_ptr(sys_status) ||
                !device_ptr(sys_nsteps))
                return WIND_ERR_ARGUMENT;
            p.constants = net.constants;
            p.rates = net.rates;
            p.species = net.species;
            p.linear = net.linear;
            p.y = y;
            p.sys_status = sys_status;
            p.sys_nsteps = sys_nsteps;
            return WIND_OK;
        }
        // host memory: validate mass-action species indices before upload
        if (net.kind == WIND_NET_MASS_ACTION && net.species) {
            const size_t cnt = (size_t)nsys * net.n_react * 4;
            for (size_t i = 0; i < cnt; i++)
                if (net.species[i] >= (uint16_t)N) return WIND_ERR_ARGUMENT;
        }
        h_y = y;
        h_status = sys_status;
        h_nsteps = sys_nsteps;
        ybytes = (size_t)nsys * N * sizeof(double);
        p.constants = upload(net.constants, net.constants ? (size_t)nsys * net.n_const : 0);
        p.rates = upload(net.rates, net.rates ? (size_t)nsys * net.n_react : 0);
        p.species = upload(net.species, net.species ? (size_t)nsys * net.n_react * 4 : 0);
        p.linear = upload(net.linear, net.linear ? (size_t)nsys * N * N : 0);
        p.y = static_cast<double*>(alloc(ybytes));
        if (failed) return WIND_ERR_NOMEM;
        if (cudaMemcpyAsync(p.y, y, ybytes, cudaMemcpyHostToDevice, stream) != cudaSuccess)
            return launch_status("state upload");
        if (sys_status) p.sys_status = static_cast<int32_t*>(alloc(nsys * sizeof(int32_t)));
        if (sys_nsteps) p.sys_nsteps = static_cast<int64_t*>(alloc(nsys * sizeof(int64_t)));
        if (failed) return WIND_ERR_NOMEM;
        return WIND_OK;
    }

    wind_status finish(int64_t* total) {
        unsigned long long cnt[CNT_SLOTS] = {};
        if (memory == WIND_MEM_HOST) {
            if (cudaMemcpyAsync(h_y, params.y, ybytes, cudaMemcpyDeviceToHost, stream) != cudaSuccess)
                return launch_status("state download");
            if (h_status &&
                cudaMemcpyAsync(h_status, params.sys_status, params.nsys * sizeof(int32_t),
                                cudaMemcpyDeviceToHost, stream) != cudaSuccess)
                return WIND_ERR_CUDA;
            if (h_nsteps &&
                cudaMemcpyAsync(h_nsteps, params.sys_nsteps, params.nsys * sizeof(int64_t),
                                cudaMemcpyDeviceToHost, stream) != cudaSuccess)
                return WIND_ERR_CUDA;
        }
        if (memory == WIND_MEM_HOST || total) {
            if (cudaMemcpyAsync(cnt, params.counters, sizeof(cnt), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
                return WIND_ERR_CUDA;
            const cudaError_t se = cudaStreamSynchronize(stream);
            if (se != cudaSuccess) return cuda_status(se, "stream synchronize");
            if (total) *total = (int64_t)cnt[CNT_STEPS];
        }
        return launch_status("finish");
    }

    void release() {
        for (int i = 0; i < nalloc; i++) cudaFreeAsync(allocs[i], stream);
        nalloc = 0;
    }
};

}  // namespace wind

namespace wind {
wind_status launch_batch(const wind_options& o, const wind_group* groups, int ngroups,
                         cudaStream_t stream);
}
