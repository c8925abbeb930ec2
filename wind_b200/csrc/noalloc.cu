// noalloc.cu -- a batch entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: host codes whose device memory is
// owned by another framework's allocator (a hydrodynamics code that hands the
// integrator slices of its own arena), processes running under a hard device
// memory budget, and code paths that must not enter the CUDA allocator at all
// while other work is in flight.  For them, wind_integrate_batch_noalloc runs
// the same kernels as wind_integrate_batch, but the only global scratch the
// kernels need -- one small block of counters per group (the work-queue
// ticket and the substep total) -- lives in the file-scope array below
// instead of in memory taken from the allocator.  The caller passes every
// input and output as device memory.
//
// Limits and rules:
//  * at most WIND_NOALLOC_MAX_GROUPS groups per call (the array holds
//    WIND_NOALLOC_MAX_GROUPS * 4 64-bit counters, 8 KiB); larger calls are
//    rejected with WIND_ERR_ARGUMENT before anything is launched;
//  * every GPU that loads this library holds the array until the process
//    exits;
//  * the array is shared by all calls on a device and keeps the last call's
//    contents: each call clears the counters it uses on its stream before its
//    kernels run, so calls issued one after another are independent, but
//    calls whose work overlaps on the GPU (different streams, or host threads
//    racing on one stream) race on the counters and must not be issued;
//  * the device address of the array is looked up once per device, with that
//    device current, on the first call made on it; make that first call
//    before any stream capture on the device.  The address is kept with the
//    CUDA context it was read in: after a device reset (a new primary
//    context, in which the module and its array load again) the next call
//    looks it up again;
//  * the groups run one after another on the caller's stream (no streams or
//    events are created);
//  * groups whose kernels need matrix scratch in global memory (mass-action
//    networks with N > 32 whose factor does not fit in shared memory, and the
//    Gauss-Jordan solver for N > 32) make the call return
//    WIND_ERR_UNSUPPORTED before anything is cleared or launched, so no
//    group's state has been touched and the call can be retried with the
//    allocating entry point.
#include <cuda.h>

#include <mutex>
#include <vector>

#include "api_internal.h"

namespace {

constexpr int kNoallocSlots = WIND_NOALLOC_MAX_GROUPS * wind::CNT_SLOTS;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_noalloc_counters[kNoallocSlots];

std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_addr[kMaxDevices] = {};
CUcontext g_noalloc_ctx[kMaxDevices] = {};

// The current CUDA context, read through the driver entry point the runtime
// hands out (no link against the driver library is needed).
CUcontext current_context() {
    using GetCtx = CUresult (*)(CUcontext*);
    static GetCtx fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<GetCtx>(f);
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

// Device address of g_noalloc_counters on the current device, looked up with
// the device current on the first call and again whenever the context changed.
wind_status noalloc_scratch(unsigned long long** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return WIND_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return WIND_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    const CUcontext ctx = current_context();
    if (!g_noalloc_addr[dev] || ctx != g_noalloc_ctx[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_counters);
        if (e != cudaSuccess || !p) return wind::cuda_status(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                                                             "noalloc scratch address");
        g_noalloc_addr[dev] = static_cast<unsigned long long*>(p);
        g_noalloc_ctx[dev] = current_context();
    }
    *out = g_noalloc_addr[dev];
    return WIND_OK;
}

}  // namespace

extern "C" int wind_integrate_batch_noalloc(const wind_options* opt_in, const wind_group* groups,
                                            int32_t ngroups, void* stream_v) {
    wind_options o;
    if (opt_in) o = *opt_in; else wind_default_options(&o);
    (void)cudaGetLastError();  // an earlier, unrelated error is not this call's
    if (wind::check_options(o) != WIND_OK) return WIND_ERR_ARGUMENT;
    if (ngroups < 0 || (ngroups > 0 && !groups)) return WIND_ERR_ARGUMENT;
    if (ngroups > WIND_NOALLOC_MAX_GROUPS) return WIND_ERR_ARGUMENT;
    for (int g = 0; g < ngroups; g++) {
        const wind_status st = wind::check_network(&groups[g].net, groups[g].nsys);
        if (st != WIND_OK) return st;
        if (groups[g].nsys > 0 && !groups[g].y) return WIND_ERR_ARGUMENT;
        if (groups[g].n_integration_steps < 1) return WIND_ERR_ARGUMENT;
        const wind_network& gn = groups[g].net;
        if (!wind::device_ptr(gn.constants) || !wind::device_ptr(gn.rates) ||
            !wind::device_ptr(gn.species) || !wind::device_ptr(gn.linear) ||
            !wind::device_ptr(groups[g].y) || !wind::device_ptr(groups[g].sys_status) ||
            !wind::device_ptr(groups[g].sys_nsteps))
            return WIND_ERR_ARGUMENT;
    }
    if (ngroups == 0) return WIND_OK;
    cudaStream_t stream = (cudaStream_t)stream_v;
    unsigned long long* scratch = nullptr;
    wind_status st = noalloc_scratch(&scratch);
    if (st != WIND_OK) return st;
    std::vector<wind::KParams> ps((size_t)ngroups);
    for (int g = 0; g < ngroups; g++) {
        const wind_group& G = groups[g];
        wind::KParams& p = ps[g];
        p = wind::KParams{};
        p.kind = G.net.kind;
        p.n_eq = G.net.n_eq;
        p.n_const = G.net.n_const;
        p.n_react = G.net.n_react;
        p.constants = G.net.constants;
        p.rates = G.net.rates;
        p.species = G.net.species;
        p.linear = G.net.linear;
        p.tnow = G.tnow;
        p.tend = G.tend;
        p.h0 = (G.tend - G.tnow) / G.n_integration_steps;
        p.atol = G.atol;
        p.rtol = G.rtol;
        p.y = G.y;
        p.nsys = G.nsys;
        p.sys_status = G.sys_status;
        p.sys_nsteps = G.sys_nsteps;
        p.counters = scratch + (size_t)g * wind::CNT_SLOTS;
        p.max_attempts = o.max_attempts > 0 ? o.max_attempts : ((int64_t)1 << 40);
        p.timeout_ns = o.timeout_s > 0 ? (uint64_t)(o.timeout_s * 1e9) : 0;
        // a group that would need global scratch is refused here, before any
        // group has been cleared or launched
        if (p.nsys > 0 && p.kind == WIND_NET_MASS_ACTION && p.n_eq > wind::WIND_TEAM_MAX_EQ) {
            wind::CtaPlan pl;
            wind_options oc = o;
            oc.solver = wind::resolve_solver(o.solver, p.kind, p.n_eq);
            const wind_status pst = wind::plan_cta(oc, p, /*allow_global=*/false, &pl);
            if (pst != WIND_OK) return pst;
        }
    }
    if (cudaMemsetAsync(scratch, 0, (size_t)ngroups * wind::CNT_SLOTS * sizeof(unsigned long long),
                        stream) != cudaSuccess)
        return wind::launch_status("noalloc counters clear");
    for (int g = 0; g < ngroups && st == WIND_OK; g++)
        st = wind::launch_integrate(o, ps[g], stream, /*allow_alloc=*/false);
    return st;
}
