// batch.cu -- several network shapes integrated together.
//
// Mass-action groups of every size go to ONE persistent launch (k_mixed:
// largest N first, each group's systems pulled from its own device work
// queue).  Groups of the builtin networks (thread-per-system kernels) run on
// forked streams beside it.  The caller's stream waits for all of them.
#include <vector>

#include "api_internal.h"

namespace wind {

wind_status launch_mixed(const wind_options& o, const std::vector<KParams>& ps, cudaStream_t stream);

// Streams and events for the builtin groups that run beside the mass-action
// launch, kept per host thread and device and reused by every call (a
// request loop calls launch_batch once per batch: creating and destroying
// them each time would sit on its latency path).  They live until the
// process exits.
struct ForkPool {
    int device = -1;
    cudaEvent_t fork = nullptr;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> done;
};

static wind_status fork_pool(size_t n, ForkPool** out) {
    thread_local std::vector<ForkPool> pools;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return launch_status("fork pool device");
    ForkPool* fp = nullptr;
    for (auto& p : pools)
        if (p.device == dev) fp = &p;
    if (!fp) {
        pools.emplace_back();
        fp = &pools.back();
        fp->device = dev;
        if (cudaEventCreateWithFlags(&fp->fork, cudaEventDisableTiming) != cudaSuccess)
            return launch_status("fork event");
    }
    while (fp->streams.size() < n) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
            return launch_status("fork stream");
        fp->streams.push_back(st);
        fp->done.push_back(ev);
    }
    *out = fp;
    return WIND_OK;
}

wind_status launch_batch(const wind_options& o, const wind_group* groups, int ngroups,
                         cudaStream_t stream) {
    if (o.solver == WIND_SOLVER_MIXED_TC) return WIND_ERR_UNSUPPORTED;
    for (int g = 0; g < ngroups; g++) {
        wind_status st = check_network(&groups[g].net, groups[g].nsys);
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
    unsigned long long* counters = nullptr;
    if (cudaMallocAsync((void**)&counters, (size_t)ngroups * CNT_SLOTS * 8, stream) != cudaSuccess)
        return WIND_ERR_NOMEM;
    cudaMemsetAsync(counters, 0, (size_t)ngroups * CNT_SLOTS * 8, stream);
    std::vector<KParams> mass, builtin;
    for (int g = 0; g < ngroups; g++) {
        const wind_group& G = groups[g];
        KParams p{};
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
        p.counters = counters + (size_t)g * CNT_SLOTS;
        p.max_attempts = o.max_attempts > 0 ? o.max_attempts : ((int64_t)1 << 40);
        p.timeout_ns = o.timeout_s > 0 ? (uint64_t)(o.timeout_s * 1e9) : 0;
        if (p.nsys == 0) continue;
        (p.kind == WIND_NET_MASS_ACTION ? mass : builtin).push_back(p);
    }
    wind_status st = WIND_OK;
    ForkPool* fp = nullptr;
    if (!builtin.empty()) {
        st = fork_pool(builtin.size(), &fp);
        if (st == WIND_OK) st = cuda_status(cudaEventRecord(fp->fork, stream), "fork record");
    }
    for (size_t g = 0; g < builtin.size() && st == WIND_OK; g++) {
        cudaStreamWaitEvent(fp->streams[g], fp->fork, 0);
        st = launch_integrate(o, builtin[g], fp->streams[g]);
        cudaEventRecord(fp->done[g], fp->streams[g]);
    }
    if (st == WIND_OK) st = launch_mixed(o, mass, stream);
    if (fp)
        for (size_t g = 0; g < builtin.size(); g++) cudaStreamWaitEvent(stream, fp->done[g], 0);
    cudaFreeAsync(counters, stream);
    return st;
}

}  // namespace wind
