// batch.cu -- several network shapes integrated together.
#include <vector>

#include "api_internal.h"

namespace wind {

// Each group runs its kernel family on its own forked stream so the groups
// overlap on the device; the caller's stream waits for all of them.
wind_status launch_batch(const wind_options& o, const wind_group* groups, int ngroups,
                         cudaStream_t stream) {
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
    cudaEvent_t fork;
    cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    cudaEventRecord(fork, stream);
    std::vector<cudaStream_t> ss(ngroups, nullptr);
    std::vector<cudaEvent_t> done(ngroups, nullptr);
    wind_status st = WIND_OK;
    for (int g = 0; g < ngroups && st == WIND_OK; g++) {
        const wind_group& G = groups[g];
        cudaStreamCreateWithFlags(&ss[g], cudaStreamNonBlocking);
        cudaEventCreateWithFlags(&done[g], cudaEventDisableTiming);
        cudaStreamWaitEvent(ss[g], fork, 0);
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
        st = launch_integrate(o, p, ss[g]);
        cudaEventRecord(done[g], ss[g]);
        cudaStreamWaitEvent(stream, done[g], 0);
    }
    cudaFreeAsync(counters, stream);
    for (int g = 0; g < ngroups; g++) {
        if (ss[g]) cudaStreamDestroy(ss[g]);
        if (done[g]) cudaEventDestroy(done[g]);
    }
    cudaEventDestroy(fork);
    return st;
}

}  // namespace wind
