// api.cu -- extern "C" entry points of libwind (include/wind.h).
//
// Host side of the integrators: argument checks, device workspace, the
// kernel dispatch table, launches and copies.  The reference's harness
// (cuda/common/harness.cu:5-106) did cudaMalloc / copy / launch / copy /
// cudaFree per call on the default stream and returned an int step count;
// here allocations are stream-ordered (cudaMallocAsync draws from the
// device's pool, so repeated calls do not hit the driver), the caller may
// pass device pointers to skip the copies, and every failure is a status.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "api_internal.h"
#include "networks.cuh"

using namespace wind;

namespace wind {

std::atomic<int64_t> g_launches{0};

static thread_local char t_last_error[160] = "";

void record_cuda_error(cudaError_t e, const char* where) {
    std::snprintf(t_last_error, sizeof(t_last_error), "%s: %s", where, cudaGetErrorName(e));
}
const char* last_error_text() { return t_last_error; }

static int builtin_n(int kind) {
    switch (kind) {
    case WIND_NET_NR_TEST: return NetNR::N;
    case WIND_NET_KATZ96: return NetKatz96::N;
    case WIND_NET_STIFFTRIG: return NetTrig::N;
    default: return -1;
    }
}
static int builtin_nc(int kind) {
    switch (kind) {
    case WIND_NET_NR_TEST: return NetNR::NC;
    case WIND_NET_KATZ96: return NetKatz96::NC;
    case WIND_NET_STIFFTRIG: return NetTrig::NC;
    default: return -1;
    }
}

int device_sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    return n;
}

wind_status check_network(const wind_network* net, int64_t nsys) {
    if (!net) return WIND_ERR_ARGUMENT;
    if (net->kind == WIND_NET_MASS_ACTION) {
        if (net->n_eq < 1 || net->n_eq > WIND_MAX_EQ) return WIND_ERR_UNSUPPORTED;
        if (net->n_react > 65535) return WIND_ERR_UNSUPPORTED;
        if (net->n_react < 0) return WIND_ERR_ARGUMENT;
        if (nsys > 0 && net->n_react > 0 && (!net->rates || !net->species)) return WIND_ERR_ARGUMENT;
        return WIND_OK;
    }
    const int n = builtin_n(net->kind);
    if (n < 0) return WIND_ERR_ARGUMENT;
    // n_eq = Ntile x N: Ntile copies of the network (the Precompiler's
    // tiling, python/ode_systems/ode_base.py:86-88, 219-281)
    if (net->n_eq < n || net->n_eq % n != 0) return WIND_ERR_ARGUMENT;
    if (net->n_eq / n > WIND_MAX_TILES) return WIND_ERR_UNSUPPORTED;
    if (net->n_const < builtin_nc(net->kind)) return WIND_ERR_ARGUMENT;
    if (nsys > 0 && !net->constants) return WIND_ERR_ARGUMENT;
    return WIND_OK;
}

// Launch the right kernel family for one homogeneous batch already on the
// device.  `p.counters` must point at zeroed device counters.
wind_status launch_integrate(const wind_options& o_in, const KParams& p, cudaStream_t stream,
                             bool allow_alloc) {
    if (p.nsys == 0) return WIND_OK;
    if (o_in.method == WIND_METHOD_SIM) return launch_sim(o_in, p, stream);
    // the tensor-core variant exists for the CTA kernels' MIXED inverse only
    if (o_in.solver == WIND_SOLVER_MIXED_TC &&
        (p.kind != WIND_NET_MASS_ACTION || p.n_eq <= WIND_TEAM_MAX_EQ || o_in.method != WIND_METHOD_SIE))
        return WIND_ERR_UNSUPPORTED;
    wind_options o = o_in;
    o.solver = resolve_solver(o.solver, p.kind, p.n_eq);
    if (p.kind != WIND_NET_MASS_ACTION) {
        const int n = builtin_n(p.kind);
        return p.n_eq == n ? launch_lane(o, p, stream) : launch_tile(o, p, n, stream);
    }
    if (p.n_eq <= WIND_TEAM_MAX_EQ) return launch_team(o, p, stream);
    // CTA kernels: global scratch for the matrices that do not fit in shared
    // memory, taken from the stream-ordered pool and returned after the launch
    CtaPlan pl;
    const wind_status pst = plan_cta(o, p, allow_alloc, &pl);
    if (pst != WIND_OK) return pst;
    if (pl.gstride == 0) return launch_cta(pl, p, stream, nullptr);
    double* scratch = nullptr;
    if (cudaMallocAsync((void**)&scratch, (size_t)pl.grid * pl.gstride * sizeof(double), stream) != cudaSuccess)
        return WIND_ERR_NOMEM;
    const wind_status st = launch_cta(pl, p, stream, scratch);
    cudaFreeAsync(scratch, stream);
    return st;
}

}  // namespace wind

// ===========================================================================
extern "C" {

void wind_default_options(wind_options* opt) {
    if (!opt) return;
    opt->method = WIND_METHOD_SIE;
    opt->solver = WIND_SOLVER_GJE_F64;
    opt->controller = WIND_CTRL_DEVICE;
    opt->spec_width = 0;
    opt->max_attempts = 0;
    opt->timeout_s = 0.0;
}

const char* wind_version(void) { return "wind_b200 0.1 (sm_100a)"; }

const char* wind_status_string(int s) {
    switch (s) {
    case WIND_OK: return "ok";
    case WIND_ERR_ARGUMENT: return "invalid argument";
    case WIND_ERR_UNSUPPORTED: return "unsupported configuration";
    case WIND_ERR_CUDA: return "CUDA runtime error";
    case WIND_ERR_NOMEM: return "out of device memory";
    case WIND_ERR_TIMEOUT: return "timed out";
    case WIND_ERR_BUSY: return "admission refused";
    case WIND_ERR_NOT_FOUND: return "unknown request";
    default: return "unknown status";
    }
}

int64_t wind_launch_count(void) { return g_launches.load(); }

const char* wind_last_error(void) { return wind::last_error_text(); }

int wind_integrate(const wind_options* opt_in, const wind_network* net, double tnow,
                   double tend, int32_t n_integration_steps, double* y, int64_t nsys,
                   double atol, double rtol, int32_t* sys_status, int64_t* sys_nsteps,
                   int64_t* total_nsteps, int32_t memory, void* stream_v) {
    wind_options o;
    if (opt_in) o = *opt_in; else wind_default_options(&o);
    (void)cudaGetLastError();  // an earlier, unrelated error is not this call's
    if (check_options(o, true) != WIND_OK) return WIND_ERR_ARGUMENT;
    if (nsys < 0 || n_integration_steps < 1) return WIND_ERR_ARGUMENT;
    if (memory != WIND_MEM_HOST && memory != WIND_MEM_DEVICE) return WIND_ERR_ARGUMENT;
    wind_status st = check_network(net, nsys);
    if (st != WIND_OK) return st;
    if (nsys > 0 && !y) return WIND_ERR_ARGUMENT;
    if (total_nsteps) *total_nsteps = 0;
    if (nsys == 0) return WIND_OK;
    cudaStream_t stream = (cudaStream_t)stream_v;

    IntegrateCall call;
    st = call.prepare(o, *net, tnow, tend, n_integration_steps, y, nsys, atol, rtol,
                      sys_status, sys_nsteps, memory, stream);
    if (st == WIND_OK) st = launch_integrate(o, call.params, stream);
    if (st == WIND_OK) st = call.finish(total_nsteps);
    call.release();
    return st;
}

}  // extern "C"

// ---- device-resident output loop and multi-group batch ---------------------
extern "C" {

int wind_integrate_output_steps(const wind_options* opt_in, const wind_network* net, double tnow,
                                double tend, int32_t n_integration_steps, int32_t n_output_steps,
                                double* y, int64_t nsys, double atol, double rtol,
                                double* out_over_time, int64_t* steps_per_output, int32_t memory,
                                void* stream_v) {
    wind_options o;
    if (opt_in) o = *opt_in; else wind_default_options(&o);
    if (n_output_steps < 1 || n_integration_steps < 1 || nsys < 0) return WIND_ERR_ARGUMENT;
    (void)cudaGetLastError();
    if (check_options(o, true) != WIND_OK) return WIND_ERR_ARGUMENT;
    if (memory != WIND_MEM_HOST && memory != WIND_MEM_DEVICE) return WIND_ERR_ARGUMENT;
    wind_status st = check_network(net, nsys);
    if (st != WIND_OK) return st;
    if (nsys > 0 && (!y || !out_over_time)) return WIND_ERR_ARGUMENT;
    if (nsys == 0) return WIND_OK;
    cudaStream_t stream = (cudaStream_t)stream_v;
    const int N = net->n_eq;
    const size_t ybytes = (size_t)nsys * N * sizeof(double);

    IntegrateCall call;
    st = call.prepare(o, *net, tnow, tend, n_integration_steps, y, nsys, atol, rtol, nullptr,
                      nullptr, memory, stream);
    // per-interval counters and the trajectory buffer live on the device
    unsigned long long* cnt = nullptr;
    double* traj = nullptr;
    if (st == WIND_OK) {
        cnt = static_cast<unsigned long long*>(
            call.alloc((size_t)n_output_steps * CNT_SLOTS * sizeof(unsigned long long)));
        traj = (memory == WIND_MEM_DEVICE) ? out_over_time
                                           : static_cast<double*>(call.alloc(ybytes * (n_output_steps + 1)));
        if (call.failed) st = WIND_ERR_NOMEM;
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr;
    if (st == WIND_OK && cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
        st = WIND_ERR_CUDA;
    // Order the capture stream after the uploads on `stream`.
    cudaEvent_t ready = nullptr;
    if (st == WIND_OK) {
        cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
        cudaEventRecord(ready, stream);
        cudaStreamWaitEvent(cap, ready, 0);
        cudaStreamSynchronize(cap);
    }
    // ode_base.py:338-378: intervals [tcur, tcur+dt], tcur += dt
    if (st == WIND_OK && cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const double dt = (tend - tnow) / n_output_steps;
        double tcur = tnow;
        cudaMemsetAsync(cnt, 0, (size_t)n_output_steps * CNT_SLOTS * sizeof(unsigned long long), cap);
        cudaMemcpyAsync(traj, call.params.y, ybytes, cudaMemcpyDeviceToDevice, cap);
        for (int k = 0; k < n_output_steps && st == WIND_OK; k++) {
            KParams p = call.params;
            p.tnow = tcur;
            p.tend = tcur + dt;
            p.h0 = (p.tend - p.tnow) / n_integration_steps;
            p.counters = cnt + (size_t)k * CNT_SLOTS;
            st = launch_integrate(o, p, cap);
            cudaMemcpyAsync(traj + (size_t)(k + 1) * nsys * N, call.params.y, ybytes,
                            cudaMemcpyDeviceToDevice, cap);
            tcur += dt;
        }
        if (cudaStreamEndCapture(cap, &graph) != cudaSuccess) st = WIND_ERR_CUDA;
        if (st == WIND_OK && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) st = WIND_ERR_CUDA;
        if (st == WIND_OK && cudaGraphLaunch(exec, cap) != cudaSuccess) st = WIND_ERR_CUDA;
        g_launches++;  // the graph launch (its kernel nodes are counted above)
        if (st == WIND_OK) {
            cudaEventRecord(ready, cap);
            cudaStreamWaitEvent(stream, ready, 0);
        }
    } else if (st == WIND_OK) {
        st = WIND_ERR_CUDA;
    }
    if (st == WIND_OK) {
        std::vector<unsigned long long> hc((size_t)n_output_steps * CNT_SLOTS);
        cudaMemcpyAsync(hc.data(), cnt, hc.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                        stream);
        if (memory == WIND_MEM_HOST)
            cudaMemcpyAsync(out_over_time, traj, ybytes * (n_output_steps + 1), cudaMemcpyDeviceToHost,
                            stream);
        st = call.finish(nullptr);
        if (st == WIND_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = WIND_ERR_CUDA;
        if (st == WIND_OK && steps_per_output) {
            if (memory == WIND_MEM_HOST) {
                for (int k = 0; k < n_output_steps; k++)
                    steps_per_output[k] = (int64_t)hc[(size_t)k * CNT_SLOTS + CNT_STEPS];
            } else {
                std::vector<int64_t> tmp(n_output_steps);
                for (int k = 0; k < n_output_steps; k++)
                    tmp[k] = (int64_t)hc[(size_t)k * CNT_SLOTS + CNT_STEPS];
                cudaMemcpy(steps_per_output, tmp.data(), tmp.size() * sizeof(int64_t), cudaMemcpyHostToDevice);
            }
        }
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap) {
        cudaStreamSynchronize(cap);
        cudaStreamDestroy(cap);
    }
    if (ready) cudaEventDestroy(ready);
    call.release();
    return st;
}

}  // extern "C"

extern "C" int wind_integrate_batch(const wind_options* opt_in, const wind_group* groups,
                                    int32_t ngroups, void* stream_v) {
    wind_options o;
    if (opt_in) o = *opt_in; else wind_default_options(&o);
    if (ngroups < 0 || (ngroups > 0 && !groups)) return WIND_ERR_ARGUMENT;
    (void)cudaGetLastError();
    if (wind::check_options(o) != WIND_OK) return WIND_ERR_ARGUMENT;
    return wind::launch_batch(o, groups, ngroups, (cudaStream_t)stream_v);
}
