// global.cu -- the SIE_host variant: every system advances with one shared
// step, accepted or refined for all at once.
//
// Replaces cudaIntegrateSIE (cuda/SIE_host/harness_kernel.cu:427-532) and its
// errorLoop (:248-425).  The reference drives the step loop from the host
// with a dozen small kernels per substep, cuBLAS SgemmBatched for the
// products and a blocking copy of one global error flag per attempt; here
// one kernel per attempt computes, for every system at once (one thread per
// system, everything in registers), the full step and the two half steps
// from the last accepted state and ORs the error test into a flag, and the
// host reads that flag and decides (the same host-driven control: the shared
// step must see every system before it moves).  Compiled networks only, as
// in the reference, whose SIE_host build integrates the generated network.
#include <algorithm>

#include "api_internal.h"
#include "lane_kernel.cuh"

namespace wind {

// One attempt over all systems: y1 = one substep of h, y2 = two of h/2 from
// yacc (GOLD substep arithmetic, solveSystem harness_kernel.cu:175-246), y2
// into ytry; *flag |= 1 when any element fails checkError
// (cuda/SIE_host/vector_kernels.cu:45-70: strict, signed relative test).
template <class Net, int SOLVER>
__global__ void __launch_bounds__(LANE_THREADS)
    k_global_attempt(const double* __restrict__ consts, int nc, const double* __restrict__ yacc,
                     double* __restrict__ ytry, int64_t nsys, double t0, double h, double atol,
                     double rtol, unsigned* flag) {
    constexpr int N = Net::N, NC = Net::NC;
    bool err = false;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nsys;
         s += (int64_t)gridDim.x * blockDim.x) {
        double c[NC];
#pragma unroll
        for (int k = 0; k < NC; k++) c[k] = consts[s * nc + k];
        xd a[N], b[N];
#pragma unroll
        for (int e = 0; e < N; e++) a[e] = b[e] = yacc[s * N + e];
        lane_take_step<Net, WIND_METHOD_SIE, WIND_CTRL_GOLD, SOLVER>(c, t0, h, 1, a);
        lane_take_step<Net, WIND_METHOD_SIE, WIND_CTRL_GOLD, SOLVER>(c, t0, h, 2, b);
#pragma unroll
        for (int e = 0; e < N; e++) {
            const xd d = a[e] - b[e];
            if (fabs(d.v) > atol) err = true;
            if (fabs((d / (b[e] + 1e-12)).v) > rtol && a[e].v > atol && b[e].v > atol) err = true;
            ytry[s * N + e] = b[e].v;
        }
    }
    if (__any_sync(0xffffffffu, err) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

using GlobalFn = void (*)(const double*, int, const double*, double*, int64_t, double, double, double,
                          double, unsigned*);

template <class Net>
static GlobalFn global_fn_solver(int solver) {
    switch (solver) {
    case WIND_SOLVER_LU_F64: return k_global_attempt<Net, WIND_SOLVER_LU_F64>;
    case WIND_SOLVER_MIXED: return k_global_attempt<Net, WIND_SOLVER_MIXED>;
    default: return k_global_attempt<Net, WIND_SOLVER_GJE_F64>;
    }
}

static GlobalFn global_fn(int kind, int solver) {
    switch (kind) {
    case WIND_NET_NR_TEST: return global_fn_solver<NetNR>(solver);
    case WIND_NET_KATZ96: return global_fn_solver<NetKatz96>(solver);
    case WIND_NET_STIFFTRIG: return global_fn_solver<NetTrig>(solver);
    default: return nullptr;
    }
}

}  // namespace wind

using namespace wind;

extern "C" int wind_integrate_global(const wind_options* opt_in, const wind_network* net, double tnow,
                                     double tend, int32_t n_integration_steps, double* y,
                                     int64_t nsys, double atol, double rtol, int64_t* total_nsteps,
                                     double* t_reached, int32_t memory, void* stream_v) {
    wind_options o;
    if (opt_in) o = *opt_in; else wind_default_options(&o);
    (void)cudaGetLastError();
    if (check_options(o) != WIND_OK || o.method != WIND_METHOD_SIE) return WIND_ERR_ARGUMENT;
    if (o.solver == WIND_SOLVER_MIXED_TC) return WIND_ERR_UNSUPPORTED;
    if (nsys < 0 || n_integration_steps < 1) return WIND_ERR_ARGUMENT;
    if (memory != WIND_MEM_HOST && memory != WIND_MEM_DEVICE) return WIND_ERR_ARGUMENT;
    wind_status st = check_network(net, nsys);
    if (st != WIND_OK) return st;
    if (net->kind == WIND_NET_MASS_ACTION) return WIND_ERR_UNSUPPORTED;
    // one thread integrates one whole system here: tiled networks (n_eq =
    // Ntile x N) go through wind_integrate
    const int base_n = net->kind == WIND_NET_KATZ96 ? NetKatz96::N : NetNR::N;
    if (net->n_eq != base_n) return WIND_ERR_UNSUPPORTED;
    if (nsys > 0 && !y) return WIND_ERR_ARGUMENT;
    if (total_nsteps) *total_nsteps = 0;
    if (t_reached) *t_reached = tnow;
    if (nsys == 0) return WIND_OK;
    cudaStream_t stream = (cudaStream_t)stream_v;
    GlobalFn fn = global_fn(net->kind, resolve_solver(o.solver, net->kind, net->n_eq));

    IntegrateCall call;
    st = call.prepare(o, *net, tnow, tend, n_integration_steps, y, nsys, atol, rtol, nullptr, nullptr,
                      memory, stream);
    const int N = net->n_eq;
    double* ytry = nullptr;
    unsigned* flag = nullptr;
    if (st == WIND_OK) {
        ytry = static_cast<double*>(call.alloc((size_t)nsys * N * sizeof(double)));
        flag = static_cast<unsigned*>(call.alloc(sizeof(unsigned)));
        if (call.failed) st = WIND_ERR_NOMEM;
    }
    double* yacc = call.params.y;
    const int64_t blocks_needed = (nsys + LANE_THREADS - 1) / LANE_THREADS;
    const int grid = (int)std::min<int64_t>(blocks_needed, (int64_t)device_sm_count() * 16);
    int64_t nsteps = 0;
    int unsolved = 0;
    double timestep = (tend - tnow) / n_integration_steps;
    // errorLoop, harness_kernel.cu:288-402
    while (st == WIND_OK && tnow < tend && unsolved < 9) {
        timestep = std::min(timestep, tend - tnow);
        nsteps += 3;
        unsigned h_flag = 0;
        if (cudaMemsetAsync(flag, 0, sizeof(unsigned), stream) != cudaSuccess) {
            st = launch_status("global flag clear");
            break;
        }
        fn<<<grid, LANE_THREADS, 0, stream>>>(call.params.constants, net->n_const, yacc, ytry, nsys,
                                              tnow, timestep, atol, rtol, flag);
        g_launches++;
        st = launch_status("k_global_attempt launch");
        if (st != WIND_OK) break;
        if (cudaMemcpyAsync(&h_flag, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            st = launch_status("global flag read");
            break;
        }
        if (h_flag) {
            unsolved++;
            timestep /= 2;
        } else {
            unsolved = 0;
            std::swap(yacc, ytry);
            tnow += timestep;
            timestep *= 2;
        }
    }
    // the accepted state must end in the call's state buffer
    if (st == WIND_OK && yacc != call.params.y)
        st = cuda_status(cudaMemcpyAsync(call.params.y, yacc, (size_t)nsys * N * sizeof(double),
                                         cudaMemcpyDeviceToDevice, stream),
                         "global state copy");
    if (st == WIND_OK) st = call.finish(nullptr);
    if (st == WIND_OK && memory == WIND_MEM_DEVICE) st = cuda_status(cudaStreamSynchronize(stream), "global sync");
    call.release();
    if (st == WIND_OK) {
        if (total_nsteps) *total_nsteps = nsteps * nsys;  // harness_kernel.cu:423
        if (t_reached) *t_reached = tnow;
    }
    return st;
}
