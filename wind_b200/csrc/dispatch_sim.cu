// dispatch_sim.cu -- launch of the fixed-step semi-implicit midpoint rule
// (WIND_METHOD_SIM, python/pysolvers/sim.py:36-90).
#include "api_internal.h"
#include "sim_kernel.cuh"

namespace wind {

int warp_nmax(int n);
size_t warp_smem_bytes(int n, int R, bool lin, int solver, int threads);

template <typename Fn>
static int sim_blocks_per_sm(Fn fn, int threads, size_t smem) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return nb;
}

wind_status launch_sim(const wind_options& o, const KParams& p, cudaStream_t stream) {
    if (p.nsys == 0) return WIND_OK;
    if (o.solver != WIND_SOLVER_LU_F64 && o.solver != WIND_SOLVER_AUTO) return WIND_ERR_UNSUPPORTED;
    if (p.n_steps < 1) return WIND_ERR_ARGUMENT;
    const int64_t sms = device_sm_count();
    if (p.kind != WIND_NET_MASS_ACTION) {
        void (*fn)(KParams) = nullptr;
        switch (p.kind) {
        case WIND_NET_NR_TEST: fn = p.n_eq == NetNR::N ? k_sim_lane<NetNR> : nullptr; break;
        case WIND_NET_KATZ96: fn = p.n_eq == NetKatz96::N ? k_sim_lane<NetKatz96> : nullptr; break;
        case WIND_NET_STIFFTRIG: fn = p.n_eq == NetTrig::N ? k_sim_lane<NetTrig> : nullptr; break;
        default: break;
        }
        if (!fn) return WIND_ERR_UNSUPPORTED;  // tiled builtin networks
        const int nb = sim_blocks_per_sm(fn, SIM_THREADS, 0);
        if (nb < 1) return WIND_ERR_UNSUPPORTED;
        const int64_t need = (p.nsys + SIM_THREADS - 1) / SIM_THREADS;
        const int64_t cap = nb * sms;
        fn<<<(int)(need < cap ? need : cap), SIM_THREADS, 0, stream>>>(p);
        g_launches++;
        return launch_status("k_sim_lane launch");
    }
    if (p.n_eq > WIND_TEAM_MAX_EQ) return WIND_ERR_UNSUPPORTED;
    const int nmax = warp_nmax(p.n_eq);
    void (*fn)(KParams) = nmax == 8 ? k_sim_warp<8> : nmax == 16 ? k_sim_warp<16> : k_sim_warp<32>;
    const size_t smem = warp_smem_bytes(p.n_eq, p.n_react, p.linear != nullptr, WIND_SOLVER_LU_F64,
                                        WARP_THREADS);
    if (smem > 227 * 1024) return WIND_ERR_UNSUPPORTED;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return launch_status("k_sim_warp shared-memory attribute");
    const int nb = sim_blocks_per_sm(fn, WARP_THREADS, smem);
    if (nb < 1) return WIND_ERR_UNSUPPORTED;
    const int teams = WARP_THREADS / nmax;
    const int64_t need = (p.nsys + teams - 1) / teams;
    const int64_t cap = nb * sms;
    fn<<<(int)(need < cap ? need : cap), WARP_THREADS, smem, stream>>>(p);
    g_launches++;
    return launch_status("k_sim_warp launch");
}

}  // namespace wind
