/*
 * wind.h -- C ABI of the B200 batched stiff-ODE integrators (SIE and RK2).
 *
 * Two layers are exported:
 *
 *  1. The drop-in entry of the reference solver libraries (declared in
 *     wind_legacy.h): `cudaIntegrateSystem`, with the reference's C++ linkage
 *     and signature (cuda/common/harness.cu:5-14), so the reference's ctypes
 *     caller (python/wind_harness.py:32-40, python/ode_systems/ode_base.py:441-469)
 *     and its dlopen driver (cuda/debug/debug.c:14-17) bind it unchanged.
 *
 *  2. The extern "C" API below: FP64 state, explicit constants stride,
 *     per-system status and step counts, a stream, and a choice of linear
 *     solver.  It replaces the same call (cuda/common/harness.cu:5-106) with
 *     the information the legacy signature cannot carry.
 *
 * Every function returns a wind_status code; none aborts or traps.
 *
 * Layouts (the reference's own, cuda/common/kernel.cu:264-273):
 *   y[s*N + i]                      state, array-of-structures per system
 *   constants[s*n_const + k]        per-system constants
 *   rates[s*R + r], species[(s*R + r)*4 + q]  mass-action reactions
 *   linear[(s*N + j)*N + k]         dense linear term, f_j += L_jk y_k
 * The Jacobian handed to solvers is the reference's transposed layout,
 * Jt[i*N + j] = d f_j / d y_i (cuda/common/kernel.cu:123,
 * cuda/c_baseline/linear_algebra/matrix_ops.c:16-20).
 */
#ifndef WIND_H
#define WIND_H

#ifdef __CUDACC_RTC__
/* compiled by NVRTC inside a runtime plug-in: no C library headers */
typedef signed char int8_t;
typedef short int16_t;
typedef int int32_t;
typedef long long int64_t;
typedef unsigned char uint8_t;
typedef unsigned short uint16_t;
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
#else
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ------------------------------------------------------ */
typedef enum wind_status {
    WIND_OK = 0,
    WIND_ERR_ARGUMENT = 1,     /* bad pointer, size or enum value            */
    WIND_ERR_UNSUPPORTED = 2,  /* combination not built (e.g. N too large)   */
    WIND_ERR_CUDA = 3,         /* a CUDA runtime call failed                 */
    WIND_ERR_NOMEM = 4,        /* device allocation failed / over the cap    */
    WIND_ERR_TIMEOUT = 5,      /* host-side wait ran out                     */
    WIND_ERR_BUSY = 6,         /* admission refused (serving)                */
    WIND_ERR_NOT_FOUND = 7     /* unknown request id (serving)               */
} wind_status;

/* ---- per-system status bits (written to sys_status[s]) ----------------- */
enum {
    WIND_SYS_OK = 0,
    WIND_SYS_NONFINITE = 1,      /* state contains NaN/Inf at the end          */
    WIND_SYS_MAX_ATTEMPTS = 2,   /* attempt budget ran out before tend         */
    WIND_SYS_STALLED = 4,        /* tnow + h == tnow: step below resolution    */
    WIND_SYS_REFINE_FALLBACK = 8,/* mixed solve fell back to the FP64 solve    */
    WIND_SYS_TIMEOUT = 16,       /* device deadline passed                     */
    WIND_SYS_BAD_INPUT = 32      /* species index >= N: system not integrated  */
};

/* ---- enums --------------------------------------------------------------- */
/* Integration method: the reference builds one library per method
 * (cuda/Makefile:68-73, -DSIE / -DRK2).
 * SIM: the semi-implicit midpoint rule with smoothing step (Bader-Deuflhard,
 *      Numerical Recipes 16.6) of python/pysolvers/sim.py:36-90 -- FIXED
 *      steps, no error control: n_integration_steps = m steps of
 *      h = (tend - tnow)/m, the Jacobian re-evaluated at every step, each
 *      (I - hJ) solve by the FP64 LU (solver LU_F64 or AUTO; the controller,
 *      atol, rtol, spec_width and max_attempts are not used).  sys_nsteps
 *      counts the m + 1 linear solves.  Accepted by wind_integrate and
 *      wind_integrate_output_steps (each output interval one m-step call)
 *      for the untiled builtin networks and mass-action networks of up to
 *      32 species; other shapes return WIND_ERR_UNSUPPORTED, the other
 *      entry points WIND_ERR_ARGUMENT. */
enum { WIND_METHOD_SIE = 0, WIND_METHOD_RK2 = 1, WIND_METHOD_SIM = 2 };

/* Step-doubling controller semantics.
 * DEVICE: the reference GPU kernel (cuda/common/kernel.cu:12-39, 191-296):
 *         strict '>' tolerance tests, refinement cap 10 (SIE) / 20 (RK2),
 *         substep h clamped with fmin, SIE update accumulated term by term.
 * GOLD:   the reference CPU twin (cuda/c_baseline/common/common_gold.c:8-153):
 *         '>=' tests, cap 10 for both methods, no clamp, matvec then update. */
enum { WIND_CTRL_DEVICE = 0, WIND_CTRL_GOLD = 1 };

/* Linear solve inside each SIE substep, (I - hJ) x = f.
 * GJE_F64: the reference's unpivoted Gauss-Jordan inverse followed by the
 *          transposed matrix-vector product, in FP64, same operation order
 *          (cuda/c_baseline/linear_algebra/gje_gold.c:5-144,
 *           cuda/linear_algebra/gauss_jordan_elimination.cu:15-212).
 * LU_F64:  partial-pivot LU solve in FP64 (the plain FP64 path).
 * MIXED:   an FP32 Gauss-Jordan inverse of I - hJ computed once per
 *          step-doubling attempt (at the half-step size) and reused as the
 *          approximate inverse of the attempt's substeps -- and of the next
 *          attempt's full step after a rejection -- inside an FP64 iterative
 *          refinement r = f - (x - h J x), x += M r, with J x evaluated in FP64
 *          from the network; stops when the predicted error is below 2^-33
 *          max|x|.  N <= 32: the inverse is pivoted; a substep FP32 cannot
 *          refine is solved by the FP64 LU.  32 < N: the inverse is unpivoted
 *          and blocked, pivoted at and above the step size where the
 *          unpivoted one failed to refine, and an FP32 LU recovery stands
 *          behind both.  Any recovery flags the system
 *          WIND_SYS_REFINE_FALLBACK.
 * AUTO:    per network shape, the faster of the two measured on B200: LU_F64
 *          for the compiled networks and N <= 32, MIXED above 32 species (one
 *          persistent launch still serves a mixed-size batch). */
/* MIXED_TC: MIXED for mass-action networks with 32 < N (wind_integrate,
 *          wind_integrate_output_steps), the blocked inverse's rank-16
 *          updates on the 5th-generation tensor cores: tcgen05.mma kind::tf32
 *          with the accumulator in tensor memory, each operand split into
 *          TF32 high and low parts (hi*hi + hi*lo + lo*hi, FP32-level
 *          products); rows beyond the first 128 on the CUDA cores.  The FP32
 *          matrix and the operand staging must fit in one CTA's shared
 *          memory together (N up to ~190).  Other shapes and entry points
 *          return WIND_ERR_UNSUPPORTED.  Measured slower than MIXED on B200
 *          (the operand staging and the halved CTAs per SM cost more than
 *          the update it moves off the CUDA cores); AUTO never picks it. */
enum { WIND_SOLVER_GJE_F64 = 0, WIND_SOLVER_LU_F64 = 1, WIND_SOLVER_MIXED = 2, WIND_SOLVER_AUTO = 3,
       WIND_SOLVER_MIXED_TC = 4 };

/* Network kinds: the ode_system plug-ins (cuda/include/device.h:1-13,
 * cuda/include/ode_gold.h:1-12).
 *   NR_TEST    2 equations, 4 constants   (python/ode_systems/NR_test.py:575-603)
 *   KATZ96     5 equations, 10 constants  (cuda/ode_system/ode_gold.c:3-93)
 *   STIFFTRIG  2 equations, 2 constants   (python/ode_systems/stifftrig.py:625-661)
 *   MASS_ACTION runtime network: per-system two-body reactions A+B -> C+D
 *              with rate k (w = k y_A y_B), plus an optional dense linear
 *              term L (f += L y).  No reference instance exists; it follows
 *              the same RHS/Jacobian contract. */
enum { WIND_NET_NR_TEST = 1, WIND_NET_KATZ96 = 2, WIND_NET_STIFFTRIG = 3,
       WIND_NET_MASS_ACTION = 4 };

enum { WIND_MEM_HOST = 0, WIND_MEM_DEVICE = 1 };

typedef struct wind_network {
    int32_t kind;               /* WIND_NET_*                                  */
    int32_t n_eq;               /* equations per system (N)                    */
    int32_t n_const;            /* constants per system (builtin kinds)        */
    int32_t n_react;            /* reactions per system (mass action)          */
    const double*   constants;  /* [nsys*n_const] or NULL                      */
    const double*   rates;      /* [nsys*n_react] or NULL                      */
    const uint16_t* species;    /* [nsys*n_react*4] or NULL                    */
    const float*    linear;     /* [nsys*N*N] or NULL                          */
} wind_network;

typedef struct wind_options {
    int32_t method;             /* WIND_METHOD_*                               */
    int32_t solver;             /* WIND_SOLVER_*                               */
    int32_t controller;         /* WIND_CTRL_*                                 */
    int32_t spec_width;         /* speculative refinement lanes per system,
                                   1,2,4,8,16 or 32; 0 = tuned default        */
    int64_t max_attempts;       /* per system per call; 0 = 1<<40              */
    double  timeout_s;          /* device deadline per call; 0 = none          */
} wind_options;

/* Fill `opt` with the defaults: SIE, GJE_F64, DEVICE, tuned width. */
void wind_default_options(wind_options* opt);

/* Integrate nsys independent systems from tnow to tend.
 * Replaces cudaIntegrateSystem (cuda/common/harness.cu:5-106) with FP64 state.
 *  y            [nsys*N] in/out
 *  sys_status   [nsys] out or NULL;  sys_nsteps [nsys] out or NULL
 *  total_nsteps out or NULL: sum of substeps, 3 per attempt
 *               (cuda/common/kernel.cu:192, cuda/common/harness.cu:105)
 *  memory       WIND_MEM_HOST: all arrays are host memory, the call copies
 *               in and out and returns after the results are back.
 *               WIND_MEM_DEVICE: all arrays are device memory on the current
 *               device; the call is asynchronous on `stream` except that
 *               total_nsteps (a host pointer) forces a synchronisation.
 *  stream       cudaStream_t, or NULL for the legacy default stream. */
int wind_integrate(const wind_options* opt, const wind_network* net,
                   double tnow, double tend, int32_t n_integration_steps,
                   double* y, int64_t nsys, double atol, double rtol,
                   int32_t* sys_status, int64_t* sys_nsteps,
                   int64_t* total_nsteps, int32_t memory, void* stream);

/* ---- mixed-size batch in one persistent launch ------------------------- */
/* One group = one network shape with its own systems, interval and
 * tolerances.  All groups of a batch share the method/solver/controller.
 * All pointers are device pointers. */
typedef struct wind_group {
    wind_network net;
    double*  y;                 /* [nsys*N] in/out (device)                    */
    int64_t  nsys;
    double   tnow, tend;
    int32_t  n_integration_steps;
    int32_t  pad_;
    double   atol, rtol;
    int32_t* sys_status;        /* [nsys] (device) or NULL                     */
    int64_t* sys_nsteps;        /* [nsys] (device) or NULL                     */
} wind_group;

/* Integrate all groups in ONE persistent kernel launch fed by a device work
 * queue (largest systems first).  Asynchronous on `stream`. */
int wind_integrate_batch(const wind_options* opt, const wind_group* groups,
                         int32_t ngroups, void* stream);

/* ---- allocation-free batch ---------------------------------------------- */
/* No counterpart in the reference (its harness allocates and frees on every
 * call, cuda/common/harness.cu:28-58,95-102).  For callers that cannot call
 * cudaMalloc -- codes whose device memory belongs to another allocator or
 * budget -- this runs the same kernels as wind_integrate_batch without
 * allocating: the per-group counters the kernels need live in a static
 * device array of WIND_NOALLOC_MAX_GROUPS*4 64-bit words (8 KiB, held by
 * every GPU that loads the library until exit).  All pointers in `groups`
 * are device pointers.  ngroups > WIND_NOALLOC_MAX_GROUPS returns
 * WIND_ERR_ARGUMENT.  Groups run one after another on `stream`.  The array
 * is shared by every call and keeps the last call's contents; each call
 * clears what it uses first, so calls in sequence are independent, while
 * calls that overlap on the GPU race and must not be issued.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress);
 * make it before any stream capture on that device (the lookup is repeated
 * only if the device's CUDA context changed, e.g. after a device reset).  A
 * group whose kernels would need matrix scratch in global memory (mass
 * action with N > 32 whose factor does not fit in shared memory, or
 * Gauss-Jordan with N > 32) makes the whole call return WIND_ERR_UNSUPPORTED
 * before any group is cleared or launched: no state is changed. */
#define WIND_NOALLOC_MAX_GROUPS 256
int wind_integrate_batch_noalloc(const wind_options* opt, const wind_group* groups,
                                 int32_t ngroups, void* stream);

/* ---- the SIE_host variant: one step shared by every system -------------- */
/* Replaces cudaIntegrateSIE (cuda/SIE_host/harness_kernel.cu:427-532, exported
 * as _Z16cudaIntegrateSIEffiPfS_iiff, bound by python/wind_harness.py:27-28)
 * and its controller errorLoop (:248-425): all nsys systems take the same
 * step; an attempt (one full SIE substep and two half substeps from the last
 * accepted state, 3 substeps counted per system) is refined for ALL systems
 * when any element of any system fails the SIE_host error test
 * (vector_kernels.cu:45-70: |y1-y2| > atol, or |(y1-y2)/(y2+1e-12)| > rtol
 * with y1 > atol and y2 > atol -- strict and signed); an accepted attempt
 * takes y2 for all systems and doubles the step.  The loop stops at tend or
 * after 9 consecutive refinements, leaving the last accepted state;
 * *t_reached (may be null) receives the time reached, *total_nsteps the
 * reference's return value (substeps per system times nsys).  Compiled
 * networks only (NR_test, Katz96, StiffTrig; mass action returns
 * WIND_ERR_UNSUPPORTED), SIE only; opt->solver selects the linear solve
 * (GJE_F64 is the reference's Gauss-Jordan in FP64), opt->controller is not
 * used.  Host or device memory as in wind_integrate. */
int wind_integrate_global(const wind_options* opt, const wind_network* net, double tnow,
                          double tend, int32_t n_integration_steps, double* y, int64_t nsys,
                          double atol, double rtol, int64_t* total_nsteps, double* t_reached,
                          int32_t memory, void* stream);

/* ---- device-resident output loop (the caller loop of
 * python/ode_systems/ode_base.py:315-397) -------------------------------- */
/* Integrate n_output_steps intervals of (tend-tnow)/n_output_steps each, with
 * the state resident on the device; after every interval the state is copied
 * to out_over_time[(k+1)*nsys*N ...] (host or device memory, `memory` flag
 * applies to y/out/steps arrays).  out_over_time[0..nsys*N) receives the
 * initial state.  steps_per_output [n_output_steps] receives the substep sum of
 * each interval (ode_base.py:341-349).  The interval launches are captured in
 * one CUDA graph and replayed. */
int wind_integrate_output_steps(const wind_options* opt, const wind_network* net,
                                double tnow, double tend,
                                int32_t n_integration_steps,
                                int32_t n_output_steps,
                                double* y, int64_t nsys, double atol, double rtol,
                                double* out_over_time, int64_t* steps_per_output,
                                int32_t memory, void* stream);

/* ---- serving: request loop with continuous batching --------------------- */
/* No counterpart in the reference (its only caller integrates one batch per
 * blocking call, python/ode_systems/ode_base.py:338-378).  A server owns a
 * worker thread on the current device.  Requests (a set of cells of one
 * network, an interval, tolerances; host arrays copied at submit) are
 * admitted in arrival order while the device footprint of admitted requests
 * stays under hbm_budget_bytes; whenever one of max_inflight launch slots is
 * free, every admitted request not yet running -- of any network size -- is
 * merged into one batch launch (wind_integrate_batch), so requests arriving
 * while others run start at once and overlap with them on the device. */
typedef struct wind_server wind_server;
#define WIND_SERVER_MAX_GROUPS 1024  /* requests merged into one launch at most */
typedef struct wind_server_config {
    int32_t method, solver, controller;
    int32_t max_inflight;        /* launch slots in flight (1..64)             */
    int64_t hbm_budget_bytes;    /* device footprint cap of admitted requests  */
    int64_t max_waiting;         /* waiting requests before submit says BUSY   */
    int32_t poll_us;             /* worker idle wait                           */
    int32_t pad_;
} wind_server_config;
typedef struct wind_request {
    wind_network net;            /* host arrays                                */
    const double* y0;            /* host [nsys*N]                              */
    int64_t nsys;
    double tnow, tend, atol, rtol;
    int32_t n_integration_steps, pad_;
} wind_request;
void wind_server_default_config(wind_server_config* cfg);
int wind_server_create(const wind_server_config* cfg, wind_server** out);
/* Copies the request; WIND_ERR_BUSY when max_waiting requests wait. */
int wind_server_submit(wind_server* srv, const wind_request* req, int64_t* id_out);
/* Waits up to timeout_s for request `id`; on completion copies the final
 * state, per-system status and substep counts (any may be NULL), the
 * submit-to-completion latency, forgets the request and returns its status;
 * WIND_ERR_TIMEOUT if it is not done yet (poll again). */
int wind_server_poll(wind_server* srv, int64_t id, double timeout_s, double* y_out,
                     int32_t* status_out, int64_t* nsteps_out, double* latency_s);
/* waiting, admitted, running, completed, launches, resident bytes */
int wind_server_stats(wind_server* srv, int64_t* out6);
/* Finishes all submitted work, then frees the server. */
int wind_server_destroy(wind_server* srv);

/* ---- runtime network plug-ins (NVRTC) ---------------------------------- */
/* Replaces the reference's build-time Precompiler (python/ode_systems/
 * ode_base.py:16-123), which splices a network's bodies into the solver
 * sources and rebuilds lib/sie.so.  `source` is the network as the
 * reference's host plug-in (cuda/include/ode_gold.h:1-12, the Precompiler's
 * ode_gold.c output):
 *     #include "ode_gold.h"
 *     void calculate_dydt(float tnow, float* equations, float* constants,
 *                         float* dydt, int Neqn_p_sys);
 *     void calculate_jacobian(float* equations, float* constants,
 *                             float* Jacobian);   (transposed, zero-filled)
 * It is compiled at run time (NVRTC, sm_100a) in FP64 -- `float` is defined
 * as `double` around it -- with every product rounded before its add, and
 * linked to the team-per-system Gauss-Jordan integrator.  n_eq <= 64 equations,
 * n_const constants per system (NUM_CONST in the plug-in); `options` are
 * extra NVRTC options separated by spaces (e.g. "-DNTILE=4"), or NULL; the
 * compiler's log is copied into log[log_size] when given.
 * Returns WIND_ERR_ARGUMENT when the source does not compile and
 * WIND_ERR_UNSUPPORTED when NVRTC is not available or n_eq > 64. */
typedef struct wind_plugin wind_plugin;
int wind_plugin_create(const char* source, int32_t n_eq, int32_t n_const, const char* options,
                       wind_plugin** out, char* log, int64_t log_size);
int wind_plugin_destroy(wind_plugin* plugin);
/* wind_integrate for a plug-in network: constants[nsys*n_const], y[nsys*n_eq];
 * the solver is the reference's Gauss-Jordan (GJE_F64; AUTO selects it),
 * either controller, SIE or RK2.  The time passed to calculate_dydt is the
 * substep's start, as in the reference's c_baseline (sie_gold.c:54-78). */
int wind_integrate_plugin(const wind_options* opt, wind_plugin* plugin, double tnow, double tend,
                          int32_t n_integration_steps, const double* constants, double* y,
                          int64_t nsys, double atol, double rtol, int32_t* sys_status,
                          int64_t* sys_nsteps, int64_t* total_nsteps, int32_t memory,
                          void* stream);

/* ---- version / diagnostics -------------------------------------------- */
const char* wind_version(void);
const char* wind_status_string(int status);
/* The CUDA error behind the calling thread's last WIND_ERR_CUDA, as
 * "<where>: <cudaError name>" ("" if none). */
const char* wind_last_error(void);
/* Kernel launches issued by this library since load (all entry points). */
int64_t wind_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* WIND_H */
