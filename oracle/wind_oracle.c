/*
 * wind_oracle.c -- CPU restatement of WIND's batched SIE / RK2 step-doubling
 * integrators, in FP64.  TEST INFRASTRUCTURE ONLY: it is the checker for the
 * CUDA path (tests, __graft_entry__.smoke, bench.py's cpu_baseline leg) and is
 * never linked into or called by the product libraries.
 *
 * Parity pinning: in GOLD controller semantics this file reproduces the
 * reference CPU twin compiled in double precision (cuda/c_baseline built with
 * -Dfloat=double, recipe oracle/build_ref.sh) bit for bit; the tests compare
 * the two on every network and on the committed golden vectors.  DEVICE
 * semantics restate the reference GPU kernel (cuda/common/kernel.cu), whose
 * differences from GOLD are listed at each switch below.
 *
 * No FMA contraction: compile with -ffp-contract=off (the recipe does), so
 * every product is rounded before it is added, as in the reference's x86-64
 * build and in the CUDA kernels (which use explicit __dmul_rn/__dadd_rn).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/wind.h"

#define ORACLE_MAXN 320

/* ------------------------------------------------------------------------ */
/* ode_system plug-ins: RHS f and transposed Jacobian Jt[i*N+j] = df_j/dy_i  */
/* ------------------------------------------------------------------------ */

/* NR_test, generated body of python/ode_systems/NR_test.py:584-590 (RHS)
 * and :575-582 (Jacobian) for Ntile=1. */
static void nr_rhs(const double* c, const double* y, double* f) {
    f[0] = c[0] * y[0] + c[1] * y[1];
    f[1] = c[2] * y[0] + c[3] * y[1];
}
static void nr_jac(const double* c, double* J) {
    J[0] = c[0];
    J[1] = c[2];
    J[2] = c[1];
    J[3] = c[3];
}

/* Katz96, cuda/ode_system/ode_gold.c:3-48 (RHS) and :50-93 (Jacobian),
 * same expression order.  J[13] = J[12] keeps the reference's sign
 * (ode_gold.c:79, device_dydt.cu:91): parity is with what it computes. */
static void katz_rhs_ne(const double* c, double ne, const double* y, double* f) {
    f[0] = c[2] * ne * y[1] - (c[0] * ne + c[1]) * y[0];
    f[1] = -c[2] * ne * y[1] + (c[0] * ne + c[1]) * y[0];
    f[2] = (c[7] + c[8]) * ne * y[3] - (c[3] * ne + c[4]) * y[2];
    f[3] = c[9] * ne * y[4] + (c[3] * ne + c[4]) * y[2]
         - (c[7] + c[8]) * ne * y[3] - (c[5] * ne + c[6]) * y[3];
    f[4] = (c[5] * ne + c[6]) * y[3] - c[9] * ne * y[4];
}
static void katz_jac_ne(const double* c, double ne, double* J) {
    J[0] = -(c[0] * ne + c[1]);
    J[1] = -J[0];
    J[6] = -c[2] * ne;
    J[5] = -J[6];
    J[12] = -(c[3] * ne + c[4]);
    J[13] = J[12];
    J[19] = c[5] * ne + c[6];
    J[17] = (c[7] + c[8]) * ne;
    J[18] = -J[17] - J[19];
    J[24] = -c[9] * ne;
    J[23] = -J[24];
}

/* the generated prefix: ne from equations 1, 3, 4 (katz96.py:485-500) */
static double katz_ne(const double* y) { return y[1] + y[3] + y[4] * 2.0; }

/* StiffTrig, python/ode_systems/stifftrig.py:639-647 (RHS), :625-637 (J). */
static void trig_rhs(const double* c, const double* y, double* f) {
    f[0] = -y[0] + c[1] * y[1];
    f[1] = -y[1] - c[0] * y[0];
}
static void trig_jac(const double* c, double* J) {
    J[0] = -1;
    J[2] = c[1];
    J[1] = -c[0];
    J[3] = -1;
}

/* Mass action with optional dense linear part (no reference instance; this is
 * the operation order every implementation of WIND_NET_MASS_ACTION follows):
 *   f_j  = sum_k L_jk y_k  (k ascending, starting from 0.0)
 *   for r ascending: w = (k_r * y_A) * y_B;
 *        f_A -= w; f_B -= w; f_C += w; f_D += w;
 *   Jt_ij = L_ji, then for r ascending with dA = k_r*y_B, dB = k_r*y_A:
 *        Jt[A][A]-=dA; Jt[A][B]-=dA; Jt[A][C]+=dA; Jt[A][D]+=dA;
 *        Jt[B][A]-=dB; Jt[B][B]-=dB; Jt[B][C]+=dB; Jt[B][D]+=dB; */
static void ma_rhs(int N, int R, const double* k, const uint16_t* sp,
                   const float* L, const double* y, double* f) {
    for (int j = 0; j < N; j++) {
        double acc = 0.0;
        if (L) {
            for (int q = 0; q < N; q++) acc += (double)L[j * N + q] * y[q];
        }
        f[j] = acc;
    }
    for (int r = 0; r < R; r++) {
        int a = sp[4 * r], b = sp[4 * r + 1], c = sp[4 * r + 2], d = sp[4 * r + 3];
        double w = k[r] * y[a] * y[b];
        f[a] -= w;
        f[b] -= w;
        f[c] += w;
        f[d] += w;
    }
}
static void ma_jac(int N, int R, const double* k, const uint16_t* sp,
                   const float* L, const double* y, double* J) {
    if (L) {
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++) J[i * N + j] = (double)L[j * N + i];
    }
    for (int r = 0; r < R; r++) {
        int a = sp[4 * r], b = sp[4 * r + 1], c = sp[4 * r + 2], d = sp[4 * r + 3];
        double da = k[r] * y[b];
        double db = k[r] * y[a];
        J[a * N + a] -= da;
        J[a * N + b] -= da;
        J[a * N + c] += da;
        J[a * N + d] += da;
        J[b * N + a] -= db;
        J[b * N + b] -= db;
        J[b * N + c] += db;
        J[b * N + d] += db;
    }
}

typedef struct {
    const wind_network* net;
    int64_t s;
} sysref;

/* Equations per copy of a builtin network; n_eq = Ntile x base_n for the
 * Precompiler's tiling (python/ode_systems/ode_base.py:86-88, 219-281): tile
 * t owns equations [t*base_n, (t+1)*base_n), every tile uses the system's
 * one set of constants, the Jacobian is block diagonal (reindex,
 * ode_base.py:86-88), and Katz96's ne comes from tile 0 (the prefix is not
 * reindexed, katz96.py:331-448). */
static int base_n(int kind) { return kind == WIND_NET_KATZ96 ? 5 : 2; }

static int net_ok(const wind_network* net) {
    if (!net || net->n_eq < 1 || net->n_eq > ORACLE_MAXN) return 0;
    if (net->kind == WIND_NET_MASS_ACTION) return 1;
    if (net->kind != WIND_NET_NR_TEST && net->kind != WIND_NET_KATZ96 &&
        net->kind != WIND_NET_STIFFTRIG)
        return 0;
    return net->n_eq % base_n(net->kind) == 0;
}

static void eval_rhs(const sysref* sr, const double* y, double* f) {
    const wind_network* n = sr->net;
    const double* c = n->constants ? n->constants + sr->s * n->n_const : NULL;
    const int b = base_n(n->kind), nt = n->n_eq / b;
    switch (n->kind) {
    case WIND_NET_NR_TEST:
        for (int t = 0; t < nt; t++) nr_rhs(c, y + t * b, f + t * b);
        break;
    case WIND_NET_KATZ96: {
        double ne = katz_ne(y);
        for (int t = 0; t < nt; t++) katz_rhs_ne(c, ne, y + t * b, f + t * b);
        break;
    }
    case WIND_NET_STIFFTRIG:
        for (int t = 0; t < nt; t++) trig_rhs(c, y + t * b, f + t * b);
        break;
    default: {
        int N = n->n_eq, R = n->n_react;
        ma_rhs(N, R, n->rates + sr->s * R, n->species + sr->s * R * 4,
               n->linear ? n->linear + sr->s * N * N : NULL, y, f);
    }
    }
}

/* Jacobian into a zero-filled buffer (gold: sie_gold.c:59 memset). */
static void eval_jac(const sysref* sr, const double* y, double* J) {
    const wind_network* n = sr->net;
    int N = n->n_eq;
    memset(J, 0, sizeof(double) * N * N);
    const double* c = n->constants ? n->constants + sr->s * n->n_const : NULL;
    if (n->kind != WIND_NET_MASS_ACTION) {
        /* each tile's block written at its place on the diagonal */
        const int b = base_n(n->kind), nt = N / b;
        double ne = n->kind == WIND_NET_KATZ96 ? katz_ne(y) : 0.0;
        for (int t = 0; t < nt; t++) {
            double Jb[25];
            memset(Jb, 0, sizeof(Jb));
            if (n->kind == WIND_NET_NR_TEST) nr_jac(c, Jb);
            else if (n->kind == WIND_NET_KATZ96) katz_jac_ne(c, ne, Jb);
            else trig_jac(c, Jb);
            for (int r = 0; r < b; r++)
                for (int q = 0; q < b; q++) J[(t * b + r) * N + t * b + q] = Jb[r * b + q];
        }
        return;
    }
    switch (n->kind) {
    default: {
        int R = n->n_react;
        ma_jac(N, R, n->rates + sr->s * R, n->species + sr->s * R * 4,
               n->linear ? n->linear + sr->s * N * N : NULL, y, J);
    }
    }
}

/* ------------------------------------------------------------------------ */
/* Unpivoted Gauss-Jordan inverse, cuda/c_baseline/linear_algebra/gje_gold.c */
/* ------------------------------------------------------------------------ */
static void gje_invert(double* M, double* Inv, int n) {
    /* setIdentity, gje_gold.c:5-16 */
    memset(Inv, 0, sizeof(double) * n * n);
    for (int i = 0; i < n; i++) Inv[i * (n + 1)] = 1;
    /* gjeUFactor, gje_gold.c:56-100: scale pivot row, eliminate below */
    for (int i = 0; i < n; i++) {
        double s = M[i * n + i];
        for (int t = 0; t < n; t++) M[i * n + t] /= s;
        for (int t = 0; t < n; t++) Inv[i * n + t] /= s;
        for (int k = i + 1; k < n; k++) {
            double f = M[k * n + i];
            for (int t = 0; t < n; t++) M[k * n + t] -= f * M[i * n + t];
            for (int t = 0; t < n; t++) Inv[k * n + t] -= f * Inv[i * n + t];
        }
    }
    /* gjeLFactor, gje_gold.c:102-134: eliminate above, bottom-up */
    for (int ri = 0; ri < n; ri++) {
        int bri = n - 1 - ri;
        for (int nri = ri + 1; nri < n; nri++) {
            int bnri = n - 1 - nri;
            double f = M[bnri * n + bri];
            for (int t = 0; t < n; t++) M[bnri * n + t] -= f * M[bri * n + t];
            for (int t = 0; t < n; t++) Inv[bnri * n + t] -= f * Inv[bri * n + t];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Substeps                                                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
    double J[ORACLE_MAXN * ORACLE_MAXN];
    double Inv[ORACLE_MAXN * ORACLE_MAXN];
    double f[ORACLE_MAXN];
    double out[ORACLE_MAXN];
} scratch_t;

/* One SIE substep of length h from y, in place.
 * GOLD: sie_gold.c:38-79 -- A = (-h)J then diag += 1, GJE inverse, out = Inv^T f
 *       (matrix_ops.c:6-27), y += h*out.
 * DEVICE: kernel.cu:69-138 -- A = (i==j) - J*h, GJE, y_j += (Inv_kj*f_k)*h
 *       accumulated for k ascending. */
static void sie_substep(const sysref* sr, int ctrl, double h, double* y,
                        scratch_t* w) {
    int n = sr->net->n_eq;
    eval_rhs(sr, y, w->f);
    eval_jac(sr, y, w->J);
    if (ctrl == WIND_CTRL_GOLD) {
        for (int e = 0; e < n * n; e++) w->J[e] = -h * w->J[e];
        for (int i = 0; i < n; i++) w->J[i * (n + 1)] += 1;
    } else {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                w->J[i * n + j] = (double)(i == j) - w->J[i * n + j] * h;
    }
    gje_invert(w->J, w->Inv, n);
    if (ctrl == WIND_CTRL_GOLD) {
        for (int r = 0; r < n; r++) w->out[r] = 0;
        for (int c = 0; c < n; c++)
            for (int r = 0; r < n; r++) w->out[r] += w->Inv[c * n + r] * w->f[c];
        for (int e = 0; e < n; e++) y[e] += h * w->out[e];
    } else {
        for (int k = 0; k < n; k++)
            for (int j = 0; j < n; j++) y[j] += w->Inv[k * n + j] * w->f[k] * h;
    }
}

/* One explicit Euler substep (rk2_gold.c:19-46, kernel.cu:128-130). */
static void euler_substep(const sysref* sr, double h, double* y, scratch_t* w) {
    int n = sr->net->n_eq;
    eval_rhs(sr, y, w->f);
    for (int e = 0; e < n; e++) y[e] += h * w->f[e];
}

/* take_step / innerstep: nsub substeps spanning [t0, t1].
 * GOLD (sie_gold.c:38-51): h = (t1-t0)/nsub, no clamp.
 * DEVICE (kernel.cu:82-88): h = (t1-t0)/nsub, then h = fmin(t1 - t, h) at
 * every substep with t advanced by h. */
static void take_step(const sysref* sr, int method, int ctrl, double t0,
                      double t1, int nsub, double* y, scratch_t* w) {
    double h = (t1 - t0) / nsub;
    double t = t0;
    for (int i = 0; i < nsub; i++) {
        if (ctrl == WIND_CTRL_DEVICE) h = fmin(t1 - t, h);
        if (method == WIND_METHOD_SIE) sie_substep(sr, ctrl, h, y, w);
        else euler_substep(sr, h, y, w);
        t += h;
    }
}

/* checkError.  GOLD common_gold.c:8-46 ('>=' tests); DEVICE kernel.cu:12-39
 * ('>' tests).  SIE relative denominator y2+1e-12, RK2 2*y2-y1+1e-12. */
static int check_error(int method, int ctrl, const double* y1, const double* y2,
                       int n, double atol, double rtol) {
    int flag = 0;
    for (int e = 0; e < n; e++) {
        double abs_err = fabs(y2[e] - y1[e]);
        double rel_err = (method == WIND_METHOD_RK2)
                             ? fabs((y2[e] - y1[e]) / (2 * y2[e] - y1[e] + 1e-12))
                             : fabs((y2[e] - y1[e]) / (y2[e] + 1e-12));
        if (ctrl == WIND_CTRL_GOLD) {
            if (abs_err >= atol) flag = 1;
            if (rel_err >= rtol && fabs(y1[e]) > atol && fabs(y2[e]) > atol) flag = 1;
        } else {
            if (abs_err > atol) flag = 1;
            if (rel_err > rtol && fabs(y1[e]) > atol && fabs(y2[e]) > atol) flag = 1;
        }
    }
    return flag;
}

/* The adaptive loop for one system: common_gold.c:48-153 / kernel.cu:191-296.
 * Returns the substep count (3 per attempt). */
static int64_t integrate_one(const sysref* sr, int method, int ctrl,
                             double tnow, double tend, double timestep,
                             double* y, double atol, double rtol,
                             int64_t max_attempts, int32_t* status, scratch_t* w) {
    int n = sr->net->n_eq;
    double y1[ORACLE_MAXN], y2[ORACLE_MAXN];
    int cap = (ctrl == WIND_CTRL_DEVICE && method == WIND_METHOD_RK2) ? 20 : 10;
    int64_t nsteps = 0, attempts = 0;
    int unsolved = 0;
    int32_t st = WIND_SYS_OK;
    while (tnow < tend) {
        if (attempts >= max_attempts) { st |= WIND_SYS_MAX_ATTEMPTS; break; }
        attempts++;
        timestep = fmin(tend - tnow, timestep);
        memcpy(y1, y, sizeof(double) * n);
        memcpy(y2, y, sizeof(double) * n);
        take_step(sr, method, ctrl, tnow, tnow + timestep, 1, y1, w);
        take_step(sr, method, ctrl, tnow, tnow + timestep, 2, y2, w);
        nsteps += 3;
        int err = check_error(method, ctrl, y1, y2, n, atol, rtol);
        if (err && unsolved < cap) {
            unsolved++;
            timestep /= 2.0;
        } else {
            unsolved = 0;
            if (method == WIND_METHOD_RK2) {
                for (int e = 0; e < n; e++) y[e] = 2 * y2[e] - y1[e];
            } else {
                memcpy(y, y2, sizeof(double) * n);
            }
            if (tnow + timestep == tnow) { st |= WIND_SYS_STALLED; break; }
            tnow += timestep;
            if (method == WIND_METHOD_RK2) timestep *= 2;
            else timestep = tend - tnow;
        }
    }
    for (int e = 0; e < n; e++)
        if (!isfinite(y[e])) st |= WIND_SYS_NONFINITE;
    if (status) *status = st;
    return nsteps;
}

/* Integrate systems [s_begin, s_end) of `net`; y is the full [nsys*N] array.
 * h0 = (tend - tnow)/n_integration_steps (harness.cu:80, sie_gold.c:105).
 * Returns the substep total of the range, or -1 on bad arguments. */
int64_t wind_oracle_integrate(int method, int ctrl, const wind_network* net,
                              double tnow, double tend, int n_integration_steps,
                              double* y, int64_t s_begin, int64_t s_end,
                              double atol, double rtol, int64_t max_attempts,
                              int32_t* status, int64_t* sys_nsteps) {
    if (!net_ok(net) || !y ||
        n_integration_steps < 1)
        return -1;
    if (max_attempts <= 0) max_attempts = (int64_t)1 << 40;
    scratch_t* w = (scratch_t*)malloc(sizeof(scratch_t));
    if (!w) return -1;
    int n = net->n_eq;
    int64_t total = 0;
    double h0 = (tend - tnow) / n_integration_steps;
    for (int64_t s = s_begin; s < s_end; s++) {
        sysref sr = {net, s};
        int32_t st = 0;
        int64_t k = integrate_one(&sr, method, ctrl, tnow, tend, h0, y + s * n,
                                  atol, rtol, max_attempts, &st, w);
        if (status) status[s] = st;
        if (sys_nsteps) sys_nsteps[s] = k;
        total += k;
    }
    free(w);
    return total;
}

/* RHS and transposed Jacobian of one system, for plug-in tests. */
int wind_oracle_rhs_jac(const wind_network* net, int64_t s, const double* y,
                        double* f, double* Jt) {
    if (!net_ok(net)) return -1;
    sysref sr = {net, s};
    if (f) eval_rhs(&sr, y, f);
    if (Jt) eval_jac(&sr, y, Jt);
    return 0;
}

/* One SIE substep of one system (tests of the solver paths). */
int wind_oracle_sie_substep(const wind_network* net, int64_t s, int ctrl,
                            double h, double* y) {
    if (!net_ok(net)) return -1;
    scratch_t* w = (scratch_t*)malloc(sizeof(scratch_t));
    if (!w) return -1;
    sysref sr = {net, s};
    sie_substep(&sr, ctrl, h, y, w);
    free(w);
    return 0;
}

/* The SIE_host variant's controller (cuda/SIE_host/harness_kernel.cu:248-425,
 * errorLoop): every system advances with ONE shared step.  Per attempt
 * (3 substeps counted per system, :292): y1 = one substep of h, y2 = two of
 * h/2 from the last accepted state (solveSystem, :175-246, with GOLD
 * substep arithmetic: h_sub = (t1 - t0)/n, y += h*(Inv f)); the error flag is
 * set when ANY element of ANY system fails checkError (vector_kernels.cu:45-70:
 * |y1 - y2| > atol, or |(y1 - y2)/(y2 + 1e-12)| > rtol with y1 > atol and
 * y2 > atol -- signed, strict).  A failed attempt halves the step for all
 * (:363-367); an accepted one takes y2 for all, advances t and doubles the
 * step (:383-400).  The loop ends at tend or after 9 consecutive refinements
 * (:289), leaving the last accepted state.  Returns the substep total over
 * all systems (nsteps * Nsystems, :423), *t_reached the time reached. */
int64_t wind_oracle_integrate_global(const wind_network* net, double tnow, double tend,
                                     int n_integration_steps, double* y, int64_t nsys,
                                     double atol, double rtol, double* t_reached) {
    if (!net_ok(net) || !y || n_integration_steps < 1 ||
        nsys < 0)
        return -1;
    int n = net->n_eq;
    scratch_t* w = (scratch_t*)malloc(sizeof(scratch_t));
    double* y1 = (double*)malloc(sizeof(double) * (size_t)(nsys > 0 ? nsys : 1) * n);
    double* y2 = (double*)malloc(sizeof(double) * (size_t)(nsys > 0 ? nsys : 1) * n);
    if (!w || !y1 || !y2) { free(w); free(y1); free(y2); return -1; }
    int64_t nsteps = 0;
    int unsolved = 0;
    double timestep = (tend - tnow) / n_integration_steps;
    while (tnow < tend && unsolved < 9) {
        timestep = fmin(timestep, tend - tnow);
        nsteps += 3;
        int flag = 0;
        for (int64_t s = 0; s < nsys; s++) {
            sysref sr = {net, s};
            double* a = y1 + s * n;
            double* b = y2 + s * n;
            memcpy(a, y + s * n, sizeof(double) * n);
            memcpy(b, y + s * n, sizeof(double) * n);
            take_step(&sr, WIND_METHOD_SIE, WIND_CTRL_GOLD, tnow, tnow + timestep, 1, a, w);
            take_step(&sr, WIND_METHOD_SIE, WIND_CTRL_GOLD, tnow, tnow + timestep, 2, b, w);
            for (int e = 0; e < n; e++) {
                if (fabs(a[e] - b[e]) > atol) flag = 1;
                if (fabs((a[e] - b[e]) / (b[e] + 1e-12)) > rtol && a[e] > atol && b[e] > atol)
                    flag = 1;
            }
        }
        if (flag) {
            unsolved++;
            timestep /= 2;
        } else {
            unsolved = 0;
            memcpy(y, y2, sizeof(double) * (size_t)nsys * n);
            tnow += timestep;
            timestep *= 2;
        }
    }
    if (t_reached) *t_reached = tnow;
    free(w);
    free(y1);
    free(y2);
    return nsteps * nsys;
}

/* ------------------------------------------------------------------------ */
/* Semi-implicit midpoint rule (Bader-Deuflhard), python/pysolvers/sim.py    */
/* ------------------------------------------------------------------------ */
/* Solve (I - h J) x = b in place on b, J in the plug-ins' transposed layout
 * (Jt[i*N+j] = df_j/dy_i), by an FP64 LU with partial pivoting.  The
 * reference inverts the matrix with numpy.linalg.inv and multiplies
 * (sim.py:61-64); both are the same solve up to rounding. */
static int lu_solve_ih(int n, double h, const double* Jt, double* A, double* b) {
    for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++) A[r * n + c] = (r == c ? 1.0 : 0.0) - h * Jt[c * n + r];
    for (int k = 0; k < n; k++) {
        int p = k;
        double best = fabs(A[k * n + k]);
        for (int r = k + 1; r < n; r++)
            if (fabs(A[r * n + k]) > best) { best = fabs(A[r * n + k]); p = r; }
        if (best == 0.0) return -1;
        if (p != k) {
            for (int c = 0; c < n; c++) {
                double t = A[k * n + c]; A[k * n + c] = A[p * n + c]; A[p * n + c] = t;
            }
            double t = b[k]; b[k] = b[p]; b[p] = t;
        }
        for (int r = k + 1; r < n; r++) {
            double m = A[r * n + k] / A[k * n + k];
            for (int c = k + 1; c < n; c++) A[r * n + c] -= m * A[k * n + c];
            b[r] -= m * b[k];
        }
    }
    for (int k = n - 1; k >= 0; k--) {
        double s = b[k];
        for (int c = k + 1; c < n; c++) s -= A[k * n + c] * b[c];
        b[k] = s / A[k * n + k];
    }
    return 0;
}

/* m steps of size h = (tend - tnow)/m of the semi-implicit midpoint rule with
 * the smoothing step (Numerical Recipes 16.6, as sim.py:36-90 implements it,
 * with the Jacobian re-evaluated at every y_k, sim.py:59):
 *   D_0 = (I - hJ(y_0))^-1 h f(y_0),                 y_1 = y_0 + D_0
 *   D_k = D_{k-1} + 2 (I - hJ(y_k))^-1 (h f(y_k) - D_{k-1}),
 *                                      y_{k+1} = y_k + D_k,  k = 1..m-1
 *   ybar = y_m + (I - hJ(y_m))^-1 (h f(y_m) - D_{m-1})
 * ybar is the result at tend.  The reference's integrate_sie(y0, c, dt, tend)
 * takes M = len(arange(0, tend + dt, dt)) - 1 interior steps after the first
 * (sim.py:51-80), so its final row equals m = M + 1 steps over (M + 1) dt.
 * Per system: nsteps = m + 1 linear solves; status NONFINITE when ybar is
 * not finite.  Returns the solve total of the range, -1 on bad arguments. */
int64_t wind_oracle_integrate_sim(const wind_network* net, double tnow, double tend, int m,
                                  double* y, int64_t s_begin, int64_t s_end,
                                  int32_t* status, int64_t* sys_nsteps) {
    if (!net_ok(net) || !y || m < 1) return -1;
    scratch_t* w = (scratch_t*)malloc(sizeof(scratch_t));
    double* d = (double*)malloc(sizeof(double) * ORACLE_MAXN);
    if (!w || !d) { free(w); free(d); return -1; }
    const int n = net->n_eq;
    const double h = (tend - tnow) / m;
    int64_t total = 0;
    for (int64_t s = s_begin; s < s_end; s++) {
        sysref sr = {net, s};
        double* ys = y + s * n;
        int32_t st = 0;
        for (int k = 0; k <= m; k++) {
            eval_rhs(&sr, ys, w->f);
            eval_jac(&sr, ys, w->J);
            for (int i = 0; i < n; i++) w->out[i] = h * w->f[i] - (k ? d[i] : 0.0);
            if (lu_solve_ih(n, h, w->J, w->Inv, w->out) != 0) {
                for (int i = 0; i < n; i++) w->out[i] = NAN;
            }
            for (int i = 0; i < n; i++) {
                if (k == 0 || k == m) d[i] = w->out[i];
                else d[i] = d[i] + 2.0 * w->out[i];
                ys[i] = ys[i] + d[i];
            }
        }
        for (int i = 0; i < n; i++)
            if (!isfinite(ys[i])) st |= WIND_SYS_NONFINITE;
        if (status) status[s] = st;
        if (sys_nsteps) sys_nsteps[s] = m + 1;
        total += m + 1;
    }
    free(w);
    free(d);
    return total;
}
