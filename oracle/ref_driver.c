/*
 * ORACLE — test infrastructure only.  Driver around the UNMODIFIED reference 2DCode
 * sources, compiled from where they lie by oracle/Makefile into oracle/_ref/.  Only the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library, and
 * only to check or time the reference; nothing in the product calls it.
 *
 * What it adds around the reference functions:
 *  - ref_set_mesh(): fills the reference globals (2DCode/MeshAttributes.h:5-42) from
 *    arrays, so meshes too large for the O(E*N) builder of
 *    2DCode/extract_mesh_attributes.c:260-295 can still be stepped by the reference code.
 *  - ref_step(): one SSP-RK2 step.  With wet_dry = 0 and rain = 0 it calls the
 *    reference's own oneTimeStep2D (2DCode/time_evolution.c:10-246).  Otherwise it
 *    runs the same gsl-vector sequence with the wet/dry calls placed where
 *    ChanNet/time_evolution.c:218-427 puts them under WDON:
 *       wetDryStatus2D, L, w1=w+dt*L, SlopeLimiter, PDop2D, wetDryStatus2D,
 *       w1+=w, L, w=0.5*w1+dt/2*L, SlopeLimiter, PDop2D
 *    and, when rain != 0, RHSZeta += rain right after each compute2DL.
 *  - ref_run(): the time loop of 2DCode/time_evolution.c:311-402 with the CFL number,
 *    first dt and the tide as parameters.
 *  - exit() in the reference is caught (shim/ref_hooks.h) and returned as -1 with the
 *    reference's own message.
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "MeshAttributes.h"
#include "gsl/gsl_vector.h"
#include "../dg-rain_b200/csrc/dgr_forcing.h"

extern void store_mesh(char *Mesh);
extern void extract_mesh_attributes();
extern void initialize();
extern void boundary_conditions();
extern void compute2DL(double time);
extern void SlopeLimiter();
extern void oneTimeStep2D(double time, double dt);
extern void time_evolution(double FinalTime);
extern void wetDryStatus2D();
extern void PDop2D();
extern double RoeFlux(double *Fhatdotn, double zeta_in, double zeta_ex, double Qx_in, double Qx_ex,
                      double Qy_in, double Qy_ex, double z_edge, double nx, double ny, double localG);
extern void Compute2DInnerProducts(double SI[9], double VI[21], int el, double time);

#undef exit
#undef printf

static jmp_buf g_jump;
static int g_jump_armed = 0;
static char g_last_msg[512];

void dgr_ref_exit(int status)
{
    if (g_jump_armed) longjmp(g_jump, status == 0 ? 1 : status);
    fprintf(stderr, "reference exit(%d) outside a guarded call: %s\n", status, g_last_msg);
    abort();
}

int dgr_ref_printf(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    int n = vsnprintf(g_last_msg, sizeof(g_last_msg), fmt, ap);
    va_end(ap);
    return n;
}

const char *ref_last_message(void) { return g_last_msg; }

#define GUARD_BEGIN                                                   \
    g_last_msg[0] = 0;                                                \
    if (setjmp(g_jump) != 0) {                                        \
        g_jump_armed = 0;                                             \
        return -1;                                                    \
    }                                                                 \
    g_jump_armed = 1;
#define GUARD_END g_jump_armed = 0;

/* ---------------------------------------------------------------- mesh ---- */

int ref_load_fort14(const char *path)
{
    GUARD_BEGIN
    minEdgLength = 9999999;
    store_mesh((char *)path);
    extract_mesh_attributes();
    GUARD_END
    return 0;
}

static void *dup_bytes(const void *src, size_t n)
{
    void *p = malloc(n ? n : 1);
    if (p && n) memcpy(p, src, n);
    return p;
}

int ref_set_mesh(int ne, int nn, int nf, const double *x, const double *y, const double *zz,
                 const double *nfric, const int *el2v, const int *ed2el, const int *ed2v,
                 const int *bdry, double min_edge_length)
{
    NumEl = ne;
    NumNodes = nn;
    NumEdges = nf;
    x_coord = dup_bytes(x, sizeof(double) * (size_t)nn);
    y_coord = dup_bytes(y, sizeof(double) * (size_t)nn);
    z = dup_bytes(zz, sizeof(double) * (size_t)nn);
    nFriction = dup_bytes(nfric, sizeof(double) * (size_t)nn);
    EltoVert = dup_bytes(el2v, sizeof(int) * 3 * (size_t)ne);
    EdgtoEls = dup_bytes(ed2el, sizeof(int) * 2 * (size_t)nf);
    EdgtoVert = dup_bytes(ed2v, sizeof(int) * 2 * (size_t)nf);
    BdryPrescribed = dup_bytes(bdry, sizeof(int) * (size_t)nf);
    minEdgLength = min_edge_length;
    return 0;
}

void ref_get_counts(int *ne, int *nn, int *nf, double *min_edge)
{
    *ne = NumEl;
    *nn = NumNodes;
    *nf = NumEdges;
    *min_edge = minEdgLength;
}

void ref_get_mesh(double *x, double *y, double *zz, double *nfric, int *el2v, int *ed2el,
                  int *ed2v, int *bdry)
{
    memcpy(x, x_coord, sizeof(double) * (size_t)NumNodes);
    memcpy(y, y_coord, sizeof(double) * (size_t)NumNodes);
    memcpy(zz, z, sizeof(double) * (size_t)NumNodes);
    memcpy(nfric, nFriction, sizeof(double) * (size_t)NumNodes);
    memcpy(el2v, EltoVert, sizeof(int) * 3 * (size_t)NumEl);
    memcpy(ed2el, EdgtoEls, sizeof(int) * 2 * (size_t)NumEdges);
    memcpy(ed2v, EdgtoVert, sizeof(int) * 2 * (size_t)NumEdges);
    memcpy(bdry, BdryPrescribed, sizeof(int) * (size_t)NumEdges);
}

/* --------------------------------------------------------------- state ---- */

int ref_initialize(void)
{
    GUARD_BEGIN
    initialize();
    GUARD_END
    return 0;
}

void ref_set_state(const double *zt, const double *qx, const double *qy, const int *wd)
{
    size_t n = 3 * (size_t)NumEl;
    memcpy(zeta, zt, n * sizeof(double));
    memcpy(Qx, qx, n * sizeof(double));
    memcpy(Qy, qy, n * sizeof(double));
    if (wd) memcpy(WD, wd, (size_t)NumEl * sizeof(int));
}

void ref_get_state(double *zt, double *qx, double *qy, int *wd)
{
    size_t n = 3 * (size_t)NumEl;
    memcpy(zt, zeta, n * sizeof(double));
    memcpy(qx, Qx, n * sizeof(double));
    memcpy(qy, Qy, n * sizeof(double));
    if (wd) memcpy(wd, WD, (size_t)NumEl * sizeof(int));
}

void ref_get_rhs(double *rz, double *rqx, double *rqy)
{
    size_t n = 3 * (size_t)NumEl;
    memcpy(rz, RHSZeta, n * sizeof(double));
    memcpy(rqx, RHSQx, n * sizeof(double));
    memcpy(rqy, RHSQy, n * sizeof(double));
}

void ref_get_fhat(double *f1, double *f2, double *f3)
{
    size_t n = 3 * (size_t)NumEl;
    memcpy(f1, Fhat1dotn, n * sizeof(double));
    memcpy(f2, Fhat2dotn, n * sizeof(double));
    memcpy(f3, Fhat3dotn, n * sizeof(double));
}

void ref_set_bc(const double *bz, const double *bq)
{
    memcpy(bzeta, bz, (size_t)NumEdges * sizeof(double));
    memcpy(bQn, bq, (size_t)NumEdges * sizeof(double));
}

void ref_get_bc(double *bz, double *bq)
{
    memcpy(bz, bzeta, (size_t)NumEdges * sizeof(double));
    memcpy(bq, bQn, (size_t)NumEdges * sizeof(double));
}

double ref_max_lambda(void) { return max_lambda; }

/* ----------------------------------------------------- single operators ---- */

int ref_boundary_conditions(void)
{
    GUARD_BEGIN
    boundary_conditions();
    GUARD_END
    return 0;
}

int ref_compute2DL(double time)
{
    GUARD_BEGIN
    compute2DL(time);
    GUARD_END
    return 0;
}

int ref_slope_limiter(void)
{
    GUARD_BEGIN
    SlopeLimiter();
    GUARD_END
    return 0;
}

int ref_pdop(void)
{
    GUARD_BEGIN
    PDop2D();
    GUARD_END
    return 0;
}

int ref_wd_status(void)
{
    GUARD_BEGIN
    wetDryStatus2D();
    GUARD_END
    return 0;
}

double ref_roe_flux(double *out3, double zi, double ze, double qxi, double qxe, double qyi,
                    double qye, double zedge, double nx, double ny, double localg)
{
    return RoeFlux(out3, zi, ze, qxi, qxe, qyi, qye, zedge, nx, ny, localg);
}

void ref_inner_products(int el, double *si9, double *vi21)
{
    Compute2DInnerProducts(si9, vi21, el, 0.0);
}

/* --------------------------------------------------------------- steps ---- */

static void add_rain(double rain)
{
    if (rain == 0.0) return;
    for (int i = 0; i < 3 * NumEl; ++i) RHSZeta[i] += rain;
}

/* One SSP-RK2 step in the gsl-vector form of 2DCode/time_evolution.c:10-246, with the
 * wet/dry calls of ChanNet/time_evolution.c:225-226,330-333,413-415 when wet_dry != 0. */
static void step_sequence(double time, double dt, int wet_dry, double rain)
{
    const size_t n = 3 * (size_t)NumEl;
    if (wet_dry) wetDryStatus2D();

    gsl_vector *gz = gsl_vector_alloc(n), *gqx = gsl_vector_alloc(n), *gqy = gsl_vector_alloc(n);
    for (size_t i = 0; i < n; ++i) {
        gsl_vector_set(gz, i, zeta[i]);
        gsl_vector_set(gqx, i, Qx[i]);
        gsl_vector_set(gqy, i, Qy[i]);
    }

    compute2DL(time);
    add_rain(rain);
    gsl_vector *rz = gsl_vector_alloc(n), *rqx = gsl_vector_alloc(n), *rqy = gsl_vector_alloc(n);
    for (size_t i = 0; i < n; ++i) {
        gsl_vector_set(rz, i, RHSZeta[i]);
        gsl_vector_set(rqx, i, RHSQx[i]);
        gsl_vector_set(rqy, i, RHSQy[i]);
    }

    gsl_vector *z1 = gsl_vector_alloc(n), *qx1 = gsl_vector_alloc(n), *qy1 = gsl_vector_alloc(n);
    for (size_t i = 0; i < n; ++i) {
        gsl_vector_set(z1, i, gsl_vector_get(gz, i));
        gsl_vector_set(qx1, i, gsl_vector_get(gqx, i));
        gsl_vector_set(qy1, i, gsl_vector_get(gqy, i));
    }
    gsl_vector_scale(rz, dt);
    gsl_vector_scale(rqx, dt);
    gsl_vector_scale(rqy, dt);
    gsl_vector_add(z1, rz);
    gsl_vector_add(qx1, rqx);
    gsl_vector_add(qy1, rqy);
    for (size_t i = 0; i < n; ++i) {
        zeta[i] = gsl_vector_get(z1, i);
        Qx[i] = gsl_vector_get(qx1, i);
        Qy[i] = gsl_vector_get(qy1, i);
    }

    SlopeLimiter();
    if (wet_dry) {
        PDop2D();
        wetDryStatus2D();
    }

    for (size_t i = 0; i < n; ++i) {
        gsl_vector_set(z1, i, zeta[i]);
        gsl_vector_set(qx1, i, Qx[i]);
        gsl_vector_set(qy1, i, Qy[i]);
    }
    gsl_vector_add(z1, gz);
    gsl_vector_add(qx1, gqx);
    gsl_vector_add(qy1, gqy);

    compute2DL(time);
    add_rain(rain);
    for (size_t i = 0; i < n; ++i) {
        gsl_vector_set(rz, i, RHSZeta[i]);
        gsl_vector_set(rqx, i, RHSQx[i]);
        gsl_vector_set(rqy, i, RHSQy[i]);
    }
    gsl_vector_scale(z1, 0.5);
    gsl_vector_scale(qx1, 0.5);
    gsl_vector_scale(qy1, 0.5);
    gsl_vector_scale(rz, dt / 2);
    gsl_vector_scale(rqx, dt / 2);
    gsl_vector_scale(rqy, dt / 2);
    gsl_vector_add(z1, rz);
    gsl_vector_add(qx1, rqx);
    gsl_vector_add(qy1, rqy);
    for (size_t i = 0; i < n; ++i) {
        zeta[i] = gsl_vector_get(z1, i);
        Qx[i] = gsl_vector_get(qx1, i);
        Qy[i] = gsl_vector_get(qy1, i);
    }

    SlopeLimiter();
    if (wet_dry) PDop2D();

    gsl_vector_free(gz);
    gsl_vector_free(gqx);
    gsl_vector_free(gqy);
    gsl_vector_free(z1);
    gsl_vector_free(qx1);
    gsl_vector_free(qy1);
    gsl_vector_free(rz);
    gsl_vector_free(rqx);
    gsl_vector_free(rqy);
}

/* use_reference_step != 0 forces the reference's own oneTimeStep2D (wet/dry off, no rain). */
int ref_step(double time, double dt, int wet_dry, double rain, int use_reference_step)
{
    GUARD_BEGIN
    if (use_reference_step)
        oneTimeStep2D(time, dt);
    else
        step_sequence(time, dt, wet_dry, rain);
    GUARD_END
    return 0;
}

/* Forcing at time t: 2DCode/boundary_conditions.c, then the tide on type-2 edges. */
static void forcing(double t, int tide_on, double amp, double period)
{
    boundary_conditions();
    if (!tide_on) return;
    const double zb = dgr_outflow_zeta(t, 1, amp, period);
    for (int e = 0; e < NumEdges; ++e)
        if (BdryPrescribed[e] == 2) bzeta[e] = zb;
}

/*
 * Time loop of 2DCode/time_evolution.c:248-402 without the file output:
 *   forcing(0); loop { time += dt; step(time, dt); forcing(time);
 *                      dt = cfl*minEdgLength/max_lambda; clip to final_time }
 * It stops after nsteps steps or when time reaches final_time.  On return *time_io and
 * *dt_io hold the clock, and dt_hist (if given) the dt used by each step.
 * A negative start clock (*time_io < 0) means: start at time 0 with dt = dt0.
 */
int ref_run(int nsteps, double final_time, double cfl, double dt0, int wet_dry, double rain,
            int tide_on, double amp, double period, double *time_io, double *dt_io,
            double *dt_hist, int *steps_done)
{
    double time = *time_io, dt = *dt_io;
    int done = 0;
    GUARD_BEGIN
    if (time < 0) {
        time = 0;
        dt = dt0;
        forcing(time, tide_on, amp, period);
    }
    while (done < nsteps && time < final_time) {
        time = time + dt;
        step_sequence(time, dt, wet_dry, rain);
        forcing(time, tide_on, amp, period);
        if (dt_hist) dt_hist[done] = dt;
        ++done;
        *time_io = time;
        *steps_done = done;
        dt = cfl * minEdgLength / max_lambda;
        if ((time + dt) > final_time) dt = final_time - time;
        *dt_io = dt;
    }
    GUARD_END
    *time_io = time;
    *dt_io = dt;
    *steps_done = done;
    return 0;
}

/* The reference's own time loop, output files included (written to the current
 * directory).  Used to check that ref_run reproduces it. */
int ref_time_evolution(double final_time)
{
    GUARD_BEGIN
    time_evolution(final_time);
    GUARD_END
    return 0;
}
