/*
 * Link-level drop-in of the 2DCode step operators over the reference's process-wide
 * arrays (2DCode/MeshAttributes.h:5-42), backed by the GPU step of libdgrain:
 *
 *   void compute2DL(double time)   2DCode/compute2DL.c:12      -> dgr_compute_L
 *   void SlopeLimiter(void)        2DCode/SlopeLimiter2D.c:10  -> dgr_slope_limiter
 *   void wetDryStatus2D(void)      2DCode/wetDry2D.c:16        -> dgr_wet_dry_status
 *   void PDop2D(void)              2DCode/wetDry2D.c:63        -> dgr_pdop
 *
 * Link this file (and -ldgrain) in place of compute2DL.c, numericalFlux2D.c,
 * 2DInnerProducts.c, SlopeLimiter2D.c and wetDry2D.c; the reference's own main.c,
 * time_evolution.c (whose oneTimeStep2D calls these operators), initialize.c,
 * boundary_conditions.c, extract_mesh_attributes.c and mathfunctions.c stay unmodified.
 * The first call builds the device context from the mesh globals that
 * extract_mesh_attributes() filled; every call copies the globals the operator reads to
 * the device and the ones it writes back, as the reference's callers expect.  A numerical
 * failure prints the operator, the status and the edge or element index, then exits with
 * EXIT_FAILURE, as the reference does.  Build with -DWDON for the reference's wet/dry flux
 * branch (dgr_params.wet_dry = 1).
 */
#include <stdio.h>
#include <stdlib.h>

#include "../../include/dgrain.h"

extern int NumEl, NumNodes, NumEdges;
extern double *x_coord, *y_coord, *z, *nFriction;
extern int *EltoVert, *EdgtoEls, *EdgtoVert, *BdryPrescribed;
extern double minEdgLength, max_lambda;
extern double *zeta, *Qx, *Qy;
extern double *Fhat1dotn, *Fhat2dotn, *Fhat3dotn;
extern double *RHSZeta, *RHSQx, *RHSQy;
extern double *bzeta, *bQn;
extern const double g, H0, VELZERO;
extern int *WD;

static dgr_ctx *g_ctx;

static void legacy_fail(const char *where, dgr_ctx *c, int rc)
{
    int code = 0, index = -1, step = -1;
    if (c && rc >= 1 && rc <= 6) dgr_last_error(c, &code, &index, &step);
    printf("%s: %s (status %d) at index %d\n", where, dgr_status_string(rc), rc, index);
    if (rc == DGR_ERR_CUDA) printf("%s\n", dgr_last_cuda_error());
    exit(EXIT_FAILURE);
}

static void legacy_release(void)
{
    if (g_ctx) dgr_destroy(g_ctx);
    g_ctx = NULL;
}

static dgr_ctx *legacy_context(void)
{
    if (g_ctx) return g_ctx;
    dgr_mesh_view m;
    m.num_el = NumEl;
    m.num_nodes = NumNodes;
    m.num_edges = NumEdges;
    m.x_coord = x_coord;
    m.y_coord = y_coord;
    m.z = z;
    m.nFriction = nFriction;
    m.EltoVert = EltoVert;
    m.EdgtoEls = EdgtoEls;
    m.EdgtoVert = EdgtoVert;
    m.BdryPrescribed = BdryPrescribed;
    m.minEdgLength = minEdgLength;
    dgr_params p;
    dgr_params_default(&p);
    p.g = g;
    p.H0 = H0;
    p.VELZERO = VELZERO;
#ifdef WDON
    p.wet_dry = 1;
#else
    p.wet_dry = 0;
#endif
    int rc = dgr_create(&m, &p, &g_ctx);
    if (rc) legacy_fail("dgr_create", NULL, rc);
    atexit(legacy_release);
    return g_ctx;
}

static void legacy_upload(dgr_ctx *c)
{
    int rc = dgr_upload_state(c, zeta, Qx, Qy, WD);
    if (rc) legacy_fail("upload", c, rc);
}

static void legacy_download(dgr_ctx *c)
{
    int rc = dgr_download_state(c, zeta, Qx, Qy, WD);
    if (rc) legacy_fail("download", c, rc);
}

void compute2DL(double time)
{
    dgr_ctx *c = legacy_context();
    legacy_upload(c);
    int rc = dgr_set_boundary(c, bzeta, bQn);
    if (rc) legacy_fail("compute2DL", c, rc);
    rc = dgr_compute_L(c, time, RHSZeta, RHSQx, RHSQy, &max_lambda);
    if (rc) legacy_fail("compute2DL", c, rc);
    rc = dgr_get_fhat(c, Fhat1dotn, Fhat2dotn, Fhat3dotn);
    if (rc) legacy_fail("compute2DL", c, rc);
}

void SlopeLimiter(void)
{
    dgr_ctx *c = legacy_context();
    legacy_upload(c);
    int rc = dgr_slope_limiter(c);
    if (rc) legacy_fail("SlopeLimiter", c, rc);
    legacy_download(c);
}

void wetDryStatus2D(void)
{
    dgr_ctx *c = legacy_context();
    legacy_upload(c);
    int rc = dgr_wet_dry_status(c);
    if (rc) legacy_fail("wetDryStatus2D", c, rc);
    legacy_download(c);
}

void PDop2D(void)
{
    dgr_ctx *c = legacy_context();
    legacy_upload(c);
    int rc = dgr_pdop(c);
    if (rc) legacy_fail("PDop2D", c, rc);
    legacy_download(c);
}
