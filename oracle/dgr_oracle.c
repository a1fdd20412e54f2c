/*
 * ORACLE — test infrastructure only; see dgr_oracle.h.
 *
 * CPU restatement of the reference 2D step.  Each function cites the reference lines it
 * restates.  Expressions keep the reference's operation order and parenthesisation
 * (including its multiplications by the zero entries of diagonal matrices) because the
 * restatement must reproduce the reference bits, not just its mathematics.
 */
#include "dgr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../dg-rain_b200/csrc/dgr_forcing.h"

struct orc_ctx {
    int ne, nn, nf;
    double *x, *y, *z, *nfric, *nel;
    int *el2v, *ed2el, *ed2v, *bdry;
    double min_edge;
    double g, h0, velzero;
    /* state and work arrays, reference layout [3*el+k] */
    double *zeta, *qx, *qy;
    int *wd;
    double *f1, *f2, *f3;
    double *rz, *rqx, *rqy;
    double *bzeta, *bqn;
    double max_lambda;
    int err_code, err_index;
    int *dec_limit, *dec_pdop;
    /* node -> element lists (built once; the reference rebuilds them per call,
     * 2DCode/SlopeLimiter2D.c:39-89, in the same element order) */
    int *n2e_ptr, *n2e;
};

static void *dup_mem(const void *p, size_t n)
{
    void *q = malloc(n ? n : 1);
    if (p && n) memcpy(q, p, n);
    return q;
}

/* sign() of 2DCode/mathfunctions.c:4-12 */
static int orc_sign(double a)
{
    if (a < 0) return -1;
    if (a == 0) return 0;
    return 1;
}

/* max()/min() macros of 2DCode/mathfunctions.h:8-14 */
static double orc_max(double a, double b) { return (a > b) ? a : b; }
static double orc_min(double a, double b) { return (a < b) ? a : b; }

/* fmax as the reference build evaluates it.  glibc's x86-64 fmax(x, y) returns
 * x > y ? x : y, a NaN operand giving the other one; so when x and y compare equal it
 * returns y, which matters for zeros of opposite sign.  gcc treats fmax as commutative
 * and passes a call's operands in either order.  The build of the reference step made by
 * oracle/Makefile (gcc -O2 -ffp-contract=off, read from its x86-64 code) keeps the
 * written order at the limiter's clamp (2DCode/SlopeLimiter2D.c:244-246) and swaps it at
 * RoeFlux's entropy fix (2DCode/numericalFlux2D.c:74-84).  These two helpers are those
 * two orders of fmax(a, b): fmax_b returns b on a tie, fmax_a returns a. */
static double fmax_b(double a, double b) { return (a > b || b != b) ? a : b; }
static double fmax_a(double a, double b) { return (b > a || a != a) ? b : a; }

orc_ctx *orc_create(int ne, int nn, int nf, const double *x, const double *y, const double *z,
                    const double *nfric, const int *el2v, const int *ed2el, const int *ed2v,
                    const int *bdry, double min_edge)
{
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
    size_t s3 = 3 * (size_t)ne;
    c->ne = ne;
    c->nn = nn;
    c->nf = nf;
    c->x = dup_mem(x, nn * sizeof(double));
    c->y = dup_mem(y, nn * sizeof(double));
    c->z = dup_mem(z, nn * sizeof(double));
    c->nfric = dup_mem(nfric, nn * sizeof(double));
    c->el2v = dup_mem(el2v, s3 * sizeof(int));
    c->ed2el = dup_mem(ed2el, 2 * (size_t)nf * sizeof(int));
    c->ed2v = dup_mem(ed2v, 2 * (size_t)nf * sizeof(int));
    c->bdry = dup_mem(bdry, (size_t)nf * sizeof(int));
    c->min_edge = min_edge;
    c->g = 9.81;
    c->h0 = 1e-3;
    c->velzero = 1e-2;
    c->zeta = calloc(s3, sizeof(double));
    c->qx = calloc(s3, sizeof(double));
    c->qy = calloc(s3, sizeof(double));
    c->wd = malloc((size_t)ne * sizeof(int));
    for (int i = 0; i < ne; ++i) c->wd[i] = -1;
    c->f1 = calloc(s3, sizeof(double));
    c->f2 = calloc(s3, sizeof(double));
    c->f3 = calloc(s3, sizeof(double));
    c->rz = calloc(s3, sizeof(double));
    c->rqx = calloc(s3, sizeof(double));
    c->rqy = calloc(s3, sizeof(double));
    c->bzeta = calloc((size_t)nf, sizeof(double));
    c->bqn = calloc((size_t)nf, sizeof(double));
    c->dec_limit = calloc((size_t)ne, sizeof(int));
    c->dec_pdop = calloc((size_t)ne, sizeof(int));
    /* node -> element CSR in ascending element order */
    c->n2e_ptr = calloc((size_t)nn + 1, sizeof(int));
    for (size_t i = 0; i < s3; ++i) c->n2e_ptr[el2v[i] + 1]++;
    for (int n = 0; n < nn; ++n) c->n2e_ptr[n + 1] += c->n2e_ptr[n];
    c->n2e = malloc(s3 * sizeof(int));
    int *fill = calloc((size_t)nn, sizeof(int));
    for (int el = 0; el < ne; ++el)
        for (int k = 0; k < 3; ++k) {
            int v = el2v[3 * el + k];
            c->n2e[c->n2e_ptr[v] + fill[v]++] = el;
        }
    free(fill);
    return c;
}

void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    free(c->x); free(c->y); free(c->z); free(c->nfric); free(c->nel);
    free(c->el2v); free(c->ed2el); free(c->ed2v); free(c->bdry);
    free(c->zeta); free(c->qx); free(c->qy); free(c->wd);
    free(c->f1); free(c->f2); free(c->f3);
    free(c->rz); free(c->rqx); free(c->rqy);
    free(c->bzeta); free(c->bqn);
    free(c->dec_limit); free(c->dec_pdop);
    free(c->n2e_ptr); free(c->n2e);
    free(c);
}

void orc_set_constants(orc_ctx *c, double g, double h0, double velzero)
{
    c->g = g;
    c->h0 = h0;
    c->velzero = velzero;
}

void orc_set_element_manning(orc_ctx *c, const double *n_el)
{
    free(c->nel);
    c->nel = n_el ? dup_mem(n_el, (size_t)c->ne * sizeof(double)) : NULL;
}

void orc_set_state(orc_ctx *c, const double *zeta, const double *qx, const double *qy, const int *wd)
{
    size_t s3 = 3 * (size_t)c->ne * sizeof(double);
    memcpy(c->zeta, zeta, s3);
    memcpy(c->qx, qx, s3);
    memcpy(c->qy, qy, s3);
    if (wd) memcpy(c->wd, wd, (size_t)c->ne * sizeof(int));
}

void orc_get_state(const orc_ctx *c, double *zeta, double *qx, double *qy, int *wd)
{
    size_t s3 = 3 * (size_t)c->ne * sizeof(double);
    memcpy(zeta, c->zeta, s3);
    memcpy(qx, c->qx, s3);
    memcpy(qy, c->qy, s3);
    if (wd) memcpy(wd, c->wd, (size_t)c->ne * sizeof(int));
}

void orc_set_bc(orc_ctx *c, const double *bzeta, const double *bqn)
{
    memcpy(c->bzeta, bzeta, (size_t)c->nf * sizeof(double));
    memcpy(c->bqn, bqn, (size_t)c->nf * sizeof(double));
}

void orc_get_bc(const orc_ctx *c, double *bzeta, double *bqn)
{
    memcpy(bzeta, c->bzeta, (size_t)c->nf * sizeof(double));
    memcpy(bqn, c->bqn, (size_t)c->nf * sizeof(double));
}

void orc_get_rhs(const orc_ctx *c, double *rz, double *rqx, double *rqy)
{
    size_t s3 = 3 * (size_t)c->ne * sizeof(double);
    memcpy(rz, c->rz, s3);
    memcpy(rqx, c->rqx, s3);
    memcpy(rqy, c->rqy, s3);
}

void orc_get_fhat(const orc_ctx *c, double *f1, double *f2, double *f3)
{
    size_t s3 = 3 * (size_t)c->ne * sizeof(double);
    memcpy(f1, c->f1, s3);
    memcpy(f2, c->f2, s3);
    memcpy(f3, c->f3, s3);
}

double orc_max_lambda(const orc_ctx *c) { return c->max_lambda; }

void orc_last_error(const orc_ctx *c, int *code, int *index)
{
    *code = c->err_code;
    *index = c->err_index;
}

void orc_get_decisions(const orc_ctx *c, int *limit, int *pdop)
{
    if (limit) memcpy(limit, c->dec_limit, (size_t)c->ne * sizeof(int));
    if (pdop) memcpy(pdop, c->dec_pdop, (size_t)c->ne * sizeof(int));
}

/* 2DCode/initialize.c:117-126: nodal values averaged onto the edge midpoints, WD = -1. */
void orc_initial_state(orc_ctx *c, const double *zeta_nodal)
{
    for (int el = 0; el < c->ne; ++el) {
        double nz[3];
        for (int k = 0; k < 3; ++k) {
            nz[k] = zeta_nodal ? zeta_nodal[c->el2v[3 * el + k]] : 0.1;
            c->qx[3 * el + k] = 0;
            c->qy[3 * el + k] = 0;
        }
        c->zeta[3 * el] = 0.5 * (nz[0] + nz[1]);
        c->zeta[3 * el + 1] = 0.5 * (nz[1] + nz[2]);
        c->zeta[3 * el + 2] = 0.5 * (nz[2] + nz[0]);
        c->wd[el] = -1;
    }
}

/* 2DCode/boundary_conditions.c:9-82 plus the tide extension on type-2 edges. */
int orc_boundary_conditions(orc_ctx *c, double t, int tide_on, double amp, double period)
{
    const double zb2 = dgr_outflow_zeta(t, tide_on, amp, period);
    for (int e = 0; e < c->nf; ++e) {
        double qn = 0, zb = 0;
        switch (c->bdry[e]) {
        case 1: qn = DGR_BC1_QN; zb = DGR_BC1_ZETA; break;
        case 2: qn = DGR_BC2_QN; zb = zb2; break;
        case 3: qn = DGR_BC3_QN; zb = DGR_BC3_ZETA; break;
        default:
            /* the reference leaves qn/zeta_b uninitialised here and stores them;
             * land edges never read them (2DCode/compute2DL.c:147-191) */
            qn = 0; zb = 0; break;
        }
        c->bzeta[e] = zb;
        c->bqn[e] = qn;
    }
    return 0;
}

/* RoeFlux, 2DCode/numericalFlux2D.c:6-108.  'g' is the global gravity used by the
 * eigen-structure; 'local_g' scales only the pressure term. */
double orc_roe_flux(double *fh, double zeta_in, double zeta_ex, double qx_in, double qx_ex,
                    double qy_in, double qy_ex, double z_edge, double nx, double ny, double local_g,
                    double g)
{
    double h_in = zeta_in + z_edge;
    double h_ex = zeta_ex + z_edge;
    double u_in = qx_in / h_in, u_ex = qx_ex / h_ex;
    double v_in = qy_in / h_in, v_ex = qy_ex / h_ex;
    double jump[3] = {zeta_in - zeta_ex, qx_in - qx_ex, qy_in - qy_ex};

    double f1x_in = h_in * u_in, f1x_ex = h_ex * u_ex;
    double f1y_in = h_in * v_in, f1y_ex = h_ex * v_ex;
    double f2x_in = h_in * u_in * u_in + 0.5 * local_g * (h_in * h_in - z_edge * z_edge);
    double f2x_ex = h_ex * u_ex * u_ex + 0.5 * local_g * (h_ex * h_ex - z_edge * z_edge);
    double f2y_in = h_in * u_in * v_in, f2y_ex = h_ex * u_ex * v_ex;
    double f3x_in = h_in * u_in * v_in, f3x_ex = h_ex * u_ex * v_ex;
    double f3y_in = h_in * v_in * v_in + 0.5 * local_g * (h_in * h_in - z_edge * z_edge);
    double f3y_ex = h_ex * v_ex * v_ex + 0.5 * local_g * (h_ex * h_ex - z_edge * z_edge);

    double fn_in[3] = {f1x_in * nx + f1y_in * ny, f2x_in * nx + f2y_in * ny, f3x_in * nx + f3y_in * ny};
    double fn_ex[3] = {f1x_ex * nx + f1y_ex * ny, f2x_ex * nx + f2y_ex * ny, f3x_ex * nx + f3y_ex * ny};

    /* Roe averages, :45-47 */
    double h_hat = 0.5 * (h_in + h_ex);
    double u_hat = (u_in * sqrt(h_in) + u_ex * sqrt(h_ex)) / (sqrt(h_in) + sqrt(h_ex));
    double v_hat = (v_in * sqrt(h_in) + v_ex * sqrt(h_ex)) / (sqrt(h_in) + sqrt(h_ex));
    double c = sqrt(g * h_hat);

    /* eigenvectors and their inverse, :49-60 */
    double r[3][3] = {{1, 0, 1}, {u_hat - c * nx, -ny, u_hat + c * nx}, {v_hat - c * ny, nx, v_hat + c * ny}};
    double ri[3][3];
    double den = -2 * c;
    ri[0][0] = (-c - nx * u_hat - ny * v_hat) / den;
    ri[0][1] = nx / den;
    ri[0][2] = ny / den;
    ri[1][0] = (-2 * c * ny * u_hat + 2 * c * nx * v_hat) / den;
    ri[1][1] = 2 * c * ny / den;
    ri[1][2] = -2 * c * nx / den;
    ri[2][0] = (-c + nx * u_hat + ny * v_hat) / den;
    ri[2][1] = -nx / den;
    ri[2][2] = -ny / den;

    /* characteristic speeds and entropy fix, :62-84 */
    double l1_in = u_in * nx + v_in * ny - sqrt(g * h_in);
    double l2_in = u_in * nx + v_in * ny;
    double l3_in = u_in * nx + v_in * ny + sqrt(g * h_in);
    double l1_ex = u_ex * nx + v_ex * ny - sqrt(g * h_ex);
    double l2_ex = u_ex * nx + v_ex * ny;
    double l3_ex = u_ex * nx + v_ex * ny + sqrt(g * h_ex);
    double lh1 = u_hat * nx + v_hat * ny - c;
    double lh2 = u_hat * nx + v_hat * ny;
    double lh3 = u_hat * nx + v_hat * ny + c;

    double e1 = fmax_a(0, (lh1 - l1_in));
    e1 = fmax_a(e1, (l1_ex - lh1));
    lh1 = fmax_a(e1, fabs(lh1));
    double e2 = fmax_a(0, (lh2 - l2_in));
    e2 = fmax_a(e2, (l2_ex - lh2));
    lh2 = fmax_a(e2, fabs(lh2));
    double e3 = fmax_a(0, (lh3 - l3_in));
    e3 = fmax_a(e3, (l3_ex - lh3));
    lh3 = fmax_a(e3, fabs(lh3));

    /* R |Lambda| R^-1 jump as three dense 3x3 products (mathfunctions.c:24-35) */
    double lam[3][3] = {{lh1, 0, 0}, {0, lh2, 0}, {0, 0, lh3}};
    double p1[3], p2[3], p3[3];
    for (int i = 0; i < 3; ++i) {
        double s = 0;
        for (int j = 0; j < 3; ++j) s += ri[i][j] * jump[j];
        p1[i] = s;
    }
    for (int i = 0; i < 3; ++i) {
        double s = 0;
        for (int j = 0; j < 3; ++j) s += lam[i][j] * p1[j];
        p2[i] = s;
    }
    for (int i = 0; i < 3; ++i) {
        double s = 0;
        for (int j = 0; j < 3; ++j) s += r[i][j] * p2[j];
        p3[i] = s;
    }
    for (int k = 0; k < 3; ++k) fh[k] = 0.5 * (fn_in[k] + fn_ex[k]) + 0.5 * p3[k];

    double m = orc_max(fabs(l1_in), fabs(l1_ex));
    m = orc_max(m, fabs(l2_in));
    m = orc_max(m, fabs(l2_ex));
    m = orc_max(m, fabs(l3_in));
    m = orc_max(m, fabs(l3_ex));
    return m;
}

/* local edge k of element el joining vertices (v0,v1): 2DCode/compute2DL.c:45-67 */
static int local_edge(const int *ev, int v0, int v1)
{
    if ((v0 == ev[0] && v1 == ev[1]) || (v0 == ev[1] && v1 == ev[0])) return 0;
    if ((v0 == ev[1] && v1 == ev[2]) || (v0 == ev[2] && v1 == ev[1])) return 1;
    if ((v0 == ev[2] && v1 == ev[0]) || (v0 == ev[0] && v1 == ev[2])) return 2;
    return -1;
}

static int set_err(orc_ctx *c, int code, int index)
{
    c->err_code = code;
    c->err_index = index;
    return code;
}

/* Compute2DInnerProducts, 2DCode/2DInnerProducts.c:8-570 (live code only). */
void orc_inner_products(const orc_ctx *c, int i, double si[9], double vi[21])
{
    const double *X = c->x, *Y = c->y;
    const int v0 = c->el2v[3 * i], v1 = c->el2v[3 * i + 1], v2 = c->el2v[3 * i + 2];
    const double xv1 = X[v0], xv2 = X[v1], xv3 = X[v2];
    const double yv1 = Y[v0], yv2 = Y[v1], yv3 = Y[v2];

    /* edge midpoints, lengths, edge Jacobians (:29-45) */
    const double x1 = (X[v0] + X[v1]) / 2, x2 = (X[v1] + X[v2]) / 2, x3 = (X[v2] + X[v0]) / 2;
    const double y1 = (Y[v0] + Y[v1]) / 2, y2 = (Y[v1] + Y[v2]) / 2, y3 = (Y[v2] + Y[v0]) / 2;
    double el_len[3], ej[3];
    el_len[0] = sqrt((xv2 - xv1) * (xv2 - xv1) + (yv2 - yv1) * (yv2 - yv1));
    el_len[1] = sqrt((xv3 - xv2) * (xv3 - xv2) + (yv3 - yv2) * (yv3 - yv2));
    el_len[2] = sqrt((xv3 - xv1) * (xv3 - xv1) + (yv3 - yv1) * (yv3 - yv1));
    for (int e = 0; e < 3; ++e) ej[e] = el_len[e] / 2;

    /* two Gauss points per edge (:48-65) */
    const double s3 = sqrt(3);
    double xe[3][2], ye[3][2];
    xe[0][0] = (s3 * x1 - x2 + x3) / s3;
    ye[0][0] = (s3 * y1 - y2 + y3) / s3;
    xe[0][1] = (s3 * x1 + x2 - x3) / s3;
    ye[0][1] = (s3 * y1 + y2 - y3) / s3;
    xe[1][0] = (x1 + s3 * x2 - x3) / s3;
    ye[1][0] = (y1 + s3 * y2 - y3) / s3;
    xe[1][1] = (-x1 + s3 * x2 + x3) / s3;
    ye[1][1] = (-y1 + s3 * y2 + y3) / s3;
    xe[2][0] = (-x1 + x2 + s3 * x3) / s3;
    ye[2][0] = (-y1 + y2 + s3 * y3) / s3;
    xe[2][1] = (x1 - x2 + s3 * x3) / s3;
    ye[2][1] = (y1 - y2 + s3 * y3) / s3;

    /* CR basis values at the Gauss points (:73-87): psi[b][e][n] */
    double psi[3][3][2];
    double den = x1 * y2 - x1 * y3 + x2 * y3 - x2 * y1 + x3 * y1 - x3 * y2;
    for (int n = 0; n < 2; ++n)
        for (int e = 0; e < 3; ++e) {
            const double xq = xe[e][n], yq = ye[e][n];
            psi[0][e][n] = -(yq * x2 - yq * x3 - xq * y2 + x3 * y2 + xq * y3 - x2 * y3) / den;
            psi[1][e][n] = -(-x1 * yq + x3 * yq - x3 * y1 + xq * y1 - xq * y3 + x1 * y3) / den;
            psi[2][e][n] = -(yq * x1 - yq * x2 - xq * y1 + x2 * y1 + xq * y2 - x1 * y2) / den;
        }

    /* edge normals (:110-116) */
    const double jac = 4 * (x2 - x3) * (y2 - y1) - 4 * (x2 - x1) * (y2 - y3);
    const int sj = orc_sign(jac);
    const double nx1 = sj * 2 * (y2 - y3) / el_len[0], ny1 = sj * 2 * (x3 - x2) / el_len[0];
    const double nx2 = sj * 2 * (y3 - y1) / el_len[1], ny2 = sj * 2 * (x1 - x3) / el_len[1];
    const double nx3 = sj * 2 * (y1 - y2) / el_len[2], ny3 = sj * 2 * (x2 - x1) / el_len[2];
    const double nxs[3] = {nx1, nx2, nx3}, nys[3] = {ny1, ny2, ny3};

    /* RT0 fit matrix (:126-134) */
    const double M11 = nx1, M12 = x1 * nx1 + y1 * ny1, M13 = ny1;
    const double M21 = nx2, M22 = x2 * nx2 + y2 * ny2, M23 = ny2;
    const double M31 = nx3, M32 = x3 * nx3 + y3 * ny3, M33 = ny3;
    const double dM = M13 * M22 * M31 - M12 * M23 * M31 - M13 * M21 * M32 + M11 * M23 * M32 +
                      M12 * M21 * M33 - M11 * M22 * M33;

    /* surface term: fit F = (a + b x, c + b y) to the three Fhat.n values (:95-146) */
    const double *F[3] = {c->f1, c->f2, c->f3};
    double a[3], b[3], cc[3];
    for (int v = 0; v < 3; ++v) {
        const double R1 = F[v][3 * i], R2 = F[v][3 * i + 1], R3 = F[v][3 * i + 2];
        a[v] = (R3 * M13 * M22 - R3 * M12 * M23 - R2 * M13 * M32 + R1 * M23 * M32 + R2 * M12 * M33 -
                R1 * M22 * M33) / dM;
        b[v] = -(R3 * M13 * M21 - R3 * M11 * M23 - R2 * M13 * M31 + R1 * M23 * M31 + R2 * M11 * M33 -
                 R1 * M21 * M33) / dM;
        cc[v] = (R3 * M12 * M21 - R3 * M11 * M22 - R2 * M12 * M31 + R1 * M22 * M31 + R2 * M11 * M32 -
                 R1 * M21 * M32) / dM;
    }
    /* F.n at the Gauss points (:154-167) and the surface integrals (:205-239) */
    for (int v = 0; v < 3; ++v) {
        double fd[3][2];
        for (int n = 0; n < 2; ++n)
            for (int e = 0; e < 3; ++e)
                fd[e][n] = (a[v] + b[v] * xe[e][n]) * nxs[e] + (cc[v] + b[v] * ye[e][n]) * nys[e];
        for (int bf = 0; bf < 3; ++bf)
            si[3 * v + bf] = ej[0] * (fd[0][0] * psi[bf][0][0] + fd[0][1] * psi[bf][0][1]) +
                             ej[1] * (fd[1][0] * psi[bf][1][0] + fd[1][1] * psi[bf][1][1]) +
                             ej[2] * (fd[2][0] * psi[bf][2][0] + fd[2][1] * psi[bf][2][1]);
    }

    /* volume term (:247-566) */
    const double weight = 1.0 / 6;
    const int n0 = v0, n1 = v1, n2 = v2;
    double midz[3], midn[3];
    midz[0] = 0.5 * (c->z[n0] + c->z[n1]);
    midz[1] = 0.5 * (c->z[n1] + c->z[n2]);
    midz[2] = 0.5 * (c->z[n2] + c->z[n0]);
    if (c->nel) {
        midn[0] = midn[1] = midn[2] = c->nel[i];
    } else {
        midn[0] = 0.5 * (c->nfric[n0] + c->nfric[n1]);
        midn[1] = 0.5 * (c->nfric[n1] + c->nfric[n2]);
        midn[2] = 0.5 * (c->nfric[n2] + c->nfric[n0]);
    }
    double gp[3][2];
    gp[0][0] = 4 / jac * (y2 - y3);
    gp[0][1] = 4 / jac * (x3 - x2);
    gp[1][0] = 4 / jac * (y3 - y1);
    gp[1][1] = 4 / jac * (x1 - x3);
    gp[2][0] = 4 / jac * (y1 - y2);
    gp[2][1] = 4 / jac * (x2 - x1);

    double zr[3], qxr[3], qyr[3], H[3], tau[3];
    for (int e = 0; e < 3; ++e) {
        zr[e] = c->zeta[3 * i + e];
        qxr[e] = c->qx[3 * i + e];
        qyr[e] = c->qy[3 * i + e];
        H[e] = zr[e] + midz[e];
        double u = qxr[e] / H[e];
        double v = qyr[e] / H[e];
        tau[e] = c->g * midn[e] * midn[e] * sqrt(u * u + v * v) / (pow(H[e], 4. / 3));
    }
    double local_g = c->g;
    if (c->wd[i] == 0) local_g = 0;
    double fx[3][3], fy[3][3]; /* [variable][edge] */
    for (int e = 0; e < 3; ++e) {
        fx[0][e] = qxr[e];
        fx[1][e] = qxr[e] * qxr[e] / H[e] + 0.5 * local_g * (H[e] * H[e] - midz[e] * midz[e]);
        fx[2][e] = qxr[e] * qyr[e] / H[e];
        fy[0][e] = qyr[e];
        fy[1][e] = qxr[e] * qyr[e] / H[e];
        fy[2][e] = qyr[e] * qyr[e] / H[e] + 0.5 * local_g * (H[e] * H[e] - midz[e] * midz[e]);
    }
    double gradz[2];
    for (int j = 0; j < 2; ++j) gradz[j] = midz[0] * gp[0][j] + midz[1] * gp[1][j] + midz[2] * gp[2][j];

    for (int v = 0; v < 3; ++v) {
        const double R1 = fx[v][0] * nx1 + fy[v][0] * ny1;
        const double R2 = fx[v][1] * nx2 + fy[v][1] * ny2;
        const double R3 = fx[v][2] * nx3 + fy[v][2] * ny3;
        a[v] = (R3 * M13 * M22 - R3 * M12 * M23 - R2 * M13 * M32 + R1 * M23 * M32 + R2 * M12 * M33 -
                R1 * M22 * M33) / dM;
        b[v] = -(R3 * M13 * M21 - R3 * M11 * M23 - R2 * M13 * M31 + R1 * M23 * M31 + R2 * M11 * M33 -
                 R1 * M21 * M33) / dM;
        cc[v] = (R3 * M12 * M21 - R3 * M11 * M22 - R2 * M12 * M31 + R1 * M22 * M31 + R2 * M11 * M32 -
                 R1 * M21 * M32) / dM;
    }
    const double aj = fabs(jac);
    /* divergence parts: VI[0..2] (a1), VI[3,6,9] (a2), VI[12,15,18] (a3) */
    double dv[3][3];
    for (int v = 0; v < 3; ++v)
        for (int bf = 0; bf < 3; ++bf)
            dv[v][bf] = aj * (0.5 * a[v] * gp[bf][0] + 0.5 * cc[v] * gp[bf][1] +
                              b[v] * weight * (gp[bf][0] * (x1 + x2 + x3) + gp[bf][1] * (y1 + y2 + y3)));
    vi[0] = dv[0][0];
    vi[1] = dv[0][1];
    vi[2] = dv[0][2];
    for (int bf = 0; bf < 3; ++bf) {
        vi[3 + 3 * bf] = dv[1][bf];
        vi[4 + 3 * bf] = local_g * aj * gradz[0] * weight * zr[bf];
        vi[5 + 3 * bf] = aj * weight * tau[bf] * qxr[bf];
        vi[12 + 3 * bf] = dv[2][bf];
        vi[13 + 3 * bf] = local_g * aj * gradz[1] * weight * zr[bf];
        vi[14 + 3 * bf] = aj * weight * tau[bf] * qyr[bf];
    }
}

/* compute2DL, 2DCode/compute2DL.c:12-413 (WDON branch :201-293 when wet_dry != 0). */
int orc_compute_L(orc_ctx *c, int wet_dry, double rain)
{
    const double g = c->g;
    c->err_code = 0;
    c->err_index = -1;
    for (int i = 0; i < c->nf; ++i) {
        const int el_in = c->ed2el[2 * i], el_ex = c->ed2el[2 * i + 1];
        const int v0 = c->ed2v[2 * i], v1 = c->ed2v[2 * i + 1];
        const int *ev_in = &c->el2v[3 * el_in], *ev_ex = &c->el2v[3 * el_ex];
        const int k_in = local_edge(ev_in, v0, v1);
        const int k_ex = local_edge(ev_ex, v0, v1);
        if (k_in < 0 || k_ex < 0) return set_err(c, ORC_ERR_EDGE_MATCH, i);

        /* normal of the "in" element (:98-132) */
        const double *X = c->x, *Y = c->y;
        double len = sqrt((X[v1] - X[v0]) * (X[v1] - X[v0]) + (Y[v1] - Y[v0]) * (Y[v1] - Y[v0]));
        double jac = X[ev_in[0]] * (Y[ev_in[1]] - Y[ev_in[2]]) + X[ev_in[1]] * (Y[ev_in[2]] - Y[ev_in[0]]) +
                     X[ev_in[2]] * (Y[ev_in[0]] - Y[ev_in[1]]);
        const int a0 = ev_in[k_in], a1 = ev_in[(k_in + 1) % 3];
        double xa = X[a0], xb = X[a1], ya = Y[a0], yb = Y[a1];
        double nx = orc_sign(jac) * (yb - ya) / len;
        double ny = orc_sign(jac) * (xa - xb) / len;
        double tx = -ny, ty = nx;

        double zi = c->zeta[3 * el_in + k_in], qxi = c->qx[3 * el_in + k_in], qyi = c->qy[3 * el_in + k_in];
        double z_edge = (c->z[v0] + c->z[v1]) / 2;
        double ze, qxe, qye;
        /* boundary ghost states (:147-199) */
        if (c->bdry[i]) {
            ze = c->bzeta[i];
            double qn_ex = c->bqn[i];
            if (ze < 0) ze = zi;
            if (qn_ex > 1000) qn_ex = qxi * nx + qyi * ny;
            double qt_ex = qxi * tx + qyi * ty;
            double d = 1. / (nx * ty - ny * tx);
            qxe = (ty * qn_ex - ny * qt_ex) * d;
            qye = (-tx * qn_ex + nx * qt_ex) * d;
        } else if (el_in == el_ex) {
            ze = c->zeta[3 * el_ex + k_ex];
            double qn_in = qxi * nx + qyi * ny;
            double qt_in = qxi * tx + qyi * ty;
            double qn_ex = -qn_in, qt_ex = qt_in;
            double d = 1. / (nx * ty - ny * tx);
            qxe = (ty * qn_ex - ny * qt_ex) * d;
            qye = (-tx * qn_ex + nx * qt_ex) * d;
        } else {
            ze = c->zeta[3 * el_ex + k_ex];
            qxe = c->qx[3 * el_ex + k_ex];
            qye = c->qy[3 * el_ex + k_ex];
        }

        double fn_in[3], fn_ex[3], lam;
        if (wet_dry && c->wd[el_in] == 0 && c->wd[el_ex] == 0) {
            /* both dry: two reflective fluxes without pressure (:203-239) */
            double qn_in = qxi * nx + qyi * ny;
            double qt_in = qxi * tx + qyi * ty;
            double qn_ex = -qn_in, qt_ex = qt_in;
            double d = 1. / (nx * ty - ny * tx);
            double qxe_ref = (ty * qn_ex - ny * qt_ex) * d;
            double qye_ref = (-tx * qn_ex + nx * qt_ex) * d;
            double lam_in = orc_roe_flux(fn_in, zi, zi, qxi, qxe_ref, qyi, qye_ref, z_edge, nx, ny, 0, g);
            qn_ex = qxe * nx + qye * ny;
            qt_ex = qxe * tx + qye * ty;
            qn_in = -qn_ex;
            qt_in = qt_ex;
            double qxi_ref = (ty * qn_in - ny * qt_in) * d;
            double qyi_ref = (-tx * qn_in + nx * qt_ex) * d;
            double lam_ex = orc_roe_flux(fn_ex, ze, ze, qxi_ref, qxe, qyi_ref, qye, z_edge, nx, ny, 0, g);
            lam = orc_max(lam_in, lam_ex);
            if (i == 0)
                c->max_lambda = lam;
            else {
                c->max_lambda = orc_max(c->max_lambda, lam_in);
                c->max_lambda = orc_max(c->max_lambda, lam_ex);
            }
        } else {
            double fh[3];
            lam = orc_roe_flux(fh, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, g, g);
            if (isnan(fh[0]) || isnan(fh[1]) || isnan(fh[2])) return set_err(c, ORC_ERR_NAN_FLUX, i);
            if (!wet_dry || c->wd[el_in] == 1) {
                fn_in[0] = fh[0]; fn_in[1] = fh[1]; fn_in[2] = fh[2];
            } else {
                double l2 = orc_roe_flux(fn_in, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, 0, g);
                if (isnan(fn_in[0]) || isnan(fn_in[1]) || isnan(fn_in[2]))
                    return set_err(c, ORC_ERR_NAN_FLUX_IN, i);
                lam = orc_max(lam, l2);
            }
            if (!wet_dry || c->wd[el_ex] == 1) {
                fn_ex[0] = fh[0]; fn_ex[1] = fh[1]; fn_ex[2] = fh[2];
            } else {
                double l2 = orc_roe_flux(fn_ex, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, 0, g);
                if (isnan(fn_ex[0]) || isnan(fn_ex[1]) || isnan(fn_ex[2]))
                    return set_err(c, ORC_ERR_NAN_FLUX_EX, i);
                lam = orc_max(lam, l2);
            }
            c->max_lambda = (i == 0) ? lam : orc_max(c->max_lambda, lam);
        }
        /* store (:319-329) */
        c->f1[3 * el_in + k_in] = fn_in[0];
        c->f2[3 * el_in + k_in] = fn_in[1];
        c->f3[3 * el_in + k_in] = fn_in[2];
        if (el_ex != el_in) {
            c->f1[3 * el_ex + k_ex] = -fn_ex[0];
            c->f2[3 * el_ex + k_ex] = -fn_ex[1];
            c->f3[3 * el_ex + k_ex] = -fn_ex[2];
        }
    }

    /* element right-hand sides (:338-411) */
    for (int k = 0; k < c->ne; ++k) {
        double si[9], vi[21];
        orc_inner_products(c, k, si, vi);
        double ze[3] = {-si[0] + vi[0], -si[1] + vi[1], -si[2] + vi[2]};
        double qx[3] = {-si[3] + vi[3] + vi[4] - vi[5], -si[4] + vi[6] + vi[7] - vi[8],
                        -si[5] + vi[9] + vi[10] - vi[11]};
        double qy[3] = {-si[6] + vi[12] + vi[13] - vi[14], -si[7] + vi[15] + vi[16] - vi[17],
                        -si[8] + vi[18] + vi[19] - vi[20]};
        const int *ev = &c->el2v[3 * k];
        double x0 = c->x[ev[0]], x1 = c->x[ev[1]], x2 = c->x[ev[2]];
        double y0 = c->y[ev[0]], y1 = c->y[ev[1]], y2 = c->y[ev[2]];
        double jac = x0 * (y1 - y2) + x1 * (y2 - y0) + x2 * (y0 - y1);
        double m11 = 6 / fabs(jac);
        double mi[3][3] = {{m11, 0, 0}, {0, m11, 0}, {0, 0, m11}};
        for (int j = 0; j < 3; ++j) {
            c->rz[3 * k + j] = mi[j][0] * ze[0] + mi[j][1] * ze[1] + mi[j][2] * ze[2];
            c->rqx[3 * k + j] = mi[j][0] * qx[0] + mi[j][1] * qx[1] + mi[j][2] * qx[2];
            c->rqy[3 * k + j] = mi[j][0] * qy[0] + mi[j][1] * qy[1] + mi[j][2] * qy[2];
        }
    }
    /* rain extension: RHSZeta += rain (absent from the reference; skipped when zero) */
    if (rain != 0.0)
        for (int i = 0; i < 3 * c->ne; ++i) c->rz[i] += rain;
    return 0;
}

/* SlopeLimiter, 2DCode/SlopeLimiter2D.c:10-359 (live code). */
int orc_slope_limiter(orc_ctx *c)
{
    const int nn = c->nn;
    double *bmax = malloc(3 * (size_t)nn * sizeof(double));
    double *bmin = malloc(3 * (size_t)nn * sizeof(double));
    double *vars[3] = {c->zeta, c->qx, c->qy};
    /* node bounds of element averages (:105-153) */
    for (int i = 0; i < nn; ++i) {
        double mx[3] = {-99999, -99999, -99999}, mn[3] = {99999, 99999, 99999};
        for (int j = c->n2e_ptr[i]; j < c->n2e_ptr[i + 1]; ++j) {
            int el = c->n2e[j];
            for (int v = 0; v < 3; ++v) {
                double avg = (vars[v][3 * el] + vars[v][3 * el + 1] + vars[v][3 * el + 2]) / 3;
                if (avg < mn[v]) mn[v] = avg;
                if (avg > mx[v]) mx[v] = avg;
            }
        }
        for (int v = 0; v < 3; ++v) {
            bmax[3 * i + v] = mx[v];
            bmin[3 * i + v] = mn[v];
        }
    }
    /* element pass (:157-343) */
    const double h0 = c->h0;
    for (int el = 0; el < c->ne; ++el) {
        const int nd[3] = {c->el2v[3 * el], c->el2v[3 * el + 1], c->el2v[3 * el + 2]};
        int modify = 0;
        for (int v = 0; v < 3; ++v) {
            double *w = vars[v];
            const double w1 = w[3 * el], w2 = w[3 * el + 1], w3 = w[3 * el + 2];
            double vx[3] = {w1 - w2 + w3, w1 + w2 - w3, -w1 + w2 + w3};
            double vmax[3], vmin[3];
            for (int k = 0; k < 3; ++k) {
                vmax[k] = bmax[3 * nd[k] + v];
                vmin[k] = bmin[3 * nd[k] + v];
            }
            const double avg = (w1 + w2 + w3) / 3;
            if (v == 0) {
                const double zz[3] = {c->z[nd[0]], c->z[nd[1]], c->z[nd[2]]};
                double h1 = vx[0] + zz[0], h2 = vx[1] + zz[1], h3 = vx[2] + zz[2];
                double m0 = vmin[0] + zz[0], m1 = vmin[1] + zz[1], m2 = vmin[2] + zz[2];
                if (h1 > h0 && h2 > h0 && h3 > h0 && m0 > h0 && m1 > h0 && m2 > h0) modify = 1;
            }
            for (int k = 0; k < 3; ++k) vx[k] = fmax_b(orc_min(vx[k], vmax[k]), vmin[k]);
            /* three passes of mass-conserving redistribution (:249-299) */
            for (int ll = 0; ll < 3; ++ll) {
                double sumloc = (vx[0] + vx[1] + vx[2]) / 3;
                double sumdiff = (sumloc - avg) * 3;
                int sd = orc_sign(sumdiff);
                double diff[3] = {(vx[0] - avg) * sd, (vx[1] - avg) * sd, (vx[2] - avg) * sd};
                double kdp = (diff[0] > 0) + (diff[1] > 0) + (diff[2] > 0);
                for (int k = 0; k < 3; ++k) {
                    double div = fmax(1, kdp);
                    double redfac, redmax;
                    if (diff[k] > 0) {
                        redfac = sumdiff * sd / div;
                        kdp -= 1;
                    } else
                        redfac = 0;
                    if (sd > 0)
                        redmax = vx[k] - vmin[k];
                    else
                        redmax = vmax[k] - vx[k];
                    redfac = orc_min(redfac, redmax);
                    sumdiff -= redfac * sd;
                    vx[k] -= redfac * sd;
                }
            }
            const double mid1 = (vx[0] + vx[1]) / 2, mid2 = (vx[1] + vx[2]) / 2, mid3 = (vx[2] + vx[0]) / 2;
            if (v == 0) {
                double h1 = vx[0] + c->z[nd[0]], h2 = vx[1] + c->z[nd[1]], h3 = vx[2] + c->z[nd[2]];
                if (h1 < h0 || h2 < h0 || h3 < h0) modify = 0;
            }
            if (modify) {
                w[3 * el] = mid1;
                w[3 * el + 1] = mid2;
                w[3 * el + 2] = mid3;
            }
        }
        c->dec_limit[el] = modify;
    }
    free(bmax);
    free(bmin);
    return 0;
}

/* BigTheta, 2DCode/wetDry2D.c:7-14 */
static int big_theta(double a) { return a > 0 ? 1 : 0; }

/* wetDryStatus2D, 2DCode/wetDry2D.c:16-60 */
void orc_wd_status(orc_ctx *c)
{
    const double h0 = c->h0;
    for (int el = 0; el < c->ne; ++el) {
        const double m0 = c->zeta[3 * el], m1 = c->zeta[3 * el + 1], m2 = c->zeta[3 * el + 2];
        const double zv[3] = {m0 - m1 + m2, m0 + m1 - m2, -m0 + m1 + m2};
        const double zn[3] = {c->z[c->el2v[3 * el]], c->z[c->el2v[3 * el + 1]], c->z[c->el2v[3 * el + 2]]};
        const double h[3] = {zv[0] + zn[0], zv[1] + zn[1], zv[2] + zn[2]};
        const double avg_h = (h[0] + h[1] + h[2]) / 3;
        int imax = 0;
        double hmax = h[0];
        for (int i = 1; i < 3; ++i)
            if (h[i] > hmax) {
                imax = i;
                hmax = h[i];
            }
        const double zeta_max = zv[imax];
        double zmin = zn[0];
        for (int i = 1; i < 3; ++i)
            if (zn[i] < zmin) zmin = zn[i];
        if (c->wd[el] == -1)
            c->wd[el] = big_theta(avg_h - h0) * big_theta(zeta_max - (h0 - zmin));
        else
            c->wd[el] = c->wd[el] * big_theta(avg_h - h0) +
                        (1 - c->wd[el]) * big_theta(avg_h - h0) * big_theta(zeta_max - (h0 - zmin));
    }
}

/* PDop2D, 2DCode/wetDry2D.c:63-260 */
int orc_pdop(orc_ctx *c)
{
    const double h0 = c->h0;
    for (int el = 0; el < c->ne; ++el) {
        int mass_branch = 0, mom_branch = 0;
        const double mz0 = c->zeta[3 * el], mz1 = c->zeta[3 * el + 1], mz2 = c->zeta[3 * el + 2];
        const double z0 = c->z[c->el2v[3 * el]], z1 = c->z[c->el2v[3 * el + 1]], z2 = c->z[c->el2v[3 * el + 2]];
        const double midz0 = 0.5 * (z0 + z1), midz1 = 0.5 * (z1 + z2), midz2 = 0.5 * (z2 + z0);
        double mh0 = mz0 + midz0, mh1 = mz1 + midz1, mh2 = mz2 + midz2;
        double ht[3] = {mh0 - mh1 + mh2, mh0 + mh1 - mh2, -mh0 + mh1 + mh2};
        const double avg_h = (ht[0] + ht[1] + ht[2]) / 3;
        if (ht[0] <= h0 || ht[1] <= h0 || ht[2] <= h0) {
            if (avg_h <= h0) {
                mass_branch = 1;
                for (int i = 0; i < 3; ++i) ht[i] = avg_h;
            } else {
                mass_branch = 2;
                int imin = 0;
                double hmin = ht[0];
                for (int i = 1; i < 3; ++i)
                    if (ht[i] < hmin) {
                        imin = i;
                        hmin = ht[i];
                    }
                /* the second search starts at index 1 even when index 1 is the minimum
                 * (:115-124); kept as is, it decides which vertices give up mass */
                int inext = 1;
                double hnext = ht[1];
                for (int i = 0; i < 3; ++i)
                    if (ht[i] < hnext && i != imin) {
                        inext = i;
                        hnext = ht[i];
                    }
                int irem = 2;
                for (int i = 0; i < 3; ++i)
                    if (i != imin && i != inext) {
                        irem = i;
                        break;
                    }
                ht[imin] = h0;
                ht[inext] = fmax(h0, hnext - 0.5 * (ht[imin] - hmin));
                ht[irem] = ht[irem] - (ht[imin] - hmin) - (ht[inext] - hnext);
            }
            if (isnan(ht[0]) || isnan(ht[1]) || isnan(ht[2])) {
                c->dec_pdop[el] = 4 * mass_branch;
                return set_err(c, ORC_ERR_NEG_DEPTH, el);
            }
            mh0 = 0.5 * (ht[0] + ht[1]);
            mh1 = 0.5 * (ht[1] + ht[2]);
            mh2 = 0.5 * (ht[2] + ht[0]);
            c->zeta[3 * el] = mh0 - midz0;
            c->zeta[3 * el + 1] = mh1 - midz1;
            c->zeta[3 * el + 2] = mh2 - midz2;
        }
        int wet[3];
        for (int i = 0; i < 3; ++i) wet[i] = (ht[i] > h0);
        if (wet[0] == 0 && wet[1] == 0 && wet[2] == 0) {
            mom_branch = 1;
            for (int i = 0; i < 3; ++i) {
                c->qx[3 * el + i] = 0;
                c->qy[3 * el + i] = 0;
            }
        } else if (wet[0] == 0 || wet[1] == 0 || wet[2] == 0) {
            mom_branch = 2;
            const double q0 = c->qx[3 * el], q1 = c->qx[3 * el + 1], q2 = c->qx[3 * el + 2];
            const double r0 = c->qy[3 * el], r1 = c->qy[3 * el + 1], r2 = c->qy[3 * el + 2];
            double qxe[3] = {q0 - q1 + q2, q0 + q1 - q2, -q0 + q1 + q2};
            double qye[3] = {r0 - r1 + r2, r0 + r1 - r2, -r0 + r1 + r2};
            double u[3], v[3];
            for (int i = 0; i < 3; ++i) {
                u[i] = qxe[i] / ht[i];
                v[i] = qye[i] / ht[i];
            }
            int npos = 0;
            double delu = 0, delv = 0;
            for (int i = 0; i < 3; ++i) {
                npos += wet[i];
                delu += u[i] * (1 - wet[i]) * (fabs(qxe[i]) > c->velzero);
                delv += v[i] * (1 - wet[i]) * (fabs(qye[i]) > c->velzero);
            }
            for (int i = 0; i < 3; ++i) {
                u[i] = wet[i] * (u[i] + delu / npos);
                v[i] = wet[i] * (v[i] + delv / npos);
                if (isnan(u[i]) || isnan(v[i])) {
                    c->dec_pdop[el] = 4 * mass_branch + mom_branch;
                    return set_err(c, ORC_ERR_NAN_VELOCITY, el);
                }
            }
            for (int i = 0; i < 3; ++i) {
                qxe[i] = ht[i] * u[i];
                qye[i] = ht[i] * v[i];
            }
            for (int i = 0; i < 3; ++i) {
                c->qx[3 * el + i] = 0.5 * (qxe[i % 3] + qxe[(i + 1) % 3]);
                c->qy[3 * el + i] = 0.5 * (qye[i % 3] + qye[(i + 1) % 3]);
            }
        }
        c->dec_pdop[el] = 4 * mass_branch + mom_branch;
    }
    return 0;
}

/* One SSP-RK2 step: 2DCode/time_evolution.c:10-246 with the wet/dry calls of
 * ChanNet/time_evolution.c:225-226,330-333,413-415.  The reference copies through gsl
 * vectors; the arithmetic per entry is w1 = w + RHS*dt, then w = 0.5*(w1 + w) + RHS*(dt/2). */
int orc_step(orc_ctx *c, double time, double dt, int wet_dry, double rain, int *limit0, int *pdop0,
             int *limit1, int *pdop1)
{
    (void)time;
    const size_t n = 3 * (size_t)c->ne;
    int rc;
    double *w0z = dup_mem(c->zeta, n * sizeof(double));
    double *w0x = dup_mem(c->qx, n * sizeof(double));
    double *w0y = dup_mem(c->qy, n * sizeof(double));
    if (wet_dry) orc_wd_status(c);

    if ((rc = orc_compute_L(c, wet_dry, rain))) goto out;
    for (size_t i = 0; i < n; ++i) {
        c->zeta[i] = w0z[i] + c->rz[i] * dt;
        c->qx[i] = w0x[i] + c->rqx[i] * dt;
        c->qy[i] = w0y[i] + c->rqy[i] * dt;
    }
    orc_slope_limiter(c);
    if (limit0) memcpy(limit0, c->dec_limit, (size_t)c->ne * sizeof(int));
    if (wet_dry) {
        if ((rc = orc_pdop(c))) goto out;
        if (pdop0) memcpy(pdop0, c->dec_pdop, (size_t)c->ne * sizeof(int));
        orc_wd_status(c);
    }

    if ((rc = orc_compute_L(c, wet_dry, rain))) goto out;
    const double half_dt = dt / 2;
    for (size_t i = 0; i < n; ++i) {
        c->zeta[i] = (c->zeta[i] + w0z[i]) * 0.5 + c->rz[i] * half_dt;
        c->qx[i] = (c->qx[i] + w0x[i]) * 0.5 + c->rqx[i] * half_dt;
        c->qy[i] = (c->qy[i] + w0y[i]) * 0.5 + c->rqy[i] * half_dt;
    }
    orc_slope_limiter(c);
    if (limit1) memcpy(limit1, c->dec_limit, (size_t)c->ne * sizeof(int));
    if (wet_dry) {
        if ((rc = orc_pdop(c))) goto out;
        if (pdop1) memcpy(pdop1, c->dec_pdop, (size_t)c->ne * sizeof(int));
    }
out:
    free(w0z);
    free(w0x);
    free(w0y);
    return rc;
}

/* One SSP(3,3) step (extension: the coefficients of DG-SWEM src/prep_DG.F:1253-1270 around
 * the 2DCode operators, limiter / PDop / status after every stage as in orc_step):
 * u1 = u + dt L(u);  u2 = 0.75 u + 0.25 (u1 + dt L(u1));  u3 = 1/3 u + 2/3 (u2 + dt L(u2)). */
int orc_step3(orc_ctx *c, double time, double dt, int wet_dry, double rain)
{
    (void)time;
    const size_t n = 3 * (size_t)c->ne;
    int rc = 0;
    double *w0z = dup_mem(c->zeta, n * sizeof(double));
    double *w0x = dup_mem(c->qx, n * sizeof(double));
    double *w0y = dup_mem(c->qy, n * sizeof(double));
    if (wet_dry) orc_wd_status(c);
    for (int st = 0; st < 3; ++st) {
        if ((rc = orc_compute_L(c, wet_dry, rain))) break;
        if (st == 0) {
            for (size_t i = 0; i < n; ++i) {
                c->zeta[i] = w0z[i] + c->rz[i] * dt;
                c->qx[i] = w0x[i] + c->rqx[i] * dt;
                c->qy[i] = w0y[i] + c->rqy[i] * dt;
            }
        } else {
            const double a = st == 1 ? 0.75 : 1.0 / 3;
            const double b = st == 1 ? 0.25 : 2.0 / 3;
            for (size_t i = 0; i < n; ++i) {
                c->zeta[i] = a * w0z[i] + b * (c->zeta[i] + c->rz[i] * dt);
                c->qx[i] = a * w0x[i] + b * (c->qx[i] + c->rqx[i] * dt);
                c->qy[i] = a * w0y[i] + b * (c->qy[i] + c->rqy[i] * dt);
            }
        }
        orc_slope_limiter(c);
        if (wet_dry) {
            if ((rc = orc_pdop(c))) break;
            if (st < 2) orc_wd_status(c);
        }
    }
    free(w0z);
    free(w0x);
    free(w0y);
    return rc;
}

/* Time loop of 2DCode/time_evolution.c:248-402 without file output. */
int orc_run(orc_ctx *c, int nsteps, double final_time, double cfl, double dt0, int wet_dry,
            double rain, int tide_on, double amp, double period, double *time_io, double *dt_io,
            double *dt_hist, int *steps_done)
{
    return orc_run_rk(c, nsteps, final_time, cfl, dt0, wet_dry, rain, tide_on, amp, period, time_io, dt_io,
                      dt_hist, steps_done, 2);
}

/* orc_run with 2 (SSP-RK2, the reference) or 3 (SSP(3,3)) stages per step; the CFL dt
 * follows the last stage's max wave speed. */
int orc_run_rk(orc_ctx *c, int nsteps, double final_time, double cfl, double dt0, int wet_dry,
               double rain, int tide_on, double amp, double period, double *time_io, double *dt_io,
               double *dt_hist, int *steps_done, int stages)
{
    double time = *time_io, dt = *dt_io;
    int done = 0, rc = 0;
    if (time < 0) {
        time = 0;
        dt = dt0;
        orc_boundary_conditions(c, time, tide_on, amp, period);
    }
    while (done < nsteps && time < final_time) {
        time = time + dt;
        rc = stages == 3 ? orc_step3(c, time, dt, wet_dry, rain)
                         : orc_step(c, time, dt, wet_dry, rain, NULL, NULL, NULL, NULL);
        if (rc) break;
        orc_boundary_conditions(c, time, tide_on, amp, period);
        if (dt_hist) dt_hist[done] = dt;
        ++done;
        dt = cfl * c->min_edge / c->max_lambda;
        if ((time + dt) > final_time) dt = final_time - time;
    }
    *time_io = time;
    *dt_io = dt;
    *steps_done = done;
    return rc;
}

/* ------------------------------------------------------------ channel coupling ---- */

/* Junction side of one coupled edge e as ChanNet/internal_BC.c:33-95 forms it: the element
 * EdgtoEls[2e], its local edge found by vertex matching (pairs (1,2), (2,3), (3,1) in that
 * order), the edge length and outward normal from the element's vertices, and the mid-edge
 * depth of the edge's own vertices. */
static int orc_cpl_edge(const double *x, const double *y, const double *z, const int *el2v, const int *ed2v,
                        const int *ed2el, int e, int *el_out, int *k_out, double *len, double *nx, double *ny,
                        double *zmid)
{
    const int el = ed2el[2 * e];
    const int a = el2v[3 * el], b = el2v[3 * el + 1], c = el2v[3 * el + 2];
    const int p = ed2v[2 * e], q = ed2v[2 * e + 1];
    const double xa = x[a], xb = x[b], xc = x[c], ya = y[a], yb = y[b], yc = y[c];
    double x0, x1, y0, y1, l;
    int k;
    if ((a == p && b == q) || (a == q && b == p)) {
        k = 0;
        x0 = xa; x1 = xb; y0 = ya; y1 = yb;
        l = sqrt((xa - xb) * (xa - xb) + (ya - yb) * (ya - yb));
    } else if ((b == p && c == q) || (b == q && c == p)) {
        k = 1;
        x0 = xb; x1 = xc; y0 = yb; y1 = yc;
        l = sqrt((xb - xc) * (xb - xc) + (yb - yc) * (yb - yc));
    } else if ((c == p && a == q) || (c == q && a == p)) {
        k = 2;
        x0 = xc; x1 = xa; y0 = yc; y1 = ya;
        l = sqrt((xa - xc) * (xa - xc) + (ya - yc) * (ya - yc));
    } else {
        return -1;
    }
    const double jac = (xb - xa) * (yc - ya) - (xc - xa) * (yb - ya);
    const int s = (jac < 0) ? -1 : (jac == 0 ? 0 : 1); /* sign() of ChanNet/mathfunctions.c:17-25 */
    *el_out = el;
    *k_out = k;
    *len = l;
    *nx = s * (y1 - y0) / l;
    *ny = s * (x0 - x1) / l;
    *zmid = 0.5 * (z[p] + z[q]);
    return 0;
}

int orc_internal_bc(int ne, int nf, const double *x, const double *y, const double *z, const int *el2v,
                    const int *ed2v, const int *ed2el, const double *zeta, const double *qx, const double *qy,
                    double *bzeta, double *bqn, int nchan, const int *in_ptr, const int *in_edges,
                    const int *out_ptr, const int *out_edges, const int *chan_nodes, const int *chan_off,
                    double *A, double *Q)
{
    (void)ne;
    for (int ch = 0; ch < nchan; ++ch) {
        double *Ac = A + 2 * (size_t)chan_off[ch], *Qc = Q + 2 * (size_t)chan_off[ch];
        const int nn = chan_nodes[ch];
        for (int side = 0; side < 2; ++side) { /* inflow list (:23-115), then outflow (:117-216) */
            const int *ptr = side ? out_ptr : in_ptr;
            const int *edges = side ? out_edges : in_edges;
            const int n = ptr[ch + 1] - ptr[ch];
            const int node_val = side ? 2 * nn - 2 : 1; /* the channel's own trace at the junction */
            double area = 0, qn_sum = 0;
            for (int j = ptr[ch]; j < ptr[ch + 1]; ++j) {
                const int e = edges[j];
                if (e < 0 || e >= nf) return -1;
                int el, k;
                double len, nx, ny, zmid;
                if (orc_cpl_edge(x, y, z, el2v, ed2v, ed2el, e, &el, &k, &len, &nx, &ny, &zmid)) return -1;
                const double h = zeta[3 * el + k] + zmid;
                const double qn = qx[3 * el + k] * nx + qy[3 * el + k] * ny;
                if (side) {
                    area += h * len;
                } else {
                    area += len * h;
                }
                qn_sum += qn * len;
                const double Hc = Ac[node_val] / (n * len);
                bzeta[e] = Hc - zmid;
                bqn[e] = side ? -Qc[node_val] / (n * len) : Qc[node_val] / (n * len);
            }
            if (n != 0) {
                if (side) {
                    Qc[2 * nn - 1] = -qn_sum;
                    Ac[2 * nn - 1] = area;
                } else {
                    Qc[0] = qn_sum;
                    Ac[0] = area;
                }
            }
        }
    }
    return 0;
}
