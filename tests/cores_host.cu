/*
 * Test harness: the per-edge and per-element differentiation cores of the library
 * (dgr_scheme.cuh forward, instantiated with dual numbers, and the hand-written reverse of
 * dgr_reverse.cuh) compiled as HOST code, so that the tangent-linear / adjoint pairs can be
 * checked on the CPU with many random inputs (dot-product test, finite differences).  Not
 * part of the library: the library's compute path runs on the GPU only.
 *
 * Every function takes the primal inputs x, a tangent direction xd and an output adjoint yb,
 * and returns the outputs y, the tangent yd = J xd and the adjoint xb = J^T yb.
 */
#include "../dg-rain_b200/csrc/dgr_dual.cuh"
#include "../dg-rain_b200/csrc/dgr_reverse.cuh"

using namespace dgr;
using ad::Dual;

namespace {

struct DualZ {
    Dual mz[3], gn[3], gz[2];
    Dual midz(int e) const { return mz[e]; }
    Dual gnn(int e) const { return gn[e]; }
    Dual gradz(int j) const { return gz[j]; }
};

}  // namespace

static int g_ftype = 0; /* numerical flux of the edge cases: 0 Roe, 1 local Lax-Friedrichs */

extern "C" {

void dgr_t_set_flux(int type) { g_ftype = type; }

/* x = zin, zex, qxin, qxex, qyin, qyex, zedge */
int dgr_t_roe(const double *x, double nx, double ny, double lg, double g, const double *xd, const double *yb,
              double *y, double *yd, double *xb)
{
    Dual in[7];
    for (int i = 0; i < 7; ++i) in[i] = Dual(x[i], xd[i]);
    Dual fh[3];
    numerical_flux<Dual>(g_ftype, fh, in[0], in[1], in[2], in[3], in[4], in[5], in[6], nx, ny, lg, g);
    for (int k = 0; k < 3; ++k) {
        y[k] = fh[k].v;
        yd[k] = fh[k].d;
    }
    RoeBar b = {0, 0, 0, 0, 0, 0, 0};
    numerical_flux_rev(g_ftype, yb, x[0], x[1], x[2], x[3], x[4], x[5], x[6], nx, ny, lg, g, b);
    const double o[7] = {b.zin, b.zex, b.qxin, b.qxex, b.qyin, b.qyex, b.zed};
    for (int i = 0; i < 7; ++i) xb[i] = o[i];
    return 0;
}

/* x = zi, qxi, qyi, ze, qxe, qye (exterior slot; ignored on boundary edges), z_edge;
 * kind: 0 interior, 1 land, 2 prescribed (bd, bz, bq); y = fin[3], fex[3] */
int dgr_t_edge(int wd_on, int kind, int bd, int wdi, int wde, double bz, double bq, const double *x, double nx,
               double ny, double g, const double *xd, const double *yb, double *y, double *yd, double *xb)
{
    Dual in[7];
    for (int i = 0; i < 7; ++i) in[i] = Dual(x[i], xd[i]);
    Dual ze, qxe, qye;
    if (kind == 2)
        ghost_state<Dual>(bd, nx, ny, in[0], in[1], in[2], bz, bq, Dual(0.0), ze, qxe, qye);
    else if (kind == 1)
        ghost_state<Dual>(0, nx, ny, in[0], in[1], in[2], 0.0, 0.0, in[0], ze, qxe, qye);
    else {
        ze = in[3];
        qxe = in[4];
        qye = in[5];
    }
    Dual fin[3], fex[3];
    int code;
    if (wd_on)
        flux_core<Dual, true>(in[0], in[1], in[2], ze, qxe, qye, in[6], nx, ny, wdi, wde, g, fin, fex, code, g_ftype);
    else
        flux_core<Dual, false>(in[0], in[1], in[2], ze, qxe, qye, in[6], nx, ny, wdi, wde, g, fin, fex, code,
                               g_ftype);
    for (int k = 0; k < 3; ++k) {
        y[k] = fin[k].v;
        yd[k] = fin[k].d;
        y[3 + k] = fex[k].v;
        yd[3 + k] = fex[k].d;
    }
    /* reverse */
    double zev = x[3], qxev = x[4], qyev = x[5];
    if (kind) ghost_state<double>(kind == 2 ? bd : 0, nx, ny, x[0], x[1], x[2], bz, bq, x[0], zev, qxev, qyev);
    EdgeBar b = {0, 0, 0, 0, 0, 0, 0};
    if (wd_on)
        flux_core_rev<true>(x[0], x[1], x[2], zev, qxev, qyev, x[6], nx, ny, wdi, wde, g, yb, yb + 3, b, g_ftype);
    else
        flux_core_rev<false>(x[0], x[1], x[2], zev, qxev, qyev, x[6], nx, ny, wdi, wde, g, yb, yb + 3, b, g_ftype);
    for (int i = 0; i < 7; ++i) xb[i] = 0;
    if (kind) {
        ghost_state_rev(kind == 2 ? bd : 0, nx, ny, bz, bq, b.ze, b.qxe, b.qye, b.zi, b.qxi, b.qyi);
    } else {
        xb[3] = b.ze;
        xb[4] = b.qxe;
        xb[5] = b.qye;
    }
    xb[0] = b.zi;
    xb[1] = b.qxi;
    xb[2] = b.qyi;
    xb[6] = b.zed;
    return code;
}

/* One element: inputs F[9] ([v][k]), S[9] (stage input [v][k]), U[9] (step input, stage
 * 2), vertex depths zv[3] and element n; outputs w[9].  Tangent/adjoint inputs in the same
 * order; geometry from the vertex coordinates xv, yv. */
int dgr_t_element(int mode, const double *xv, const double *yv, const double *zv, double nel, double g, double lg,
                  double rain, double dt, const double *F, const double *S, const double *U, const double *Fd,
                  const double *Sd, const double *Ud, const double *zvd, double neld, const double *wbar, double *w,
                  double *wdot, double *Fb, double *Sb, double *Ub, double *zvb, double *nelb)
{
    double G[NG];
    const double nfv[3] = {0.03, 0.03, 0.03};
    element_geometry(xv, yv, zv, nfv, nel, g, [&G](int j, double val) { G[j] = val; });
    const auto geo = [&G](int j) { return G[j]; };
    /* forward-mode */
    DualZ zg;
    for (int e = 0; e < 3; ++e) {
        zg.mz[e] = Dual(G[G_MIDZ + e], 0.5 * (zvd[e] + zvd[(e + 1) % 3]));
        zg.gn[e] = Dual(G[G_GNN + e], 2.0 * g * nel * neld);
    }
    for (int j = 0; j < 2; ++j)
        zg.gz[j] = Dual(G[G_GRADZ + j],
                        zg.mz[0].d * G[G_GP + j] + zg.mz[1].d * G[G_GP + 2 + j] + zg.mz[2].d * G[G_GP + 4 + j]);
    Dual Fv[3][3], zr[3], qxr[3], qyr[3], Uv[3][3];
    for (int v = 0; v < 3; ++v)
        for (int k = 0; k < 3; ++k) {
            Fv[v][k] = Dual(F[3 * v + k], Fd[3 * v + k]);
            Uv[v][k] = Dual(U[3 * v + k], Ud[3 * v + k]);
        }
    for (int k = 0; k < 3; ++k) {
        zr[k] = Dual(S[k], Sd[k]);
        qxr[k] = Dual(S[3 + k], Sd[3 + k]);
        qyr[k] = Dual(S[6 + k], Sd[6 + k]);
    }
    const auto uin = [&Uv](int v, int k) { return Uv[v][k]; };
    Dual wo[3][3], av[3];
    if (mode == 1)
        element_core<MODE_STAGE1, Dual>(Fv, zr, qxr, qyr, geo, zg, uin, lg, rain, dt, wo, av);
    else if (mode == 2)
        element_core<MODE_STAGE2, Dual>(Fv, zr, qxr, qyr, geo, zg, uin, lg, rain, dt, wo, av);
    else
        element_core<MODE_RHS, Dual>(Fv, zr, qxr, qyr, geo, zg, uin, lg, rain, dt, wo, av);
    for (int i = 0; i < 9; ++i) {
        w[i] = wo[i / 3][i % 3].v;
        wdot[i] = wo[i / 3][i % 3].d;
    }
    /* reverse */
    double wb[3][3], Fbar[3][3] = {{0}}, Sbar[3][3] = {{0}}, midzb[3] = {0, 0, 0}, gnnb[3] = {0, 0, 0},
                     gradzb[2] = {0, 0};
    for (int i = 0; i < 9; ++i) wb[i / 3][i % 3] = wbar[i];
    const double zrv[3] = {S[0], S[1], S[2]}, qxv[3] = {S[3], S[4], S[5]}, qyv[3] = {S[6], S[7], S[8]};
    const PlaneZGeo pz{G, 1};
    if (mode == 1)
        element_core_rev<MODE_STAGE1>(wb, zrv, qxv, qyv, geo, pz, lg, dt, Fbar, Sbar, midzb, gnnb, gradzb);
    else if (mode == 2)
        element_core_rev<MODE_STAGE2>(wb, zrv, qxv, qyv, geo, pz, lg, dt, Fbar, Sbar, midzb, gnnb, gradzb);
    else
        element_core_rev<MODE_RHS>(wb, zrv, qxv, qyv, geo, pz, lg, dt, Fbar, Sbar, midzb, gnnb, gradzb);
    for (int i = 0; i < 9; ++i) {
        Fb[i] = Fbar[i / 3][i % 3];
        Sb[i] = Sbar[i / 3][i % 3];
        Ub[i] = mode == 2 ? 0.5 * wbar[i] : 0.0;
    }
    double mb[3];
    for (int k = 0; k < 3; ++k) mb[k] = midzb[k] + G[G_GP + 2 * k] * gradzb[0] + G[G_GP + 2 * k + 1] * gradzb[1];
    for (int k = 0; k < 3; ++k) zvb[k] = 0;
    for (int e = 0; e < 3; ++e) {
        zvb[e] += 0.5 * mb[e];
        zvb[(e + 1) % 3] += 0.5 * mb[e];
    }
    *nelb = (gnnb[0] + gnnb[1] + gnnb[2]) * 2.0 * g * nel;
    return 0;
}

/* Limiter (+ PDop): inputs w[9], bmax[9], bmin[9] ([v][k]), zn[3]; outputs w[9];
 * dec = modify, mass branch, momentum branch, code. */
int dgr_t_limit(int pdop, const double *w, const double *bmax, const double *bmin, const double *zn, double h0,
                double velzero, const double *wd_, const double *bmaxd, const double *bmind, const double *znd,
                const double *wbar, double *out, double *outd, double *wb_out, double *bmaxb, double *bminb,
                double *znb, int *dec)
{
    Dual wv[3][3], znv[3];
    for (int i = 0; i < 9; ++i) wv[i / 3][i % 3] = Dual(w[i], wd_[i]);
    for (int k = 0; k < 3; ++k) znv[k] = Dual(zn[k], znd[k]);
    const auto bnd_d = [&](int v, int k, int is_min) {
        return is_min ? Dual(bmin[3 * v + k], bmind[3 * v + k]) : Dual(bmax[3 * v + k], bmaxd[3 * v + k]);
    };
    LimitDecisions d;
    if (pdop)
        limit_core<true, true, Dual>(wv, bnd_d, znv, h0, velzero, d);
    else
        limit_core<true, false, Dual>(wv, bnd_d, znv, h0, velzero, d);
    for (int i = 0; i < 9; ++i) {
        out[i] = wv[i / 3][i % 3].v;
        outd[i] = wv[i / 3][i % 3].d;
    }
    double w0[3][3], wb[3][3], bxb[3][3] = {{0}}, bnb[3][3] = {{0}}, zb[3] = {0, 0, 0};
    for (int i = 0; i < 9; ++i) {
        w0[i / 3][i % 3] = w[i];
        wb[i / 3][i % 3] = wbar[i];
    }
    const auto bnd = [&](int v, int k, int is_min) { return is_min ? bmin[3 * v + k] : bmax[3 * v + k]; };
    LimitDecisions d2;
    if (pdop)
        d2 = limit_core_rev<true, true>(w0, bnd, zn, h0, velzero, wb, bxb, bnb, zb);
    else
        d2 = limit_core_rev<true, false>(w0, bnd, zn, h0, velzero, wb, bxb, bnb, zb);
    for (int i = 0; i < 9; ++i) {
        wb_out[i] = wb[i / 3][i % 3];
        bmaxb[i] = bxb[i / 3][i % 3];
        bminb[i] = bnb[i / 3][i % 3];
    }
    for (int k = 0; k < 3; ++k) znb[k] = zb[k];
    dec[0] = d.modify;
    dec[1] = d.mass_branch;
    dec[2] = d.mom_branch;
    dec[3] = d.code;
    dec[4] = (d2.modify == d.modify && d2.mass_branch == d.mass_branch && d2.mom_branch == d.mom_branch) ? 1 : 0;
    return 0;
}

/* the Manning power x^(4./3) as the host compiles it (pow43_exact: cbrt refined by one
 * Newton step with exact residuals, log-based exponent correction) */
void dgr_t_pow43(const double *x, double *y, int n)
{
    for (int i = 0; i < n; ++i) y[i] = pow43(x[i]);
}

}  // extern "C"
