/*
 * Arithmetic of the DG-RAIN 2D step for one edge or one element, templated on the scalar:
 * T = double is the forward step (the kernels in dgr_kernels.cuh), T = ad::Dual is its
 * tangent-linear model.  Loads and stores stay in the kernels; these functions see values
 * only, so one source defines the discrete scheme that the forward runs, the TLM
 * linearises and the hand-written reverse (dgr_reverse.cuh) transposes.
 *
 * Expressions are the reference's, in its order (see dgr_device.cuh): instantiated with
 * double they are the same IEEE operations as 2DCode's C.
 */
#pragma once

#include <type_traits>

#include "dgr_device.cuh"

namespace dgr {

/* element geometry planes */
enum {
    G_NX = 0,     /* nx1..nx3              2DCode/2DInnerProducts.c:110-116 */
    G_NY = 3,     /* ny1..ny3 */
    G_M12 = 6,    /* x_k*nx_k + y_k*ny_k   :126-128 */
    G_DM = 9,     /* Cramer determinant    :134 */
    G_XE = 10,    /* Gauss points x, [edge][2]   :52-65 */
    G_YE = 16,
    G_EJ = 22,    /* edge Jacobians        :42-45 */
    G_PSI = 25,   /* basis at Gauss points [basis][edge][2]  :73-87 */
    G_MIDZ = 43,  /* mid-edge depth        :268-270 */
    G_GNN = 46,   /* g*n*n per edge        :318 */
    G_GP = 49,    /* grad psi [basis][2]   :303-308 */
    G_GRADZ = 55, /* grad z                :343-347 */
    G_AJ = 57,    /* |jac|                 :522 */
    G_P = 58,     /* grad psi . (sum of midpoints)  :523-524 */
    G_AJW = 61,   /* |jac| * (1/6)         :536 */
    G_M11 = 62,   /* 6/|jac| of the vertex Jacobian, 2DCode/compute2DL.c:380-382 */
    NG = 63
};

/* Storage of the planes: tiles of 32 consecutive elements, each tile's NG planes one after
 * another (element el, plane j at ((el / 32) * NG + j) * 32 + el % 32).  A warp reads 256
 * contiguous bytes per plane as with whole planes, and a block's geometry is one
 * contiguous range.  DGR_GEO_TILED=0 (measurement builds): whole planes of stride ldE. */
#ifndef DGR_GEO_TILED
#define DGR_GEO_TILED 1
#endif
DGR_HD size_t geo_offset(int el, int ldE)
{
    return DGR_GEO_TILED ? (size_t)(el >> 5) * (NG * 32) + (el & 31) : (size_t)el;
}
DGR_HD int geo_stride(int ldE) { return DGR_GEO_TILED ? 32 : ldE; }

/* Per-element factors of 2DCode/2DInnerProducts.c and 2DCode/compute2DL.c:373-382 from the
 * vertex coordinates, depths and Manning n (nel >= 0: per-element n, else the node
 * average), each with the reference's own expression; set(j, value) stores plane j. */
template <class SetG>
DGR_HD void element_geometry(const double xv[3], const double yv[3], const double zv[3], const double nfv[3],
                             double nel, double g, const SetG &set)
{
    const double xv1 = xv[0], xv2 = xv[1], xv3 = xv[2];
    const double yv1 = yv[0], yv2 = yv[1], yv3 = yv[2];
    const double x1 = (xv[0] + xv[1]) / 2, x2 = (xv[1] + xv[2]) / 2, x3 = (xv[2] + xv[0]) / 2;
    const double y1 = (yv[0] + yv[1]) / 2, y2 = (yv[1] + yv[2]) / 2, y3 = (yv[2] + yv[0]) / 2;
    double len[3];
    len[0] = sqrt((xv2 - xv1) * (xv2 - xv1) + (yv2 - yv1) * (yv2 - yv1));
    len[1] = sqrt((xv3 - xv2) * (xv3 - xv2) + (yv3 - yv2) * (yv3 - yv2));
    len[2] = sqrt((xv3 - xv1) * (xv3 - xv1) + (yv3 - yv1) * (yv3 - yv1));
    for (int e = 0; e < 3; ++e) set(G_EJ + e, len[e] / 2);
    const double s3 = sqrt(3.0);
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
    for (int e = 0; e < 3; ++e)
        for (int n = 0; n < 2; ++n) {
            set(G_XE + 2 * e + n, xe[e][n]);
            set(G_YE + 2 * e + n, ye[e][n]);
        }
    const double den = x1 * y2 - x1 * y3 + x2 * y3 - x2 * y1 + x3 * y1 - x3 * y2;
    for (int e = 0; e < 3; ++e)
        for (int n = 0; n < 2; ++n) {
            const double xq = xe[e][n], yq = ye[e][n];
            set(G_PSI + 0 * 6 + 2 * e + n, -(yq * x2 - yq * x3 - xq * y2 + x3 * y2 + xq * y3 - x2 * y3) / den);
            set(G_PSI + 1 * 6 + 2 * e + n, -(-x1 * yq + x3 * yq - x3 * y1 + xq * y1 - xq * y3 + x1 * y3) / den);
            set(G_PSI + 2 * 6 + 2 * e + n, -(yq * x1 - yq * x2 - xq * y1 + x2 * y1 + xq * y2 - x1 * y2) / den);
        }
    const double jac = 4 * (x2 - x3) * (y2 - y1) - 4 * (x2 - x1) * (y2 - y3);
    const int sj = sgn(jac);
    const double nx1 = sj * 2 * (y2 - y3) / len[0], ny1 = sj * 2 * (x3 - x2) / len[0];
    const double nx2 = sj * 2 * (y3 - y1) / len[1], ny2 = sj * 2 * (x1 - x3) / len[1];
    const double nx3 = sj * 2 * (y1 - y2) / len[2], ny3 = sj * 2 * (x2 - x1) / len[2];
    set(G_NX, nx1);
    set(G_NX + 1, nx2);
    set(G_NX + 2, nx3);
    set(G_NY, ny1);
    set(G_NY + 1, ny2);
    set(G_NY + 2, ny3);
    const double M11 = nx1, M12 = x1 * nx1 + y1 * ny1, M13 = ny1;
    const double M21 = nx2, M22 = x2 * nx2 + y2 * ny2, M23 = ny2;
    const double M31 = nx3, M32 = x3 * nx3 + y3 * ny3, M33 = ny3;
    set(G_M12, M12);
    set(G_M12 + 1, M22);
    set(G_M12 + 2, M32);
    set(G_DM, M13 * M22 * M31 - M12 * M23 * M31 - M13 * M21 * M32 + M11 * M23 * M32 + M12 * M21 * M33 -
                  M11 * M22 * M33);
    const double midz[3] = {0.5 * (zv[0] + zv[1]), 0.5 * (zv[1] + zv[2]), 0.5 * (zv[2] + zv[0])};
    double midn[3];
    if (nel >= 0.0) {
        midn[0] = midn[1] = midn[2] = nel;
    } else {
        midn[0] = 0.5 * (nfv[0] + nfv[1]);
        midn[1] = 0.5 * (nfv[1] + nfv[2]);
        midn[2] = 0.5 * (nfv[2] + nfv[0]);
    }
    for (int e = 0; e < 3; ++e) {
        set(G_MIDZ + e, midz[e]);
        set(G_GNN + e, g * midn[e] * midn[e]);
    }
    double gp[3][2];
    gp[0][0] = 4 / jac * (y2 - y3);
    gp[0][1] = 4 / jac * (x3 - x2);
    gp[1][0] = 4 / jac * (y3 - y1);
    gp[1][1] = 4 / jac * (x1 - x3);
    gp[2][0] = 4 / jac * (y1 - y2);
    gp[2][1] = 4 / jac * (x2 - x1);
    for (int b = 0; b < 3; ++b) {
        set(G_GP + 2 * b, gp[b][0]);
        set(G_GP + 2 * b + 1, gp[b][1]);
        set(G_P + b, gp[b][0] * (x1 + x2 + x3) + gp[b][1] * (y1 + y2 + y3));
    }
    for (int j = 0; j < 2; ++j) set(G_GRADZ + j, midz[0] * gp[0][j] + midz[1] * gp[1][j] + midz[2] * gp[2][j]);
    const double aj = fabs(jac);
    set(G_AJ, aj);
    set(G_AJW, aj * (1.0 / 6));
    const double jv = xv[0] * (yv[1] - yv[2]) + xv[1] * (yv[2] - yv[0]) + xv[2] * (yv[0] - yv[1]);
    set(G_M11, 6 / fabs(jv));
}

/* Depth- and Manning-dependent element factors read from the geometry planes. */
struct PlaneZGeo {
    const double *G;
    int ld;
    DGR_HD double midz(int e) const { return G[(size_t)(G_MIDZ + e) * ld]; }
    DGR_HD double gnn(int e) const { return G[(size_t)(G_GNN + e) * ld]; }
    DGR_HD double gradz(int j) const { return G[(size_t)(G_GRADZ + j) * ld]; }
};

/* Exterior discharge of a boundary edge from the interior one: normal part qn_ex,
 * tangential part kept (2DCode/compute2DL.c:149-191). */
template <class T>
DGR_HD void ghost_discharge(double nx, double ny, const T &qn_ex, const T &qt_ex, T &qxe, T &qye)
{
    const double tx = -ny, ty = nx;
    const double d = 1. / (nx * ty - ny * tx);
    qxe = (ty * qn_ex - ny * qt_ex) * d;
    qye = (-tx * qn_ex + nx * qt_ex) * d;
}

/* Ghost state of a boundary edge.  bd != 0: prescribed elevation / normal discharge with
 * the reference's sentinels (bzeta < 0: take the interior elevation; bqn > 1000: take the
 * interior normal discharge), :149-164.  bd == 0: land, the normal discharge reflected,
 * :175-191; ze_slot is the elevation the reference reads for the exterior side (the same
 * slot as the interior trace). */
template <class T>
DGR_HD void ghost_state(int bd, double nx, double ny, const T &zi, const T &qxi, const T &qyi, double bz, double bq,
                        const T &ze_slot, T &ze, T &qxe, T &qye)
{
    const double tx = -ny, ty = nx;
    if (bd) {
        ze = bz;
        if (bz < 0) ze = zi;
        T qn_ex = bq;
        if (bq > 1000) qn_ex = qxi * nx + qyi * ny;
        const T qt_ex = qxi * tx + qyi * ty;
        ghost_discharge(nx, ny, qn_ex, qt_ex, qxe, qye);
    } else {
        ze = ze_slot;
        const T qn_in = qxi * nx + qyi * ny;
        const T qt_in = qxi * tx + qyi * ty;
        ghost_discharge(nx, ny, T(-qn_in), qt_in, qxe, qye);
    }
}

/*
 * Numerical flux of one edge (2DCode/compute2DL.c:201-293) from the interior and exterior
 * traces: Fhat.n for the "in" side (fin) and the "ex" side (fex), the max wave speed as the
 * return value, and in `code` the first NaN flux (1: shared flux, 2: in side, 3: ex side).
 * With WD: both dry -> two reflective g = 0 fluxes; one side dry -> that side gets the
 * g = 0 flux.
 */
template <class T, bool WD, class Div = PlainDiv>
DGR_HD T flux_core(const T &zi, const T &qxi, const T &qyi, const T &ze, const T &qxe, const T &qye,
                   const T &z_edge, double nx, double ny, int wdi, int wde, double g, T fin[3], T fex[3],
                   int &code, int ftype = 0, Div *dv = nullptr)
{
    const double tx = -ny, ty = nx;
    T lam = 0.0;
    code = 0;
    if (WD && wdi == 0 && wde == 0) { /* both dry, :203-239 */
        T qn_in = qxi * nx + qyi * ny;
        T qt_in = qxi * tx + qyi * ty;
        T qn_ex = -qn_in, qt_ex = qt_in;
        const double d = 1. / (nx * ty - ny * tx);
        const T qxe_ref = (ty * qn_ex - ny * qt_ex) * d;
        const T qye_ref = (-tx * qn_ex + nx * qt_ex) * d;
        const T lam_in = numerical_flux<T, Div>(ftype, fin, zi, zi, qxi, qxe_ref, qyi, qye_ref,
                                                  z_edge, nx, ny, 0.0, g, dv);
        qn_ex = qxe * nx + qye * ny;
        qt_ex = qxe * tx + qye * ty;
        qn_in = -qn_ex;
        qt_in = qt_ex;
        const T qxi_ref = (ty * qn_in - ny * qt_in) * d;
        const T qyi_ref = (-tx * qn_in + nx * qt_ex) * d;
        const T lam_ex = numerical_flux<T, Div>(ftype, fex, ze, ze, qxi_ref, qxe, qyi_ref, qye,
                                                  z_edge, nx, ny, 0.0, g, dv);
        lam = rmax(lam_in, lam_ex);
    } else {
        T fh[3];
        lam = numerical_flux<T, Div>(ftype, fh, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, g, g, dv);
        if (isnan(fh[0]) || isnan(fh[1]) || isnan(fh[2])) code = 1;
        if (!WD || wdi == 1) {
            fin[0] = fh[0];
            fin[1] = fh[1];
            fin[2] = fh[2];
        } else {
            const T l2 =
                numerical_flux<T, Div>(ftype, fin, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, 0.0, g, dv);
            if (!code && (isnan(fin[0]) || isnan(fin[1]) || isnan(fin[2]))) code = 2;
            lam = rmax(lam, l2);
        }
        if (!WD || wde == 1) {
            fex[0] = fh[0];
            fex[1] = fh[1];
            fex[2] = fh[2];
        } else {
            const T l2 =
                numerical_flux<T, Div>(ftype, fex, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, 0.0, g, dv);
            if (!code && (isnan(fex[0]) || isnan(fex[1]) || isnan(fex[2]))) code = 3;
            lam = rmax(lam, l2);
        }
    }
    return lam;
}

/* Element stage modes: the RHS alone; SSP-RK2 stages 1 and 2; SSP(3,3) stages 2 and 3
 * (its stage 1 is MODE_STAGE1). */
enum { MODE_RHS = 0, MODE_STAGE1 = 1, MODE_STAGE2 = 2, MODE_RK3_2 = 3, MODE_RK3_3 = 4 };

/* The stage combination w = cu*u + cs*(s + dt*rhs) as coefficients of (u, s, dt*rhs), used
 * by the reverse: RK2 stage 2 is (0.5, 0.5, 0.5). */
DGR_HD void stage_coefficients(int mode, double &cu, double &cs, double &cr)
{
    cu = 0.0;
    cs = 1.0;
    cr = 1.0;
    if (mode == MODE_STAGE2) { cu = 0.5; cs = 0.5; cr = 0.5; }
    else if (mode == MODE_RK3_2) { cu = 0.75; cs = 0.25; cr = 0.25; }
    else if (mode == MODE_RK3_3) { cu = 1.0 / 3; cs = 2.0 / 3; cr = 2.0 / 3; }
    else if (mode == MODE_RHS) { cs = 0.0; }
}

/*
 * One element: surface and volume integrals of 2DCode/2DInnerProducts.c:8-570, the
 * right-hand side of 2DCode/compute2DL.c:338-411 and the SSP-RK2 combination of
 * 2DCode/time_evolution.c:76-88 (stage 1: w = s + RHS*dt) or :176-217 (stage 2:
 * w = (s + u)*0.5 + RHS*(dt/2)); MODE_RHS returns the RHS.
 *   F[v][k]     Fhat.n of variable v on local edge k, outward for this element
 *   zr, qxr, qyr  stage input at the three edge midpoints
 *   geo(j)      state-independent geometry plane j (double)
 *   zg.midz(e), zg.gnn(e), zg.gradz(j)  the depth- and Manning-dependent factors (T)
 *   uin(v, k)   step input u^n (stage 2 only)
 * Returns w[3][3] and the element means avg[3].
 */
template <int MODE, class T, class Geo, class ZGeo, class UIn, bool RCP = false>
DGR_HD void element_core(const T F[3][3], const T zr[3], const T qxr[3], const T qyr[3], const Geo &geo,
                         const ZGeo &zg, const UIn &uin, double local_g, double rain, double dt, T w[3][3],
                         T avg[3], bool *rcp_ok = nullptr)
{
    const double nx[3] = {geo(G_NX), geo(G_NX + 1), geo(G_NX + 2)};
    const double ny[3] = {geo(G_NY), geo(G_NY + 1), geo(G_NY + 2)};
    const double M12 = geo(G_M12), M22 = geo(G_M12 + 1), M32 = geo(G_M12 + 2), dM = geo(G_DM);
    const double M11 = nx[0], M13 = ny[0], M21 = nx[1], M23 = ny[1], M31 = nx[2], M33 = ny[2];
    /* RCP (T = double): the eighteen divisions by dM of the six fits share one reciprocal
     * (div_rcp, the same bits); *rcp_ok is cleared where that is not valid, and the caller
     * then redoes the element with plain divisions */
    double y_dm = 0.0;
    bool ok = true;
    if constexpr (RCP) {
        y_dm = 1.0 / dM;
        ok = rcp_divisor_ok(dM);
    }
    const auto fit = [&](const T &R1, const T &R2, const T &R3, T &a, T &b, T &c) {
        if constexpr (RCP)
            rt0_fit_rcp(R1, R2, R3, M11, M12, M13, M21, M22, M23, M31, M32, M33, dM, y_dm, a, b, c, ok);
        else
            rt0_fit(R1, R2, R3, M11, M12, M13, M21, M22, M23, M31, M32, M33, dM, a, b, c);
    };

    /* surface integrals SI[9] (:95-239), edge by edge: the three fits first, then per edge
     * its two Gauss points and basis values, each variable's normal fluxes there and their
     * products, added to si in the reference's order (edge 0, 1, 2); every value is the
     * reference's expression, only evaluated in this order (fewer values live at once) */
    T si[9];
    {
        T fa[3], fb[3], fc[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) fit(F[v][0], F[v][1], F[v][2], fa[v], fb[v], fc[v]);
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            const double ej = geo(G_EJ + e);
            const double xq[2] = {geo(G_XE + 2 * e), geo(G_XE + 2 * e + 1)};
            const double yq[2] = {geo(G_YE + 2 * e), geo(G_YE + 2 * e + 1)};
            double ps[3][2];
#pragma unroll
            for (int bf = 0; bf < 3; ++bf) {
                ps[bf][0] = geo(G_PSI + 6 * bf + 2 * e);
                ps[bf][1] = geo(G_PSI + 6 * bf + 2 * e + 1);
            }
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                const T fd0 = (fa[v] + fb[v] * xq[0]) * nx[e] + (fc[v] + fb[v] * yq[0]) * ny[e];
                const T fd1 = (fa[v] + fb[v] * xq[1]) * nx[e] + (fc[v] + fb[v] * yq[1]) * ny[e];
#pragma unroll
                for (int bf = 0; bf < 3; ++bf) {
                    const T term = ej * (fd0 * ps[bf][0] + fd1 * ps[bf][1]);
                    si[3 * v + bf] = e == 0 ? term : si[3 * v + bf] + term;
                }
            }
        }
    }

    /* volume integrals VI[21] (:247-566) */
    T H[3], tau[3], R[3][3]; /* R[variable][edge] = volume flux . n */
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const T midz = zg.midz(e);
        H[e] = zr[e] + midz;
        /* the five divisions by H: plain, or (RCP) through one reciprocal of H */
        T yH = 0.0;
        if constexpr (RCP) {
            yH = 1.0 / H[e];
            ok = ok && rcp_divisor_ok(H[e]);
        }
        const auto byH = [&](const T &x) -> T {
            if constexpr (RCP)
                return div_rcp(x, H[e], yH, ok);
            else
                return x / H[e];
        };
        const T u = byH(qxr[e]);
        const T v = byH(qyr[e]);
        tau[e] = zg.gnn(e) * sqrt(u * u + v * v) / pow43(H[e]);
        const T pr = 0.5 * local_g * (H[e] * H[e] - midz * midz);
        const T qxy = byH(qxr[e] * qyr[e]);
        R[0][e] = qxr[e] * nx[e] + qyr[e] * ny[e];
        R[1][e] = (byH(qxr[e] * qxr[e]) + pr) * nx[e] + qxy * ny[e];
        R[2][e] = qxy * nx[e] + (byH(qyr[e] * qyr[e]) + pr) * ny[e];
    }
    const double aj = geo(G_AJ), ajw = geo(G_AJW);
    const double weight = 1.0 / 6;
    T dv[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        T a, b, c;
        fit(R[v][0], R[v][1], R[v][2], a, b, c);
#pragma unroll
        for (int bf = 0; bf < 3; ++bf)
            dv[v][bf] = aj * (0.5 * a * geo(G_GP + 2 * bf) + 0.5 * c * geo(G_GP + 2 * bf + 1) +
                              b * weight * geo(G_P + bf));
    }
    const T bedx = local_g * aj * zg.gradz(0) * weight;
    const T bedy = local_g * aj * zg.gradz(1) * weight;

    /* right-hand side (2DCode/compute2DL.c:344-409) */
    T X[3][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        X[0][j] = -si[j] + dv[0][j];
        X[1][j] = -si[3 + j] + dv[1][j] + bedx * zr[j] - ajw * tau[j] * qxr[j];
        X[2][j] = -si[6 + j] + dv[2][j] + bedy * zr[j] - ajw * tau[j] * qyr[j];
    }
    const double m11 = geo(G_M11);
    T rhs[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        rhs[v][0] = m11 * X[v][0] + 0.0 * X[v][1] + 0.0 * X[v][2];
        rhs[v][1] = 0.0 * X[v][0] + m11 * X[v][1] + 0.0 * X[v][2];
        rhs[v][2] = 0.0 * X[v][0] + 0.0 * X[v][1] + m11 * X[v][2];
    }
    if (rain != 0.0) { /* extension: rain on the elevation equation */
        rhs[0][0] += rain;
        rhs[0][1] += rain;
        rhs[0][2] += rain;
    }

    if constexpr (RCP) *rcp_ok = ok;
    if (MODE == MODE_RHS) {
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int k = 0; k < 3; ++k) w[v][k] = rhs[v][k];
        return;
    }
    const T s[3][3] = {{zr[0], zr[1], zr[2]}, {qxr[0], qxr[1], qxr[2]}, {qyr[0], qyr[1], qyr[2]}};
    if (MODE == MODE_STAGE1) {
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int k = 0; k < 3; ++k) w[v][k] = s[v][k] + rhs[v][k] * dt;
    } else if (MODE == MODE_STAGE2) {
        const double hdt = dt / 2;
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int k = 0; k < 3; ++k) w[v][k] = (s[v][k] + uin(v, k)) * 0.5 + rhs[v][k] * hdt;
    } else { /* SSP(3,3): u_i = a u^n + b (u_{i-1} + dt L(u_{i-1})), prep_DG.F:1253-1270 */
        const double a = MODE == MODE_RK3_2 ? 0.75 : 1.0 / 3;
        const double b = MODE == MODE_RK3_2 ? 0.25 : 2.0 / 3;
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int k = 0; k < 3; ++k) w[v][k] = a * uin(v, k) + b * (s[v][k] + rhs[v][k] * dt);
    }
    if constexpr (RCP) { /* the means' divisions by 3 through the reciprocal RN(1/3) */
        bool ok_avg = true;
#pragma unroll
        for (int v = 0; v < 3; ++v) avg[v] = div_rcp(w[v][0] + w[v][1] + w[v][2], 3.0, 1.0 / 3, ok_avg);
        *rcp_ok = ok && ok_avg;
    } else {
#pragma unroll
        for (int v = 0; v < 3; ++v) avg[v] = (w[v][0] + w[v][1] + w[v][2]) / 3;
    }
}

/* Decisions of one element's limiter and PDop pass (recorded for the adjoint tests). */
struct LimitDecisions {
    int modify;      /* the limited values replaced the element's (SlopeLimiter2D.c:189-200, 307-311) */
    int mass_branch; /* PDop mass: 0 none, 1 all to the mean, 2 min/next/rest (wetDry2D.c:93-156) */
    int mom_branch;  /* PDop momentum: 0 none, 1 all dry, 2 partly dry (:170-253) */
    int code;        /* 4: NaN depth, 5: NaN velocity */
};

/* The limiter's path for one variable, recorded for the adjoint (48 bits): clamp of
 * vertex k in bits 2k..2k+1 (0 none, 1 to the node max, 2 to the node min); sign of the
 * redistribution pass ll plus one in bits 6+2ll..; per pass ll and vertex k four bits at
 * 12 + 4(3ll+k): bit 0 diff > 0, bit 1 the cap redmax taken, bits 2-3 the divisor. */
struct LimitTrace {
    unsigned long long bits[3];
};

/*
 * One element: vertex-based limiter (2DCode/SlopeLimiter2D.c:157-343), then the
 * positive-depth operator (2DCode/wetDry2D.c:63-260), in place on w[variable][midpoint].
 * bnd(v, k, is_min) is the node max (is_min = 0) or min (1) of variable v's element means
 * at the element's vertex k; zn are the vertex depths.  With TRACE the limiter's path is
 * recorded in *trace (values are unaffected).
 */
template <bool LIMIT, bool PDOP, class T, class Bnd, bool TRACE = false, class Div = PlainDiv>
DGR_HD void limit_core(T w[3][3], const Bnd &bnd, const T zn[3], double h0, double velzero, LimitDecisions &dec,
                       LimitTrace *trace = nullptr, Div *dv = nullptr)
{
    /* divisions by 3 and by the vertex depths: plain, or (Div = RcpDiv) through shared
     * reciprocals (div_rcp, the same bits; dv->ok reports where that is not valid) */
    constexpr bool rcp = std::is_same<Div, RcpDiv>::value;
    const auto div3 = [&](const T &x) -> T {
        if constexpr (rcp)
            return dv->div(x, RcpDiv::By{3.0, 1.0 / 3});
        else
            return x / 3;
    };
    dec.modify = 0;
    dec.mass_branch = 0;
    dec.mom_branch = 0;
    dec.code = 0;
    if (LIMIT) {
        int modify = 0;
        T out[3][3];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const T w1 = w[v][0], w2 = w[v][1], w3 = w[v][2];
            T vx[3] = {w1 - w2 + w3, w1 + w2 - w3, -w1 + w2 + w3};
            T vmax[3], vmin[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                vmax[k] = bnd(v, k, 0);
                vmin[k] = bnd(v, k, 1);
            }
            const T avg = div3(w1 + w2 + w3);
            if (v == 0) { /* :189-200 */
                const T h1 = vx[0] + zn[0], h2 = vx[1] + zn[1], h3 = vx[2] + zn[2];
                const T m0 = vmin[0] + zn[0], m1 = vmin[1] + zn[1], m2 = vmin[2] + zn[2];
                if (h1 > h0 && h2 > h0 && h3 > h0 && m0 > h0 && m1 > h0 && m2 > h0) modify = 1;
            }
            unsigned long long tb = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (TRACE) {
                    const T r1 = rmin(vx[k], vmax[k]);
                    unsigned long long c = (vx[k] < vmax[k]) ? 0 : 1;
                    if (fmax_takes_b(val(r1), val(vmin[k]))) c = 2;
                    tb |= c << (2 * k);
                }
                vx[k] = fmax_b(rmin(vx[k], vmax[k]), vmin[k]);
            }
            /* the three passes stay a loop: unrolled, the 27 copies of the pass body overflow
             * the instruction cache (measured: 8 % off the limiter kernel rolled) */
#pragma unroll 1
            for (int ll = 0; ll < 3; ++ll) { /* :254-299 */
                const T sumloc = div3(vx[0] + vx[1] + vx[2]);
                T sumdiff = (sumloc - avg) * 3;
                const int sd = sgn(sumdiff);
                const double sdd = (double)sd;
                if (TRACE) tb |= (unsigned long long)(sd + 1) << (6 + 2 * ll);
                const T diff[3] = {(vx[0] - avg) * sdd, (vx[1] - avg) * sdd, (vx[2] - avg) * sdd};
                double kdp = (double)((diff[0] > 0) + (diff[1] > 0) + (diff[2] > 0));
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double div = fmax(1.0, kdp);
                    T redfac;
                    if (diff[k] > 0) {
                        if constexpr (rcp) {
                            const T x = sumdiff * sdd;
                            redfac = div == 1.0 ? x : (div == 2.0 ? x * 0.5 : div3(x));
                        } else {
                            redfac = div_by_count(T(sumdiff * sdd), div);
                        }
                        kdp -= 1;
                    } else {
                        redfac = 0;
                    }
                    const T redmax = (sd > 0) ? vx[k] - vmin[k] : vmax[k] - vx[k];
                    if (TRACE)
                        tb |= (unsigned long long)((diff[k] > 0 ? 1 : 0) | (redfac < redmax ? 0 : 2) |
                                                   ((int)div << 2))
                              << (12 + 4 * (3 * ll + k));
                    redfac = rmin(redfac, redmax);
                    sumdiff -= redfac * sdd;
                    vx[k] -= redfac * sdd;
                }
            }
            if (TRACE) trace->bits[v] = tb;
            out[v][0] = (vx[0] + vx[1]) / 2;
            out[v][1] = (vx[1] + vx[2]) / 2;
            out[v][2] = (vx[2] + vx[0]) / 2;
            if (v == 0) { /* :307-311 */
                const T h1 = vx[0] + zn[0], h2 = vx[1] + zn[1], h3 = vx[2] + zn[2];
                if (h1 < h0 || h2 < h0 || h3 < h0) modify = 0;
            }
        }
        if (modify) {
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int k = 0; k < 3; ++k) w[v][k] = out[v][k];
        }
        dec.modify = modify;
    }

    if (PDOP) {
        const T midz0 = 0.5 * (zn[0] + zn[1]), midz1 = 0.5 * (zn[1] + zn[2]), midz2 = 0.5 * (zn[2] + zn[0]);
        T mh0 = w[0][0] + midz0, mh1 = w[0][1] + midz1, mh2 = w[0][2] + midz2;
        T ht[3] = {mh0 - mh1 + mh2, mh0 + mh1 - mh2, -mh0 + mh1 + mh2};
        const T avg_h = div3(ht[0] + ht[1] + ht[2]);
        int code = 0;
        if (ht[0] <= h0 || ht[1] <= h0 || ht[2] <= h0) { /* :93-156 */
            if (avg_h <= h0) {
                dec.mass_branch = 1;
                ht[0] = avg_h;
                ht[1] = avg_h;
                ht[2] = avg_h;
            } else {
                dec.mass_branch = 2;
                int imin = 0;
                T hmin = ht[0];
                if (ht[1] < hmin) { imin = 1; hmin = ht[1]; }
                if (ht[2] < hmin) { imin = 2; hmin = ht[2]; }
                int inext = 1; /* the reference starts this search at index 1 (:115-124) */
                T hnext = ht[1];
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (ht[i] < hnext && i != imin) { inext = i; hnext = ht[i]; }
                int irem = 2;
                if (0 != imin && 0 != inext) irem = 0;
                else if (1 != imin && 1 != inext) irem = 1;
                T hh[3] = {ht[0], ht[1], ht[2]};
                hh[imin] = h0;
                hh[inext] = fmax(h0, hnext - 0.5 * (hh[imin] - hmin));
                hh[irem] = hh[irem] - (hh[imin] - hmin) - (hh[inext] - hnext);
                ht[0] = hh[0];
                ht[1] = hh[1];
                ht[2] = hh[2];
            }
            if (isnan(ht[0]) || isnan(ht[1]) || isnan(ht[2])) code = 4;
            mh0 = 0.5 * (ht[0] + ht[1]);
            mh1 = 0.5 * (ht[1] + ht[2]);
            mh2 = 0.5 * (ht[2] + ht[0]);
            w[0][0] = mh0 - midz0;
            w[0][1] = mh1 - midz1;
            w[0][2] = mh2 - midz2;
        }
        const int wet[3] = {ht[0] > h0, ht[1] > h0, ht[2] > h0};
        if (!code) {
            if (wet[0] == 0 && wet[1] == 0 && wet[2] == 0) { /* :170-178 */
                dec.mom_branch = 1;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    w[1][i] = 0;
                    w[2][i] = 0;
                }
            } else if (wet[0] == 0 || wet[1] == 0 || wet[2] == 0) { /* :180-253 */
                dec.mom_branch = 2;
                const T q0 = w[1][0], q1 = w[1][1], q2 = w[1][2];
                const T r0 = w[2][0], r1 = w[2][1], r2 = w[2][2];
                T qxe[3] = {q0 - q1 + q2, q0 + q1 - q2, -q0 + q1 + q2};
                T qye[3] = {r0 - r1 + r2, r0 + r1 - r2, -r0 + r1 + r2};
                T u[3], vv[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    if constexpr (rcp) {
                        const auto by_h = dv->by(ht[i]);
                        u[i] = dv->div(qxe[i], by_h);
                        vv[i] = dv->div(qye[i], by_h);
                    } else {
                        u[i] = qxe[i] / ht[i];
                        vv[i] = qye[i] / ht[i];
                    }
                }
                int npos = 0;
                T delu = 0, delv = 0;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    npos += wet[i];
                    delu += u[i] * (double)(1 - wet[i]) * (double)(fabs(qxe[i]) > velzero);
                    delv += vv[i] * (double)(1 - wet[i]) * (double)(fabs(qye[i]) > velzero);
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    u[i] = (double)wet[i] * (u[i] + delu / (double)npos);
                    vv[i] = (double)wet[i] * (vv[i] + delv / (double)npos);
                    if (!code && (isnan(u[i]) || isnan(vv[i]))) code = 5;
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    qxe[i] = ht[i] * u[i];
                    qye[i] = ht[i] * vv[i];
                }
                w[1][0] = 0.5 * (qxe[0] + qxe[1]);
                w[1][1] = 0.5 * (qxe[1] + qxe[2]);
                w[1][2] = 0.5 * (qxe[2] + qxe[0]);
                w[2][0] = 0.5 * (qye[0] + qye[1]);
                w[2][1] = 0.5 * (qye[1] + qye[2]);
                w[2][2] = 0.5 * (qye[2] + qye[0]);
            }
        }
        dec.code = code;
    }
}

/* BigTheta, 2DCode/wetDry2D.c:7-14 */
DGR_HD int big_theta(double a) { return a > 0 ? 1 : 0; }

/* wetDryStatus2D for one element (2DCode/wetDry2D.c:18-57). */
DGR_HD int wd_status(const double mz[3], const double zn[3], int wd_prev, double h0, RcpDiv *dv = nullptr)
{
    const double zv[3] = {mz[0] - mz[1] + mz[2], mz[0] + mz[1] - mz[2], -mz[0] + mz[1] + mz[2]};
    const double h[3] = {zv[0] + zn[0], zv[1] + zn[1], zv[2] + zn[2]};
    const double avg_h = dv ? dv->div(h[0] + h[1] + h[2], RcpDiv::By{3.0, 1.0 / 3}) : (h[0] + h[1] + h[2]) / 3;
    int imax = 0;
    double hmax = h[0];
    if (h[1] > hmax) { imax = 1; hmax = h[1]; }
    if (h[2] > hmax) { imax = 2; hmax = h[2]; }
    const double zeta_max = zv[imax];
    double zmin = zn[0];
    if (zn[1] < zmin) zmin = zn[1];
    if (zn[2] < zmin) zmin = zn[2];
    if (wd_prev == -1) return big_theta(avg_h - h0) * big_theta(zeta_max - (h0 - zmin));
    return wd_prev * big_theta(avg_h - h0) + (1 - wd_prev) * big_theta(avg_h - h0) * big_theta(zeta_max - (h0 - zmin));
}

}  // namespace dgr
