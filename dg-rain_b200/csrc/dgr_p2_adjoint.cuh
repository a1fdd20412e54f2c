/*
 * Tangent-linear (two-lane) and adjoint (hand-written reverse) kernels of the p = 2 modal
 * step of dgr_p2.cuh.
 *
 * Parameters of the derivatives, as for p = 1: the state, the node depths z (enter the
 * vertex depths of each element, hence its linear depth and depth gradient, and the depth
 * at every edge Gauss point) and the per-element Manning n (g n^2).
 *
 * Adjoint work arrays (p = 2):
 *   fbar [18][ldF]  per edge and side, per Gauss point (edge orientation) and variable:
 *                   first the adjoint of the stored flux, written by the one element that
 *                   gathers it; then, in place, the adjoint of the side's trace values,
 *                   written by the edge's own thread (plane 9 side + 3 gp + v)
 *   zvb  [3][ldE]   depth adjoint per element vertex slot
 *   zeb  [2][ldF]   depth adjoint of each edge's two end vertices (those of its "in" element)
 * No atomics: every slot has one writer per launch, so gradients are bitwise reproducible.
 */
#pragma once

#include "dgr_p2.cuh"
#include "dgr_tlm.cuh"

/* minimum resident blocks per SM of the p = 2 reverse kernels (128 registers at 128
 * threads; the measured sweep made the backward sweep 19 % faster than uncapped) */
#ifndef DGR_P2_MINB_ADJ_ELEMENT
#define DGR_P2_MINB_ADJ_ELEMENT 4
#endif
#ifndef DGR_P2_MINB_ADJ_EDGE
#define DGR_P2_MINB_ADJ_EDGE 4
#endif

namespace dgr {

/* ==================================================================== tangent ==== */

/* depth-dependent element planes in two-lane arithmetic: values from the geometry planes,
 * second lanes from the vertex-depth lanes zvx and the element-n lane by the set-up's
 * expressions (k_p2_setup) */
template <class T>
struct P2LaneZ {
    T z[3], gx, gy, gn;
    DGR_HD T zv(int k) const { return z[k]; }
    DGR_HD T dzx() const { return gx; }
    DGR_HD T dzy() const { return gy; }
    DGR_HD T gnn() const { return gn; }
};

template <class T>
DGR_HD P2LaneZ<T> p2_lane_z(const double *G, int ld, const double zvx[3], double nel, double nelx, double g)
{
    const T *tag = nullptr;
    P2LaneZ<T> z;
#pragma unroll
    for (int k = 0; k < 3; ++k) z.z[k] = lane(tag, G[(size_t)(P2G_ZV + k) * ld], zvx[k]);
    const double zr = (zvx[1] - zvx[0]) / 2, zs = (zvx[2] - zvx[0]) / 2;
    z.gx = lane(tag, G[(size_t)P2G_DZX * ld], zr * G[(size_t)P2G_RX * ld] + zs * G[(size_t)P2G_SX * ld]);
    z.gy = lane(tag, G[(size_t)P2G_DZY * ld], zr * G[(size_t)P2G_RY * ld] + zs * G[(size_t)P2G_SY * ld]);
    const double gnn = G[(size_t)P2G_GNN * ld];
    z.gn = nel >= 0.0 ? gnn_lane(tag, gnn, g, nel, nelx) : T(gnn);
    return z;
}

/* Tangent (T = Dual) or frozen-decision perturbation (T = Pert) of the p = 2 edge fluxes;
 * the "_x" arrays hold the second lanes. */
template <class T>
__global__ void __launch_bounds__(128) k_p2_tlm_edge(P2Ref ref, MeshDev m, const double *__restrict__ p2g,
                                                     const double *__restrict__ S, const double *__restrict__ Sx,
                                                     const double *__restrict__ bzeta,
                                                     const double *__restrict__ bqn, const double *__restrict__ zx,
                                                     double *__restrict__ flux, double *__restrict__ flux_x, double g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nf) return;
    const T *tag = nullptr;
    const int el_in = m.e_in[i], el_ex = m.e_ex[i], info = m.e_info[i];
    const int k_in = info & 3, bd = (info >> 4) & 7;
    const double nx = m.e_geo[i], ny = m.e_geo[m.ldF + i];
    const int ld = m.ldE;
    int va, vb;
    edge_vertices(m, el_in, k_in, va, vb);
    const T za = lane(tag, p2g[(size_t)(P2G_ZV + k_in) * ld + el_in], zx[va]);
    const T zb = lane(tag, p2g[(size_t)(P2G_ZV + (k_in + 1) % 3) * ld + el_in], zx[vb]);
    const auto st = [S, Sx, ld, tag](int plane, int el) { return lane(tag, S[plane * ld + el], Sx[plane * ld + el]); };
    T fh[P2_NGP][3];
    int code;
    p2_edge_core<T>(ref, st, el_in, el_ex, info, nx, ny, za, zb, bd ? bzeta[i] : 0.0, bd ? bqn[i] : 0.0, g, fh, code,
                    m.flux);
    const int lf = m.ldF;
#pragma unroll
    for (int gp = 0; gp < P2_NGP; ++gp)
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            flux[(3 * gp + v) * lf + i] = val(fh[gp][v]);
            flux_x[(3 * gp + v) * lf + i] = second(fh[gp][v]);
        }
}

template <int MODE, class T>
__global__ void __launch_bounds__(128) k_p2_tlm_element(P2Ref ref, MeshDev m, const double *__restrict__ p2g,
                                                        const double *__restrict__ S, const double *__restrict__ Sx,
                                                        const double *U, const double *Ux,
                                                        const double *__restrict__ flux,
                                                        const double *__restrict__ flux_x,
                                                        const double *__restrict__ zx,
                                                        const double *__restrict__ n_el,
                                                        const double *__restrict__ nelx, double *out, double *out_x,
                                                        const DevClock *clk, double g,
                                                        const double *__restrict__ dt_n)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const T *tag = nullptr;
    const int ld = m.ldE;
    const int sid = m.el_sid ? m.el_sid[el] : 0;
    T s[3][P2_NM];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < P2_NM; ++k) s[v][k] = lane(tag, S[(P2_NM * v + k) * ld + el], Sx[(P2_NM * v + k) * ld + el]);
    T F[3][P2_NGP][3];
    const int lf = m.ldF;
    p2_gather_flux<T>(m, el, [flux, flux_x, lf, tag](int plane, int e) {
        return lane(tag, flux[plane * lf + e], flux_x[plane * lf + e]);
    }, F);
    const double *G = p2g + el;
    const auto geo = [G, ld](int j) { return G[(size_t)j * ld]; };
    const double zvx[3] = {zx[m.el2v[el]], zx[m.el2v[ld + el]], zx[m.el2v[2 * ld + el]]};
    const P2LaneZ<T> zg = p2_lane_z<T>(G, ld, zvx, n_el ? n_el[el] : -1.0, nelx ? nelx[el] : 0.0, g);
    const auto uin = [U, Ux, ld, el, tag](int v, int k) {
        return lane(tag, U[(P2_NM * v + k) * ld + el], Ux[(P2_NM * v + k) * ld + el]);
    };
    T w[3][P2_NM];
    p2_element_core<MODE, T>(ref, s, F, geo, zg, uin, g, clk[sid].rain, dt_n[sid], w);
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < P2_NM; ++k) {
            out[(P2_NM * v + k) * ld + el] = val(w[v][k]);
            out_x[(P2_NM * v + k) * ld + el] = second(w[v][k]);
        }
}

/* ==================================================================== reverse ==== */

/*
 * Reverse of the area integrals of p2_element_core for one element.
 *   S      stage input (values); Xb: adjoint of the accumulated integrals acc[v][m]
 *   Sb     accumulates the stage input's adjoint; zvb, dzb[2], gnnb: the depth-dependent
 *          planes' adjoints
 * Forward values are recomputed by the forward's expressions; the kink of the friction
 * speed |u| at 0 takes derivative 0 (as ad::Dual's sqrt).
 */
DGR_HD void p2_area_rev(const P2Ref &ref, const double S[3][P2_NM], const double Xb[3][P2_NM], double rx, double ry,
                        double sx, double sy, double detJ, const double zv[3], double dzx, double dzy, double gnn,
                        double g, double Sb[3][P2_NM], double zvb[3], double dzb[2], double &gnnb)
{
    /* a loop, as the forward's area loop (instruction cache) */
#pragma unroll 1
    for (int q = 0; q < P2_NQ; ++q) {
        double uq[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            double a = 0.0;
#pragma unroll
            for (int m = 0; m < P2_NM; ++m) a += ref.phi[q][m] * S[v][m];
            uq[v] = a;
        }
        const double zq = ref.lam[q][0] * zv[0] + ref.lam[q][1] * zv[1] + ref.lam[q][2] * zv[2];
        const double H = uq[0] + zq;
        /* these quotients only scale derivatives (no decision depends on them): products
         * with one reciprocal per divisor, whose last bit does not matter */
        const double iH = 1.0 / H;
        const double u = uq[1] * iH, vv = uq[2] * iH;
        const double sp = sqrt(u * u + vv * vv);
        const double iP = 1.0 / pow43(H);
        const double tau = gnn * sp * iP;
        const double wj = 2.0 * ref.wq[q] * detJ;
        /* adjoints of fx, fy, src */
        double fxb[3] = {0, 0, 0}, fyb[3] = {0, 0, 0}, srcb[3] = {0, 0, 0};
#pragma unroll
        for (int m = 0; m < P2_NM; ++m) {
            const double gx = ref.dr[q][m] * rx + ref.ds[q][m] * sx;
            const double gy = ref.dr[q][m] * ry + ref.ds[q][m] * sy;
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                const double a = wj * Xb[v][m];
                fxb[v] += a * gx;
                fyb[v] += a * gy;
                srcb[v] += a * ref.phi[q][m];
            }
        }
        double q1b = 0, q2b = 0, zb = 0, ub = 0, vb = 0, Hb = 0, zqb = 0;
        /* fx = (q1, q1 u + p, q1 vv), fy = (q2, q1 vv, q2 vv + p) */
        q1b += fxb[0];
        q2b += fyb[0];
        q1b += fxb[1] * u;
        ub += fxb[1] * uq[1];
        const double pb = fxb[1] + fyb[2];
        const double qxyb = fxb[2] + fyb[1];
        q2b += fyb[2] * vv;
        vb += fyb[2] * uq[2];
        q1b += qxyb * vv;
        vb += qxyb * uq[1];
        /* src = (rain, g zeta dzx - tau q1, g zeta dzy - tau q2) */
        zb += g * dzx * srcb[1] + g * dzy * srcb[2];
        dzb[0] += g * uq[0] * srcb[1];
        dzb[1] += g * uq[0] * srcb[2];
        const double taub = -(srcb[1] * uq[1] + srcb[2] * uq[2]);
        q1b -= tau * srcb[1];
        q2b -= tau * srcb[2];
        /* tau = gnn sp / H^(4/3) */
        gnnb += taub * sp * iP;
        Hb -= taub * tau * (4.0 / 3.0) * iH;
        if (sp != 0.0) {
            const double spb = taub * gnn * iP;
            const double isp = 1.0 / sp;
            ub += spb * u * isp;
            vb += spb * vv * isp;
        }
        /* p = g (H^2 - zq^2) / 2 */
        Hb += pb * g * H;
        zqb -= pb * g * zq;
        /* u = q1 / H, vv = q2 / H */
        q1b += ub * iH;
        q2b += vb * iH;
        Hb -= (ub * u + vb * vv) * iH;
        zb += Hb;
        zqb += Hb;
#pragma unroll
        for (int k = 0; k < 3; ++k) zvb[k] += ref.lam[q][k] * zqb;
        const double uqb[3] = {zb, q1b, q2b};
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int m = 0; m < P2_NM; ++m) Sb[v][m] += ref.phi[q][m] * uqb[v];
    }
}

/* depth gradient of the linear depth to the vertex depths (transpose of k_p2_setup's) */
DGR_HD void p2_dz_rev(double rx, double ry, double sx, double sy, const double dzb[2], double zvb[3])
{
    const double zrb = dzb[0] * rx + dzb[1] * ry, zsb = dzb[0] * sx + dzb[1] * sy;
    zvb[1] += zrb / 2;
    zvb[2] += zsb / 2;
    zvb[0] -= zrb / 2 + zsb / 2;
}

/*
 * Element reverse of one stage: lamO = adjoint of the stage output.  Writes
 *   lamS   the stage input's adjoint: added for stage 1 (lamS is lamU there), else set;
 *   lamU   cu * lamO into the step input's adjoint (set, or added with u_accumulate);
 *   fbar   the adjoints of the element's gathered edge fluxes, per edge side, in the edge's
 *          Gauss point order;
 * and accumulates the depth (zvb) and Manning (nbar) adjoints.  lamO may be lamU (last
 * stage): every element reads its own columns before writing them.
 */
template <int MODE>
__global__ void __launch_bounds__(128, DGR_P2_MINB_ADJ_ELEMENT) k_p2_adj_element(P2Ref ref, MeshDev m, const double *__restrict__ p2g,
                                                        const double *__restrict__ S, const double *lamO, double *lamS,
                                                        double *lamU, int u_accumulate, double *__restrict__ fbar,
                                                        double *__restrict__ zvb, double *__restrict__ nbar,
                                                        const double *__restrict__ n_el, double g,
                                                        const double *__restrict__ dt_n)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE;
    const double *G = p2g + el;
    const double detJ = G[0], rx = G[(size_t)P2G_RX * ld], ry = G[(size_t)P2G_RY * ld];
    const double sx = G[(size_t)P2G_SX * ld], sy = G[(size_t)P2G_SY * ld];
    double cu, cs, cr;
    stage_coefficients(MODE, cu, cs, cr);
    const double rk = MODE == MODE_RHS ? 1.0 : cr * dt_n[m.el_sid ? m.el_sid[el] : 0];
    double wb[3][P2_NM], Xb[3][P2_NM];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < P2_NM; ++k) wb[v][k] = lamO[(P2_NM * v + k) * ld + el];
#pragma unroll
    for (int k = 0; k < P2_NM; ++k) {
        const double minv = 1.0 / (detJ * ref.mass[k]);
#pragma unroll
        for (int v = 0; v < 3; ++v) Xb[v][k] = (wb[v][k] * rk) * minv;
    }
    /* edge integrals: acc[v][m] -= wl F[k][gp][v] phie[k][gp][m] */
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double half = G[(size_t)(P2G_LEN + k) * ld] / 2;
        const int ee = m.elem_edge[k * ld + el];
        const int e = ee >> 1, side = ee & 1;
        const int info = side ? m.e_info[e] : 0;
#pragma unroll
        for (int gp = 0; gp < P2_NGP; ++gp) {
            const double wl = ref.wg[gp] * half;
            const int gi = side ? p2_match_point(info, gp) : gp;
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                double a = 0.0;
#pragma unroll
                for (int mm = 0; mm < P2_NM; ++mm) a += Xb[v][mm] * ref.phie[k][gp][mm];
                const double fb = -wl * a;
                fbar[(9 * side + 3 * gi + v) * m.ldF + e] = side ? -fb : fb;
            }
        }
    }
    /* area integrals */
    double s[3][P2_NM], Sb[3][P2_NM];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < P2_NM; ++k) {
            s[v][k] = S[(P2_NM * v + k) * ld + el];
            Sb[v][k] = cs * wb[v][k];
        }
    const double zv[3] = {G[(size_t)P2G_ZV * ld], G[(size_t)(P2G_ZV + 1) * ld], G[(size_t)(P2G_ZV + 2) * ld]};
    const double gnn = G[(size_t)P2G_GNN * ld];
    double zvbl[3] = {0, 0, 0}, dzb[2] = {0, 0}, gnnb = 0;
    p2_area_rev(ref, s, Xb, rx, ry, sx, sy, detJ, zv, G[(size_t)P2G_DZX * ld], G[(size_t)P2G_DZY * ld], gnn, g, Sb,
                zvbl, dzb, gnnb);
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < P2_NM; ++k) {
            const int idx = (P2_NM * v + k) * ld + el;
            if (MODE == MODE_STAGE1) {
                lamS[idx] += Sb[v][k];
            } else {
                lamS[idx] = Sb[v][k];
                lamU[idx] = (u_accumulate ? lamU[idx] : 0.0) + cu * wb[v][k];
            }
        }
    p2_dz_rev(rx, ry, sx, sy, dzb, zvbl);
#pragma unroll
    for (int k = 0; k < 3; ++k) zvb[k * ld + el] += zvbl[k];
    if (n_el && n_el[el] >= 0.0) nbar[el] += gnnb * 2.0 * g * n_el[el];
}

/*
 * Edge reverse: the flux adjoints of both sides (fbar, edge point order) through the Roe
 * flux and the ghost states at each Gauss point; the trace adjoints of each side replace
 * the flux adjoints in fbar, and the adjoints of the Gauss-point depths go to the edge's
 * end vertices (zeb).
 */
template <int FT = -1>
__global__ void __launch_bounds__(128, DGR_P2_MINB_ADJ_EDGE) k_p2_adj_edge(P2Ref ref, MeshDev m, const double *__restrict__ p2g,
                                                            const double *__restrict__ S,
                                                            const double *__restrict__ bzeta,
                                                            const double *__restrict__ bqn, double *__restrict__ fbar,
                                                            double *__restrict__ zeb, double g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nf) return;
    const int el_in = m.e_in[i], el_ex = m.e_ex[i], info = m.e_info[i];
    const int k_in = info & 3, k_ex = (info >> 2) & 3, bd = (info >> 4) & 7;
    const bool boundary = bd || el_in == el_ex;
    const double nx = m.e_geo[i], ny = m.e_geo[m.ldF + i];
    const int ld = m.ldE, lf = m.ldF;
    const double za = p2g[(size_t)(P2G_ZV + k_in) * ld + el_in];
    const double zb = p2g[(size_t)(P2G_ZV + (k_in + 1) % 3) * ld + el_in];
    const double bz = bd ? bzeta[i] : 0.0, bq = bd ? bqn[i] : 0.0;
    double zab = 0, zbb = 0;
    /* a loop (instruction cache; nothing here is indexed by the point but the tables and
     * the global adjoints): 1.7 % off the calibration backward */
#pragma unroll 1
    for (int gp = 0; gp < P2_NGP; ++gp) {
        const double t = ref.te[gp];
        const double z_g = za * ((1.0 - t) / 2) + zb * ((1.0 + t) / 2);
        double ui[3], ue[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            double a = 0.0;
#pragma unroll
            for (int mm = 0; mm < P2_NM; ++mm) a += ref.phie[k_in][gp][mm] * S[(P2_NM * v + mm) * ld + el_in];
            ui[v] = a;
        }
        const int ge = p2_match_point(info, gp);
        if (boundary) {
            ghost_state<double>(bd, nx, ny, ui[0], ui[1], ui[2], bz, bq, ui[0], ue[0], ue[1], ue[2]);
        } else {
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                double a = 0.0;
#pragma unroll
                for (int mm = 0; mm < P2_NM; ++mm) a += ref.phie[k_ex][ge][mm] * S[(P2_NM * v + mm) * ld + el_ex];
                ue[v] = a;
            }
        }
        double fhb[3];
#pragma unroll
        for (int v = 0; v < 3; ++v)
            fhb[v] = fbar[(3 * gp + v) * lf + i] + (boundary ? 0.0 : fbar[(9 + 3 * gp + v) * lf + i]);
        RoeBar b = {0, 0, 0, 0, 0, 0, 0};
        numerical_flux_rev(FT >= 0 ? FT : m.flux, fhb, ui[0], ue[0], ui[1], ue[1], ui[2], ue[2], z_g, nx, ny, g, g, b);
        if (boundary) ghost_state_rev(bd, nx, ny, bz, bq, b.zex, b.qxex, b.qyex, b.zin, b.qxin, b.qyin);
        fbar[(3 * gp) * lf + i] = b.zin;
        fbar[(3 * gp + 1) * lf + i] = b.qxin;
        fbar[(3 * gp + 2) * lf + i] = b.qyin;
        if (!boundary) {
            fbar[(9 + 3 * gp) * lf + i] = b.zex;
            fbar[(9 + 3 * gp + 1) * lf + i] = b.qxex;
            fbar[(9 + 3 * gp + 2) * lf + i] = b.qyex;
        }
        zab += b.zed * ((1.0 - t) / 2);
        zbb += b.zed * ((1.0 + t) / 2);
    }
    zeb[i] += zab;
    zeb[lf + i] += zbb;
}

/* trace adjoints (fbar after k_p2_adj_edge) of an element's three edges to its modes */
static __global__ void __launch_bounds__(128) k_p2_adj_trace(P2Ref ref, MeshDev m, const double *__restrict__ fbar,
                                                             double *__restrict__ lamS)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE;
    double a[3][P2_NM];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < P2_NM; ++k) a[v][k] = lamS[(P2_NM * v + k) * ld + el];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * ld + el];
        const int e = ee >> 1, side = ee & 1;
        const int info = side ? m.e_info[e] : 0;
#pragma unroll
        for (int gp = 0; gp < P2_NGP; ++gp) {
            const int gi = side ? p2_match_point(info, gp) : gp;
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                const double t = fbar[(9 * side + 3 * gi + v) * m.ldF + e];
#pragma unroll
                for (int mm = 0; mm < P2_NM; ++mm) a[v][mm] += ref.phie[k][gp][mm] * t;
            }
        }
    }
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < P2_NM; ++k) lamS[(P2_NM * v + k) * ld + el] = a[v][k];
}

/* edge end-vertex depth adjoints to the vertex slots of each edge's "in" element */
static __global__ void __launch_bounds__(256) k_p2_adj_zfold(MeshDev m, const double *__restrict__ zeb,
                                                             double *__restrict__ zvb)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * ld + el];
        if (ee & 1) continue;
        zvb[k * ld + el] += zeb[ee >> 1];
        zvb[((k + 1) % 3) * ld + el] += zeb[m.ldF + (ee >> 1)];
    }
}

}  // namespace dgr
