/*
 * p = 2 modal discontinuous Galerkin step (extension; 2DCode has p = 1 only).
 *
 * The basis is DG-SWEM's orthogonal (Dubiner) basis on the reference triangle with
 * vertices (-1,-1), (1,-1), (-1,1) (src/orthobasis_area.F:18-175): with the collapsed
 * coordinate a = 2(1+r)/(1-s) - 1,
 *     phi_ij(r, s) = P_i^(0,0)(a) ((1-s)/2)^i P_j^(2i+1,0)(s),
 * in its hierarchical order (0,0), (0,1), (1,0), (0,2), (1,1), (2,0).  For p = 2 these are,
 * in closed form with A = r + (1+s)/2 = a (1-s)/2 and B = (1-s)/2,
 *     1, (3s+1)/2, A, (5s^2+2s-1)/2, A (5s+3)/2, (3A^2 - B^2)/2.
 * The mass matrix is diagonal.  Each variable (zeta, Qx, Qy) has 6 coefficients per
 * element: state planes 6v + m.
 *
 * Weak form per element T and mode m (the 2DCode equations: H = zeta + z with z the depth,
 * pressure g (H^2 - z^2)/2, bed term g zeta grad z, Manning friction -tau Q):
 *     M_mm dU_m/dt = int_T F(U) . grad phi_m + int_T S(U) phi_m - int_dT Fhat.n phi_m.
 * Area integrals: the 7-point degree-5 rule (Radon); edge integrals: 3-point Gauss; the
 * numerical flux is the Roe flux of 2DCode (roe_flux) at each edge Gauss point.  The depth
 * is linear per element (the node depths), which keeps a lake at rest exactly at rest.
 * No limiter and no wet/dry treatment: the p = 2 step is for flows that stay wet.
 */
#pragma once

#include "dgr_kernels.cuh"

namespace dgr {

/* Minimum resident blocks per SM requested for the p = 2 kernels (register caps 65536 /
 * (block size x blocks): 128 for the element kernel, 102 for the edge kernel at 128
 * threads).  Chosen by a measured sweep (1.3 M triangles, SSP(3,3): 14 % faster than the
 * uncapped 242 / 150 registers despite the spills); overridable at build time. */
#ifndef DGR_P2_MINB_EDGE
#define DGR_P2_MINB_EDGE 5
#endif
#ifndef DGR_P2_MINB_ELEMENT
#define DGR_P2_MINB_ELEMENT 4
#endif

constexpr int P2_NM = 6;       /* modes per variable */
constexpr int P2_NQ = 7;       /* area quadrature points */
constexpr int P2_NGP = 3;      /* Gauss points per edge */
constexpr int P2_PLANES = 18;  /* state planes: 3 variables x 6 modes */
constexpr int P2_FLUX = 9;     /* flux planes per edge: 3 points x 3 variables */

/* Reference-element tables (passed by value: the kernel parameter space is constant memory). */
struct P2Ref {
    double wq[P2_NQ];              /* area weights, summing to 1 */
    double lam[P2_NQ][3];          /* barycentric coordinates of the area points */
    double phi[P2_NQ][P2_NM];      /* basis at the area points */
    double dr[P2_NQ][P2_NM];       /* d/dr */
    double ds[P2_NQ][P2_NM];       /* d/ds */
    double te[P2_NGP];             /* Gauss points on [-1, 1] */
    double wg[P2_NGP];             /* Gauss weights */
    double phie[3][P2_NGP][P2_NM]; /* basis at the Gauss points of local edge k, running from
                                      vertex k to vertex k+1 */
    double mass[P2_NM];            /* int_ref phi_m^2 dr ds */
};

/* per-element geometry planes of the p = 2 step */
enum {
    P2G_DETJ = 0, /* |d(x,y)/d(r,s)| = area / 2 */
    P2G_RX = 1,   /* dr/dx, dr/dy, ds/dx, ds/dy */
    P2G_RY = 2,
    P2G_SX = 3,
    P2G_SY = 4,
    P2G_LEN = 5,  /* lengths of local edges 0..2 */
    P2G_ZV = 8,   /* vertex depths 0..2 */
    P2G_DZX = 11, /* depth gradient */
    P2G_DZY = 12,
    P2G_GNN = 13, /* g n^2 (per-element n, else the mean of the vertex n) */
    P2G_N = 14
};

/* local Gauss point of a side-1 element that matches point g of the edge's "in" orientation:
 * consistently oriented neighbours run a shared edge in opposite directions (bit 7 of
 * e_info marks the same direction) */
DGR_HD int p2_match_point(int info, int g) { return (info & 128) ? g : P2_NGP - 1 - g; }

/* ------------------------------------------------------------------ edges ---- */

/* Roe flux at the 3 Gauss points of one edge, Fhat.n for the "in" element's outward normal
 * at its own Gauss points; returns the max wave speed.  Sx = the second lane of the state
 * (tangents / perturbed values) for the two-lane arithmetics, unused for T = double. */
template <class T, class Load>
DGR_HD T p2_edge_core(const P2Ref &ref, const Load &st, int el_in, int el_ex, int info, double nx, double ny,
                      const T &za, const T &zb, double bz, double bq, double g, T fh[P2_NGP][3], int &code,
                      int ftype = 0)
{
    const int k_in = info & 3, k_ex = (info >> 2) & 3, bd = (info >> 4) & 7;
    const bool boundary = bd || el_in == el_ex;
    T lam = 0.0;
    code = 0;
#pragma unroll
    for (int gp = 0; gp < P2_NGP; ++gp) {
        const double t = ref.te[gp];
        const T z_g = za * ((1.0 - t) / 2) + zb * ((1.0 + t) / 2);
        T ui[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            T a = 0.0;
#pragma unroll
            for (int m = 0; m < P2_NM; ++m) a += ref.phie[k_in][gp][m] * st(P2_NM * v + m, el_in);
            ui[v] = a;
        }
        T ue[3];
        if (boundary) {
            ghost_state<T>(bd, nx, ny, ui[0], ui[1], ui[2], bz, bq, ui[0], ue[0], ue[1], ue[2]);
        } else {
            const int ge = p2_match_point(info, gp);
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                T a = 0.0;
#pragma unroll
                for (int m = 0; m < P2_NM; ++m) a += ref.phie[k_ex][ge][m] * st(P2_NM * v + m, el_ex);
                ue[v] = a;
            }
        }
        const T l = numerical_flux<T>(ftype, fh[gp], ui[0], ue[0], ui[1], ue[1], ui[2], ue[2], z_g, nx, ny, g, g);
        if (isnan(fh[gp][0]) || isnan(fh[gp][1]) || isnan(fh[gp][2])) code = 1;
        lam = rmax(lam, l);
    }
    return lam;
}

/* ---------------------------------------------------------------- elements ---- */

/*
 * One element of the p = 2 step: the right-hand side of the weak form above and the RK
 * stage combination of element_core (modes MODE_STAGE1 .. MODE_RK3_3; MODE_RHS returns the
 * RHS).  S[v][m]: stage input; F[k][g][v]: Fhat.n, outward for this element, at its own
 * Gauss points of local edge k; geo(j): geometry plane j; zg: the depth-dependent planes as
 * T (zv0..2, dzx, dzy, gnn); uin(v, m): step input (stages > 1).
 */
template <int MODE, class T, class Geo, class ZGeo, class UIn>
DGR_HD void p2_element_core(const P2Ref &ref, const T S[3][P2_NM], const T F[3][P2_NGP][3], const Geo &geo,
                            const ZGeo &zg, const UIn &uin, double g, double rain, double dt, T w[3][P2_NM])
{
    const double detJ = geo(P2G_DETJ), rx = geo(P2G_RX), ry = geo(P2G_RY), sx = geo(P2G_SX), sy = geo(P2G_SY);
    const T zv[3] = {zg.zv(0), zg.zv(1), zg.zv(2)};
    const T dzx = zg.dzx(), dzy = zg.dzy(), gnn = zg.gnn();
    T acc[3][P2_NM];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int m = 0; m < P2_NM; ++m) acc[v][m] = 0.0;

    /* area integrals; the point loop stays a loop (its mode and variable indices are still
     * compile-time): unrolled, seven copies of its body overflow the instruction cache
     * (measured: 8 % off the p = 2 step rolled) */
#pragma unroll 1
    for (int q = 0; q < P2_NQ; ++q) {
        T uq[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            T a = 0.0;
#pragma unroll
            for (int m = 0; m < P2_NM; ++m) a += ref.phi[q][m] * S[v][m];
            uq[v] = a;
        }
        const T zq = ref.lam[q][0] * zv[0] + ref.lam[q][1] * zv[1] + ref.lam[q][2] * zv[2];
        const T H = uq[0] + zq;
        const T u = uq[1] / H, vv = uq[2] / H;
        const T p = 0.5 * g * (H * H - zq * zq);
        const T qxy = uq[1] * vv;
        const T fx[3] = {uq[1], uq[1] * u + p, qxy};
        const T fy[3] = {uq[2], qxy, uq[2] * vv + p};
        const T tau = gnn * sqrt(u * u + vv * vv) / pow43(H);
        const T src[3] = {T(rain), g * uq[0] * dzx - tau * uq[1], g * uq[0] * dzy - tau * uq[2]};
        const double wj = 2.0 * ref.wq[q] * detJ;
#pragma unroll
        for (int m = 0; m < P2_NM; ++m) {
            const double gx = ref.dr[q][m] * rx + ref.ds[q][m] * sx;
            const double gy = ref.dr[q][m] * ry + ref.ds[q][m] * sy;
#pragma unroll
            for (int v = 0; v < 3; ++v) acc[v][m] += wj * (fx[v] * gx + fy[v] * gy + src[v] * ref.phi[q][m]);
        }
    }
    /* edge integrals */
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double half = geo(P2G_LEN + k) / 2;
#pragma unroll
        for (int gp = 0; gp < P2_NGP; ++gp) {
            const double wl = ref.wg[gp] * half;
#pragma unroll
            for (int m = 0; m < P2_NM; ++m)
#pragma unroll
                for (int v = 0; v < 3; ++v) acc[v][m] -= wl * (F[k][gp][v] * ref.phie[k][gp][m]);
        }
    }
    T rhs[3][P2_NM];
#pragma unroll
    for (int m = 0; m < P2_NM; ++m) {
        const double minv = 1.0 / (detJ * ref.mass[m]);
#pragma unroll
        for (int v = 0; v < 3; ++v) rhs[v][m] = acc[v][m] * minv;
    }
    if (MODE == MODE_RHS) {
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int m = 0; m < P2_NM; ++m) w[v][m] = rhs[v][m];
        return;
    }
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int m = 0; m < P2_NM; ++m) {
            if (MODE == MODE_STAGE1) {
                w[v][m] = S[v][m] + rhs[v][m] * dt;
            } else if (MODE == MODE_STAGE2) {
                w[v][m] = (S[v][m] + uin(v, m)) * 0.5 + rhs[v][m] * (dt / 2);
            } else {
                const double a = MODE == MODE_RK3_2 ? 0.75 : 1.0 / 3;
                const double b = MODE == MODE_RK3_2 ? 0.25 : 2.0 / 3;
                w[v][m] = a * uin(v, m) + b * (S[v][m] + rhs[v][m] * dt);
            }
        }
}

/* depth-dependent element planes read as doubles (forward) */
struct P2PlaneZ {
    const double *G;
    int ld;
    DGR_HD double zv(int k) const { return G[(size_t)(P2G_ZV + k) * ld]; }
    DGR_HD double dzx() const { return G[(size_t)P2G_DZX * ld]; }
    DGR_HD double dzy() const { return G[(size_t)P2G_DZY * ld]; }
    DGR_HD double gnn() const { return G[(size_t)P2G_GNN * ld]; }
};

/* --------------------------------------------------------------- kernels ---- */

/* FT: the numerical flux as a compile-time constant, or -1 to take it from the mesh */
template <int BS, int FT = -1>
__global__ void __launch_bounds__(BS, DGR_P2_MINB_EDGE) k_p2_edge(P2Ref ref, MeshDev m, const double *__restrict__ p2g,
                                                const double *__restrict__ S, const double *__restrict__ bzeta,
                                                const double *__restrict__ bqn, double *__restrict__ flux,
                                                DevClock *clk, int lam_slot, int phase, double g)
{
    const int i = blockIdx.x * BS + threadIdx.x;
    const bool valid = i < m.nf;
    const int sid = (valid && m.ed_sid) ? m.ed_sid[i] : 0;
    double lam = 0.0;
    if (valid) {
        DevClock *ck = clk + sid;
        if (!ck->done) {
            const int el_in = m.e_in[i], el_ex = m.e_ex[i], info = m.e_info[i];
            const int k_in = info & 3;
            const int bd = (info >> 4) & 7;
            const double nx = m.e_geo[i], ny = m.e_geo[m.ldF + i];
            const int ld = m.ldE;
            const double za = p2g[(size_t)(P2G_ZV + k_in) * ld + el_in];
            const double zb = p2g[(size_t)(P2G_ZV + (k_in + 1) % 3) * ld + el_in];
            const auto st = [S, ld](int plane, int el) { return S[plane * ld + el]; };
            double fh[P2_NGP][3];
            int code;
            lam = p2_edge_core<double>(ref, st, el_in, el_ex, info, nx, ny, za, zb, bd ? bzeta[i] : 0.0,
                                       bd ? bqn[i] : 0.0, g, fh, code, FT >= 0 ? FT : m.flux);
            if (code) atomicMin(&ck->err, err_key(ck->step, phase, code, i - ck->ed_off));
#pragma unroll
            for (int gp = 0; gp < P2_NGP; ++gp)
#pragma unroll
                for (int v = 0; v < 3; ++v) flux[(3 * gp + v) * m.ldF + i] = fh[gp][v];
            if (!(lam >= 0.0)) lam = 0.0;
        }
    }
    block_max_speed(lam, sid, valid, clk, lam_slot);
}

/* the three edges' fluxes of one element, outward and at its own Gauss points */
template <class T, class FluxLoad>
DGR_HD void p2_gather_flux(const MeshDev &m, int el, const FluxLoad &fl, T F[3][P2_NGP][3])
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * m.ldE + el];
        const int e = ee >> 1, side = ee & 1;
        const int info = side ? m.e_info[e] : 0;
#pragma unroll
        for (int gp = 0; gp < P2_NGP; ++gp) {
            /* this element's point gp is point gi of the edge's "in" orientation */
            const int gi = side ? p2_match_point(info, gp) : gp;
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                const T f = fl(3 * gi + v, e);
                F[k][gp][v] = side ? -f : f;
            }
        }
    }
}

template <int MODE, int BS>
__global__ void __launch_bounds__(BS, DGR_P2_MINB_ELEMENT) k_p2_element(P2Ref ref, MeshDev m, const double *__restrict__ p2g,
                                                   const double *__restrict__ S, const double *__restrict__ U,
                                                   const double *__restrict__ flux, double *__restrict__ out,
                                                   const DevClock *clk, double g)
{
    const int el = blockIdx.x * BS + threadIdx.x;
    if (el >= m.ne) return;
    const DevClock *ck = clk + (m.el_sid ? m.el_sid[el] : 0);
    if (ck->done) return;
    const int ld = m.ldE;
    double s[3][P2_NM];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < P2_NM; ++k) s[v][k] = S[(P2_NM * v + k) * ld + el];
    double F[3][P2_NGP][3];
    const int lf = m.ldF;
    p2_gather_flux<double>(m, el, [flux, lf](int plane, int e) { return flux[plane * lf + e]; }, F);
    const double *G = p2g + el;
    const auto geo = [G, ld](int j) { return G[(size_t)j * ld]; };
    const P2PlaneZ zg{G, ld};
    const auto uin = [U, ld, el](int v, int k) { return U[(P2_NM * v + k) * ld + el]; };
    double w[3][P2_NM];
    p2_element_core<MODE, double>(ref, s, F, geo, zg, uin, g, ck->rain, MODE == MODE_RHS ? 0.0 : ck->dt, w);
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < P2_NM; ++k) out[(P2_NM * v + k) * ld + el] = w[v][k];
}

/* Per-element p = 2 geometry from the vertex coordinates, depths and Manning n. */
static __global__ void __launch_bounds__(256) k_p2_setup(int ne, int ldE, const int *__restrict__ el2v_aos,
                                                         const double *__restrict__ x, const double *__restrict__ y,
                                                         const double *__restrict__ z,
                                                         const double *__restrict__ nfric,
                                                         const double *__restrict__ n_el, double g, double *p2g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    const int v0 = el2v_aos[3 * i], v1 = el2v_aos[3 * i + 1], v2 = el2v_aos[3 * i + 2];
    double *G = p2g + i;
#define SETP(j, val) G[(size_t)(j) * ldE] = (val)
    const double xr = (x[v1] - x[v0]) / 2, xs = (x[v2] - x[v0]) / 2;
    const double yr = (y[v1] - y[v0]) / 2, ys = (y[v2] - y[v0]) / 2;
    const double det = xr * ys - xs * yr;
    SETP(P2G_DETJ, fabs(det));
    SETP(P2G_RX, ys / det);
    SETP(P2G_RY, -xs / det);
    SETP(P2G_SX, -yr / det);
    SETP(P2G_SY, xr / det);
    const int vv[3] = {v0, v1, v2};
    for (int k = 0; k < 3; ++k) {
        const int a = vv[k], b = vv[(k + 1) % 3];
        SETP(P2G_LEN + k, sqrt((x[b] - x[a]) * (x[b] - x[a]) + (y[b] - y[a]) * (y[b] - y[a])));
        SETP(P2G_ZV + k, z[vv[k]]);
    }
    /* grad z of the linear depth: z = z0 + (z1 - z0)(1+r)/2 + (z2 - z0)(1+s)/2 */
    const double zr = (z[v1] - z[v0]) / 2, zs = (z[v2] - z[v0]) / 2;
    SETP(P2G_DZX, zr * (ys / det) + zs * (-yr / det));
    SETP(P2G_DZY, zr * (-xs / det) + zs * (xr / det));
    const double n = (n_el && n_el[i] >= 0.0) ? n_el[i] : (nfric[v0] + nfric[v1] + nfric[v2]) / 3;
    SETP(P2G_GNN, g * n * n);
#undef SETP
}

}  // namespace dgr
