/*
 * sm_100a kernels of the DG-RAIN 2D step.
 *
 * Layout in HBM (all FP64 unless noted, "planar" = one contiguous plane of ld entries per
 * component so that consecutive threads read consecutive addresses):
 *   state U, W        planar [9][ldE]: plane 3*v+k = variable v (zeta, Qx, Qy) at edge
 *                     midpoint k of every element
 *   element geometry  planar [NG][ldE], state-independent factors of
 *                     2DCode/2DInnerProducts.c computed once with the reference's formulas
 *   el2v, elem_edge   int planar [3][ldE]: vertices; (edge << 1 | side) of each local edge
 *   edge data         e_in/e_ex/e_info int [nf], e_geo planar [3][ldF] (nx, ny, z_edge)
 *   flux              planar [6][ldF]: Fhat.n of the "in" side (3) and the "ex" side (3)
 *   avg, bounds       planar [3][ldE] element means; planar [6][ldN] node max/min
 *
 * Per RK stage: edge flux -> element RHS + RK update -> node bounds -> limiter + PDop +
 * wet/dry status.  Every kernel has one thread per edge, element or node; no atomics
 * touch the data path (the edge flux is stored once per edge and gathered by both
 * elements), only the max wave speed and the first-error word are reduced atomically.
 */
#pragma once

#include "dgr_device.cuh"
#include "dgr_forcing.h"

/* Minimum resident blocks per SM requested from the compiler for the edge kernel
 * (register cap 65536 / (256 x blocks)); chosen by measurement, overridable at build time.
 * The element kernels are capped at 128 registers and the limiter kernels at 85
 * (launch bounds 512/BS and 768/BS blocks of BS threads). */
#ifndef DGR_MINB_EDGE
#define DGR_MINB_EDGE 3
#endif

namespace dgr {

/* Loads of data that the same launch may have written on another SM (used by the
 * persistent fused kernel, COH = true): served from L2, never from a stale L1 line or the
 * read-only path.  The one-item-per-thread kernels use plain loads (COH = false). */
template <bool COH, class T>
DGR_DEV T ldm(const T *p)
{
    if (COH) return __ldcg(p);
    return *p;
}

/* element geometry planes */
enum {
    G_NX = 0,     /* nx1..nx3              2DInnerProducts.c:110-116 */
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

/* Clock and forcing of one scenario (one mesh of an ensemble; a single mesh is an
 * ensemble of one).  Every scenario advances with its own CFL dt. */
struct DevClock {
    double time;        /* current time */
    double dt;          /* dt of the step in progress, then of the next step */
    double final_time;
    double bc2_zeta;    /* type-2 boundary elevation of the step in progress */
    unsigned long long lam_bits[2]; /* max wave speed per stage, bits of a double >= 0 */
    unsigned long long err;         /* first failure key; ~0 = none */
    int step;           /* steps done in the current run */
    int nsteps;         /* step limit of the current run */
    int done;           /* 1: the run has finished, later kernels do nothing */
    int dt_pending;     /* 1: dt of the next step is still to be derived from lam_bits[1] */
    /* per-scenario constants */
    double min_edge;    /* minEdgLength of this scenario's mesh */
    double rain;        /* m/s on the elevation equation (extension) */
    double tide_amp, tide_period;
    int tide_on;
    int el_off, ed_off; /* first element / edge of the scenario in the flattened mesh */
    int pad_;
};

struct MeshDev {
    int ne, nn, nf;
    int ldE, ldF, ldN;
    const int *el2v;      /* [3][ldE] */
    const int *elem_edge; /* [3][ldE] */
    const int *e_in, *e_ex, *e_info; /* [nf]; info = k_in | k_ex<<2 | bdry<<4 */
    const double *e_geo;  /* [3][ldF] */
    const double *geo;    /* [NG][ldE] */
    const int *n2e_ptr, *n2e;
    const double *zn;     /* node depth [nn] */
    const int *el_sid;    /* scenario of each element, NULL for a single mesh */
    const int *ed_sid;    /* scenario of each edge, NULL for a single mesh */
};

struct PhysParams {
    double g, h0, velzero, cfl, dt0;
};

/* ------------------------------------------------------------------ edges ---- */

/* One edge (2DCode/compute2DL.c:17-331): traces, ghost state, Roe flux(es); stores Fhat.n
 * for both sides and returns the edge's max wave speed (0 for a finished scenario). */
template <bool WD, bool COH = false>
DGR_DEV double edge_flux_item(const MeshDev &m, const double *S, const int *wd, const double *bzeta,
                              const double *bqn, double *flux, DevClock *clk, int phase, double g, int i)
{
    double lam = 0.0;
    DevClock *ck = clk + (m.ed_sid ? m.ed_sid[i] : 0);
    if (!ldm<COH>(&ck->done)) {
        const int el_in = m.e_in[i], el_ex = m.e_ex[i], info = m.e_info[i];
        const int k_in = info & 3, k_ex = (info >> 2) & 3, bd = (info >> 4) & 7;
        const double nx = m.e_geo[i], ny = m.e_geo[m.ldF + i], z_edge = m.e_geo[2 * m.ldF + i];
        const double tx = -ny, ty = nx;
        const int ld = m.ldE;
        const double zi = ldm<COH>(&S[k_in * ld + el_in]), qxi = ldm<COH>(&S[(3 + k_in) * ld + el_in]),
                     qyi = ldm<COH>(&S[(6 + k_in) * ld + el_in]);
        double ze, qxe, qye;
        if (bd) { /* :149-164 */
            ze = ldm<COH>(&bzeta[i]);
            double qn_ex = ldm<COH>(&bqn[i]);
            if (ze < 0) ze = zi;
            if (qn_ex > 1000) qn_ex = qxi * nx + qyi * ny;
            const double qt_ex = qxi * tx + qyi * ty;
            const double d = 1. / (nx * ty - ny * tx);
            qxe = (ty * qn_ex - ny * qt_ex) * d;
            qye = (-tx * qn_ex + nx * qt_ex) * d;
        } else if (el_in == el_ex) { /* land: reflect the normal discharge, :175-191 */
            ze = ldm<COH>(&S[k_ex * ld + el_ex]);
            const double qn_in = qxi * nx + qyi * ny;
            const double qt_in = qxi * tx + qyi * ty;
            const double qn_ex = -qn_in, qt_ex = qt_in;
            const double d = 1. / (nx * ty - ny * tx);
            qxe = (ty * qn_ex - ny * qt_ex) * d;
            qye = (-tx * qn_ex + nx * qt_ex) * d;
        } else {
            ze = ldm<COH>(&S[k_ex * ld + el_ex]);
            qxe = ldm<COH>(&S[(3 + k_ex) * ld + el_ex]);
            qye = ldm<COH>(&S[(6 + k_ex) * ld + el_ex]);
        }

        double fin[3], fex[3];
        int code = 0;
        const int wdi = WD ? ldm<COH>(&wd[el_in]) : 1, wde = WD ? ldm<COH>(&wd[el_ex]) : 1;
        if (WD && wdi == 0 && wde == 0) { /* both dry, :203-239 */
            double qn_in = qxi * nx + qyi * ny;
            double qt_in = qxi * tx + qyi * ty;
            double qn_ex = -qn_in, qt_ex = qt_in;
            const double d = 1. / (nx * ty - ny * tx);
            const double qxe_ref = (ty * qn_ex - ny * qt_ex) * d;
            const double qye_ref = (-tx * qn_ex + nx * qt_ex) * d;
            const double lam_in = roe_flux(fin, zi, zi, qxi, qxe_ref, qyi, qye_ref, z_edge, nx, ny, 0.0, g);
            qn_ex = qxe * nx + qye * ny;
            qt_ex = qxe * tx + qye * ty;
            qn_in = -qn_ex;
            qt_in = qt_ex;
            const double qxi_ref = (ty * qn_in - ny * qt_in) * d;
            const double qyi_ref = (-tx * qn_in + nx * qt_ex) * d;
            const double lam_ex = roe_flux(fex, ze, ze, qxi_ref, qxe, qyi_ref, qye, z_edge, nx, ny, 0.0, g);
            lam = rmax(lam_in, lam_ex);
        } else {
            double fh[3];
            lam = roe_flux(fh, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, g, g);
            if (isnan(fh[0]) || isnan(fh[1]) || isnan(fh[2])) code = 1;
            if (!WD || wdi == 1) {
                fin[0] = fh[0]; fin[1] = fh[1]; fin[2] = fh[2];
            } else {
                const double l2 = roe_flux(fin, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, 0.0, g);
                if (!code && (isnan(fin[0]) || isnan(fin[1]) || isnan(fin[2]))) code = 2;
                lam = rmax(lam, l2);
            }
            if (!WD || wde == 1) {
                fex[0] = fh[0]; fex[1] = fh[1]; fex[2] = fh[2];
            } else {
                const double l2 = roe_flux(fex, zi, ze, qxi, qxe, qyi, qye, z_edge, nx, ny, 0.0, g);
                if (!code && (isnan(fex[0]) || isnan(fex[1]) || isnan(fex[2]))) code = 3;
                lam = rmax(lam, l2);
            }
        }
        if (code) atomicMin(&ck->err, err_key(ldm<COH>(&ck->step), phase, code, i - ck->ed_off));
        const int lf = m.ldF;
        flux[i] = fin[0];
        flux[lf + i] = fin[1];
        flux[2 * lf + i] = fin[2];
        flux[3 * lf + i] = fex[0];
        flux[4 * lf + i] = fex[1];
        flux[5 * lf + i] = fex[2];
        if (!(lam >= 0.0)) lam = 0.0; /* NaN speeds are reported through the flux check */
        }
    return lam;
}

/* Max of the wave speed per scenario: one atomic per block when the block's edges all
 * belong to one scenario (always for a single mesh), else one per lane. */
DGR_DEV void block_max_speed(double lam, int sid, bool valid, DevClock *clk, int lam_slot)
{
    __shared__ double red[32];
    __shared__ int s_sid0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_sid0 = sid;
    __syncthreads();
    const int one_scenario = __syncthreads_and(!valid || sid == s_sid0);
    if (one_scenario) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lam = fmax(lam, __shfl_xor_sync(0xffffffffu, lam, o));
        if (lane == 0) red[wid] = lam;
        __syncthreads();
        if (wid == 0) {
            lam = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) lam = fmax(lam, __shfl_xor_sync(0xffffffffu, lam, o));
            if (lane == 0 && lam > 0.0)
                atomicMax(&clk[s_sid0].lam_bits[lam_slot], (unsigned long long)__double_as_longlong(lam));
        }
        __syncthreads();
    } else if (valid && lam > 0.0) {
        atomicMax(&clk[sid].lam_bits[lam_slot], (unsigned long long)__double_as_longlong(lam));
    }
}

template <bool WD>
__global__ void __launch_bounds__(256, DGR_MINB_EDGE) k_edge_flux(MeshDev m, const double *__restrict__ S,
                                                                  const int *__restrict__ wd,
                                                                  const double *__restrict__ bzeta,
                                                                  const double *__restrict__ bqn,
                                                                  double *__restrict__ flux, DevClock *clk,
                                                                  int lam_slot, int phase, double g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < m.nf;
    const int sid = (valid && m.ed_sid) ? m.ed_sid[i] : 0;
    const double lam = valid ? edge_flux_item<WD>(m, S, wd, bzeta, bqn, flux, clk, phase, g, i) : 0.0;
    block_max_speed(lam, sid, valid, clk, lam_slot);
}

/* ---------------------------------------------------------------- elements ---- */

enum { MODE_RHS = 0, MODE_STAGE1 = 1, MODE_STAGE2 = 2 };

/* One element: surface and volume integrals of 2DCode/2DInnerProducts.c:8-570, the
 * right-hand side of 2DCode/compute2DL.c:338-411 and the SSP-RK2 combination of
 * 2DCode/time_evolution.c:76-88 (stage 1: w1 = w + RHS*dt) or :176-217 (stage 2:
 * w = (w1 + w)*0.5 + RHS*(dt/2)).  S is the stage input, U the step input (stage 2 only).
 * MODE_RHS writes the RHS. */
template <int MODE, bool COH = false>
DGR_DEV void element_item(const MeshDev &m, const double *S, const double *U, const int *wd, const double *flux,
                          double *out, double *avg, const DevClock *clk, double g, int el)
{
    const DevClock *ck = clk + (m.el_sid ? m.el_sid[el] : 0);
    if (ldm<COH>(&ck->done)) return;
    const double rain = ck->rain;
    const int ld = m.ldE;
    const double *G = m.geo + el;
#define GEO(j) G[(size_t)(j) * ld]

    /* gathered numerical fluxes, sign flipped on the "ex" side (:319-329) */
    double F[3][3]; /* [variable][local edge] */
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * ld + el];
        const int e = ee >> 1;
        const int side = ee & 1;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double f = ldm<COH>(&flux[(3 * side + v) * m.ldF + e]);
            F[v][k] = side ? -f : f;
        }
    }

    const double nx[3] = {GEO(G_NX), GEO(G_NX + 1), GEO(G_NX + 2)};
    const double ny[3] = {GEO(G_NY), GEO(G_NY + 1), GEO(G_NY + 2)};
    const double M12 = GEO(G_M12), M22 = GEO(G_M12 + 1), M32 = GEO(G_M12 + 2), dM = GEO(G_DM);
    const double M11 = nx[0], M13 = ny[0], M21 = nx[1], M23 = ny[1], M31 = nx[2], M33 = ny[2];

    /* surface integrals SI[9] (:95-239) */
    double si[9];
    {
        const double ej0 = GEO(G_EJ), ej1 = GEO(G_EJ + 1), ej2 = GEO(G_EJ + 2);
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            double a, b, c;
            rt0_fit(F[v][0], F[v][1], F[v][2], M11, M12, M13, M21, M22, M23, M31, M32, M33, dM, a, b, c);
            double fd[3][2];
#pragma unroll
            for (int e = 0; e < 3; ++e)
#pragma unroll
                for (int n = 0; n < 2; ++n)
                    fd[e][n] = (a + b * GEO(G_XE + 2 * e + n)) * nx[e] + (c + b * GEO(G_YE + 2 * e + n)) * ny[e];
#pragma unroll
            for (int bf = 0; bf < 3; ++bf) {
                const int p = G_PSI + 6 * bf;
                si[3 * v + bf] = ej0 * (fd[0][0] * GEO(p) + fd[0][1] * GEO(p + 1)) +
                                 ej1 * (fd[1][0] * GEO(p + 2) + fd[1][1] * GEO(p + 3)) +
                                 ej2 * (fd[2][0] * GEO(p + 4) + fd[2][1] * GEO(p + 5));
            }
        }
    }

    /* volume integrals VI[21] (:247-566) */
    double zr[3], qxr[3], qyr[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        zr[k] = ldm<COH>(&S[k * ld + el]);
        qxr[k] = ldm<COH>(&S[(3 + k) * ld + el]);
        qyr[k] = ldm<COH>(&S[(6 + k) * ld + el]);
    }
    const double local_g = (ldm<COH>(&wd[el]) == 0) ? 0.0 : g;
    double H[3], tau[3], R[3][3]; /* R[variable][edge] = volume flux . n */
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const double midz = GEO(G_MIDZ + e);
        H[e] = zr[e] + midz;
        const double u = qxr[e] / H[e];
        const double v = qyr[e] / H[e];
        tau[e] = GEO(G_GNN + e) * sqrt(u * u + v * v) / pow43(H[e]);
        const double pr = 0.5 * local_g * (H[e] * H[e] - midz * midz);
        const double qxy = qxr[e] * qyr[e] / H[e];
        R[0][e] = qxr[e] * nx[e] + qyr[e] * ny[e];
        R[1][e] = (qxr[e] * qxr[e] / H[e] + pr) * nx[e] + qxy * ny[e];
        R[2][e] = qxy * nx[e] + (qyr[e] * qyr[e] / H[e] + pr) * ny[e];
    }
    const double aj = GEO(G_AJ), ajw = GEO(G_AJW);
    const double weight = 1.0 / 6;
    double dv[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        double a, b, c;
        rt0_fit(R[v][0], R[v][1], R[v][2], M11, M12, M13, M21, M22, M23, M31, M32, M33, dM, a, b, c);
#pragma unroll
        for (int bf = 0; bf < 3; ++bf)
            dv[v][bf] = aj * (0.5 * a * GEO(G_GP + 2 * bf) + 0.5 * c * GEO(G_GP + 2 * bf + 1) +
                              b * weight * GEO(G_P + bf));
    }
    const double bedx = local_g * aj * GEO(G_GRADZ) * weight;
    const double bedy = local_g * aj * GEO(G_GRADZ + 1) * weight;

    /* right-hand side (2DCode/compute2DL.c:344-409) */
    double X[3][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        X[0][j] = -si[j] + dv[0][j];
        X[1][j] = -si[3 + j] + dv[1][j] + bedx * zr[j] - ajw * tau[j] * qxr[j];
        X[2][j] = -si[6 + j] + dv[2][j] + bedy * zr[j] - ajw * tau[j] * qyr[j];
    }
    const double m11 = GEO(G_M11);
    double rhs[3][3];
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
#undef GEO

    if (MODE == MODE_RHS) {
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int k = 0; k < 3; ++k) out[(3 * v + k) * ld + el] = rhs[v][k];
        return;
    }
    const double dt = ldm<COH>(&ck->dt);
    double w[3][3];
    if (MODE == MODE_STAGE1) {
        w[0][0] = zr[0] + rhs[0][0] * dt;
        w[0][1] = zr[1] + rhs[0][1] * dt;
        w[0][2] = zr[2] + rhs[0][2] * dt;
        w[1][0] = qxr[0] + rhs[1][0] * dt;
        w[1][1] = qxr[1] + rhs[1][1] * dt;
        w[1][2] = qxr[2] + rhs[1][2] * dt;
        w[2][0] = qyr[0] + rhs[2][0] * dt;
        w[2][1] = qyr[1] + rhs[2][1] * dt;
        w[2][2] = qyr[2] + rhs[2][2] * dt;
    } else {
        const double hdt = dt / 2;
        const double s[3][3] = {{zr[0], zr[1], zr[2]}, {qxr[0], qxr[1], qxr[2]}, {qyr[0], qyr[1], qyr[2]}};
#pragma unroll
        for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int k = 0; k < 3; ++k) w[v][k] = (s[v][k] + ldm<COH>(&U[(3 * v + k) * ld + el])) * 0.5 + rhs[v][k] * hdt;
    }
#pragma unroll
    for (int v = 0; v < 3; ++v) {
#pragma unroll
        for (int k = 0; k < 3; ++k) out[(3 * v + k) * ld + el] = w[v][k];
        avg[v * ld + el] = (w[v][0] + w[v][1] + w[v][2]) / 3;
    }
}

template <int MODE, int BS>
__global__ void __launch_bounds__(BS, 512 / BS) k_element(MeshDev m, const double *__restrict__ S,
                                                          const double *__restrict__ U, const int *__restrict__ wd,
                                                          const double *__restrict__ flux, double *__restrict__ out,
                                                          double *__restrict__ avg, const DevClock *clk, double g)
{
    const int el = blockIdx.x * BS + threadIdx.x;
    if (el < m.ne) element_item<MODE>(m, S, U, wd, flux, out, avg, clk, g, el);
}

/* ------------------------------------------------------------------ nodes ---- */

/* Node max/min of element averages, 2DCode/SlopeLimiter2D.c:105-153 (the reference's
 * +-99999 starting values included). */
template <bool COH = false>
DGR_DEV void node_item(const MeshDev &m, const double *avg, double *bounds, int n)
{
    double mx0 = -99999, mx1 = -99999, mx2 = -99999, mn0 = 99999, mn1 = 99999, mn2 = 99999;
    const int b = m.n2e_ptr[n], e = m.n2e_ptr[n + 1];
    for (int j = b; j < e; ++j) {
        const int el = m.n2e[j];
        const double a0 = ldm<COH>(&avg[el]), a1 = ldm<COH>(&avg[m.ldE + el]), a2 = ldm<COH>(&avg[2 * m.ldE + el]);
        if (a0 < mn0) mn0 = a0;
        if (a0 > mx0) mx0 = a0;
        if (a1 < mn1) mn1 = a1;
        if (a1 > mx1) mx1 = a1;
        if (a2 < mn2) mn2 = a2;
        if (a2 > mx2) mx2 = a2;
    }
    const int l = m.ldN;
    bounds[n] = mx0;
    bounds[l + n] = mx1;
    bounds[2 * l + n] = mx2;
    bounds[3 * l + n] = mn0;
    bounds[4 * l + n] = mn1;
    bounds[5 * l + n] = mn2;
}

__global__ void __launch_bounds__(256) k_node_bounds(MeshDev m, const double *__restrict__ avg,
                                                     double *__restrict__ bounds)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < m.nn) node_item(m, avg, bounds, n);
}

/* Element means of a state (used by the stand-alone limiter call). */
__global__ void __launch_bounds__(256) k_avg(MeshDev m, const double *__restrict__ S, double *__restrict__ avg)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE;
#pragma unroll
    for (int v = 0; v < 3; ++v)
        avg[v * ld + el] = (S[(3 * v) * ld + el] + S[(3 * v + 1) * ld + el] + S[(3 * v + 2) * ld + el]) / 3;
}

/* --------------------------------------------------------------- wet/dry ---- */

/* BigTheta, 2DCode/wetDry2D.c:7-14 */
DGR_DEV int big_theta(double a) { return a > 0 ? 1 : 0; }

/* wetDryStatus2D for one element (2DCode/wetDry2D.c:18-57). */
DGR_DEV int wd_status(const double mz[3], const double zn[3], int wd_prev, double h0)
{
    const double zv[3] = {mz[0] - mz[1] + mz[2], mz[0] + mz[1] - mz[2], -mz[0] + mz[1] + mz[2]};
    const double h[3] = {zv[0] + zn[0], zv[1] + zn[1], zv[2] + zn[2]};
    const double avg_h = (h[0] + h[1] + h[2]) / 3;
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

__global__ void __launch_bounds__(256) k_wd_status(MeshDev m, const double *__restrict__ S, int *wd,
                                                   const DevClock *clk, double h0)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    if (clk[m.el_sid ? m.el_sid[el] : 0].done) return;
    const int ld = m.ldE;
    const double mz[3] = {S[el], S[ld + el], S[2 * ld + el]};
    const double zn[3] = {m.zn[m.el2v[el]], m.zn[m.el2v[ld + el]], m.zn[m.el2v[2 * ld + el]]};
    wd[el] = wd_status(mz, zn, wd[el], h0);
}

/* ---------------------------------------------------------- limit + PDop ---- */

/*
 * One element: vertex-based limiter (2DCode/SlopeLimiter2D.c:157-343), then the
 * positive-depth operator (2DCode/wetDry2D.c:63-260), then the wet/dry status
 * (2DCode/wetDry2D.c:16-60) that the reference calls next.  wd_in is the status the
 * element had; the new status goes to wd_out.
 */
template <bool LIMIT, bool PDOP, bool STATUS, bool COH = false>
DGR_DEV void limit_item(const MeshDev &m, double *S, const double *bounds, const int *wd_in, int *wd_out,
                        DevClock *clk, double h0, double velzero, int phase, int *dec_limit, int *dec_pdop, int el)
{
    DevClock *ck = clk + (m.el_sid ? m.el_sid[el] : 0);
    if (ldm<COH>(&ck->done)) return;
    const int ld = m.ldE;
    const int nd[3] = {m.el2v[el], m.el2v[ld + el], m.el2v[2 * ld + el]};
    const double zn[3] = {m.zn[nd[0]], m.zn[nd[1]], m.zn[nd[2]]};
    double w[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) w[v][k] = ldm<COH>(&S[(3 * v + k) * ld + el]);

    int modify = 0;
    if (LIMIT) {
        const int lb = m.ldN;
        double out[3][3];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double w1 = w[v][0], w2 = w[v][1], w3 = w[v][2];
            double vx[3] = {w1 - w2 + w3, w1 + w2 - w3, -w1 + w2 + w3};
            double vmax[3], vmin[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                vmax[k] = ldm<COH>(&bounds[v * lb + nd[k]]);
                vmin[k] = ldm<COH>(&bounds[(3 + v) * lb + nd[k]]);
            }
            const double avg = (w1 + w2 + w3) / 3;
            if (v == 0) { /* :189-200 */
                const double h1 = vx[0] + zn[0], h2 = vx[1] + zn[1], h3 = vx[2] + zn[2];
                const double m0 = vmin[0] + zn[0], m1 = vmin[1] + zn[1], m2 = vmin[2] + zn[2];
                if (h1 > h0 && h2 > h0 && h3 > h0 && m0 > h0 && m1 > h0 && m2 > h0) modify = 1;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) vx[k] = fmax(rmin(vx[k], vmax[k]), vmin[k]);
#pragma unroll
            for (int ll = 0; ll < 3; ++ll) { /* :254-299 */
                const double sumloc = (vx[0] + vx[1] + vx[2]) / 3;
                double sumdiff = (sumloc - avg) * 3;
                const int sd = sgn(sumdiff);
                const double sdd = (double)sd;
                const double diff[3] = {(vx[0] - avg) * sdd, (vx[1] - avg) * sdd, (vx[2] - avg) * sdd};
                double kdp = (double)((diff[0] > 0) + (diff[1] > 0) + (diff[2] > 0));
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double div = fmax(1.0, kdp);
                    double redfac;
                    if (diff[k] > 0) {
                        redfac = div_by_count(sumdiff * sdd, div);
                        kdp -= 1;
                    } else {
                        redfac = 0;
                    }
                    const double redmax = (sd > 0) ? vx[k] - vmin[k] : vmax[k] - vx[k];
                    redfac = rmin(redfac, redmax);
                    sumdiff -= redfac * sdd;
                    vx[k] -= redfac * sdd;
                }
            }
            out[v][0] = (vx[0] + vx[1]) / 2;
            out[v][1] = (vx[1] + vx[2]) / 2;
            out[v][2] = (vx[2] + vx[0]) / 2;
            if (v == 0) { /* :307-311 */
                const double h1 = vx[0] + zn[0], h2 = vx[1] + zn[1], h3 = vx[2] + zn[2];
                if (h1 < h0 || h2 < h0 || h3 < h0) modify = 0;
            }
        }
        if (modify) {
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int k = 0; k < 3; ++k) w[v][k] = out[v][k];
        }
        if (dec_limit) dec_limit[el] = modify;
    }

    int mass_branch = 0, mom_branch = 0;
    if (PDOP) {
        const double midz0 = 0.5 * (zn[0] + zn[1]), midz1 = 0.5 * (zn[1] + zn[2]), midz2 = 0.5 * (zn[2] + zn[0]);
        double mh0 = w[0][0] + midz0, mh1 = w[0][1] + midz1, mh2 = w[0][2] + midz2;
        double ht[3] = {mh0 - mh1 + mh2, mh0 + mh1 - mh2, -mh0 + mh1 + mh2};
        const double avg_h = (ht[0] + ht[1] + ht[2]) / 3;
        int code = 0;
        if (ht[0] <= h0 || ht[1] <= h0 || ht[2] <= h0) { /* :93-156 */
            if (avg_h <= h0) {
                mass_branch = 1;
                ht[0] = avg_h;
                ht[1] = avg_h;
                ht[2] = avg_h;
            } else {
                mass_branch = 2;
                int imin = 0;
                double hmin = ht[0];
                if (ht[1] < hmin) { imin = 1; hmin = ht[1]; }
                if (ht[2] < hmin) { imin = 2; hmin = ht[2]; }
                int inext = 1; /* the reference starts this search at index 1 (:115-124) */
                double hnext = ht[1];
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (ht[i] < hnext && i != imin) { inext = i; hnext = ht[i]; }
                int irem = 2;
                if (0 != imin && 0 != inext) irem = 0;
                else if (1 != imin && 1 != inext) irem = 1;
                double hh[3] = {ht[0], ht[1], ht[2]};
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
                mom_branch = 1;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    w[1][i] = 0;
                    w[2][i] = 0;
                }
            } else if (wet[0] == 0 || wet[1] == 0 || wet[2] == 0) { /* :180-253 */
                mom_branch = 2;
                const double q0 = w[1][0], q1 = w[1][1], q2 = w[1][2];
                const double r0 = w[2][0], r1 = w[2][1], r2 = w[2][2];
                double qxe[3] = {q0 - q1 + q2, q0 + q1 - q2, -q0 + q1 + q2};
                double qye[3] = {r0 - r1 + r2, r0 + r1 - r2, -r0 + r1 + r2};
                double u[3], vv[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    u[i] = qxe[i] / ht[i];
                    vv[i] = qye[i] / ht[i];
                }
                int npos = 0;
                double delu = 0, delv = 0;
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
        if (code) atomicMin(&ck->err, err_key(ldm<COH>(&ck->step), phase, code, el - ck->el_off));
        if (dec_pdop) dec_pdop[el] = 4 * mass_branch + mom_branch;
    }

#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) S[(3 * v + k) * ld + el] = w[v][k];
    if (STATUS) wd_out[el] = wd_status(w[0], zn, ldm<COH>(&wd_in[el]), h0);
}

template <bool LIMIT, bool PDOP, bool STATUS, int BS>
__global__ void __launch_bounds__(BS, 768 / BS) k_limit(MeshDev m, double *__restrict__ S,
                                                        const double *__restrict__ bounds,
                                                        const int *__restrict__ wd_in, int *__restrict__ wd_out,
                                                        DevClock *clk, double h0, double velzero, int phase,
                                                        int *__restrict__ dec_limit, int *__restrict__ dec_pdop)
{
    const int el = blockIdx.x * BS + threadIdx.x;
    if (el < m.ne)
        limit_item<LIMIT, PDOP, STATUS>(m, S, bounds, wd_in, wd_out, clk, h0, velzero, phase, dec_limit, dec_pdop,
                                        el);
}

/* ------------------------------------------------------------------ clock ---- */

/*
 * Start of one step of the device time loop (2DCode/time_evolution.c:311-401), for every
 * scenario: finish the CFL dt of the previous step, stop when time has reached
 * final_time, evaluate the boundary values for this step (boundary_conditions() at the
 * current time), then advance the clock.  One block; thread s owns scenario s's clock,
 * then all threads write the prescribed edges.
 */
DGR_DEV void clock_begin_body(DevClock *clk, int nscen, const PhysParams &p, const int *__restrict__ bnd_edges,
                              const int *__restrict__ bnd_type, const int *__restrict__ bnd_sid, int nbnd,
                              double *__restrict__ bzeta, double *__restrict__ bqn)
{
    for (int s = threadIdx.x; s < nscen; s += blockDim.x) {
        DevClock *c = clk + s;
        if (c->done) continue;
        if (c->dt_pending) {
            const double lam = __longlong_as_double((long long)c->lam_bits[1]);
            double dt = p.cfl * c->min_edge / lam;
            if ((c->time + dt) > c->final_time) dt = c->final_time - c->time;
            c->dt = dt;
            c->dt_pending = 0;
        }
        if (c->step >= c->nsteps || !(c->time < c->final_time) || c->err != ~0ull) {
            c->done = 1;
            continue;
        }
        c->bc2_zeta = dgr_outflow_zeta(c->time, c->tide_on, c->tide_amp, c->tide_period);
        c->time = c->time + c->dt;
        c->lam_bits[0] = 0;
        c->lam_bits[1] = 0;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nbnd; j += blockDim.x) {
        const DevClock *c = clk + (bnd_sid ? bnd_sid[j] : 0);
        if (c->done) continue;
        const int e = bnd_edges[j];
        const int t = bnd_type[j];
        double zb = 0, qn = 0;
        if (t == 1) { zb = DGR_BC1_ZETA; qn = DGR_BC1_QN; }
        else if (t == 2) { zb = c->bc2_zeta; qn = DGR_BC2_QN; }
        else if (t == 3) { zb = DGR_BC3_ZETA; qn = DGR_BC3_QN; }
        bzeta[e] = zb;
        bqn[e] = qn;
    }
}

__global__ void __launch_bounds__(256) k_clock_begin(DevClock *clk, int nscen, PhysParams p,
                                                     const int *__restrict__ bnd_edges,
                                                     const int *__restrict__ bnd_type,
                                                     const int *__restrict__ bnd_sid, int nbnd,
                                                     double *__restrict__ bzeta, double *__restrict__ bqn)
{
    clock_begin_body(clk, nscen, p, bnd_edges, bnd_type, bnd_sid, nbnd, bzeta, bqn);
}

/* End of a step: step counters and the pending CFL updates.  A scenario whose step just
 * failed stops here, so its step count is the number of steps that completed. */
template <bool COH = false>
DGR_DEV void clock_end_item(DevClock *clk, int s)
{
    if (clk[s].done) return;
    if (ldm<COH>(&clk[s].err) != ~0ull) {
        clk[s].done = 1;
        return;
    }
    clk[s].step += 1;
    clk[s].dt_pending = 1;
}

__global__ void k_clock_end(DevClock *clk, int nscen)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nscen) clock_end_item(clk, s);
}

/* After a run: derive each scenario's next dt so the host sees it. */
__global__ void k_clock_finish(DevClock *clk, int nscen, PhysParams p)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nscen) return;
    DevClock *c = clk + s;
    if (c->dt_pending) {
        const double lam = __longlong_as_double((long long)c->lam_bits[1]);
        double dt = p.cfl * c->min_edge / lam;
        if ((c->time + dt) > c->final_time) dt = c->final_time - c->time;
        c->dt = dt;
        c->dt_pending = 0;
    }
}

/* Host-driven step (oneTimeStep2D, single mesh): set the step's dt, clear per-step words. */
__global__ void k_clock_set(DevClock *clk, double time, double dt)
{
    clk->time = time;
    clk->dt = dt;
    clk->done = 0;
    clk->lam_bits[0] = 0;
    clk->lam_bits[1] = 0;
}

/* Device-side boundary_conditions() at time t for the stand-alone call. */
__global__ void k_forcing(const DevClock *clk, double t, const int *__restrict__ bnd_edges,
                          const int *__restrict__ bnd_type, const int *__restrict__ bnd_sid, int nbnd,
                          double *__restrict__ bzeta, double *__restrict__ bqn)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nbnd) return;
    const DevClock *c = clk + (bnd_sid ? bnd_sid[j] : 0);
    const double zb2 = dgr_outflow_zeta(t, c->tide_on, c->tide_amp, c->tide_period);
    const int e = bnd_edges[j];
    const int tt = bnd_type[j];
    double zb = 0, qn = 0;
    if (tt == 1) { zb = DGR_BC1_ZETA; qn = DGR_BC1_QN; }
    else if (tt == 2) { zb = zb2; qn = DGR_BC2_QN; }
    else if (tt == 3) { zb = DGR_BC3_ZETA; qn = DGR_BC3_QN; }
    bzeta[e] = zb;
    bqn[e] = qn;
}

/* ------------------------------------------------------ persistent fused kernel ---- */

struct FusedArgs {
    MeshDev m;
    double *U, *W, *flux, *avg, *bounds, *bzeta, *bqn;
    int *wdA, *wdB;
    DevClock *clk;
    int nscen;
    const int *bnd_edges, *bnd_type, *bnd_sid;
    int nbnd;
    PhysParams p;
    int *dec;         /* [4][ne] decisions, or nullptr */
    unsigned *bar;    /* [0] arrivals, [1] generation, [2] time-out flag */
};

/* Polls of a grid-barrier wait before it gives up (about a second with the 64 ns sleeps). */
constexpr unsigned kBarrierSpins = 1u << 24;

/* Grid-wide barrier of a cooperative launch (every block resident).  The wait is bounded:
 * a block that polls kBarrierSpins times records a time-out, and every block leaves the
 * kernel at its next barrier check, so a broken invariant ends the launch with an error
 * flag instead of hanging the GPU.  Returns false once a time-out is recorded. */
DGR_DEV bool grid_barrier(unsigned *bar)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = bar + 1;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned spins = 0;
            while (*vgen == gen) {
                if (++spins > kBarrierSpins) {
                    atomicExch(bar + 2, 1u);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile unsigned *)(bar + 2) == 0u;
}

/*
 * One persistent cooperative kernel for RK stages stage_begin..stage_end-1 (and, with
 * with_clock, the clock and boundary values of the step): the edge, element, node and
 * limiter phases of the one-item-per-thread kernels, each a grid-stride loop, separated by
 * grid barriers.  Arrays written by one phase and read by a later one are read through L2
 * (COH loads).  Same items, same arithmetic: results are identical to the separate kernels.
 */
template <bool WD, int BS>
__global__ void __launch_bounds__(BS, 512 / BS) k_step_fused(FusedArgs a, int stage_begin, int stage_end,
                                                             int with_clock)
{
    if (with_clock) {
        if (blockIdx.x == 0)
            clock_begin_body(a.clk, a.nscen, a.p, a.bnd_edges, a.bnd_type, a.bnd_sid, a.nbnd, a.bzeta, a.bqn);
        if (!grid_barrier(a.bar)) return;
    }
    const int stride = gridDim.x * BS;
    const int ne = a.m.ne;
    for (int stage = stage_begin; stage < stage_end; ++stage) {
        const double *S = stage == 0 ? a.U : a.W;
        double *OUT = stage == 0 ? a.W : a.U;
        const int *wd_in = (stage == 0 || !WD) ? a.wdA : a.wdB;
        int *wd_out = stage == 0 ? a.wdB : a.wdA;
        int *dl = a.dec ? a.dec + (size_t)(2 * stage) * ne : nullptr;
        int *dp = a.dec ? a.dec + (size_t)(2 * stage + 1) * ne : nullptr;
        for (int base = blockIdx.x * BS; base < a.m.nf; base += stride) {
            const int i = base + threadIdx.x;
            const bool valid = i < a.m.nf;
            const int sid = (valid && a.m.ed_sid) ? a.m.ed_sid[i] : 0;
            const double lam =
                valid ? edge_flux_item<WD, true>(a.m, S, wd_in, a.bzeta, a.bqn, a.flux, a.clk, 2 * stage, a.p.g, i)
                      : 0.0;
            block_max_speed(lam, sid, valid, a.clk, stage);
        }
        if (!grid_barrier(a.bar)) return;
        for (int el = blockIdx.x * BS + threadIdx.x; el < ne; el += stride) {
            if (stage == 0)
                element_item<MODE_STAGE1, true>(a.m, S, a.U, wd_in, a.flux, OUT, a.avg, a.clk, a.p.g, el);
            else
                element_item<MODE_STAGE2, true>(a.m, S, a.U, wd_in, a.flux, OUT, a.avg, a.clk, a.p.g, el);
        }
        if (!grid_barrier(a.bar)) return;
        for (int n = blockIdx.x * BS + threadIdx.x; n < a.m.nn; n += stride) node_item<true>(a.m, a.avg, a.bounds, n);
        if (!grid_barrier(a.bar)) return;
        for (int el = blockIdx.x * BS + threadIdx.x; el < ne; el += stride)
            limit_item<true, WD, WD, true>(a.m, OUT, a.bounds, wd_in, wd_out, a.clk, a.p.h0, a.p.velzero,
                                           2 * stage + 1, dl, dp, el);
        if (stage + 1 < stage_end || with_clock)
            if (!grid_barrier(a.bar)) return;
    }
    if (with_clock && blockIdx.x == 0)
        for (int sc = threadIdx.x; sc < a.nscen; sc += BS) clock_end_item<true>(a.clk, sc);
}

/* ---------------------------------------------------------------- set-up ---- */

/* local edge of element (a,b,c) joining v0-v1 (2DCode/compute2DL.c:45-67) */
DGR_DEV int local_edge(int a, int b, int c, int v0, int v1)
{
    if ((v0 == a && v1 == b) || (v0 == b && v1 == a)) return 0;
    if ((v0 == b && v1 == c) || (v0 == c && v1 == b)) return 1;
    if ((v0 == c && v1 == a) || (v0 == a && v1 == c)) return 2;
    return -1;
}

/* Per-edge state-independent data: local edge numbers, the "in" element's unit normal
 * (2DCode/compute2DL.c:98-132) and the mid-edge depth (:144). */
__global__ void k_edge_setup(int nf, int ldE, int ldF, const int *__restrict__ ed2el, const int *__restrict__ ed2v,
                             const int *__restrict__ el2v_aos, const int *__restrict__ bdry,
                             const double *__restrict__ x, const double *__restrict__ y,
                             const double *__restrict__ z, int *e_in, int *e_ex, int *e_info, double *e_geo,
                             int *elem_edge, int *bad_edge)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const int el_in = ed2el[2 * i], el_ex = ed2el[2 * i + 1];
    const int v0 = ed2v[2 * i], v1 = ed2v[2 * i + 1];
    const int a = el2v_aos[3 * el_in], b = el2v_aos[3 * el_in + 1], c = el2v_aos[3 * el_in + 2];
    const int k_in = local_edge(a, b, c, v0, v1);
    const int k_ex = local_edge(el2v_aos[3 * el_ex], el2v_aos[3 * el_ex + 1], el2v_aos[3 * el_ex + 2], v0, v1);
    if (k_in < 0 || k_ex < 0) {
        atomicMin(bad_edge, i);
        return;
    }
    const double len = sqrt((x[v1] - x[v0]) * (x[v1] - x[v0]) + (y[v1] - y[v0]) * (y[v1] - y[v0]));
    const double jac = x[a] * (y[b] - y[c]) + x[b] * (y[c] - y[a]) + x[c] * (y[a] - y[b]);
    const int ev[3] = {a, b, c};
    const int p0 = ev[k_in], p1 = ev[(k_in + 1) % 3];
    const double x0 = x[p0], x1 = x[p1], y0 = y[p0], y1 = y[p1];
    const double nx = sgn(jac) * (y1 - y0) / len;
    const double ny = sgn(jac) * (x0 - x1) / len;
    e_in[i] = el_in;
    e_ex[i] = el_ex;
    e_info[i] = k_in | (k_ex << 2) | ((bdry[i] & 7) << 4);
    e_geo[i] = nx;
    e_geo[ldF + i] = ny;
    e_geo[2 * ldF + i] = (z[v0] + z[v1]) / 2;
    elem_edge[k_in * ldE + el_in] = i << 1;
    if (el_ex != el_in) elem_edge[k_ex * ldE + el_ex] = (i << 1) | 1;
}

/* Per-element state-independent factors of 2DCode/2DInnerProducts.c and
 * 2DCode/compute2DL.c:373-382, each with the reference's own expression. */
__global__ void k_element_setup(int ne, int ldE, const int *__restrict__ el2v_aos, const double *__restrict__ x,
                                const double *__restrict__ y, const double *__restrict__ z,
                                const double *__restrict__ nfric, const double *__restrict__ n_el, double g,
                                int *el2v, double *geo)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ne) return;
    const int v0 = el2v_aos[3 * i], v1 = el2v_aos[3 * i + 1], v2 = el2v_aos[3 * i + 2];
    el2v[i] = v0;
    el2v[ldE + i] = v1;
    el2v[2 * ldE + i] = v2;
    double *G = geo + i;
#define SETG(j, val) G[(size_t)(j) * ldE] = (val)
    const double xv1 = x[v0], xv2 = x[v1], xv3 = x[v2];
    const double yv1 = y[v0], yv2 = y[v1], yv3 = y[v2];
    const double x1 = (x[v0] + x[v1]) / 2, x2 = (x[v1] + x[v2]) / 2, x3 = (x[v2] + x[v0]) / 2;
    const double y1 = (y[v0] + y[v1]) / 2, y2 = (y[v1] + y[v2]) / 2, y3 = (y[v2] + y[v0]) / 2;
    double len[3];
    len[0] = sqrt((xv2 - xv1) * (xv2 - xv1) + (yv2 - yv1) * (yv2 - yv1));
    len[1] = sqrt((xv3 - xv2) * (xv3 - xv2) + (yv3 - yv2) * (yv3 - yv2));
    len[2] = sqrt((xv3 - xv1) * (xv3 - xv1) + (yv3 - yv1) * (yv3 - yv1));
    for (int e = 0; e < 3; ++e) SETG(G_EJ + e, len[e] / 2);
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
            SETG(G_XE + 2 * e + n, xe[e][n]);
            SETG(G_YE + 2 * e + n, ye[e][n]);
        }
    const double den = x1 * y2 - x1 * y3 + x2 * y3 - x2 * y1 + x3 * y1 - x3 * y2;
    for (int e = 0; e < 3; ++e)
        for (int n = 0; n < 2; ++n) {
            const double xq = xe[e][n], yq = ye[e][n];
            SETG(G_PSI + 0 * 6 + 2 * e + n, -(yq * x2 - yq * x3 - xq * y2 + x3 * y2 + xq * y3 - x2 * y3) / den);
            SETG(G_PSI + 1 * 6 + 2 * e + n, -(-x1 * yq + x3 * yq - x3 * y1 + xq * y1 - xq * y3 + x1 * y3) / den);
            SETG(G_PSI + 2 * 6 + 2 * e + n, -(yq * x1 - yq * x2 - xq * y1 + x2 * y1 + xq * y2 - x1 * y2) / den);
        }
    const double jac = 4 * (x2 - x3) * (y2 - y1) - 4 * (x2 - x1) * (y2 - y3);
    const int sj = sgn(jac);
    const double nx1 = sj * 2 * (y2 - y3) / len[0], ny1 = sj * 2 * (x3 - x2) / len[0];
    const double nx2 = sj * 2 * (y3 - y1) / len[1], ny2 = sj * 2 * (x1 - x3) / len[1];
    const double nx3 = sj * 2 * (y1 - y2) / len[2], ny3 = sj * 2 * (x2 - x1) / len[2];
    SETG(G_NX, nx1); SETG(G_NX + 1, nx2); SETG(G_NX + 2, nx3);
    SETG(G_NY, ny1); SETG(G_NY + 1, ny2); SETG(G_NY + 2, ny3);
    const double M11 = nx1, M12 = x1 * nx1 + y1 * ny1, M13 = ny1;
    const double M21 = nx2, M22 = x2 * nx2 + y2 * ny2, M23 = ny2;
    const double M31 = nx3, M32 = x3 * nx3 + y3 * ny3, M33 = ny3;
    SETG(G_M12, M12); SETG(G_M12 + 1, M22); SETG(G_M12 + 2, M32);
    SETG(G_DM, M13 * M22 * M31 - M12 * M23 * M31 - M13 * M21 * M32 + M11 * M23 * M32 + M12 * M21 * M33 -
                   M11 * M22 * M33);
    const double midz[3] = {0.5 * (z[v0] + z[v1]), 0.5 * (z[v1] + z[v2]), 0.5 * (z[v2] + z[v0])};
    double midn[3];
    if (n_el && n_el[i] >= 0.0) {
        midn[0] = midn[1] = midn[2] = n_el[i];
    } else {
        midn[0] = 0.5 * (nfric[v0] + nfric[v1]);
        midn[1] = 0.5 * (nfric[v1] + nfric[v2]);
        midn[2] = 0.5 * (nfric[v2] + nfric[v0]);
    }
    for (int e = 0; e < 3; ++e) {
        SETG(G_MIDZ + e, midz[e]);
        SETG(G_GNN + e, g * midn[e] * midn[e]);
    }
    double gp[3][2];
    gp[0][0] = 4 / jac * (y2 - y3);
    gp[0][1] = 4 / jac * (x3 - x2);
    gp[1][0] = 4 / jac * (y3 - y1);
    gp[1][1] = 4 / jac * (x1 - x3);
    gp[2][0] = 4 / jac * (y1 - y2);
    gp[2][1] = 4 / jac * (x2 - x1);
    for (int b = 0; b < 3; ++b) {
        SETG(G_GP + 2 * b, gp[b][0]);
        SETG(G_GP + 2 * b + 1, gp[b][1]);
        SETG(G_P + b, gp[b][0] * (x1 + x2 + x3) + gp[b][1] * (y1 + y2 + y3));
    }
    for (int j = 0; j < 2; ++j) SETG(G_GRADZ + j, midz[0] * gp[0][j] + midz[1] * gp[1][j] + midz[2] * gp[2][j]);
    const double aj = fabs(jac);
    SETG(G_AJ, aj);
    SETG(G_AJW, aj * (1.0 / 6));
    const double x0v = x[v0], x1v = x[v1], x2v = x[v2], y0v = y[v0], y1v = y[v1], y2v = y[v2];
    const double jv = x0v * (y1v - y2v) + x1v * (y2v - y0v) + x2v * (y0v - y1v);
    SETG(G_M11, 6 / fabs(jv));
#undef SETG
}

/* the Manning power on n arguments (diagnostic entry point) */
__global__ void k_pow43(int n, const double *__restrict__ x, double *__restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = pow43(x[i]);
}

/* reference layout [3*el+k] <-> planar [3*v+k][ld] */
__global__ void k_aos_to_planar(int ne, int ld, const double *__restrict__ a0, const double *__restrict__ a1,
                                const double *__restrict__ a2, double *__restrict__ S)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= ne) return;
    const double *src[3] = {a0, a1, a2};
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) S[(3 * v + k) * ld + el] = src[v][3 * el + k];
}

__global__ void k_planar_to_aos(int ne, int ld, const double *__restrict__ S, double *__restrict__ a0,
                                double *__restrict__ a1, double *__restrict__ a2)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= ne) return;
    double *dst[3] = {a0, a1, a2};
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) dst[v][3 * el + k] = S[(3 * v + k) * ld + el];
}

/* edge fluxes back into the reference's element slots Fhat[3*el+k] */
__global__ void k_flux_to_slots(MeshDev m, const double *__restrict__ flux, double *f1, double *f2, double *f3)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    double *dst[3] = {f1, f2, f3};
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * m.ldE + el];
        const int e = ee >> 1, side = ee & 1;
        for (int v = 0; v < 3; ++v) {
            const double f = flux[(3 * side + v) * m.ldF + e];
            dst[v][3 * el + k] = side ? -f : f;
        }
    }
}

}  // namespace dgr
