/*
 * Tangent-linear (forward-mode, ad::Dual) and adjoint (reverse, hand-written) kernels of
 * the 2D step, one thread per edge, element or node like the forward kernels.
 *
 * Parameters of the derivatives: the state, the node depths z (enter the mid-edge depth,
 * the element mid-edge depths and depth gradient, and the vertex depths of the limiter and
 * PDop) and the per-element Manning n (enters g n^2 of the friction term).
 *
 * Layouts: tangents mirror the primal arrays (state [9][ldE], flux [6][ldF], means
 * [3][ldE], node bounds [6][ldN], z [nn], n [ne]).  Adjoint work arrays:
 *   Rbar  [9][ldE]   adjoint of an element's pre-limiter stage output
 *   bbar  [18][ldE]  adjoint of the node bounds the element's limiter read:
 *                    plane 6k+v = max of variable v at vertex k, 6k+3+v = min
 *   bnode [6][ldN], barg [6][ldN]  per node: summed bound adjoints and the element that
 *                    supplied each max/min (-1: the +-99999 start value)
 *   fbar  [6][ldF]   adjoint of the stored Fhat.n, per edge and side (each slot written by
 *                    the one element that gathers it: a conflict-free transposed gather)
 *   zvb   [3][ldE]   depth adjoint per element vertex slot, zeb [ldF] per edge, gathered to
 *                    nodes at the end of a sweep
 * No atomics: every adjoint slot has exactly one writer per launch, so gradients are
 * bitwise reproducible.
 */
#pragma once

#include "dgr_dual.cuh"
#include "dgr_kernels.cuh"
#include "dgr_reverse.cuh"

/* Minimum resident blocks per SM of the reverse kernels (register caps 65536 / (threads x
 * blocks)); chosen by measurement, overridable at build time. */
#ifndef DGR_ADJ_EDGE_BS /* threads per block of the reverse edge kernel */
#define DGR_ADJ_EDGE_BS 256
#endif
#ifndef DGR_ADJ_MINB_EDGE
#define DGR_ADJ_MINB_EDGE (512 / DGR_ADJ_EDGE_BS)
#endif
#ifndef DGR_ADJ_MINB_ELEMENT
#define DGR_ADJ_MINB_ELEMENT 4
#endif
#ifndef DGR_ADJ_MINB_LIMIT
#define DGR_ADJ_MINB_LIMIT 4
#endif

namespace dgr {

using ad::Dual;

/* Depth and Manning factors of one element in two-lane arithmetic (T = Dual or Pert):
 * values from the geometry planes, second lanes from the vertex-depth lanes zvx (tangents
 * or perturbed depths) and the element-n lane nelx, by the set-up's own expressions. */
template <class T>
struct LaneZGeo {
    T mz[3], gn[3], gz[2];
    DGR_HD T midz(int e) const { return mz[e]; }
    DGR_HD T gnn(int e) const { return gn[e]; }
    DGR_HD T gradz(int j) const { return gz[j]; }
};

template <class T, class Geo>
DGR_HD LaneZGeo<T> lane_zgeo(const Geo &geo, const double zvx[3], double nel, double nelx, double g)
{
    LaneZGeo<T> z;
    const T *tag = nullptr;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        z.mz[e] = lane(tag, geo(G_MIDZ + e), 0.5 * (zvx[e] + zvx[(e + 1) % 3]));
        /* per-element n only; the node-average n is not a parameter */
        z.gn[e] = nel >= 0.0 ? gnn_lane(tag, geo(G_GNN + e), g, nel, nelx) : T(geo(G_GNN + e));
    }
#pragma unroll
    for (int j = 0; j < 2; ++j)
        z.gz[j] = lane(tag, geo(G_GRADZ + j),
                       second(z.mz[0]) * geo(G_GP + j) + second(z.mz[1]) * geo(G_GP + 2 + j) +
                           second(z.mz[2]) * geo(G_GP + 4 + j));
    return z;
}

/* Reverse of the depth factors: mid-edge depths and the depth gradient to the vertices. */
template <class Geo>
DGR_HD void zgeo_rev(const Geo &geo, const double midzb[3], const double gradzb[2], double zvb[3])
{
    double mb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) mb[k] = midzb[k] + geo(G_GP + 2 * k) * gradzb[0] + geo(G_GP + 2 * k + 1) * gradzb[1];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        zvb[e] += 0.5 * mb[e];
        zvb[(e + 1) % 3] += 0.5 * mb[e];
    }
}

/* vertices of an edge: local edge k of its "in" element joins local vertices k, k+1 */
DGR_DEV void edge_vertices(const MeshDev &m, int el_in, int k_in, int &va, int &vb)
{
    va = m.el2v[k_in * m.ldE + el_in];
    vb = m.el2v[((k_in + 1) % 3) * m.ldE + el_in];
}

/* ================================================================ forward helpers ==== */

/* Limiter + PDop + status reading the pre-limiter values from R and writing the result to
 * S (limit_item with separate input and output arrays, used by the adjoint's recorded
 * recomputation; same arithmetic).  Without wet/dry the flags pass through unchanged, as
 * the plain step keeps using the same array. */
template <bool WD>
__global__ void __launch_bounds__(128) k_limit_to(MeshDev m, const double *__restrict__ R, double *__restrict__ S,
                                                  const double *__restrict__ bounds, const int *__restrict__ wd_in,
                                                  int *__restrict__ wd_out, DevClock *clk, double h0, double velzero,
                                                  int phase)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    DevClock *ck = clk;
    if (ck->done) return;
    const int ld = m.ldE;
    const int nd[3] = {m.el2v[el], m.el2v[ld + el], m.el2v[2 * ld + el]};
    const double zn[3] = {m.zn[nd[0]], m.zn[nd[1]], m.zn[nd[2]]};
    double w[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) w[v][k] = R[(3 * v + k) * ld + el];
    const int lb = m.ldN;
    const auto bnd = [bounds, lb, &nd](int v, int k, int is_min) { return bounds[(3 * is_min + v) * lb + nd[k]]; };
    LimitDecisions dec;
    limit_core<true, WD, double>(w, bnd, zn, h0, velzero, dec);
    if (WD && dec.code) atomicMin(&ck->err, err_key(ck->step, phase, dec.code, el));
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) S[(3 * v + k) * ld + el] = w[v][k];
    wd_out[el] = WD ? wd_status(w[0], zn, wd_in[el], h0) : wd_in[el];
}

/* Start of step n of a recorded run, every scenario: with replay, dt is the recorded one;
 * records each scenario's boundary-value time and dt of the step (histories [step][nscen]),
 * then clock_begin_body. */
static __global__ void __launch_bounds__(256) k_adj_clock_begin(DevClock *clk, int nscen, PhysParams p,
                                                         const int *__restrict__ bnd_edges,
                                                         const int *__restrict__ bnd_type,
                                                         const int *__restrict__ bnd_sid, int nbnd,
                                                         double *__restrict__ bzeta, double *__restrict__ bqn,
                                                         double *dt_hist, double *time_hist, int n, int replay)
{
    const size_t row = (size_t)n * nscen;
    for (int s = threadIdx.x; s < nscen; s += blockDim.x) {
        if (replay) {
            clk[s].dt = dt_hist[row + s];
            clk[s].dt_pending = 0;
        }
        time_hist[row + s] = clk[s].time;
    }
    __syncthreads();
    clock_begin_body(clk, nscen, p, bnd_edges, bnd_type, bnd_sid, nbnd, bzeta, bqn);
    /* thread s advanced scenario s's clock in clock_begin_body */
    if (!replay)
        for (int s = threadIdx.x; s < nscen; s += blockDim.x) dt_hist[row + s] = clk[s].dt;
}

/* boundary_conditions() at the recorded time of step n (each prescribed edge at its
 * scenario's time) */
static __global__ void __launch_bounds__(256) k_adj_forcing(const DevClock *clk, const double *__restrict__ time_hist, int n,
                                                     int nscen, const int *__restrict__ bnd_edges,
                                                     const int *__restrict__ bnd_type,
                                                     const int *__restrict__ bnd_sid, int nbnd,
                                                     double *__restrict__ bzeta, double *__restrict__ bqn)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nbnd) return;
    const int sid = bnd_sid ? bnd_sid[j] : 0;
    const DevClock *ck = clk + sid;
    const double zb2 = dgr_outflow_zeta(time_hist[(size_t)n * nscen + sid], ck->tide_on, ck->tide_amp, ck->tide_period);
    const int e = bnd_edges[j];
    const int tt = bnd_type[j];
    double zb = 0, qn = 0;
    if (tt == 1) { zb = DGR_BC1_ZETA; qn = DGR_BC1_QN; }
    else if (tt == 2) { zb = zb2; qn = DGR_BC2_QN; }
    else if (tt == 3) { zb = DGR_BC3_ZETA; qn = DGR_BC3_QN; }
    bzeta[e] = zb;
    bqn[e] = qn;
}

/* Gauge residuals of the state after step n: r_g = sum_k w_gk zeta_k(el_g) - target_g
 * (target null: 0), nw weights per gauge over the elevation planes 0..nw-1 (the three
 * midpoint values at p = 1, the six modes at p = 2).  One thread per gauge; the objective
 * is summed later in a fixed order. */
static __global__ void k_misfit(const double *__restrict__ S, int ld, int nw, int ng, const int *__restrict__ g_el,
                         const double *__restrict__ g_w, const double *__restrict__ target, double *__restrict__ resid)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
        const int el = g_el[g];
        double z = g_w[nw * g] * S[el];
        for (int k = 1; k < nw; ++k) z += g_w[nw * g + k] * S[(size_t)k * ld + el];
        resid[g] = target ? z - target[g] : z;
    }
}

/* J = sum_n sum_g r^2 into out[0] and, with rx: the tangent sum 2 r rx (squared = 0) or
 * the objective sum rx^2 of the perturbed lane (squared = 1) into out[1]; sequential for a
 * fixed order. */
static __global__ void k_misfit_sum(const double *__restrict__ resid, const double *__restrict__ rx, long long count,
                                    int squared, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double J = 0, J2 = 0;
    for (long long i = 0; i < count; ++i) {
        J += resid[i] * resid[i];
        if (rx) J2 += squared ? rx[i] * rx[i] : 2.0 * resid[i] * rx[i];
    }
    out[0] = J;
    out[1] = J2;
}

/* adjoint of the misfit of step n: lam(zeta_k) += 2 r_g w_gk at the gauges.  One thread per
 * gauge element (u_el, CSR u_ptr/u_g of its gauges in ascending order), so gauges that share
 * an element are added in a fixed order. */
static __global__ void k_misfit_rev(double *__restrict__ lam, int ld, int nw, int nu, const int *__restrict__ u_el,
                                    const int *__restrict__ u_ptr, const int *__restrict__ u_g,
                                    const double *__restrict__ g_w, const double *__restrict__ resid)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nu) return;
    const int el = u_el[u];
    for (int k = 0; k < nw; ++k) {
        double a = lam[(size_t)k * ld + el];
        for (int j = u_ptr[u]; j < u_ptr[u + 1]; ++j) {
            const int g = u_g[j];
            a += 2.0 * resid[g] * g_w[nw * g + k];
        }
        lam[(size_t)k * ld + el] = a;
    }
}

/* ==================================================================== tangent ==== */

/* Tangent (T = Dual) or frozen-decision perturbation (T = Pert) of the edge flux: the
 * "_x" arrays hold the second lane of their primal (tangents or perturbed values). */
template <bool WD, class T>
__global__ void __launch_bounds__(256) k_tlm_edge(MeshDev m, const double *__restrict__ S,
                                                  const double *__restrict__ Sx, const int *__restrict__ wd,
                                                  const double *__restrict__ bzeta, const double *__restrict__ bqn,
                                                  const double *__restrict__ zx, double *__restrict__ flux,
                                                  double *__restrict__ flux_x, double g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nf) return;
    const T *tag = nullptr;
    const int el_in = m.e_in[i], el_ex = m.e_ex[i], info = m.e_info[i];
    const int k_in = info & 3, k_ex = (info >> 2) & 3, bd = (info >> 4) & 7;
    const double nx = m.e_geo[i], ny = m.e_geo[m.ldF + i];
    const int ld = m.ldE;
    int va, vb;
    edge_vertices(m, el_in, k_in, va, vb);
    const T z_edge = lane(tag, m.e_geo[2 * m.ldF + i], 0.5 * (zx[va] + zx[vb]));
    const auto st = [S, Sx, ld, tag](int plane, int el) { return lane(tag, S[plane * ld + el], Sx[plane * ld + el]); };
    const T zi = st(k_in, el_in), qxi = st(3 + k_in, el_in), qyi = st(6 + k_in, el_in);
    T ze, qxe, qye;
    if (bd)
        ghost_state<T>(bd, nx, ny, zi, qxi, qyi, bzeta[i], bqn[i], T(0.0), ze, qxe, qye);
    else if (el_in == el_ex)
        ghost_state<T>(0, nx, ny, zi, qxi, qyi, 0.0, 0.0, st(k_ex, el_ex), ze, qxe, qye);
    else {
        ze = st(k_ex, el_ex);
        qxe = st(3 + k_ex, el_ex);
        qye = st(6 + k_ex, el_ex);
    }
    const int wdi = WD ? wd[el_in] : 1, wde = WD ? wd[el_ex] : 1;
    T fin[3], fex[3];
    int code;
    flux_core<T, WD>(zi, qxi, qyi, ze, qxe, qye, z_edge, nx, ny, wdi, wde, g, fin, fex, code, m.flux);
    const int lf = m.ldF;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        flux[k * lf + i] = val(fin[k]);
        flux_x[k * lf + i] = second(fin[k]);
        flux[(3 + k) * lf + i] = val(fex[k]);
        flux_x[(3 + k) * lf + i] = second(fex[k]);
    }
}

template <int MODE, class T>
__global__ void __launch_bounds__(128) k_tlm_element(MeshDev m, const double *__restrict__ S,
                                                     const double *__restrict__ Sx, const double *U,
                                                     const double *Ux, const int *__restrict__ wd,
                                                     const double *__restrict__ flux,
                                                     const double *__restrict__ flux_x,
                                                     const double *__restrict__ zx, const double *__restrict__ n_el,
                                                     const double *__restrict__ nelx, double *out, double *out_x,
                                                     double *__restrict__ avg, double *__restrict__ avg_x,
                                                     const DevClock *clk, double g, const double *__restrict__ dt_n)
{
    prefetch_geometry(m, blockIdx.x * blockDim.x, min((int)blockDim.x, m.ne - (int)(blockIdx.x * blockDim.x)));
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const T *tag = nullptr;
    const int sid = m.el_sid ? m.el_sid[el] : 0;
    const int ld = m.ldE;
    const double *G = m.geo + geo_offset(el, ld);
    const int gs = geo_stride(ld);
    T F[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * ld + el];
        const int e = ee >> 1, side = ee & 1;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const T f = lane(tag, flux[(3 * side + v) * m.ldF + e], flux_x[(3 * side + v) * m.ldF + e]);
            F[v][k] = side ? -f : f;
        }
    }
    T zr[3], qxr[3], qyr[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        zr[k] = lane(tag, S[k * ld + el], Sx[k * ld + el]);
        qxr[k] = lane(tag, S[(3 + k) * ld + el], Sx[(3 + k) * ld + el]);
        qyr[k] = lane(tag, S[(6 + k) * ld + el], Sx[(6 + k) * ld + el]);
    }
    const double local_g = (wd[el] == 0) ? 0.0 : g;
    const auto geo = [G, gs](int j) { return G[(size_t)j * gs]; };
    const double zvx[3] = {zx[m.el2v[el]], zx[m.el2v[ld + el]], zx[m.el2v[2 * ld + el]]};
    const LaneZGeo<T> zg = lane_zgeo<T>(geo, zvx, n_el ? n_el[el] : -1.0, nelx ? nelx[el] : 0.0, g);
    const auto uin = [U, Ux, ld, el, tag](int v, int k) {
        return lane(tag, U[(3 * v + k) * ld + el], Ux[(3 * v + k) * ld + el]);
    };
    T w[3][3], a[3];
    element_core<MODE, T>(F, zr, qxr, qyr, geo, zg, uin, local_g, clk[sid].rain, dt_n[sid], w, a);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            out[(3 * v + k) * ld + el] = val(w[v][k]);
            out_x[(3 * v + k) * ld + el] = second(w[v][k]);
        }
        avg[v * ld + el] = val(a[v]);
        avg_x[v * ld + el] = second(a[v]);
    }
}

static __global__ void __launch_bounds__(256) k_tlm_node(MeshDev m, const double *__restrict__ avg,
                                                  const double *__restrict__ avg_d, double *__restrict__ bounds,
                                                  double *__restrict__ bounds_d)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.nn) return;
    double mx[3] = {-99999, -99999, -99999}, mn[3] = {99999, 99999, 99999};
    double mxd[3] = {0, 0, 0}, mnd[3] = {0, 0, 0};
    for (int j = m.n2e_ptr[n]; j < m.n2e_ptr[n + 1]; ++j) {
        const int el = m.n2e[j];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double a = avg[v * m.ldE + el];
            if (a < mn[v]) {
                mn[v] = a;
                mnd[v] = avg_d[v * m.ldE + el];
            }
            if (a > mx[v]) {
                mx[v] = a;
                mxd[v] = avg_d[v * m.ldE + el];
            }
        }
    }
    const int l = m.ldN;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        bounds[v * l + n] = mx[v];
        bounds[(3 + v) * l + n] = mn[v];
        bounds_d[v * l + n] = mxd[v];
        bounds_d[(3 + v) * l + n] = mnd[v];
    }
}

template <bool WD, class T>
__global__ void __launch_bounds__(128) k_tlm_limit(MeshDev m, double *__restrict__ S, double *__restrict__ Sx,
                                                   const double *__restrict__ bounds,
                                                   const double *__restrict__ bounds_x,
                                                   const double *__restrict__ zx, const int *__restrict__ wd_in,
                                                   int *__restrict__ wd_out, double h0, double velzero)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const T *tag = nullptr;
    const int ld = m.ldE;
    const int nd[3] = {m.el2v[el], m.el2v[ld + el], m.el2v[2 * ld + el]};
    const T zn[3] = {lane(tag, m.zn[nd[0]], zx[nd[0]]), lane(tag, m.zn[nd[1]], zx[nd[1]]),
                     lane(tag, m.zn[nd[2]], zx[nd[2]])};
    T w[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) w[v][k] = lane(tag, S[(3 * v + k) * ld + el], Sx[(3 * v + k) * ld + el]);
    const int lb = m.ldN;
    const auto bnd = [bounds, bounds_x, lb, &nd, tag](int v, int k, int is_min) {
        const int idx = (3 * is_min + v) * lb + nd[k];
        return lane(tag, bounds[idx], bounds_x[idx]);
    };
    LimitDecisions dec;
    limit_core<true, WD, T>(w, bnd, zn, h0, velzero, dec);
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            S[(3 * v + k) * ld + el] = val(w[v][k]);
            Sx[(3 * v + k) * ld + el] = second(w[v][k]);
        }
    if (WD) {
        const double w0[3] = {val(w[0][0]), val(w[0][1]), val(w[0][2])};
        const double znv[3] = {val(zn[0]), val(zn[1]), val(zn[2])};
        wd_out[el] = wd_status(w0, znv, wd_in[el], h0);
    }
}

/* ==================================================================== adjoint ==== */

/* limiter + PDop reverse of one element */
template <bool WD>
__global__ void __launch_bounds__(128, DGR_ADJ_MINB_LIMIT) k_adj_limit(MeshDev m, const double *__restrict__ R,
                                                   const double *__restrict__ bounds,
                                                   const double *__restrict__ lamO, double *__restrict__ Rbar,
                                                   double *__restrict__ bbar, double *__restrict__ zvb, double h0,
                                                   double velzero)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE;
    const int nd[3] = {m.el2v[el], m.el2v[ld + el], m.el2v[2 * ld + el]};
    const double zn[3] = {m.zn[nd[0]], m.zn[nd[1]], m.zn[nd[2]]};
    double w[3][3], wb[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            w[v][k] = R[(3 * v + k) * ld + el];
            wb[v][k] = lamO[(3 * v + k) * ld + el];
        }
    const int lb = m.ldN;
    const auto bnd = [bounds, lb, &nd](int v, int k, int is_min) { return bounds[(3 * is_min + v) * lb + nd[k]]; };
    double bmaxb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, bminb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double znb[3] = {0, 0, 0};
    limit_core_rev<true, WD>(w, bnd, zn, h0, velzero, wb, bmaxb, bminb, znb);
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            Rbar[(3 * v + k) * ld + el] = wb[v][k];
            bbar[(6 * k + v) * ld + el] = bmaxb[v][k];
            bbar[(6 * k + 3 + v) * ld + el] = bminb[v][k];
        }
#pragma unroll
    for (int k = 0; k < 3; ++k) zvb[k * ld + el] += znb[k];
}

/* node bounds reverse: which element supplied each max/min, and the bound adjoints summed
 * over the elements around the node (in the node's element order) */
static __global__ void __launch_bounds__(256) k_adj_node(MeshDev m, const double *__restrict__ avg,
                                                  const double *__restrict__ bbar, double *__restrict__ bnode,
                                                  int *__restrict__ barg)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.nn) return;
    const int ld = m.ldE;
    double mx[3] = {-99999, -99999, -99999}, mn[3] = {99999, 99999, 99999};
    int imx[3] = {-1, -1, -1}, imn[3] = {-1, -1, -1};
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int j = m.n2e_ptr[n]; j < m.n2e_ptr[n + 1]; ++j) {
        const int el = m.n2e[j];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double a = avg[v * ld + el];
            if (a < mn[v]) {
                mn[v] = a;
                imn[v] = el;
            }
            if (a > mx[v]) {
                mx[v] = a;
                imx[v] = el;
            }
        }
        const int k = (m.el2v[el] == n) ? 0 : ((m.el2v[ld + el] == n) ? 1 : 2);
#pragma unroll
        for (int q = 0; q < 6; ++q) s[q] += bbar[(6 * k + q) * ld + el];
    }
    const int l = m.ldN;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        bnode[q * l + n] = s[q];
        barg[q * l + n] = q < 3 ? imx[q] : imn[q - 3];
    }
}

/* element reverse: RK combination, RHS, friction and bed terms.  Stage-input adjoint:
 * stage 1 (MODE_STAGE1, input u^n) adds into lamS = lamU; later stages write lamS and put
 * cu * (output adjoint) into the step-input adjoint lamU, written at the last stage
 * (u_accumulate = 0, where lamU's old content has been consumed) and added at the middle
 * stage of RK3 (u_accumulate = 1).  Also writes the per-edge-side flux adjoints and
 * accumulates the depth / Manning adjoints. */
template <int MODE>
__global__ void __launch_bounds__(128, DGR_ADJ_MINB_ELEMENT) k_adj_element(MeshDev m, const double *__restrict__ S,
                                                     const int *__restrict__ wd, const double *__restrict__ Rbar,
                                                     const double *__restrict__ bnode, const int *__restrict__ barg,
                                                     double *lamS, double *lamU, int u_accumulate,
                                                     double *__restrict__ fbar, double *__restrict__ zvb,
                                                     double *__restrict__ nbar, const double *__restrict__ n_el,
                                                     double g, const double *__restrict__ dt_n)
{
    prefetch_geometry(m, blockIdx.x * blockDim.x, min((int)blockDim.x, m.ne - (int)(blockIdx.x * blockDim.x)));
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE, lb = m.ldN;
    double ab[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int nd = m.el2v[k * ld + el];
#pragma unroll
        for (int q = 0; q < 6; ++q)
            if (barg[q * lb + nd] == el) ab[q % 3] += bnode[q * lb + nd];
    }
    double wb[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) wb[v][k] = Rbar[(3 * v + k) * ld + el] + ab[v] / 3;
    double zr[3], qxr[3], qyr[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        zr[k] = S[k * ld + el];
        qxr[k] = S[(3 + k) * ld + el];
        qyr[k] = S[(6 + k) * ld + el];
    }
    const double local_g = (wd[el] == 0) ? 0.0 : g;
    const double *G = m.geo + geo_offset(el, ld);
    const int gs = geo_stride(ld);
    const auto geo = [G, gs](int j) { return G[(size_t)j * gs]; };
    const PlaneZGeo zg{G, gs};
    double Fb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Sb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double midzb[3] = {0, 0, 0}, gnnb[3] = {0, 0, 0}, gradzb[2] = {0, 0};
    element_core_rev<MODE>(wb, zr, qxr, qyr, geo, zg, local_g, dt_n[m.el_sid ? m.el_sid[el] : 0], Fb, Sb, midzb, gnnb, gradzb);
    double cu, cs, cr;
    stage_coefficients(MODE, cu, cs, cr);
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int idx = (3 * v + k) * ld + el;
            if (MODE == MODE_STAGE1) {
                lamS[idx] += Sb[v][k];
            } else {
                lamS[idx] = Sb[v][k];
                lamU[idx] = (u_accumulate ? lamU[idx] : 0.0) + cu * wb[v][k];
            }
        }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * ld + el];
        const int e = ee >> 1, side = ee & 1;
#pragma unroll
        for (int v = 0; v < 3; ++v) fbar[(3 * side + v) * m.ldF + e] = side ? -Fb[v][k] : Fb[v][k];
    }
    double zv[3] = {0, 0, 0};
    zgeo_rev(geo, midzb, gradzb, zv);
#pragma unroll
    for (int k = 0; k < 3; ++k) zvb[k * ld + el] += zv[k];
    if (n_el && n_el[el] >= 0.0) nbar[el] += (gnnb[0] + gnnb[1] + gnnb[2]) * 2.0 * g * n_el[el];
}

/* edge reverse: Roe flux(es), ghost states; adds the trace adjoints into the slots of the
 * adjacent elements (each slot belongs to one edge side) and the mid-edge depth adjoint */
template <bool WD, int FT = -1>
__global__ void __launch_bounds__(DGR_ADJ_EDGE_BS, DGR_ADJ_MINB_EDGE) k_adj_edge(MeshDev m, const double *__restrict__ S, const int *__restrict__ wd,
                                                  const double *__restrict__ bzeta, const double *__restrict__ bqn,
                                                  const double *__restrict__ fbar, double *__restrict__ lamS,
                                                  double *__restrict__ zeb, double g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nf) return;
    const int el_in = m.e_in[i], el_ex = m.e_ex[i], info = m.e_info[i];
    const int k_in = info & 3, k_ex = (info >> 2) & 3, bd = (info >> 4) & 7;
    const double nx = m.e_geo[i], ny = m.e_geo[m.ldF + i], z_edge = m.e_geo[2 * m.ldF + i];
    const int ld = m.ldE;
    const double zi = S[k_in * ld + el_in], qxi = S[(3 + k_in) * ld + el_in], qyi = S[(6 + k_in) * ld + el_in];
    const bool boundary = bd || el_in == el_ex;
    const double bz = bd ? bzeta[i] : 0.0, bq = bd ? bqn[i] : 0.0;
    double ze, qxe, qye;
    if (boundary)
        ghost_state<double>(bd, nx, ny, zi, qxi, qyi, bz, bq, S[k_ex * ld + el_ex], ze, qxe, qye);
    else {
        ze = S[k_ex * ld + el_ex];
        qxe = S[(3 + k_ex) * ld + el_ex];
        qye = S[(6 + k_ex) * ld + el_ex];
    }
    const int wdi = WD ? wd[el_in] : 1, wde = WD ? wd[el_ex] : 1;
    const int lf = m.ldF;
    double finb[3], fexb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        finb[k] = fbar[k * lf + i];
        fexb[k] = boundary ? 0.0 : fbar[(3 + k) * lf + i]; /* no element gathers a boundary edge's ex side */
    }
    EdgeBar b = {0, 0, 0, 0, 0, 0, 0};
    flux_core_rev<WD>(zi, qxi, qyi, ze, qxe, qye, z_edge, nx, ny, wdi, wde, g, finb, fexb, b, FT >= 0 ? FT : m.flux);
    if (boundary) {
        ghost_state_rev(bd, nx, ny, bz, bq, b.ze, b.qxe, b.qye, b.zi, b.qxi, b.qyi);
    } else {
        lamS[k_ex * ld + el_ex] += b.ze;
        lamS[(3 + k_ex) * ld + el_ex] += b.qxe;
        lamS[(6 + k_ex) * ld + el_ex] += b.qye;
    }
    lamS[k_in * ld + el_in] += b.zi;
    lamS[(3 + k_in) * ld + el_in] += b.qxi;
    lamS[(6 + k_in) * ld + el_in] += b.qyi;
    zeb[i] += b.zed;
}

/* mid-edge depth adjoints to the vertex slots of each edge's "in" element */
static __global__ void __launch_bounds__(256) k_adj_zfold(MeshDev m, const double *__restrict__ zeb, double *__restrict__ zvb)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * ld + el];
        if (ee & 1) continue;
        const double h = 0.5 * zeb[ee >> 1];
        zvb[k * ld + el] += h;
        zvb[((k + 1) % 3) * ld + el] += h;
    }
}

/* vertex-slot depth adjoints to the nodes */
static __global__ void __launch_bounds__(256) k_adj_znode(MeshDev m, const double *__restrict__ zvb, double *__restrict__ zbar)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.nn) return;
    const int ld = m.ldE;
    double s = 0;
    for (int j = m.n2e_ptr[n]; j < m.n2e_ptr[n + 1]; ++j) {
        const int el = m.n2e[j];
        const int k = (m.el2v[el] == n) ? 0 : ((m.el2v[ld + el] == n) ? 1 : 2);
        s += zvb[k * ld + el];
    }
    zbar[n] = s;
}

/* z_edge of every edge from the node depths (after a bathymetry change) */
static __global__ void __launch_bounds__(256) k_edge_zsetup(MeshDev m, double *e_geo)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nf) return;
    int va, vb;
    edge_vertices(m, m.e_in[i], m.e_info[i] & 3, va, vb);
    e_geo[2 * m.ldF + i] = (m.zn[va] + m.zn[vb]) / 2;
}

}  // namespace dgr
