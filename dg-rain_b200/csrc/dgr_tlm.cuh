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

namespace dgr {

using ad::Dual;

/* Depth and Manning factors of one element as Duals: values from the geometry planes,
 * derivatives from the vertex-depth tangents and the element-n tangent. */
struct DualZGeo {
    Dual mz[3], gn[3], gz[2];
    DGR_HD Dual midz(int e) const { return mz[e]; }
    DGR_HD Dual gnn(int e) const { return gn[e]; }
    DGR_HD Dual gradz(int j) const { return gz[j]; }
};

template <class Geo>
DGR_HD DualZGeo dual_zgeo(const Geo &geo, const double zvd[3], double nel, double neld, double g)
{
    DualZGeo z;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        z.mz[e] = Dual(geo(G_MIDZ + e), 0.5 * (zvd[e] + zvd[(e + 1) % 3]));
        /* g n n: d = 2 g n dn (per-element n only) */
        z.gn[e] = Dual(geo(G_GNN + e), nel >= 0.0 ? 2.0 * g * nel * neld : 0.0);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j)
        z.gz[j] = Dual(geo(G_GRADZ + j),
                       z.mz[0].d * geo(G_GP + j) + z.mz[1].d * geo(G_GP + 2 + j) + z.mz[2].d * geo(G_GP + 4 + j));
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

/* Start of step n of a recorded run (single mesh): with replay, dt is the recorded one;
 * records the boundary-value time and dt of the step, then clock_begin_body. */
static __global__ void __launch_bounds__(256) k_adj_clock_begin(DevClock *clk, PhysParams p, const int *__restrict__ bnd_edges,
                                                         const int *__restrict__ bnd_type, int nbnd,
                                                         double *__restrict__ bzeta, double *__restrict__ bqn,
                                                         double *dt_hist, double *time_hist, int n, int replay)
{
    if (threadIdx.x == 0) {
        if (replay) {
            clk->dt = dt_hist[n];
            clk->dt_pending = 0;
        }
        time_hist[n] = clk->time;
    }
    __syncthreads();
    clock_begin_body(clk, 1, p, bnd_edges, bnd_type, nullptr, nbnd, bzeta, bqn);
    if (threadIdx.x == 0 && !replay) dt_hist[n] = clk->dt;
}

/* boundary_conditions() at the recorded time of step n */
static __global__ void __launch_bounds__(256) k_adj_forcing(const DevClock *clk, const double *__restrict__ time_hist, int n,
                                                     const int *__restrict__ bnd_edges,
                                                     const int *__restrict__ bnd_type, int nbnd,
                                                     double *__restrict__ bzeta, double *__restrict__ bqn)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nbnd) return;
    const double zb2 = dgr_outflow_zeta(time_hist[n], clk->tide_on, clk->tide_amp, clk->tide_period);
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
 * (target null: 0).  One warp; the objective is summed later in a fixed order. */
static __global__ void k_misfit(const double *__restrict__ S, int ld, int ng, const int *__restrict__ g_el,
                         const double *__restrict__ g_w, const double *__restrict__ target, double *__restrict__ resid)
{
    for (int g = threadIdx.x; g < ng; g += blockDim.x) {
        const int el = g_el[g];
        const double z = g_w[3 * g] * S[el] + g_w[3 * g + 1] * S[ld + el] + g_w[3 * g + 2] * S[2 * ld + el];
        resid[g] = target ? z - target[g] : z;
    }
}

/* J = sum_n sum_g r^2 and, with rd, dJ = sum 2 r rd; sequential for a fixed order. */
static __global__ void k_misfit_sum(const double *__restrict__ resid, const double *__restrict__ rd, long long count, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double J = 0, dJ = 0;
    for (long long i = 0; i < count; ++i) {
        J += resid[i] * resid[i];
        if (rd) dJ += 2.0 * resid[i] * rd[i];
    }
    out[0] = J;
    out[1] = dJ;
}

/* adjoint of the misfit of step n: lam(zeta) += 2 r_g w_gk at the gauges (gauges sharing an
 * element are taken one after another) */
static __global__ void k_misfit_rev(double *__restrict__ lam, int ld, int ng, const int *__restrict__ g_el,
                             const double *__restrict__ g_w, const double *__restrict__ resid)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int g = 0; g < ng; ++g) {
        const int el = g_el[g];
        const double r2 = 2.0 * resid[g];
        lam[el] += r2 * g_w[3 * g];
        lam[ld + el] += r2 * g_w[3 * g + 1];
        lam[2 * ld + el] += r2 * g_w[3 * g + 2];
    }
}

/* ==================================================================== tangent ==== */

template <bool WD>
__global__ void __launch_bounds__(256) k_tlm_edge(MeshDev m, const double *__restrict__ S,
                                                  const double *__restrict__ Sd, const int *__restrict__ wd,
                                                  const double *__restrict__ bzeta, const double *__restrict__ bqn,
                                                  const double *__restrict__ zd, double *__restrict__ flux,
                                                  double *__restrict__ flux_d, double g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nf) return;
    const int el_in = m.e_in[i], el_ex = m.e_ex[i], info = m.e_info[i];
    const int k_in = info & 3, k_ex = (info >> 2) & 3, bd = (info >> 4) & 7;
    const double nx = m.e_geo[i], ny = m.e_geo[m.ldF + i];
    const int ld = m.ldE;
    int va, vb;
    edge_vertices(m, el_in, k_in, va, vb);
    const Dual z_edge(m.e_geo[2 * m.ldF + i], 0.5 * (zd[va] + zd[vb]));
    const auto st = [S, Sd, ld](int plane, int el) { return Dual(S[plane * ld + el], Sd[plane * ld + el]); };
    const Dual zi = st(k_in, el_in), qxi = st(3 + k_in, el_in), qyi = st(6 + k_in, el_in);
    Dual ze, qxe, qye;
    if (bd)
        ghost_state<Dual>(bd, nx, ny, zi, qxi, qyi, bzeta[i], bqn[i], Dual(0.0), ze, qxe, qye);
    else if (el_in == el_ex)
        ghost_state<Dual>(0, nx, ny, zi, qxi, qyi, 0.0, 0.0, st(k_ex, el_ex), ze, qxe, qye);
    else {
        ze = st(k_ex, el_ex);
        qxe = st(3 + k_ex, el_ex);
        qye = st(6 + k_ex, el_ex);
    }
    const int wdi = WD ? wd[el_in] : 1, wde = WD ? wd[el_ex] : 1;
    Dual fin[3], fex[3];
    int code;
    flux_core<Dual, WD>(zi, qxi, qyi, ze, qxe, qye, z_edge, nx, ny, wdi, wde, g, fin, fex, code);
    const int lf = m.ldF;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        flux[k * lf + i] = fin[k].v;
        flux_d[k * lf + i] = fin[k].d;
        flux[(3 + k) * lf + i] = fex[k].v;
        flux_d[(3 + k) * lf + i] = fex[k].d;
    }
}

template <int MODE>
__global__ void __launch_bounds__(128) k_tlm_element(MeshDev m, const double *__restrict__ S,
                                                     const double *__restrict__ Sd, const double *U,
                                                     const double *Ud, const int *__restrict__ wd,
                                                     const double *__restrict__ flux,
                                                     const double *__restrict__ flux_d,
                                                     const double *__restrict__ zd, const double *__restrict__ n_el,
                                                     const double *__restrict__ neld, double *out, double *out_d,
                                                     double *__restrict__ avg, double *__restrict__ avg_d,
                                                     const DevClock *clk, double g, const double *dt_hist, int n)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE;
    const double *G = m.geo + el;
    Dual F[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * ld + el];
        const int e = ee >> 1, side = ee & 1;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const Dual f(flux[(3 * side + v) * m.ldF + e], flux_d[(3 * side + v) * m.ldF + e]);
            F[v][k] = side ? -f : f;
        }
    }
    Dual zr[3], qxr[3], qyr[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        zr[k] = Dual(S[k * ld + el], Sd[k * ld + el]);
        qxr[k] = Dual(S[(3 + k) * ld + el], Sd[(3 + k) * ld + el]);
        qyr[k] = Dual(S[(6 + k) * ld + el], Sd[(6 + k) * ld + el]);
    }
    const double local_g = (wd[el] == 0) ? 0.0 : g;
    const auto geo = [G, ld](int j) { return G[(size_t)j * ld]; };
    const double zvd[3] = {zd[m.el2v[el]], zd[m.el2v[ld + el]], zd[m.el2v[2 * ld + el]]};
    const DualZGeo zg = dual_zgeo(geo, zvd, n_el ? n_el[el] : -1.0, neld ? neld[el] : 0.0, g);
    const auto uin = [U, Ud, ld, el](int v, int k) {
        return Dual(U[(3 * v + k) * ld + el], Ud[(3 * v + k) * ld + el]);
    };
    Dual w[3][3], a[3];
    element_core<MODE, Dual>(F, zr, qxr, qyr, geo, zg, uin, local_g, clk->rain, dt_hist[n], w, a);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            out[(3 * v + k) * ld + el] = w[v][k].v;
            out_d[(3 * v + k) * ld + el] = w[v][k].d;
        }
        avg[v * ld + el] = a[v].v;
        avg_d[v * ld + el] = a[v].d;
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

template <bool WD>
__global__ void __launch_bounds__(128) k_tlm_limit(MeshDev m, double *__restrict__ S, double *__restrict__ Sd,
                                                   const double *__restrict__ bounds,
                                                   const double *__restrict__ bounds_d,
                                                   const double *__restrict__ zd, const int *__restrict__ wd_in,
                                                   int *__restrict__ wd_out, double h0, double velzero)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE;
    const int nd[3] = {m.el2v[el], m.el2v[ld + el], m.el2v[2 * ld + el]};
    const Dual zn[3] = {Dual(m.zn[nd[0]], zd[nd[0]]), Dual(m.zn[nd[1]], zd[nd[1]]), Dual(m.zn[nd[2]], zd[nd[2]])};
    Dual w[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) w[v][k] = Dual(S[(3 * v + k) * ld + el], Sd[(3 * v + k) * ld + el]);
    const int lb = m.ldN;
    const auto bnd = [bounds, bounds_d, lb, &nd](int v, int k, int is_min) {
        const int idx = (3 * is_min + v) * lb + nd[k];
        return Dual(bounds[idx], bounds_d[idx]);
    };
    LimitDecisions dec;
    limit_core<true, WD, Dual>(w, bnd, zn, h0, velzero, dec);
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            S[(3 * v + k) * ld + el] = w[v][k].v;
            Sd[(3 * v + k) * ld + el] = w[v][k].d;
        }
    if (WD) {
        const double w0[3] = {w[0][0].v, w[0][1].v, w[0][2].v};
        const double znv[3] = {zn[0].v, zn[1].v, zn[2].v};
        wd_out[el] = wd_status(w0, znv, wd_in[el], h0);
    }
}

/* ==================================================================== adjoint ==== */

/* limiter + PDop reverse of one element */
template <bool WD>
__global__ void __launch_bounds__(128) k_adj_limit(MeshDev m, const double *__restrict__ R,
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

/* element reverse: RK combination, RHS, friction and bed terms; writes the stage-input
 * adjoint (stage 2: lamS = adjoint of the stage input, lamU = 0.5 * adjoint of the output;
 * stage 1: lamS += adjoint of the stage input), the per-edge-side flux adjoints and the
 * depth / Manning adjoints */
template <int MODE>
__global__ void __launch_bounds__(128) k_adj_element(MeshDev m, const double *__restrict__ S,
                                                     const int *__restrict__ wd, const double *__restrict__ Rbar,
                                                     const double *__restrict__ bnode, const int *__restrict__ barg,
                                                     double *lamS, double *lamU, double *__restrict__ fbar,
                                                     double *__restrict__ zvb, double *__restrict__ nbar,
                                                     const double *__restrict__ n_el, double g,
                                                     const double *__restrict__ dt_hist, int n)
{
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
    const double *G = m.geo + el;
    const auto geo = [G, ld](int j) { return G[(size_t)j * ld]; };
    const PlaneZGeo zg{G, ld};
    double Fb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Sb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double midzb[3] = {0, 0, 0}, gnnb[3] = {0, 0, 0}, gradzb[2] = {0, 0};
    element_core_rev<MODE>(wb, zr, qxr, qyr, geo, zg, local_g, dt_hist[n], Fb, Sb, midzb, gnnb, gradzb);
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int idx = (3 * v + k) * ld + el;
            if (MODE == MODE_STAGE2) {
                lamS[idx] = Sb[v][k];
                lamU[idx] = 0.5 * wb[v][k];
            } else {
                lamS[idx] += Sb[v][k];
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
template <bool WD>
__global__ void __launch_bounds__(256) k_adj_edge(MeshDev m, const double *__restrict__ S, const int *__restrict__ wd,
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
    flux_core_rev<WD>(zi, qxi, qyi, ze, qxe, qye, z_edge, nx, ny, wdi, wde, g, finb, fexb, b);
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
