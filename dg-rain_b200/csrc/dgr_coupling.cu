/*
 * Channel <-> junction coupling of ChanNet (ChanNet/internal_BC.c:17-218) on the device.
 *
 * A channel end is the first node of a 1D channel (its "inflow" list of junction edges) or
 * its last node (the "outflow" list).  One coupling pass, for every end and every edge of
 * its list in list order:
 *   junction side (:85-95, :183-190): the edge's mid-edge state of its element
 *     EdgtoEls[2e], depth juncH = zeta + z_mid and normal discharge Qn = Qx nx + Qy ny;
 *     the end's sums  area += len * juncH,  qn += Qn * len;
 *   the edge's prescribed values (:99-108, :193-203), from the channel's own trace at the
 *     junction node (A, Q):  bzeta = A / (n len) - z_mid,  bQn = +-Q / (n len);
 * and then the channel's ghost trace at that node (:110-114, :205-212): A = area, Q = qn
 * (inflow) or -qn (outflow).  The edges' lengths, normals and mid-edge depths are formed
 * once, with internal_BC's own expressions, by k_cpl_setup; each pass is one thread per
 * end summing its edges in order, so the sums are the reference's bit for bit.
 *
 * The channels' 1D solver is the caller's: the pass takes each end's (A, Q) and returns
 * its ghost (A, Q).  Each coupled edge must be a prescribed boundary edge of the mesh and
 * belong to one end (the reference would let a later end overwrite an earlier one).
 */
#include <algorithm>
#include <vector>

#include "dgr_internal.cuh"
#include "dgr_ptr.h"

using namespace dgr;

namespace {

/* length, unit normal, mid-edge depth and state slot (k * ldE + el) of coupled edge j */
__global__ void __launch_bounds__(128) k_cpl_setup(int n, int ldE, const int *__restrict__ edges,
                                                   const int *__restrict__ e_in, const int *__restrict__ e_info,
                                                   const int *__restrict__ el2v, const double *__restrict__ x,
                                                   const double *__restrict__ y, const double *__restrict__ z,
                                                   int *__restrict__ slot, double *__restrict__ geo)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int e = edges[j];
    const int el = e_in[e], k = e_info[e] & 3; /* EdgtoEls[2e] and its matched local edge */
    const int a = el2v[el], b = el2v[ldE + el], c = el2v[2 * ldE + el];
    const double xa = x[a], xb = x[b], xc = x[c], ya = y[a], yb = y[b], yc = y[c];
    double x0, x1, y0, y1, len;
    int p, q;
    if (k == 0) {
        x0 = xa; x1 = xb; y0 = ya; y1 = yb; p = a; q = b;
        len = sqrt((xa - xb) * (xa - xb) + (ya - yb) * (ya - yb));
    } else if (k == 1) {
        x0 = xb; x1 = xc; y0 = yb; y1 = yc; p = b; q = c;
        len = sqrt((xb - xc) * (xb - xc) + (yb - yc) * (yb - yc));
    } else {
        x0 = xc; x1 = xa; y0 = yc; y1 = ya; p = c; q = a;
        len = sqrt((xa - xc) * (xa - xc) + (ya - yc) * (ya - yc));
    }
    const double jac = (xb - xa) * (yc - ya) - (xc - xa) * (yb - ya);
    const int s = (jac < 0) ? -1 : (jac == 0 ? 0 : 1); /* sign() of ChanNet/mathfunctions.c:17-25 */
    slot[j] = k * ldE + el;
    geo[j] = len;
    geo[n + j] = s * (y1 - y0) / len;
    geo[2 * n + j] = s * (x0 - x1) / len;
    geo[3 * n + j] = 0.5 * (z[p] + z[q]);
}

/* one coupling pass: the ends' traces in, their ghosts out (nends each) */
__global__ void __launch_bounds__(128) k_cpl_pass(int nends, int nedges, int ldE, const int *__restrict__ ptr,
                                                  const int *__restrict__ outflow, const int *__restrict__ edges,
                                                  const int *__restrict__ slot, const double *__restrict__ geo,
                                                  const double *__restrict__ U, double *__restrict__ bzeta,
                                                  double *__restrict__ bqn, const double *a_in, const double *q_in,
                                                  double *a_ghost, double *q_ghost)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nends) return;
    const int out = outflow[c];
    const int j0 = ptr[c], j1 = ptr[c + 1], n = j1 - j0;
    const double a_end = a_in[c], q_end = q_in[c];
    double area = 0, qn_sum = 0;
    for (int j = j0; j < j1; ++j) {
        const double len = geo[j], nx = geo[nedges + j], ny = geo[2 * nedges + j], zmid = geo[3 * nedges + j];
        const int s = slot[j];
        const double h = U[s] + zmid;
        const double qn = U[3 * ldE + s] * nx + U[6 * ldE + s] * ny;
        area += len * h;
        qn_sum += qn * len;
        const int e = edges[j];
        bzeta[e] = a_end / (n * len) - zmid;
        bqn[e] = out ? -q_end / (n * len) : q_end / (n * len);
    }
    a_ghost[c] = area;
    q_ghost[c] = out ? -qn_sum : qn_sum;
}

#define CPL_TRY(x)           \
    do {                     \
        const int r_ = (x);  \
        if (r_) {            \
            free_coupling(c); \
            return r_;       \
        }                    \
    } while (0)

void free_coupling(dgr_ctx *c)
{
    void *ptrs[] = {c->cpl_ptr, c->cpl_out, c->cpl_edge, c->cpl_slot, c->cpl_geo, c->cpl_io};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (c->h_cpl_io) cudaFreeHost(c->h_cpl_io);
    c->cpl_ptr = c->cpl_out = c->cpl_edge = c->cpl_slot = nullptr;
    c->cpl_geo = c->cpl_io = c->h_cpl_io = nullptr;
    c->cpl_nends = c->cpl_nedges = 0;
}

}  // namespace

void coupling_release(dgr_ctx *c) { free_coupling(c); }

extern "C" int dgr_set_channel_ends(dgr_ctx *c, int nends, const int *end_ptr, const int *end_edges,
                                    const int *end_outflow)
{
    if (!c || c->nscen != 1 || c->p.order != 1 || nends < 0) return DGR_ERR_INVALID;
    if (nends > 0 && (!end_ptr || !end_edges || !end_outflow)) return DGR_ERR_INVALID;
    /* validate on the host: lists ordered, non-empty, prescribed boundary edges, each edge once */
    std::vector<char> prescribed(c->nf, 0), used(c->nf, 0);
    for (int e : c->h_bnd)
        if (e >= 0 && e < c->nf) prescribed[e] = 1;
    if (nends > 0 && end_ptr[0] != 0) return DGR_ERR_INVALID;
    for (int k = 0; k < nends; ++k) {
        if (end_ptr[k + 1] <= end_ptr[k]) return DGR_ERR_INVALID;
        if (end_outflow[k] != 0 && end_outflow[k] != 1) return DGR_ERR_INVALID;
        for (int j = end_ptr[k]; j < end_ptr[k + 1]; ++j) {
            const int e = end_edges[j];
            if (e < 0 || e >= c->nf || !prescribed[e] || used[e]) return DGR_ERR_INVALID;
            used[e] = 1;
        }
    }
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    free_coupling(c);
    if (nends == 0) return DGR_OK;
    const int ne = end_ptr[nends];
    CPL_TRY(dalloc(&c->cpl_ptr, (size_t)nends + 1));
    CPL_TRY(dalloc(&c->cpl_out, (size_t)nends));
    CPL_TRY(dalloc(&c->cpl_edge, (size_t)ne));
    CPL_TRY(dalloc(&c->cpl_slot, (size_t)ne));
    CPL_TRY(dalloc(&c->cpl_geo, 4 * (size_t)ne));
    CPL_TRY(dalloc(&c->cpl_io, 4 * (size_t)nends));
    CK(cudaHostAlloc((void **)&c->h_cpl_io, 4 * (size_t)nends * sizeof(double), cudaHostAllocDefault));
    CK(cudaMemcpy(c->cpl_ptr, end_ptr, sizeof(int) * (nends + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->cpl_out, end_outflow, sizeof(int) * nends, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->cpl_edge, end_edges, sizeof(int) * ne, cudaMemcpyHostToDevice));
    k_cpl_setup<<<blocks(ne, 128), 128, 0, c->stream>>>(ne, c->ldE, c->cpl_edge, c->e_in, c->e_info, c->el2v, c->x,
                                                        c->y, c->zn, c->cpl_slot, c->cpl_geo);
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    c->cpl_nends = nends;
    c->cpl_nedges = ne;
    return DGR_OK;
}

extern "C" int dgr_couple_channel_ends(dgr_ctx *c, const double *a_end, const double *q_end, double *a_ghost,
                                       double *q_ghost)
{
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    const int n = c->cpl_nends;
    if (n == 0) return DGR_OK;
    if (!a_end || !q_end || !a_ghost || !q_ghost) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    CK(cudaStreamSynchronize(s)); /* the pinned mirror may still feed the previous pass */
    std::copy(a_end, a_end + n, c->h_cpl_io);
    std::copy(q_end, q_end + n, c->h_cpl_io + n);
    CK(cudaMemcpyAsync(c->cpl_io, c->h_cpl_io, 2 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
    double *io = c->cpl_io;
    k_cpl_pass<<<blocks(n, 128), 128, 0, s>>>(n, c->cpl_nedges, c->ldE, c->cpl_ptr, c->cpl_out, c->cpl_edge,
                                              c->cpl_slot, c->cpl_geo, c->U, c->bzeta, c->bqn, io, io + n,
                                              io + 2 * n, io + 3 * n);
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_cpl_io + 2 * n, c->cpl_io + 2 * n, 2 * (size_t)n * sizeof(double),
                       cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::copy(c->h_cpl_io + 2 * n, c->h_cpl_io + 3 * n, a_ghost);
    std::copy(c->h_cpl_io + 3 * n, c->h_cpl_io + 4 * n, q_ghost);
    return DGR_OK;
}

extern "C" int dgr_couple_channel_ends_device(dgr_ctx *c, const double *d_a_end, const double *d_q_end,
                                              double *d_a_ghost, double *d_q_ghost)
{
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    const int n = c->cpl_nends;
    if (n == 0) return DGR_OK;
    if (!d_a_end || !d_q_end || !d_a_ghost || !d_q_ghost) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    for (const void *p : {(const void *)d_a_end, (const void *)d_q_end, (const void *)d_a_ghost,
                          (const void *)d_q_ghost})
        if (!dgr_device_addressable(p, c->device)) return DGR_ERR_INVALID; /* before any launch */
    k_cpl_pass<<<blocks(n, 128), 128, 0, c->stream>>>(n, c->cpl_nedges, c->ldE, c->cpl_ptr, c->cpl_out,
                                                      c->cpl_edge, c->cpl_slot, c->cpl_geo, c->U, c->bzeta, c->bqn,
                                                      d_a_end, d_q_end, d_a_ghost, d_q_ghost);
    c->launches++;
    CK(cudaGetLastError());
    return DGR_OK;
}

extern "C" int dgr_get_stream(dgr_ctx *c, void **stream)
{
    if (!c || !stream) return DGR_ERR_INVALID;
    *stream = (void *)c->stream;
    return DGR_OK;
}

extern "C" int dgr_get_boundary(dgr_ctx *c, double *bzeta, double *bQn)
{
    if (!c || c->nscen != 1 || !bzeta || !bQn) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaMemcpy(bzeta, c->bzeta, sizeof(double) * c->nf, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(bQn, c->bqn, sizeof(double) * c->nf, cudaMemcpyDeviceToHost));
    return DGR_OK;
}
