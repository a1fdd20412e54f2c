/*
 * Device context and C ABI of include/dgrain.h (the part that needs CUDA).
 *
 * Step orchestration (wet/dry on; the order of ChanNet/time_evolution.c:218-427 around
 * the 2DCode operators):
 *
 *   [wetDryStatus2D on U into WA, only when the flags are stale]
 *   stage 1: edge(U, WA) -> element(U -> W) -> node bounds -> limit+PDop(W), WB = status(W, WA)
 *   stage 2: edge(W, WB) -> element(W, U -> U) -> node bounds -> limit+PDop(U), WA = status(U, WB)
 *
 * The last status call is the one the reference makes at the start of the next step;
 * doing it here saves a launch.  The reference's global WD after a step is WB, which is
 * what dgr_download_state returns.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/dgrain.h"
#include "dgr_kernels.cuh"

using namespace dgr;

static thread_local char g_cuda_err[256] = "";

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            snprintf(g_cuda_err, sizeof g_cuda_err, "%s:%d %s: %s", __FILE__, __LINE__, #call, \
                     cudaGetErrorString(e_));                                                 \
            return DGR_ERR_CUDA;                                                              \
        }                                                                                     \
    } while (0)

extern "C" const char *dgr_last_cuda_error(void) { return g_cuda_err; }

static int pad32(int n) { return (n + 31) & ~31; }

struct dgr_ctx {
    dgr_params p;
    int device;
    int ne, nn, nf, nbnd;
    int ldE, ldF, ldN;
    double min_edge;
    cudaStream_t stream;
    cudaEvent_t ev0, ev1;
    /* mesh */
    double *x, *y, *zn, *nfric, *n_el;
    int *el2v_aos, *el2v, *elem_edge, *e_in, *e_ex, *e_info, *n2e_ptr, *n2e, *bnd_edges, *bnd_type;
    int *bdry;
    double *e_geo, *geo;
    /* state and work */
    double *U, *W, *flux, *avg, *bounds, *bzeta, *bqn, *bstage;
    int *wdA, *wdB;
    int *dec;  /* [4][ne]: limit s0, pdop s0, limit s1, pdop s1 */
    DevClock *clk;
    DevClock *h_clk; /* pinned mirror */
    double *h_stage; /* pinned staging for compact boundary values */
    std::vector<int> *h_bnd; /* prescribed edge ids, host copy */
    int wd_fresh;    /* WA already holds the status for the next step */
    int wd_cur_is_B; /* reference-semantic WD lives in WB */
    long long launches;
    double last_ms;
    cudaGraph_t graph;
    cudaGraphExec_t graph_exec;
    int graph_kernels;
};

static MeshDev mesh_dev(const dgr_ctx *c)
{
    MeshDev m;
    m.ne = c->ne;
    m.nn = c->nn;
    m.nf = c->nf;
    m.ldE = c->ldE;
    m.ldF = c->ldF;
    m.ldN = c->ldN;
    m.el2v = c->el2v;
    m.elem_edge = c->elem_edge;
    m.e_in = c->e_in;
    m.e_ex = c->e_ex;
    m.e_info = c->e_info;
    m.e_geo = c->e_geo;
    m.geo = c->geo;
    m.n2e_ptr = c->n2e_ptr;
    m.n2e = c->n2e;
    m.zn = c->zn;
    m.minlen_cfl_unused = nullptr;
    return m;
}

static PhysParams phys(const dgr_ctx *c)
{
    PhysParams q;
    q.g = c->p.g;
    q.h0 = c->p.H0;
    q.velzero = c->p.VELZERO;
    q.rain = c->p.rain;
    q.cfl = c->p.cfl;
    q.dt0 = c->p.dt0;
    q.min_edge = c->min_edge;
    q.tide_amp = c->p.tide_amp;
    q.tide_period = c->p.tide_period;
    q.tide_on = c->p.tide_on;
    return q;
}

static double bits_to_double(unsigned long long b)
{
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
}

static unsigned blocks(int n, int t) { return (unsigned)((n + t - 1) / t); }

extern "C" int dgr_params_default(dgr_params *p)
{
    if (!p) return DGR_ERR_INVALID;
    memset(p, 0, sizeof *p);
    p->g = 9.81;
    p->H0 = 1e-3;
    p->VELZERO = 1e-2;
    p->cfl = 0.1;
    p->dt0 = 1e-7;
    p->wet_dry = 1;
    p->tide_on = 0;
    p->tide_amp = 0.5;
    p->tide_period = 44712.0;
    p->rain = 0.0;
    p->device = 0;
    p->record_decisions = 0;
    return DGR_OK;
}

template <class T>
static int dalloc(T **p, size_t n)
{
    *p = nullptr;
    CK(cudaMalloc((void **)p, (n ? n : 1) * sizeof(T)));
    return DGR_OK;
}

static void release(dgr_ctx *c)
{
    if (!c) return;
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    void *ptrs[] = {c->x, c->y, c->zn, c->nfric, c->n_el, c->el2v_aos, c->el2v, c->elem_edge, c->e_in,
                    c->e_ex, c->e_info, c->n2e_ptr, c->n2e, c->bnd_edges, c->bnd_type, c->bdry, c->e_geo,
                    c->geo, c->U, c->W, c->flux, c->avg, c->bounds, c->bzeta, c->bqn, c->bstage, c->wdA, c->wdB,
                    c->dec, c->clk};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (c->h_clk) cudaFreeHost(c->h_clk);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c->h_bnd;
    delete c;
}

static int upload_geometry(dgr_ctx *c)
{
    const dim3 t(128);
    k_element_setup<<<blocks(c->ne, 128), t, 0, c->stream>>>(c->ne, c->ldE, c->el2v_aos, c->x, c->y, c->zn,
                                                             c->nfric, c->n_el, c->p.g, c->el2v, c->geo);
    c->launches++;
    CK(cudaGetLastError());
    return DGR_OK;
}

static int check_mesh_view(const dgr_mesh_view *m)
{
    if (!m || m->num_el <= 0 || m->num_nodes <= 0 || m->num_edges <= 0) return DGR_ERR_INVALID;
    if (!m->x_coord || !m->y_coord || !m->z || !m->nFriction || !m->EltoVert || !m->EdgtoEls ||
        !m->EdgtoVert || !m->BdryPrescribed)
        return DGR_ERR_INVALID;
    if ((long long)m->num_edges >= (1LL << 30) || (long long)m->num_el >= (1LL << 30)) return DGR_ERR_TOO_LARGE;
    for (long long i = 0; i < 3LL * m->num_el; ++i)
        if (m->EltoVert[i] < 0 || m->EltoVert[i] >= m->num_nodes) return DGR_ERR_MESH;
    for (long long i = 0; i < 2LL * m->num_edges; ++i) {
        if (m->EdgtoEls[i] < 0 || m->EdgtoEls[i] >= m->num_el) return DGR_ERR_MESH;
        if (m->EdgtoVert[i] < 0 || m->EdgtoVert[i] >= m->num_nodes) return DGR_ERR_MESH;
    }
    for (int i = 0; i < m->num_edges; ++i)
        if (m->BdryPrescribed[i] < 0 || m->BdryPrescribed[i] > 3) return DGR_ERR_MESH;
    return DGR_OK;
}

#define TRY(x)              \
    do {                    \
        int r_ = (x);       \
        if (r_) {           \
            release(c);     \
            return r_;      \
        }                   \
    } while (0)

extern "C" int dgr_create(const dgr_mesh_view *m, const dgr_params *params, dgr_ctx **out)
{
    if (!out) return DGR_ERR_INVALID;
    *out = nullptr;
    int rc = check_mesh_view(m);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        snprintf(g_cuda_err, sizeof g_cuda_err, "no CUDA device visible");
        return DGR_ERR_NO_DEVICE;
    }
    dgr_ctx *c = new dgr_ctx();
    memset((void *)c, 0, sizeof *c);
    if (params)
        c->p = *params;
    else
        dgr_params_default(&c->p);
    c->device = c->p.device;
    if (c->device < 0 || c->device >= ndev) {
        release(c);
        return DGR_ERR_INVALID;
    }
    TRY(cudaSetDevice(c->device) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    c->ne = m->num_el;
    c->nn = m->num_nodes;
    c->nf = m->num_edges;
    c->ldE = pad32(c->ne);
    c->ldF = pad32(c->nf);
    c->ldN = pad32(c->nn);
    c->min_edge = m->minEdgLength;
    TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaEventCreate(&c->ev0) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaEventCreate(&c->ev1) == cudaSuccess ? 0 : DGR_ERR_CUDA);

    const size_t ne = c->ne, nn = c->nn, nf = c->nf, lE = c->ldE, lF = c->ldF, lN = c->ldN;
    TRY(dalloc(&c->x, nn));
    TRY(dalloc(&c->y, nn));
    TRY(dalloc(&c->zn, nn));
    TRY(dalloc(&c->nfric, nn));
    TRY(dalloc(&c->el2v_aos, 3 * ne));
    TRY(dalloc(&c->el2v, 3 * lE));
    TRY(dalloc(&c->elem_edge, 3 * lE));
    TRY(dalloc(&c->e_in, nf));
    TRY(dalloc(&c->e_ex, nf));
    TRY(dalloc(&c->e_info, nf));
    TRY(dalloc(&c->bdry, nf));
    TRY(dalloc(&c->e_geo, 3 * lF));
    TRY(dalloc(&c->geo, (size_t)NG * lE));
    TRY(dalloc(&c->U, 9 * lE));
    TRY(dalloc(&c->W, 9 * lE));
    TRY(dalloc(&c->flux, 6 * lF));
    TRY(dalloc(&c->avg, 3 * lE));
    TRY(dalloc(&c->bounds, 6 * lN));
    TRY(dalloc(&c->bzeta, nf));
    TRY(dalloc(&c->bqn, nf));
    TRY(dalloc(&c->wdA, ne));
    TRY(dalloc(&c->wdB, ne));
    TRY(dalloc(&c->dec, 4 * ne));
    TRY(dalloc(&c->clk, 1));
    TRY(cudaHostAlloc((void **)&c->h_clk, sizeof(DevClock), cudaHostAllocDefault) == cudaSuccess ? 0 : DGR_ERR_CUDA);

    cudaStream_t s = c->stream;
    TRY(cudaMemcpyAsync(c->x, m->x_coord, nn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemcpyAsync(c->y, m->y_coord, nn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemcpyAsync(c->zn, m->z, nn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemcpyAsync(c->nfric, m->nFriction, nn * 8, cudaMemcpyHostToDevice, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemcpyAsync(c->el2v_aos, m->EltoVert, 3 * ne * 4, cudaMemcpyHostToDevice, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemcpyAsync(c->bdry, m->BdryPrescribed, nf * 4, cudaMemcpyHostToDevice, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemsetAsync(c->elem_edge, 0xff, 3 * lE * 4, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemsetAsync(c->bzeta, 0, nf * 8, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemsetAsync(c->bqn, 0, nf * 8, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemsetAsync(c->U, 0, 9 * lE * 8, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemsetAsync(c->W, 0, 9 * lE * 8, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemsetAsync(c->dec, 0, 4 * ne * 4, s) == cudaSuccess ? 0 : DGR_ERR_CUDA);

    /* connectivity arrays go through a temporary device copy */
    int *d_ed2el = nullptr, *d_ed2v = nullptr, *d_bad = nullptr;
    TRY(dalloc(&d_ed2el, 2 * nf));
    TRY(dalloc(&d_ed2v, 2 * nf));
    TRY(dalloc(&d_bad, 1));
    int big = 0x7fffffff;
    cudaMemcpyAsync(d_ed2el, m->EdgtoEls, 2 * nf * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_ed2v, m->EdgtoVert, 2 * nf * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_bad, &big, 4, cudaMemcpyHostToDevice, s);
    k_edge_setup<<<blocks(c->nf, 256), 256, 0, s>>>(c->nf, c->ldE, c->ldF, d_ed2el, d_ed2v, c->el2v_aos, c->bdry,
                                                     c->x, c->y, c->zn, c->e_in, c->e_ex, c->e_info, c->e_geo,
                                                     c->elem_edge, d_bad);
    c->launches++;
    TRY(upload_geometry(c));
    int bad = 0;
    std::vector<int> ee(3 * lE);
    cudaMemcpyAsync(&bad, d_bad, 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(ee.data(), c->elem_edge, 3 * lE * 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e1 = cudaStreamSynchronize(s);
    cudaFree(d_ed2el);
    cudaFree(d_ed2v);
    cudaFree(d_bad);
    if (e1 != cudaSuccess) {
        snprintf(g_cuda_err, sizeof g_cuda_err, "setup: %s", cudaGetErrorString(e1));
        release(c);
        return DGR_ERR_CUDA;
    }
    if (bad != 0x7fffffff) {
        release(c);
        return DGR_ERR_EDGE_MATCH;
    }
    for (int k = 0; k < 3; ++k)
        for (size_t el = 0; el < ne; ++el)
            if (ee[k * lE + el] < 0) {
                release(c);
                return DGR_ERR_MESH; /* an element edge that no EdgtoEls entry covers */
            }

    /* node -> element lists, ascending element order */
    std::vector<int> ptr(nn + 1, 0), lst(3 * ne);
    for (size_t i = 0; i < 3 * ne; ++i) ptr[m->EltoVert[i] + 1]++;
    for (size_t n = 0; n < nn; ++n) ptr[n + 1] += ptr[n];
    {
        std::vector<int> fill(nn, 0);
        for (size_t el = 0; el < ne; ++el)
            for (int k = 0; k < 3; ++k) {
                int v = m->EltoVert[3 * el + k];
                lst[ptr[v] + fill[v]++] = (int)el;
            }
    }
    /* prescribed boundary edges */
    std::vector<int> be, bt;
    for (size_t i = 0; i < nf; ++i)
        if (m->BdryPrescribed[i]) {
            be.push_back((int)i);
            bt.push_back(m->BdryPrescribed[i]);
        }
    c->nbnd = (int)be.size();
    c->h_bnd = new std::vector<int>(be);
    TRY(dalloc(&c->n2e_ptr, nn + 1));
    TRY(dalloc(&c->n2e, 3 * ne));
    TRY(dalloc(&c->bnd_edges, be.size()));
    TRY(dalloc(&c->bnd_type, bt.size()));
    TRY(dalloc(&c->bstage, 2 * be.size()));
    TRY(cudaHostAlloc((void **)&c->h_stage, sizeof(double) * 2 * (be.size() + 1), cudaHostAllocDefault) == cudaSuccess
            ? 0
            : DGR_ERR_CUDA);
    TRY(cudaMemcpy(c->n2e_ptr, ptr.data(), (nn + 1) * 4, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemcpy(c->n2e, lst.data(), 3 * ne * 4, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    if (!be.empty()) {
        TRY(cudaMemcpy(c->bnd_edges, be.data(), be.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : DGR_ERR_CUDA);
        TRY(cudaMemcpy(c->bnd_type, bt.data(), bt.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    }
    /* clock and flags */
    DevClock hc;
    memset(&hc, 0, sizeof hc);
    hc.err = ~0ull;
    hc.final_time = 1e300;
    TRY(cudaMemcpy(c->clk, &hc, sizeof hc, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    std::vector<int> wd(ne, -1);
    TRY(cudaMemcpy(c->wdA, wd.data(), ne * 4, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    TRY(cudaMemcpy(c->wdB, wd.data(), ne * 4, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : DGR_ERR_CUDA);
    c->wd_fresh = 0;
    c->wd_cur_is_B = 0;
    *out = c;
    return DGR_OK;
}

extern "C" int dgr_destroy(dgr_ctx *c)
{
    if (!c) return DGR_ERR_INVALID;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    release(c);
    return DGR_OK;
}

static void drop_graph(dgr_ctx *c)
{
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
}

extern "C" int dgr_get_params(const dgr_ctx *c, dgr_params *out)
{
    if (!c || !out) return DGR_ERR_INVALID;
    *out = c->p;
    return DGR_OK;
}

extern "C" int dgr_set_params(dgr_ctx *c, const dgr_params *p)
{
    if (!c || !p) return DGR_ERR_INVALID;
    if (p->g != c->p.g || p->H0 != c->p.H0 || p->VELZERO != c->p.VELZERO || p->wet_dry != c->p.wet_dry ||
        p->device != c->p.device)
        return DGR_ERR_INVALID;
    c->p.rain = p->rain;
    c->p.tide_on = p->tide_on;
    c->p.tide_amp = p->tide_amp;
    c->p.tide_period = p->tide_period;
    c->p.cfl = p->cfl;
    c->p.dt0 = p->dt0;
    c->p.record_decisions = p->record_decisions;
    drop_graph(c);
    return DGR_OK;
}

extern "C" int dgr_set_element_manning(dgr_ctx *c, const double *n_el)
{
    if (!c) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    if (n_el) {
        if (!c->n_el) {
            int r = dalloc(&c->n_el, c->ne);
            if (r) return r;
        }
        CK(cudaMemcpyAsync(c->n_el, n_el, (size_t)c->ne * 8, cudaMemcpyHostToDevice, c->stream));
    } else if (c->n_el) {
        CK(cudaStreamSynchronize(c->stream));
        cudaFree(c->n_el);
        c->n_el = nullptr;
    }
    int r = upload_geometry(c);
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    return DGR_OK;
}

/* ------------------------------------------------------------------ state ---- */

extern "C" int dgr_upload_state(dgr_ctx *c, const double *zeta, const double *Qx, const double *Qy, const int *WD)
{
    if (!c || !zeta || !Qx || !Qy) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    const size_t n3 = 3 * (size_t)c->ne;
    double *st = c->W; /* staging: W is free between steps */
    cudaStream_t s = c->stream;
    CK(cudaMemcpyAsync(st, zeta, n3 * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(st + n3, Qx, n3 * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(st + 2 * n3, Qy, n3 * 8, cudaMemcpyHostToDevice, s));
    k_aos_to_planar<<<blocks(c->ne, 256), 256, 0, s>>>(c->ne, c->ldE, st, st + n3, st + 2 * n3, c->U);
    c->launches++;
    if (WD) CK(cudaMemcpyAsync(c->wdA, WD, (size_t)c->ne * 4, cudaMemcpyHostToDevice, s));
    /* clear the error word */
    const unsigned long long none = ~0ull;
    CK(cudaMemcpyAsync(&c->clk->err, &none, 8, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    c->wd_fresh = 0;
    c->wd_cur_is_B = 0;
    return DGR_OK;
}

extern "C" int dgr_download_state(dgr_ctx *c, double *zeta, double *Qx, double *Qy, int *WD)
{
    if (!c || !zeta || !Qx || !Qy) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    const size_t n3 = 3 * (size_t)c->ne;
    double *st = c->W;
    cudaStream_t s = c->stream;
    k_planar_to_aos<<<blocks(c->ne, 256), 256, 0, s>>>(c->ne, c->ldE, c->U, st, st + n3, st + 2 * n3);
    c->launches++;
    CK(cudaMemcpyAsync(zeta, st, n3 * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(Qx, st + n3, n3 * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(Qy, st + 2 * n3, n3 * 8, cudaMemcpyDeviceToHost, s));
    if (WD) CK(cudaMemcpyAsync(WD, c->wd_cur_is_B ? c->wdB : c->wdA, (size_t)c->ne * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return DGR_OK;
}

__global__ void k_scatter_bnd(int nb, const int *be, const double *vals, double *bzeta, double *bqn)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    bzeta[be[j]] = vals[j];
    bqn[be[j]] = vals[nb + j];
}

extern "C" int dgr_set_boundary(dgr_ctx *c, const double *bzeta, const double *bQn)
{
    if (!c || !bzeta || !bQn) return DGR_ERR_INVALID;
    if (c->nbnd == 0) return DGR_OK;
    CK(cudaSetDevice(c->device));
    /* only prescribed edges are read by the flux; copy those through a compact stage
     * (the pinned stage may still feed the previous copy: wait for the stream first) */
    CK(cudaStreamSynchronize(c->stream));
    const std::vector<int> &be = *c->h_bnd;
    for (int j = 0; j < c->nbnd; ++j) {
        c->h_stage[j] = bzeta[be[j]];
        c->h_stage[c->nbnd + j] = bQn[be[j]];
    }
    double *tmp = c->bstage;
    CK(cudaMemcpyAsync(tmp, c->h_stage, sizeof(double) * 2 * c->nbnd, cudaMemcpyHostToDevice, c->stream));
    k_scatter_bnd<<<blocks(c->nbnd, 256), 256, 0, c->stream>>>(c->nbnd, c->bnd_edges, tmp, c->bzeta, c->bqn);
    c->launches++;
    CK(cudaGetLastError());
    return DGR_OK;
}

extern "C" int dgr_boundary_conditions(dgr_ctx *c, double time)
{
    if (!c) return DGR_ERR_INVALID;
    if (c->nbnd == 0) return DGR_OK;
    CK(cudaSetDevice(c->device));
    k_forcing<<<blocks(c->nbnd, 256), 256, 0, c->stream>>>(phys(c), time, c->bnd_edges, c->bnd_type, c->nbnd,
                                                           c->bzeta, c->bqn);
    c->launches++;
    CK(cudaGetLastError());
    return DGR_OK;
}

/* --------------------------------------------------------------- launches ---- */

static const int *wd_current(const dgr_ctx *c) { return c->wd_cur_is_B ? c->wdB : c->wdA; }

/* one RK stage; stage 0 reads U writes W, stage 1 reads W and U writes U */
static void launch_stage(dgr_ctx *c, int stage, int phase_base, bool count)
{
    const MeshDev m = mesh_dev(c);
    cudaStream_t s = c->stream;
    const bool wd = c->p.wet_dry != 0;
    const double g = c->p.g;
    const double *S = stage == 0 ? c->U : c->W;
    double *OUT = stage == 0 ? c->W : c->U;
    const int *wd_in = stage == 0 ? c->wdA : c->wdB;
    int *wd_out = stage == 0 ? c->wdB : c->wdA;
    if (!wd) wd_in = c->wdA;
    int *dl = c->p.record_decisions ? c->dec + (size_t)(2 * stage) * c->ne : nullptr;
    int *dp = c->p.record_decisions ? c->dec + (size_t)(2 * stage + 1) * c->ne : nullptr;

    if (wd)
        k_edge_flux<true><<<blocks(c->nf, 256), 256, 0, s>>>(m, S, wd_in, c->bzeta, c->bqn, c->flux, c->clk, stage,
                                                             phase_base, g);
    else
        k_edge_flux<false><<<blocks(c->nf, 256), 256, 0, s>>>(m, S, wd_in, c->bzeta, c->bqn, c->flux, c->clk, stage,
                                                              phase_base, g);
    if (stage == 0)
        k_element<MODE_STAGE1><<<blocks(c->ne, 128), 128, 0, s>>>(m, S, c->U, wd_in, c->flux, OUT, c->avg, c->clk, g,
                                                                  c->p.rain);
    else
        k_element<MODE_STAGE2><<<blocks(c->ne, 128), 128, 0, s>>>(m, S, c->U, wd_in, c->flux, OUT, c->avg, c->clk, g,
                                                                  c->p.rain);
    k_node_bounds<<<blocks(c->nn, 256), 256, 0, s>>>(m, c->avg, c->bounds, c->clk);
    if (wd)
        k_limit<true, true, true><<<blocks(c->ne, 128), 128, 0, s>>>(m, OUT, c->bounds, wd_in, wd_out, c->clk,
                                                                     c->p.H0, c->p.VELZERO, phase_base + 1, dl, dp);
    else
        k_limit<true, false, false><<<blocks(c->ne, 128), 128, 0, s>>>(m, OUT, c->bounds, wd_in, wd_out, c->clk,
                                                                       c->p.H0, c->p.VELZERO, phase_base + 1, dl, dp);
    if (count) c->launches += 4;
}

static void launch_wd_refresh(dgr_ctx *c)
{
    if (c->p.wet_dry && !c->wd_fresh) {
        /* the flags the caller sees (WA after an upload, WB after a step) seed the status */
        if (c->wd_cur_is_B)
            cudaMemcpyAsync(c->wdA, c->wdB, (size_t)c->ne * 4, cudaMemcpyDeviceToDevice, c->stream);
        k_wd_status<<<blocks(c->ne, 256), 256, 0, c->stream>>>(mesh_dev(c), c->U, c->wdA, c->clk, c->p.H0);
        c->launches++;
        c->wd_fresh = 1;
    }
}

static int read_clock(dgr_ctx *c)
{
    CK(cudaMemcpyAsync(c->h_clk, c->clk, sizeof(DevClock), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DGR_OK;
}

static int decode_err(unsigned long long key, int *code, int *index, int *step)
{
    if (key == ~0ull) {
        if (code) *code = 0;
        if (index) *index = -1;
        if (step) *step = -1;
        return 0;
    }
    int cd = (int)((key >> 32) & 15);
    if (code) *code = cd;
    if (index) *index = (int)(key & 0xffffffffu);
    if (step) *step = (int)(key >> 40);
    return cd;
}

extern "C" int dgr_step(dgr_ctx *c, double time, double dt, double *max_lambda)
{
    if (!c) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    CK(cudaEventRecord(c->ev0, s));
    k_clock_set<<<1, 1, 0, s>>>(c->clk, time, dt);
    c->launches++;
    launch_wd_refresh(c);
    launch_stage(c, 0, 0, true);
    launch_stage(c, 1, 2, true);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, s));
    if (c->p.wet_dry) {
        c->wd_fresh = 1;
        c->wd_cur_is_B = 1;
    }
    int r = read_clock(c);
    if (r) return r;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    if (max_lambda) *max_lambda = bits_to_double(c->h_clk->lam_bits[1]);
    return decode_err(c->h_clk->err, nullptr, nullptr, nullptr);
}

extern "C" int dgr_compute_L(dgr_ctx *c, double time, double *rz, double *rqx, double *rqy, double *max_lambda)
{
    (void)time;
    if (!c) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const MeshDev m = mesh_dev(c);
    k_clock_set<<<1, 1, 0, s>>>(c->clk, 0.0, 0.0);
    const int *wd = wd_current(c);
    if (c->p.wet_dry)
        k_edge_flux<true><<<blocks(c->nf, 256), 256, 0, s>>>(m, c->U, wd, c->bzeta, c->bqn, c->flux, c->clk, 0, 0,
                                                             c->p.g);
    else
        k_edge_flux<false><<<blocks(c->nf, 256), 256, 0, s>>>(m, c->U, wd, c->bzeta, c->bqn, c->flux, c->clk, 0, 0,
                                                              c->p.g);
    k_element<MODE_RHS><<<blocks(c->ne, 128), 128, 0, s>>>(m, c->U, c->U, wd, c->flux, c->W, c->avg, c->clk, c->p.g,
                                                           c->p.rain);
    c->launches += 3;
    CK(cudaGetLastError());
    if (rz && rqx && rqy) {
        const size_t n3 = 3 * (size_t)c->ne;
        double *tmp = nullptr; /* stream-ordered staging for the reference layout */
        CK(cudaMallocAsync((void **)&tmp, 3 * n3 * 8, s));
        k_planar_to_aos<<<blocks(c->ne, 256), 256, 0, s>>>(c->ne, c->ldE, c->W, tmp, tmp + n3, tmp + 2 * n3);
        c->launches++;
        CK(cudaMemcpyAsync(rz, tmp, n3 * 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(rqx, tmp + n3, n3 * 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(rqy, tmp + 2 * n3, n3 * 8, cudaMemcpyDeviceToHost, s));
        CK(cudaFreeAsync(tmp, s));
    }
    int r = read_clock(c);
    if (r) return r;
    if (max_lambda) *max_lambda = bits_to_double(c->h_clk->lam_bits[0]);
    return decode_err(c->h_clk->err, nullptr, nullptr, nullptr);
}

extern "C" int dgr_get_fhat(dgr_ctx *c, double *f1, double *f2, double *f3)
{
    if (!c || !f1 || !f2 || !f3) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    const size_t n3 = 3 * (size_t)c->ne;
    double *tmp = nullptr;
    CK(cudaMallocAsync((void **)&tmp, 3 * n3 * 8, c->stream));
    k_flux_to_slots<<<blocks(c->ne, 256), 256, 0, c->stream>>>(mesh_dev(c), c->flux, tmp, tmp + n3, tmp + 2 * n3);
    c->launches++;
    CK(cudaMemcpyAsync(f1, tmp, n3 * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(f2, tmp + n3, n3 * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(f3, tmp + 2 * n3, n3 * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaFreeAsync(tmp, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DGR_OK;
}

extern "C" int dgr_slope_limiter(dgr_ctx *c)
{
    if (!c) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const MeshDev m = mesh_dev(c);
    k_clock_set<<<1, 1, 0, s>>>(c->clk, 0.0, 0.0);
    k_avg<<<blocks(c->ne, 256), 256, 0, s>>>(m, c->U, c->avg);
    k_node_bounds<<<blocks(c->nn, 256), 256, 0, s>>>(m, c->avg, c->bounds, c->clk);
    int *dl = c->p.record_decisions ? c->dec : nullptr;
    k_limit<true, false, false><<<blocks(c->ne, 128), 128, 0, s>>>(m, c->U, c->bounds, c->wdA, c->wdA, c->clk,
                                                                   c->p.H0, c->p.VELZERO, 0, dl, nullptr);
    c->launches += 4;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    c->wd_fresh = 0;
    return DGR_OK;
}

extern "C" int dgr_pdop(dgr_ctx *c)
{
    if (!c) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    k_clock_set<<<1, 1, 0, s>>>(c->clk, 0.0, 0.0);
    int *dp = c->p.record_decisions ? c->dec + c->ne : nullptr;
    k_limit<false, true, false><<<blocks(c->ne, 128), 128, 0, s>>>(mesh_dev(c), c->U, c->bounds, c->wdA, c->wdA,
                                                                   c->clk, c->p.H0, c->p.VELZERO, 1, nullptr, dp);
    c->launches += 2;
    CK(cudaGetLastError());
    int r = read_clock(c);
    if (r) return r;
    c->wd_fresh = 0;
    return decode_err(c->h_clk->err, nullptr, nullptr, nullptr);
}

extern "C" int dgr_wet_dry_status(dgr_ctx *c)
{
    if (!c) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    int *wd = c->wd_cur_is_B ? c->wdB : c->wdA;
    k_clock_set<<<1, 1, 0, s>>>(c->clk, 0.0, 0.0);
    k_wd_status<<<blocks(c->ne, 256), 256, 0, s>>>(mesh_dev(c), c->U, wd, c->clk, c->p.H0);
    c->launches += 2;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    c->wd_fresh = 0;
    return DGR_OK;
}

/* ---------------------------------------------------------- device loop ---- */

/* Capture one step (clock, two stages, clock end) into a graph. */
static int build_graph(dgr_ctx *c)
{
    drop_graph(c);
    cudaStream_t s = c->stream;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    k_clock_begin<<<1, 256, 0, s>>>(c->clk, phys(c), c->bnd_edges, c->bnd_type, c->nbnd, c->bzeta, c->bqn);
    /* the stage launches below see wd roles of a fresh step */
    launch_stage(c, 0, 0, false);
    launch_stage(c, 1, 2, false);
    k_clock_end<<<1, 1, 0, s>>>(c->clk);
    cudaError_t e = cudaStreamEndCapture(s, &c->graph);
    if (e != cudaSuccess) {
        snprintf(g_cuda_err, sizeof g_cuda_err, "capture: %s", cudaGetErrorString(e));
        return DGR_ERR_CUDA;
    }
    CK(cudaGraphInstantiate(&c->graph_exec, c->graph, 0));
    c->graph_kernels = 10;
    return DGR_OK;
}

__global__ void k_clock_init(DevClock *clk, double time, double dt, double final_time, int nsteps)
{
    clk->time = time;
    clk->dt = dt;
    clk->final_time = final_time;
    clk->step = 0;
    clk->nsteps = nsteps;
    clk->done = 0;
    clk->dt_pending = 0;
}

extern "C" int dgr_run(dgr_ctx *c, int nsteps, double final_time, double *time_io, double *dt_io, int *steps_done)
{
    if (!c || !time_io || !dt_io || nsteps < 0) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    double t0 = *time_io, dt = *dt_io;
    const bool fresh_run = t0 < 0;
    if (fresh_run) {
        t0 = 0.0;
        dt = c->p.dt0;
    }
    if (!c->graph_exec) {
        int r = build_graph(c);
        if (r) return r;
    }
    CK(cudaEventRecord(c->ev0, s));
    k_clock_init<<<1, 1, 0, s>>>(c->clk, t0, dt, final_time, nsteps);
    c->launches++;
    launch_wd_refresh(c);
    for (int i = 0; i < nsteps; ++i) CK(cudaGraphLaunch(c->graph_exec, s));
    c->launches += (long long)nsteps * c->graph_kernels;
    k_clock_finish<<<1, 1, 0, s>>>(c->clk, phys(c));
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, s));
    int r = read_clock(c);
    if (r) return r;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    if (c->p.wet_dry && c->h_clk->step > 0) {
        c->wd_fresh = 1;
        c->wd_cur_is_B = 1;
    }
    *time_io = c->h_clk->time;
    *dt_io = c->h_clk->dt;
    if (steps_done) *steps_done = c->h_clk->step;
    return decode_err(c->h_clk->err, nullptr, nullptr, nullptr);
}

extern "C" int dgr_last_error(dgr_ctx *c, int *code, int *index, int *step)
{
    if (!c) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    int r = read_clock(c);
    if (r) return r;
    decode_err(c->h_clk->err, code, index, step);
    return DGR_OK;
}

extern "C" int dgr_get_decisions(dgr_ctx *c, int stage, int *limit, int *pdop)
{
    if (!c || stage < 0 || stage > 1) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->ne;
    if (limit) CK(cudaMemcpyAsync(limit, c->dec + 2 * stage * n, n * 4, cudaMemcpyDeviceToHost, c->stream));
    if (pdop) CK(cudaMemcpyAsync(pdop, c->dec + (2 * stage + 1) * n, n * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DGR_OK;
}

extern "C" long long dgr_kernel_launches(const dgr_ctx *c) { return c ? c->launches : -1; }
extern "C" double dgr_last_device_ms(const dgr_ctx *c) { return c ? c->last_ms : -1.0; }

extern "C" void *dgr_host_alloc(size_t bytes)
{
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    return p;
}

extern "C" void dgr_host_free(void *p)
{
    if (p) cudaFreeHost(p);
}

/*
 * Per-kernel device timing of whole steps: CUDA events around every launch of
 * nsteps host-driven steps (dt of the last run, or dt0).  kernel_ms[0..3] receive the
 * average ms of one launch of: edge flux, element RHS+RK, node bounds, limiter+PDop.
 */
extern "C" int dgr_profile_step(dgr_ctx *c, int nsteps, double *kernel_ms, int n)
{
    if (!c || nsteps <= 0 || !kernel_ms || n < 4) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const MeshDev m = mesh_dev(c);
    const bool wd = c->p.wet_dry != 0;
    const double g = c->p.g;
    cudaEvent_t ev[9];
    for (int i = 0; i < 9; ++i) CK(cudaEventCreate(&ev[i]));
    double acc[4] = {0, 0, 0, 0};
    const double dt = (c->h_clk->dt > 0) ? c->h_clk->dt : c->p.dt0;
    int rc = DGR_OK;
    for (int it = 0; it < nsteps && rc == DGR_OK; ++it) {
        k_clock_set<<<1, 1, 0, s>>>(c->clk, 0.0, dt);
        launch_wd_refresh(c);
        for (int stage = 0; stage < 2; ++stage) {
            const double *S = stage == 0 ? c->U : c->W;
            double *OUT = stage == 0 ? c->W : c->U;
            const int *wd_in = (stage == 0 || !wd) ? c->wdA : c->wdB;
            int *wd_out = stage == 0 ? c->wdB : c->wdA;
            cudaEventRecord(ev[0], s);
            if (wd)
                k_edge_flux<true><<<blocks(c->nf, 256), 256, 0, s>>>(m, S, wd_in, c->bzeta, c->bqn, c->flux, c->clk,
                                                                     stage, 2 * stage, g);
            else
                k_edge_flux<false><<<blocks(c->nf, 256), 256, 0, s>>>(m, S, wd_in, c->bzeta, c->bqn, c->flux, c->clk,
                                                                      stage, 2 * stage, g);
            cudaEventRecord(ev[1], s);
            if (stage == 0)
                k_element<MODE_STAGE1><<<blocks(c->ne, 128), 128, 0, s>>>(m, S, c->U, wd_in, c->flux, OUT, c->avg,
                                                                          c->clk, g, c->p.rain);
            else
                k_element<MODE_STAGE2><<<blocks(c->ne, 128), 128, 0, s>>>(m, S, c->U, wd_in, c->flux, OUT, c->avg,
                                                                          c->clk, g, c->p.rain);
            cudaEventRecord(ev[2], s);
            k_node_bounds<<<blocks(c->nn, 256), 256, 0, s>>>(m, c->avg, c->bounds, c->clk);
            cudaEventRecord(ev[3], s);
            if (wd)
                k_limit<true, true, true><<<blocks(c->ne, 128), 128, 0, s>>>(
                    m, OUT, c->bounds, wd_in, wd_out, c->clk, c->p.H0, c->p.VELZERO, 2 * stage + 1, nullptr, nullptr);
            else
                k_limit<true, false, false><<<blocks(c->ne, 128), 128, 0, s>>>(
                    m, OUT, c->bounds, wd_in, wd_out, c->clk, c->p.H0, c->p.VELZERO, 2 * stage + 1, nullptr, nullptr);
            cudaEventRecord(ev[4], s);
            c->launches += 4;
            if (cudaEventSynchronize(ev[4]) != cudaSuccess) {
                rc = DGR_ERR_CUDA;
                break;
            }
            for (int k = 0; k < 4; ++k) {
                float ms = 0;
                cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
                acc[k] += ms;
            }
        }
        if (wd) {
            c->wd_fresh = 1;
            c->wd_cur_is_B = 1;
        }
    }
    for (int i = 0; i < 9; ++i) cudaEventDestroy(ev[i]);
    if (rc) return rc;
    CK(cudaGetLastError());
    for (int k = 0; k < 4; ++k) kernel_ms[k] = acc[k] / (2.0 * nsteps);
    return DGR_OK;
}

extern "C" int dgr_pow43_batch(const double *x, double *y, int n, int device)
{
    if (!x || !y || n < 0) return DGR_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DGR_ERR_NO_DEVICE;
    CK(cudaSetDevice(device));
    double *d = nullptr;
    CK(cudaMalloc((void **)&d, 2 * (size_t)(n ? n : 1) * sizeof(double)));
    cudaMemcpy(d, x, (size_t)n * 8, cudaMemcpyHostToDevice);
    if (n) k_pow43<<<blocks(n, 256), 256>>>(n, d, d + n);
    cudaError_t e = cudaMemcpy(y, d + n, (size_t)n * 8, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        snprintf(g_cuda_err, sizeof g_cuda_err, "pow43: %s", cudaGetErrorString(e));
        return DGR_ERR_CUDA;
    }
    return DGR_OK;
}
