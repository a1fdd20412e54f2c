/*
 * Device context and C ABI of include/dgrain.h (the part that needs CUDA).
 *
 * A context holds S >= 1 scenarios: the disjoint union of their meshes, flattened into
 * one mesh (elements, nodes and edges renumbered with per-scenario offsets), with a
 * scenario id per element and per edge and one clock per scenario.  A single mesh is
 * the case S = 1.  Each scenario's numbers are exactly those of running it alone.
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
 *
 * Schedules of the device loop ("fusion depth"), chosen by dgr_autotune or
 * dgr_set_schedule:
 *   0: ten kernels per step (clock, 4 per stage, clock end), one thread per item;
 *   1: one persistent cooperative kernel per RK stage between the clock kernels;
 *   2: one persistent cooperative kernel per step, clock included;
 * and the block size (elements per block) of the element and limiter work.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "dgr_internal.cuh"

using namespace dgr;

static thread_local char g_cuda_err[256] = "";
char *dgr_cuda_err_buffer() { return g_cuda_err; }

extern "C" const char *dgr_last_cuda_error(void) { return g_cuda_err; }

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
    p->rk_stages = 2;
    p->order = 1;
    return DGR_OK;
}

void drop_graph(dgr_ctx *c)
{
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
    if (c->stage_graph_exec) cudaGraphExecDestroy(c->stage_graph_exec);
    if (c->stage_graph) cudaGraphDestroy(c->stage_graph);
    c->stage_graph_exec = nullptr;
    c->stage_graph = nullptr;
    c->stage_graph_tried = 0;
}

static void release(dgr_ctx *c)
{
    if (!c) return;
    drop_graph(c);
    void *ptrs[] = {c->x, c->y, c->zn, c->nfric, c->n_el, c->el2v_aos, c->el2v, c->elem_edge, c->e_in, c->redo,
                    c->e_ex, c->e_info, c->n2e_ptr, c->n2e, c->bnd_edges, c->bnd_type, c->bnd_sid, c->bdry,
                    c->el_sid, c->ed_sid, c->e_geo, c->geo, c->U, c->W, c->flux, c->avg, c->bounds, c->bzeta,
                    c->bqn, c->bstage, c->wdA, c->wdB, c->wdC, c->dec, c->bar, c->clk, c->p2g,
                    c->gauge_el, c->gauge_sid, c->gauge_w, c->gauge_series};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    adjoint_release(c);
    coupling_release(c);
    if (c->h_clk) cudaFreeHost(c->h_clk);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int upload_geometry(dgr_ctx *c)
{
    k_element_setup<<<blocks(c->ne, 128), 128, 0, c->stream>>>(c->ne, c->ldE, c->el2v_aos, c->x, c->y, c->zn,
                                                               c->nfric, c->n_el, c->p.g, c->el2v, c->geo);
    c->launches++;
    if (c->p.order == 2) {
        k_p2_setup<<<blocks(c->ne, 256), 256, 0, c->stream>>>(c->ne, c->ldE, c->el2v_aos, c->x, c->y, c->zn,
                                                              c->nfric, c->n_el, c->p.g, c->p2g);
        c->launches++;
    }
    CK(cudaGetLastError());
    return DGR_OK;
}

/* The p = 2 basis at (r, s) with its derivatives, in the closed forms of dgr_p2.cuh. */
static void p2_basis(double r, double sv, double phi[P2_NM], double dr[P2_NM], double ds[P2_NM])
{
    const double A = r + (1.0 + sv) / 2, B = (1.0 - sv) / 2;
    const double f[P2_NM] = {1.0, (3.0 * sv + 1.0) / 2, A, (5.0 * sv * sv + 2.0 * sv - 1.0) / 2,
                             A * (5.0 * sv + 3.0) / 2, (3.0 * A * A - B * B) / 2};
    const double fr[P2_NM] = {0.0, 0.0, 1.0, 0.0, (5.0 * sv + 3.0) / 2, 3.0 * A};
    const double fs[P2_NM] = {0.0, 1.5, 0.5, 5.0 * sv + 1.0, (5.0 * sv + 3.0) / 4 + 5.0 * A / 2, (3.0 * A + B) / 2};
    for (int m = 0; m < P2_NM; ++m) {
        phi[m] = f[m];
        dr[m] = fr[m];
        ds[m] = fs[m];
    }
}

/* Reference tables of the p = 2 step: Radon's 7-point degree-5 area rule (centroid 9/40;
 * a = (6 -+ sqrt 15)/21 with weights (155 -+ sqrt 15)/1200), 3-point Gauss-Legendre on the
 * edges, the basis there, and the diagonal mass matrix. */
static P2Ref make_p2_ref()
{
    P2Ref R;
    const double s15 = sqrt(15.0);
    const double a1 = (6.0 - s15) / 21, a2 = (6.0 + s15) / 21;
    const double w1 = (155.0 - s15) / 1200, w2 = (155.0 + s15) / 1200;
    const double L[P2_NQ][3] = {{1.0 / 3, 1.0 / 3, 1.0 / 3}, {1.0 - 2 * a1, a1, a1}, {a1, 1.0 - 2 * a1, a1},
                                {a1, a1, 1.0 - 2 * a1},      {1.0 - 2 * a2, a2, a2}, {a2, 1.0 - 2 * a2, a2},
                                {a2, a2, 1.0 - 2 * a2}};
    const double W[P2_NQ] = {9.0 / 40, w1, w1, w1, w2, w2, w2};
    for (int m = 0; m < P2_NM; ++m) R.mass[m] = 0.0;
    for (int q = 0; q < P2_NQ; ++q) {
        R.wq[q] = W[q];
        for (int k = 0; k < 3; ++k) R.lam[q][k] = L[q][k];
        const double r = -L[q][0] + L[q][1] - L[q][2], sv = -L[q][0] - L[q][1] + L[q][2];
        p2_basis(r, sv, R.phi[q], R.dr[q], R.ds[q]);
        for (int m = 0; m < P2_NM; ++m) R.mass[m] += 2.0 * W[q] * R.phi[q][m] * R.phi[q][m];
    }
    const double g3 = sqrt(3.0 / 5);
    const double te[P2_NGP] = {-g3, 0.0, g3}, wg[P2_NGP] = {5.0 / 9, 8.0 / 9, 5.0 / 9};
    for (int gp = 0; gp < P2_NGP; ++gp) {
        R.te[gp] = te[gp];
        R.wg[gp] = wg[gp];
        const double t = te[gp];
        /* local edge k runs from vertex k to k+1: (t, -1), (-t, t), (-1, -t) */
        const double rs[3][2] = {{t, -1.0}, {-t, t}, {-1.0, -t}};
        for (int k = 0; k < 3; ++k) {
            double dr[P2_NM], ds[P2_NM];
            p2_basis(rs[k][0], rs[k][1], R.phie[k][gp], dr, ds);
        }
    }
    return R;
}

static int check_mesh_view(const dgr_mesh_view *m)
{
    if (!m || m->num_el <= 0 || m->num_nodes <= 0 || m->num_edges <= 0) return DGR_ERR_INVALID;
    if (!m->x_coord || !m->y_coord || !m->z || !m->nFriction || !m->EltoVert || !m->EdgtoEls ||
        !m->EdgtoVert || !m->BdryPrescribed)
        return DGR_ERR_INVALID;
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
#define TRYC(x) TRY((x) == cudaSuccess ? DGR_OK : DGR_ERR_CUDA)

/* Copies one host array per scenario into a flattened device array, adding `add[s]` to
 * every entry of scenario s (connectivity renumbering); add == nullptr copies as is. */
template <class T>
static int upload_concat(cudaStream_t s, T *dst, int nscen, const T *const *src, const std::vector<int> &count,
                         int mult, const std::vector<int> *add)
{
    size_t off = 0;
    std::vector<T> tmp;
    for (int k = 0; k < nscen; ++k) {
        const size_t n = (size_t)count[k] * mult;
        if (add && (*add)[k] != 0) {
            tmp.assign(src[k], src[k] + n);
            for (auto &v : tmp) v += (T)(*add)[k];
            CK(cudaMemcpy(dst + off, tmp.data(), n * sizeof(T), cudaMemcpyHostToDevice));
        } else {
            CK(cudaMemcpyAsync(dst + off, src[k], n * sizeof(T), cudaMemcpyHostToDevice, s));
        }
        off += n;
    }
    CK(cudaStreamSynchronize(s));
    return DGR_OK;
}

static int create_impl(int nscen, const dgr_mesh_view *views, const dgr_scenario_params *sp, const dgr_params *params,
                       dgr_ctx **out)
{
    if (!out || nscen <= 0 || !views) return DGR_ERR_INVALID;
    *out = nullptr;
    long long tot_e = 0, tot_n = 0, tot_f = 0;
    for (int k = 0; k < nscen; ++k) {
        int rc = check_mesh_view(&views[k]);
        if (rc) return rc;
        tot_e += views[k].num_el;
        tot_n += views[k].num_nodes;
        tot_f += views[k].num_edges;
    }
    if (tot_f >= (1LL << 30) || tot_e >= (1LL << 30) || tot_n >= (1LL << 30)) return DGR_ERR_TOO_LARGE;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        snprintf(dgr_cuda_err_buffer(), 256, "no CUDA device visible");
        return DGR_ERR_NO_DEVICE;
    }
    dgr_ctx *c = new dgr_ctx();
    if (params)
        c->p = *params;
    else
        dgr_params_default(&c->p);
    c->device = c->p.device;
    if (c->p.rk_stages == 0) c->p.rk_stages = 2; /* a zero-filled struct means the reference's RK2 */
    if (c->p.order == 0) c->p.order = 1;
    if ((c->p.rk_stages != 2 && c->p.rk_stages != 3) || (c->p.order != 1 && c->p.order != 2) ||
        (c->p.order == 2 && c->p.wet_dry) || (c->p.flux < 0 || c->p.flux > 2)) {
        delete c;
        return DGR_ERR_INVALID;
    }
    c->nm = c->p.order == 2 ? P2_NM : 3;
    c->nfp = c->p.order == 2 ? P2_FLUX : 6;
    if (c->p.order == 2) c->p2ref = make_p2_ref();
    c->bs = 64; /* measured: 0.573 ms per element launch against 0.591 (128) and 0.618 (256) at 4M */
    c->fusion = 0;
    c->bar_polls = kBarrierSpins;
    c->bar_phantom = 0;
    if (c->device < 0 || c->device >= ndev) {
        release(c);
        return DGR_ERR_INVALID;
    }
    TRYC(cudaSetDevice(c->device));
    TRYC(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device));
    c->nscen = nscen;
    c->ne = (int)tot_e;
    c->nn = (int)tot_n;
    c->nf = (int)tot_f;
    c->ldE = pad32(c->ne);
    c->ldF = pad32(c->nf);
    c->ldN = pad32(c->nn);
    std::vector<int> ne_s(nscen), nn_s(nscen), nf_s(nscen);
    c->el_off.assign(nscen + 1, 0);
    c->nd_off.assign(nscen + 1, 0);
    c->ed_off.assign(nscen + 1, 0);
    for (int k = 0; k < nscen; ++k) {
        ne_s[k] = views[k].num_el;
        nn_s[k] = views[k].num_nodes;
        nf_s[k] = views[k].num_edges;
        c->el_off[k + 1] = c->el_off[k] + ne_s[k];
        c->nd_off[k + 1] = c->nd_off[k] + nn_s[k];
        c->ed_off[k + 1] = c->ed_off[k] + nf_s[k];
    }
    std::vector<int> el_add(c->el_off.begin(), c->el_off.end() - 1), nd_add(c->nd_off.begin(), c->nd_off.end() - 1);

    TRYC(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    TRYC(cudaEventCreate(&c->ev0));
    TRYC(cudaEventCreate(&c->ev1));

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
    const size_t nst = 3 * (size_t)c->nm;
    TRY(dalloc(&c->U, nst * lE));
    TRY(dalloc(&c->W, nst * lE));
    TRY(dalloc(&c->flux, (size_t)c->nfp * lF));
    if (c->p.order == 2) TRY(dalloc(&c->p2g, (size_t)P2G_N * lE));
    TRY(dalloc(&c->avg, 3 * lE));
    TRY(dalloc(&c->bounds, 6 * lN));
    TRY(dalloc(&c->bzeta, nf));
    TRY(dalloc(&c->bqn, nf));
    TRY(dalloc(&c->wdA, ne));
    TRY(dalloc(&c->wdB, ne));
    TRY(dalloc(&c->wdC, ne));
    TRY(dalloc(&c->dec, 6 * ne));
    TRY(dalloc(&c->bar, 6)); /* barrier words [0..2]; [4..5] the checked build's bad-index word */
    TRY(dalloc(&c->redo, 2 + (size_t)nf));
    TRY(dalloc(&c->clk, nscen));
    TRYC(cudaHostAlloc((void **)&c->h_clk, sizeof(DevClock) * nscen, cudaHostAllocDefault));

    cudaStream_t s = c->stream;
    {
        std::vector<const double *> px(nscen), py(nscen), pz(nscen), pn(nscen);
        std::vector<const int *> pev(nscen), pbd(nscen);
        for (int k = 0; k < nscen; ++k) {
            px[k] = views[k].x_coord;
            py[k] = views[k].y_coord;
            pz[k] = views[k].z;
            pn[k] = views[k].nFriction;
            pev[k] = views[k].EltoVert;
            pbd[k] = views[k].BdryPrescribed;
        }
        TRY(upload_concat(s, c->x, nscen, px.data(), nn_s, 1, nullptr));
        TRY(upload_concat(s, c->y, nscen, py.data(), nn_s, 1, nullptr));
        TRY(upload_concat(s, c->zn, nscen, pz.data(), nn_s, 1, nullptr));
        TRY(upload_concat(s, c->nfric, nscen, pn.data(), nn_s, 1, nullptr));
        TRY(upload_concat(s, c->el2v_aos, nscen, pev.data(), ne_s, 3, &nd_add));
        TRY(upload_concat(s, c->bdry, nscen, pbd.data(), nf_s, 1, nullptr));
    }
    TRYC(cudaMemsetAsync(c->elem_edge, 0xff, 3 * lE * 4, s));
    TRYC(cudaMemsetAsync(c->bzeta, 0, nf * 8, s));
    TRYC(cudaMemsetAsync(c->bqn, 0, nf * 8, s));
    TRYC(cudaMemsetAsync(c->U, 0, nst * lE * 8, s));
    TRYC(cudaMemsetAsync(c->W, 0, nst * lE * 8, s));
    TRYC(cudaMemsetAsync(c->dec, 0, 6 * ne * 4, s));
    TRYC(cudaMemsetAsync(c->bar, 0, 16, s));
    TRYC(cudaMemsetAsync(c->bar + 4, 0xff, 8, s));
    TRYC(cudaMemsetAsync(c->redo, 0, 8, s));

    /* per-element Manning n of the scenarios that give one (negative: node average) */
    bool any_nel = false;
    for (int k = 0; k < nscen; ++k) any_nel |= (sp && sp[k].n_el);
    if (any_nel) {
        std::vector<double> nel(ne, -1.0);
        for (int k = 0; k < nscen; ++k)
            if (sp[k].n_el) std::copy(sp[k].n_el, sp[k].n_el + ne_s[k], nel.begin() + c->el_off[k]);
        TRY(dalloc(&c->n_el, ne));
        TRYC(cudaMemcpy(c->n_el, nel.data(), ne * 8, cudaMemcpyHostToDevice));
    }
    if (nscen > 1) {
        std::vector<int> esid(ne), fsid(nf);
        for (int k = 0; k < nscen; ++k) {
            std::fill(esid.begin() + c->el_off[k], esid.begin() + c->el_off[k + 1], k);
            std::fill(fsid.begin() + c->ed_off[k], fsid.begin() + c->ed_off[k + 1], k);
        }
        TRY(dalloc(&c->el_sid, ne));
        TRY(dalloc(&c->ed_sid, nf));
        TRYC(cudaMemcpy(c->el_sid, esid.data(), ne * 4, cudaMemcpyHostToDevice));
        TRYC(cudaMemcpy(c->ed_sid, fsid.data(), nf * 4, cudaMemcpyHostToDevice));
    }

    /* connectivity goes through a temporary device copy */
    int *d_ed2el = nullptr, *d_ed2v = nullptr, *d_bad = nullptr;
    TRY(dalloc(&d_ed2el, 2 * nf));
    TRY(dalloc(&d_ed2v, 2 * nf));
    TRY(dalloc(&d_bad, 1));
    {
        std::vector<const int *> pe(nscen), pv(nscen);
        for (int k = 0; k < nscen; ++k) {
            pe[k] = views[k].EdgtoEls;
            pv[k] = views[k].EdgtoVert;
        }
        int r1 = upload_concat(s, d_ed2el, nscen, pe.data(), nf_s, 2, &el_add);
        int r2 = upload_concat(s, d_ed2v, nscen, pv.data(), nf_s, 2, &nd_add);
        if (r1 || r2) {
            cudaFree(d_ed2el);
            cudaFree(d_ed2v);
            cudaFree(d_bad);
            release(c);
            return r1 ? r1 : r2;
        }
    }
    const int big = 0x7fffffff;
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
        snprintf(dgr_cuda_err_buffer(), 256, "setup: %s", cudaGetErrorString(e1));
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

    /* node -> element lists (ascending element order) and prescribed edges */
    std::vector<int> ptr(nn + 1, 0), lst(3 * ne), be, bt, bsid;
    for (int k = 0; k < nscen; ++k)
        for (long long i = 0; i < 3LL * ne_s[k]; ++i) ptr[views[k].EltoVert[i] + c->nd_off[k] + 1]++;
    for (size_t n = 0; n < nn; ++n) ptr[n + 1] += ptr[n];
    {
        std::vector<int> fill(nn, 0);
        for (int k = 0; k < nscen; ++k)
            for (int el = 0; el < ne_s[k]; ++el)
                for (int j = 0; j < 3; ++j) {
                    const int v = views[k].EltoVert[3 * el + j] + c->nd_off[k];
                    lst[ptr[v] + fill[v]++] = el + c->el_off[k];
                }
    }
    for (int k = 0; k < nscen; ++k)
        for (int i = 0; i < nf_s[k]; ++i)
            if (views[k].BdryPrescribed[i]) {
                be.push_back(i + c->ed_off[k]);
                bt.push_back(views[k].BdryPrescribed[i]);
                bsid.push_back(k);
            }
    c->nbnd = (int)be.size();
    c->h_bnd = be;
    TRY(dalloc(&c->n2e_ptr, nn + 1));
    TRY(dalloc(&c->n2e, 3 * ne));
    TRY(dalloc(&c->bnd_edges, be.size()));
    TRY(dalloc(&c->bnd_type, bt.size()));
    TRY(dalloc(&c->bnd_sid, bsid.size()));
    TRY(dalloc(&c->bstage, 2 * be.size()));
    TRYC(cudaHostAlloc((void **)&c->h_stage, sizeof(double) * 2 * (be.size() + 1), cudaHostAllocDefault));
    TRYC(cudaMemcpy(c->n2e_ptr, ptr.data(), (nn + 1) * 4, cudaMemcpyHostToDevice));
    TRYC(cudaMemcpy(c->n2e, lst.data(), 3 * ne * 4, cudaMemcpyHostToDevice));
    if (!be.empty()) {
        TRYC(cudaMemcpy(c->bnd_edges, be.data(), be.size() * 4, cudaMemcpyHostToDevice));
        TRYC(cudaMemcpy(c->bnd_type, bt.data(), bt.size() * 4, cudaMemcpyHostToDevice));
        TRYC(cudaMemcpy(c->bnd_sid, bsid.data(), bsid.size() * 4, cudaMemcpyHostToDevice));
    }
    /* clocks */
    for (int k = 0; k < nscen; ++k) {
        DevClock &h = c->h_clk[k];
        memset(&h, 0, sizeof h);
        h.err = ~0ull;
        h.final_time = 1e300;
        h.min_edge = views[k].minEdgLength;
        h.rain = sp ? sp[k].rain : c->p.rain;
        h.tide_on = sp ? sp[k].tide_on : c->p.tide_on;
        h.tide_amp = sp ? sp[k].tide_amp : c->p.tide_amp;
        h.tide_period = sp ? sp[k].tide_period : c->p.tide_period;
        h.el_off = c->el_off[k];
        h.ed_off = c->ed_off[k];
    }
    TRYC(cudaMemcpy(c->clk, c->h_clk, sizeof(DevClock) * nscen, cudaMemcpyHostToDevice));
    std::vector<int> wd(ne, -1);
    TRYC(cudaMemcpy(c->wdA, wd.data(), ne * 4, cudaMemcpyHostToDevice));
    TRYC(cudaMemcpy(c->wdB, wd.data(), ne * 4, cudaMemcpyHostToDevice));
    TRYC(cudaMemcpy(c->wdC, wd.data(), ne * 4, cudaMemcpyHostToDevice));
    c->wd_fresh = 0;
    c->wd_stepped = 0;
    *out = c;
    return DGR_OK;
}

extern "C" int dgr_create(const dgr_mesh_view *m, const dgr_params *params, dgr_ctx **out)
{
    return create_impl(1, m, nullptr, params, out);
}

extern "C" int dgr_ensemble_create(int nscen, const dgr_mesh_view *meshes, const dgr_scenario_params *sp,
                                   const dgr_params *params, dgr_ctx **out)
{
    return create_impl(nscen, meshes, sp, params, out);
}

extern "C" int dgr_ensemble_size(const dgr_ctx *c) { return c ? c->nscen : -1; }

extern "C" int dgr_destroy(dgr_ctx *c)
{
    if (!c) return DGR_ERR_INVALID;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    release(c);
    return DGR_OK;
}

extern "C" int dgr_get_params(const dgr_ctx *c, dgr_params *out)
{
    if (!c || !out) return DGR_ERR_INVALID;
    *out = c->p;
    return DGR_OK;
}

int read_clock(dgr_ctx *c)
{
    CK(cudaMemcpyAsync(c->h_clk, c->clk, sizeof(DevClock) * c->nscen, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DGR_OK;
}

int write_clock(dgr_ctx *c)
{
    CK(cudaMemcpyAsync(c->clk, c->h_clk, sizeof(DevClock) * c->nscen, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DGR_OK;
}

extern "C" int dgr_set_params(dgr_ctx *c, const dgr_params *p)
{
    if (!c || !p) return DGR_ERR_INVALID;
    if (p->g != c->p.g || p->H0 != c->p.H0 || p->VELZERO != c->p.VELZERO || p->wet_dry != c->p.wet_dry ||
        p->device != c->p.device || (p->order == 0 ? 1 : p->order) != c->p.order || p->flux != c->p.flux)
        return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    c->p.rain = p->rain;
    c->p.tide_on = p->tide_on;
    c->p.tide_amp = p->tide_amp;
    c->p.tide_period = p->tide_period;
    c->p.cfl = p->cfl;
    c->p.dt0 = p->dt0;
    c->p.record_decisions = p->record_decisions;
    const int stages = p->rk_stages == 0 ? 2 : p->rk_stages;
    if (stages != 2 && stages != 3) return DGR_ERR_INVALID;
    if (stages != c->p.rk_stages) {
        if (c->wd_stepped) /* the current flags sit in the old scheme's after-step buffer */
            CK(cudaMemcpyAsync(c->wdA, wd_after_step(c), (size_t)c->ne * 4, cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->wd_stepped = 0;
        c->wd_fresh = 0;
        c->p.rk_stages = stages;
    }
    if (c->nscen == 1) { /* a single mesh takes its forcing from the run parameters */
        int r = read_clock(c);
        if (r) return r;
        c->h_clk[0].rain = p->rain;
        c->h_clk[0].tide_on = p->tide_on;
        c->h_clk[0].tide_amp = p->tide_amp;
        c->h_clk[0].tide_period = p->tide_period;
        r = write_clock(c);
        if (r) return r;
    }
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

/* state of scenarios [s0, s1) from the reference layout (their arrays concatenated) */
int upload_scenarios(dgr_ctx *c, int s0, int s1, const double *zeta, const double *Qx, const double *Qy,
                     const int *WD)
{
    if (!zeta || !Qx || !Qy || s0 < 0 || s1 > c->nscen || s0 >= s1) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    const int n = c->el_off[s1] - c->el_off[s0];
    const size_t n3 = (size_t)c->nm * n; /* coefficients per variable */
    double *st = c->W; /* staging: W is free between steps */
    cudaStream_t s = c->stream;
    CK(cudaMemcpyAsync(st, zeta, n3 * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(st + n3, Qx, n3 * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(st + 2 * n3, Qy, n3 * 8, cudaMemcpyHostToDevice, s));
    k_aos_to_planar_nm<<<blocks(n, 256), 256, 0, s>>>(n, c->ldE, c->nm, st, st + n3, st + 2 * n3,
                                                      c->U + c->el_off[s0]);
    c->launches++;
    /* the other scenarios' current flags must sit in WA as well before WA is marked current */
    if (c->wd_stepped && c->nscen > 1)
        for (int k = 0; k < c->nscen; ++k)
            if (k < s0 || k >= s1)
                CK(cudaMemcpyAsync(c->wdA + c->el_off[k], wd_after_step(c) + c->el_off[k],
                                   (size_t)(c->el_off[k + 1] - c->el_off[k]) * 4, cudaMemcpyDeviceToDevice, s));
    if (WD) CK(cudaMemcpyAsync(c->wdA + c->el_off[s0], WD, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    /* clear the scenarios' error words and run state */
    int r = read_clock(c);
    if (r) return r;
    for (int k = s0; k < s1; ++k) {
        c->h_clk[k].err = ~0ull;
        c->h_clk[k].done = 0;
    }
    r = write_clock(c);
    if (r) return r;
    CK(cudaMemsetAsync(c->bar + 4, 0xff, 8, c->stream)); /* no bad index recorded */
    c->wd_fresh = 0;
    c->wd_stepped = 0;
    return DGR_OK;
}

static int upload_slice(dgr_ctx *c, int sc, const double *zeta, const double *Qx, const double *Qy, const int *WD)
{
    return upload_scenarios(c, sc, sc + 1, zeta, Qx, Qy, WD);
}

static int download_slice(dgr_ctx *c, int sc, double *zeta, double *Qx, double *Qy, int *WD)
{
    if (!zeta || !Qx || !Qy || sc < 0 || sc >= c->nscen) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    const int n = c->el_off[sc + 1] - c->el_off[sc];
    const size_t n3 = (size_t)c->nm * n;
    double *st = c->W;
    cudaStream_t s = c->stream;
    k_planar_to_aos_nm<<<blocks(n, 256), 256, 0, s>>>(n, c->ldE, c->nm, c->U + c->el_off[sc], st, st + n3,
                                                      st + 2 * n3);
    c->launches++;
    CK(cudaMemcpyAsync(zeta, st, n3 * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(Qx, st + n3, n3 * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(Qy, st + 2 * n3, n3 * 8, cudaMemcpyDeviceToHost, s));
    if (WD)
        CK(cudaMemcpyAsync(WD, (c->wd_stepped ? wd_after_step(c) : c->wdA) + c->el_off[sc], (size_t)n * 4,
                           cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return DGR_OK;
}

extern "C" int dgr_upload_state(dgr_ctx *c, const double *zeta, const double *Qx, const double *Qy, const int *WD)
{
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    return upload_slice(c, 0, zeta, Qx, Qy, WD);
}

extern "C" int dgr_download_state(dgr_ctx *c, double *zeta, double *Qx, double *Qy, int *WD)
{
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    return download_slice(c, 0, zeta, Qx, Qy, WD);
}

extern "C" int dgr_save_restart(dgr_ctx *c, const char *path, double time, double dt)
{
    NvtxRange nv("dgr_save_restart");
    if (!c || c->nscen != 1 || !path) return DGR_ERR_INVALID;
    const size_t n = (size_t)c->nm * c->ne;
    std::vector<double> st(3 * n);
    std::vector<int> wd(c->ne);
    int r = download_slice(c, 0, st.data(), st.data() + n, st.data() + 2 * n, wd.data());
    if (r) return r;
    return dgr_write_restart(path, c->ne, c->nm, st.data(), st.data() + n, st.data() + 2 * n, wd.data(), time, dt);
}

extern "C" int dgr_load_restart(dgr_ctx *c, const char *path, double *time, double *dt)
{
    NvtxRange nv("dgr_load_restart");
    if (!c || c->nscen != 1 || !path || !time || !dt) return DGR_ERR_INVALID;
    const size_t n = (size_t)c->nm * c->ne;
    std::vector<double> st(3 * n);
    std::vector<int> wd(c->ne);
    int r = dgr_read_restart(path, c->ne, c->nm, st.data(), st.data() + n, st.data() + 2 * n, wd.data(), time, dt);
    if (r) return r;
    return upload_slice(c, 0, st.data(), st.data() + n, st.data() + 2 * n, wd.data());
}

extern "C" int dgr_ensemble_upload_state(dgr_ctx *c, int scenario, const double *zeta, const double *Qx,
                                         const double *Qy, const int *WD)
{
    if (!c) return DGR_ERR_INVALID;
    return upload_slice(c, scenario, zeta, Qx, Qy, WD);
}

extern "C" int dgr_ensemble_download_state(dgr_ctx *c, int scenario, double *zeta, double *Qx, double *Qy, int *WD)
{
    if (!c) return DGR_ERR_INVALID;
    return download_slice(c, scenario, zeta, Qx, Qy, WD);
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
    if (!c || !bzeta || !bQn || c->nscen != 1) return DGR_ERR_INVALID;
    if (c->nbnd == 0) return DGR_OK;
    CK(cudaSetDevice(c->device));
    /* only prescribed edges are read by the flux; copy those through a compact stage
     * (the pinned stage may still feed the previous copy: wait for the stream first) */
    CK(cudaStreamSynchronize(c->stream));
    const std::vector<int> &be = c->h_bnd;
    for (int j = 0; j < c->nbnd; ++j) {
        c->h_stage[j] = bzeta[be[j]];
        c->h_stage[c->nbnd + j] = bQn[be[j]];
    }
    CK(cudaMemcpyAsync(c->bstage, c->h_stage, sizeof(double) * 2 * c->nbnd, cudaMemcpyHostToDevice, c->stream));
    k_scatter_bnd<<<blocks(c->nbnd, 256), 256, 0, c->stream>>>(c->nbnd, c->bnd_edges, c->bstage, c->bzeta, c->bqn);
    c->launches++;
    CK(cudaGetLastError());
    return DGR_OK;
}

extern "C" int dgr_boundary_conditions(dgr_ctx *c, double time)
{
    if (!c) return DGR_ERR_INVALID;
    if (c->nbnd == 0) return DGR_OK;
    CK(cudaSetDevice(c->device));
    k_forcing<<<blocks(c->nbnd, 256), 256, 0, c->stream>>>(c->clk, time, c->bnd_edges, c->bnd_type, c->bnd_sid,
                                                           c->nbnd, c->bzeta, c->bqn);
    c->launches++;
    CK(cudaGetLastError());
    return DGR_OK;
}

/* --------------------------------------------------------------- launches ---- */

static const int *wd_current(const dgr_ctx *c) { return c->wd_stepped ? wd_after_step(c) : c->wdA; }

template <int MODE>
static void launch_element(dgr_ctx *c, const double *S, const int *wd, double *OUT)
{
    const MeshDev m = mesh_dev(c);
    cudaStream_t s = c->stream;
    switch (c->bs) {
    case 64:
        k_element<MODE, 64><<<blocks(c->ne, 64), 64, 0, s>>>(m, S, c->U, wd, c->flux, OUT, c->avg, c->clk, c->p.g);
        break;
    case 256:
        k_element<MODE, 256><<<blocks(c->ne, 256), 256, 0, s>>>(m, S, c->U, wd, c->flux, OUT, c->avg, c->clk, c->p.g);
        break;
    default:
        k_element<MODE, 128><<<blocks(c->ne, 128), 128, 0, s>>>(m, S, c->U, wd, c->flux, OUT, c->avg, c->clk, c->p.g);
    }
}

/* the plain-division redo of the items k_limit queued (nothing queued: the blocks return
 * at once); no launch when the limiter takes plain divisions itself */
template <bool L, bool P, bool ST>
static void launch_limit_redo(dgr_ctx *c, double *S, const int *wd_in, int *wd_out, int phase, int *dl, int *dp)
{
    if (!DGR_LIMIT_RCP) return;
    k_limit_redo<L, P, ST><<<c->num_sms, 128, 0, c->stream>>>(mesh_dev(c), S, c->bounds, wd_in, wd_out, c->clk,
                                                              c->p.H0, c->p.VELZERO, phase, dl, dp);
    c->launches++;
}

template <bool L, bool P, bool ST>
static void launch_limit(dgr_ctx *c, double *S, const int *wd_in, int *wd_out, int phase, int *dl, int *dp)
{
    const MeshDev m = mesh_dev(c);
    cudaStream_t s = c->stream;
    const double h0 = c->p.H0, vz = c->p.VELZERO;
    switch (c->bs) {
    case 64:
        k_limit<L, P, ST, 64><<<blocks(c->ne, 64), 64, 0, s>>>(m, S, c->bounds, wd_in, wd_out, c->clk, h0, vz, phase,
                                                               dl, dp);
        break;
    case 256:
        k_limit<L, P, ST, 256><<<blocks(c->ne, 256), 256, 0, s>>>(m, S, c->bounds, wd_in, wd_out, c->clk, h0, vz,
                                                                  phase, dl, dp);
        break;
    default:
        k_limit<L, P, ST, 128><<<blocks(c->ne, 128), 128, 0, s>>>(m, S, c->bounds, wd_in, wd_out, c->clk, h0, vz,
                                                                  phase, dl, dp);
    }
    launch_limit_redo<L, P, ST>(c, S, wd_in, wd_out, phase, dl, dp);
}

template <bool WD, int FT>
static void launch_edge_ft(dgr_ctx *c, const double *S, const int *wd, int lam_slot, int phase)
{
    const MeshDev m = mesh_dev(c);
    k_edge_flux<WD, FT><<<blocks(c->nf, DGR_EDGE_BS), DGR_EDGE_BS, 0, c->stream>>>(m, S, wd, c->bzeta, c->bqn, c->flux, c->clk,
                                                                   lam_slot, phase, c->p.g);
    if (DGR_EDGE_RCP) {
        k_edge_redo<WD, FT><<<c->num_sms, 256, 0, c->stream>>>(m, S, wd, c->bzeta, c->bqn, c->flux, c->clk,
                                                               lam_slot, phase, c->p.g);
        c->launches++;
    }
}

/* the edge kernel compiled for the context's wet/dry mode and numerical flux */
void launch_edge(dgr_ctx *c, const double *S, const int *wd, int lam_slot, int phase)
{
    const bool w = c->p.wet_dry != 0;
    switch (c->p.flux) {
    case 1: w ? launch_edge_ft<true, 1>(c, S, wd, lam_slot, phase) : launch_edge_ft<false, 1>(c, S, wd, lam_slot, phase); break;
    case 2: w ? launch_edge_ft<true, 2>(c, S, wd, lam_slot, phase) : launch_edge_ft<false, 2>(c, S, wd, lam_slot, phase); break;
    default: w ? launch_edge_ft<true, 0>(c, S, wd, lam_slot, phase) : launch_edge_ft<false, 0>(c, S, wd, lam_slot, phase);
    }
}

/* p = 2 edge fluxes of state S: the Roe flux compiled alone, the other fluxes by run-time
 * choice */
void launch_p2_edge(dgr_ctx *c, const double *S, int lam_slot, int phase)
{
    const MeshDev m = mesh_dev(c);
    if (c->p.flux == 0)
        k_p2_edge<128, 0><<<blocks(c->nf, 128), 128, 0, c->stream>>>(c->p2ref, m, c->p2g, S, c->bzeta, c->bqn,
                                                                     c->flux, c->clk, lam_slot, phase, c->p.g);
    else
        k_p2_edge<128, -1><<<blocks(c->nf, 128), 128, 0, c->stream>>>(c->p2ref, m, c->p2g, S, c->bzeta, c->bqn,
                                                                      c->flux, c->clk, lam_slot, phase, c->p.g);
}

/* one RK stage of the p = 2 step: edge fluxes at the Gauss points, element update */
static void launch_p2_stage(dgr_ctx *c, int stage, bool count)
{
    const StageIO io = stage_io(c, stage);
    const MeshDev m = mesh_dev(c);
    cudaStream_t s = c->stream;
    launch_p2_edge(c, io.S, stage, 2 * stage);
    const unsigned nb = blocks(c->ne, 128);
    switch (io.mode) {
    case MODE_STAGE1:
        k_p2_element<MODE_STAGE1, 128><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, c->U, c->flux, io.OUT, c->clk,
                                                          c->p.g);
        break;
    case MODE_STAGE2:
        k_p2_element<MODE_STAGE2, 128><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, c->U, c->flux, io.OUT, c->clk,
                                                          c->p.g);
        break;
    case MODE_RK3_2:
        k_p2_element<MODE_RK3_2, 128><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, c->U, c->flux, io.OUT, c->clk,
                                                         c->p.g);
        break;
    default:
        k_p2_element<MODE_RK3_3, 128><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, c->U, c->flux, io.OUT, c->clk,
                                                         c->p.g);
    }
    if (count) c->launches += 2;
}

/* one RK stage as four kernels (buffers of stage_io) */
void launch_stage(dgr_ctx *c, int stage, bool count)
{
    if (c->p.order == 2) {
        launch_p2_stage(c, stage, count);
        return;
    }
    const bool wd = c->p.wet_dry != 0;
    const StageIO io = stage_io(c, stage);
    int *dl = c->p.record_decisions ? c->dec + (size_t)(2 * stage) * c->ne : nullptr;
    int *dp = c->p.record_decisions ? c->dec + (size_t)(2 * stage + 1) * c->ne : nullptr;
    {
        NvtxRange r("k_edge_flux");
        launch_edge(c, io.S, io.wd_in, stage, 2 * stage);
    }
    {
        NvtxRange r("k_element");
        switch (io.mode) {
        case MODE_STAGE1: launch_element<MODE_STAGE1>(c, io.S, io.wd_in, io.OUT); break;
        case MODE_STAGE2: launch_element<MODE_STAGE2>(c, io.S, io.wd_in, io.OUT); break;
        case MODE_RK3_2: launch_element<MODE_RK3_2>(c, io.S, io.wd_in, io.OUT); break;
        default: launch_element<MODE_RK3_3>(c, io.S, io.wd_in, io.OUT);
        }
    }
    {
        NvtxRange r("k_node_bounds");
        k_node_bounds<<<blocks(c->nn, DGR_NODE_BS), DGR_NODE_BS, 0, c->stream>>>(mesh_dev(c), c->avg, c->bounds);
    }
    {
        NvtxRange r("k_limit");
        if (wd)
            launch_limit<true, true, true>(c, io.OUT, io.wd_in, io.wd_out, 2 * stage + 1, dl, dp);
        else
            launch_limit<true, false, false>(c, io.OUT, io.wd_in, io.wd_out, 2 * stage + 1, dl, dp);
    }
    if (count) c->launches += 4; /* edge flux, element, node bounds, limiter (redo launches count themselves) */
}

void launch_wd_refresh(dgr_ctx *c)
{
    if (c->p.wet_dry && !c->wd_fresh) {
        /* the flags the caller sees (WA after an upload, WB after a step) seed the status */
        if (c->wd_stepped)
            cudaMemcpyAsync(c->wdA, wd_after_step(c), (size_t)c->ne * 4, cudaMemcpyDeviceToDevice, c->stream);
        k_wd_status<<<blocks(c->ne, 256), 256, 0, c->stream>>>(mesh_dev(c), c->U, c->wdA, c->clk, c->p.H0);
        c->launches++;
        c->wd_fresh = 1;
    }
}

/* persistent fused kernel: grid of co-resident blocks, cooperative launch */
static FusedArgs fused_args(dgr_ctx *c)
{
    FusedArgs a;
    a.m = mesh_dev(c);
    a.U = c->U;
    a.W = c->W;
    a.flux = c->flux;
    a.avg = c->avg;
    a.bounds = c->bounds;
    a.bzeta = c->bzeta;
    a.bqn = c->bqn;
    a.wdA = c->wdA;
    a.wdB = c->wdB;
    a.wdC = c->wdC;
    a.clk = c->clk;
    a.nscen = c->nscen;
    a.bnd_edges = c->bnd_edges;
    a.bnd_type = c->bnd_type;
    a.bnd_sid = c->bnd_sid;
    a.nbnd = c->nbnd;
    a.p = phys(c);
    a.dec = c->p.record_decisions ? c->dec : nullptr;
    a.bar = c->bar;
    a.bar_polls = c->bar_polls;
    a.bar_phantom = c->bar_phantom;
    return a;
}

template <bool WD, int BS>
static cudaError_t launch_fused_bs(dgr_ctx *c, int stage_begin, int stage_end, int with_clock)
{
    auto fn = k_step_fused<WD, BS>;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, BS, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int need = (int)blocks(std::max(std::max(c->ne, c->nf), c->nn), BS);
    const int grid = std::max(1, std::min(per_sm * c->num_sms, need));
    FusedArgs a = fused_args(c);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(BS);
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    /* arrivals and generation start at zero; the time-out flag (bar[2]) is left alone, so a
     * time-out of any launch of a run is still seen when the run ends */
    e = cudaMemsetAsync(c->bar, 0, 8, c->stream);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernelEx(&cfg, fn, a, stage_begin, stage_end, with_clock);
}

static cudaError_t launch_fused(dgr_ctx *c, int stage_begin, int stage_end, int with_clock)
{
    const bool wd = c->p.wet_dry != 0;
    switch (c->bs) {
    case 64:
        return wd ? launch_fused_bs<true, 64>(c, stage_begin, stage_end, with_clock)
                  : launch_fused_bs<false, 64>(c, stage_begin, stage_end, with_clock);
    case 256:
        return wd ? launch_fused_bs<true, 256>(c, stage_begin, stage_end, with_clock)
                  : launch_fused_bs<false, 256>(c, stage_begin, stage_end, with_clock);
    default:
        return wd ? launch_fused_bs<true, 128>(c, stage_begin, stage_end, with_clock)
                  : launch_fused_bs<false, 128>(c, stage_begin, stage_end, with_clock);
    }
}

/* One step of the device loop with the current schedule. */
static cudaError_t launch_step(dgr_ctx *c)
{
    cudaStream_t s = c->stream;
    const PhysParams p = phys(c);
    const int ns = c->p.rk_stages;
    if (c->fusion == 2 && c->p.order == 1) {
        cudaError_t e = launch_fused(c, 0, ns, 1);
        if (e != cudaSuccess) return e;
    } else {
        k_clock_begin<<<1, 256, 0, s>>>(c->clk, c->nscen, p, c->bnd_edges, c->bnd_type, c->bnd_sid, c->nbnd,
                                        c->bzeta, c->bqn);
        for (int st = 0; st < ns; ++st) {
            if (c->fusion == 1 && c->p.order == 1) {
                cudaError_t e = launch_fused(c, st, st + 1, 0);
                if (e != cudaSuccess) return e;
            } else {
                launch_stage(c, st, false);
            }
        }
        k_clock_end<<<blocks(c->nscen, 256), 256, 0, s>>>(c->clk, c->nscen);
    }
    if (c->gauge_n)
        k_gauge_record<<<blocks(c->gauge_n, 128), 128, 0, s>>>(c->U, c->ldE, c->nm, c->gauge_n, c->gauge_el,
                                                               c->gauge_sid, c->gauge_w, c->clk, c->gauge_cap,
                                                               c->gauge_series);
    return cudaGetLastError();
}

static int kernels_per_step(const dgr_ctx *c)
{
    const int ns = c->p.rk_stages;
    const int rec = c->gauge_n ? 1 : 0;
    if (c->p.order == 2) return 2 + 2 * ns + rec;
    return rec + (c->fusion == 2 ? 1 : (c->fusion == 1 ? 2 + ns : 2 + (4 + DGR_EDGE_RCP + DGR_LIMIT_RCP) * ns));
}

int decode_err(unsigned long long key, int *code, int *index, int *step)
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

/* Checked build: the first out-of-range gather recorded by the kernels, as
 * (kernel << 32 | item), or ~0. */
static unsigned long long bad_index(const dgr_ctx *c)
{
    unsigned long long bad = ~0ull;
#ifdef DGR_CHECKED
    if (cudaMemcpy(&bad, c->bar + 4, 8, cudaMemcpyDeviceToHost) != cudaSuccess) bad = ~0ull;
#else
    (void)c;
#endif
    return bad;
}

int first_error(const dgr_ctx *c)
{
    if (bad_index(c) != ~0ull) return DGR_ERR_BAD_INDEX;
    for (int k = 0; k < c->nscen; ++k) {
        const int cd = decode_err(c->h_clk[k].err, nullptr, nullptr, nullptr);
        if (cd) return cd;
    }
    return DGR_OK;
}

static int check_barrier(dgr_ctx *c)
{
    if (c->fusion == 0) return DGR_OK;
    unsigned flag = 0;
    CK(cudaMemcpy(&flag, c->bar + 2, 4, cudaMemcpyDeviceToHost));
    return flag ? DGR_ERR_TIMEOUT : DGR_OK;
}

/* The RK stages of one host-driven step (dgr_step) captured into a graph of their own,
 * on the first call after the context's launches last changed (drop_graph); where the
 * capture fails the stages run eagerly, without another attempt until then. */
static void build_stage_graph(dgr_ctx *c)
{
    c->stage_graph_tried = 1;
    cudaStream_t s = c->stream;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    const long long l0 = c->launches; /* captured launches are counted when they run */
    for (int st = 0; st < c->p.rk_stages; ++st) launch_stage(c, st, false);
    c->launches = l0;
    cudaError_t e = cudaGetLastError();
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess || e2 != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return;
    }
    if (cudaGraphInstantiate(&c->stage_graph_exec, g, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        c->stage_graph_exec = nullptr;
        return;
    }
    c->stage_graph = g;
}

extern "C" int dgr_step(dgr_ctx *c, double time, double dt, double *max_lambda)
{
    NvtxRange nv("dgr_step");
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    CK(cudaEventRecord(c->ev0, s));
    if (!c->stage_graph_exec && !c->stage_graph_tried) build_stage_graph(c);
    k_clock_set<<<1, 1, 0, s>>>(c->clk, time, dt);
    c->launches++;
    launch_wd_refresh(c);
    if (c->stage_graph_exec) {
        CK(cudaGraphLaunch(c->stage_graph_exec, s));
        c->launches += (long long)c->p.rk_stages * (c->p.order == 2 ? 2 : 4 + DGR_EDGE_RCP + DGR_LIMIT_RCP);
    } else {
        for (int st = 0; st < c->p.rk_stages; ++st) launch_stage(c, st, true);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, s));
    if (c->p.wet_dry) {
        c->wd_fresh = 1;
        c->wd_stepped = 1;
    }
    int r = read_clock(c);
    if (r) return r;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    if (max_lambda) *max_lambda = bits_to_double(c->h_clk[0].lam_bits[c->p.rk_stages - 1]);
    return decode_err(c->h_clk[0].err, nullptr, nullptr, nullptr);
}

extern "C" int dgr_compute_L(dgr_ctx *c, double time, double *rz, double *rqx, double *rqy, double *max_lambda)
{
    (void)time;
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    k_clock_set<<<1, 1, 0, s>>>(c->clk, 0.0, 0.0);
    if (c->p.order == 2) {
        const MeshDev m = mesh_dev(c);
        launch_p2_edge(c, c->U, 0, 0);
        k_p2_element<MODE_RHS, 128><<<blocks(c->ne, 128), 128, 0, s>>>(c->p2ref, m, c->p2g, c->U, c->U, c->flux,
                                                                       c->W, c->clk, c->p.g);
    } else {
        const int *wd = wd_current(c);
        launch_edge(c, c->U, wd, 0, 0);
        k_element<MODE_RHS, 128><<<blocks(c->ne, 128), 128, 0, s>>>(mesh_dev(c), c->U, c->U, wd, c->flux, c->W,
                                                                    c->avg, c->clk, c->p.g);
    }
    c->launches += 3;
    CK(cudaGetLastError());
    if (rz && rqx && rqy) {
        const size_t n3 = (size_t)c->nm * c->ne;
        double *tmp = nullptr; /* stream-ordered staging for the reference layout */
        CK(cudaMallocAsync((void **)&tmp, 3 * n3 * 8, s));
        k_planar_to_aos_nm<<<blocks(c->ne, 256), 256, 0, s>>>(c->ne, c->ldE, c->nm, c->W, tmp, tmp + n3,
                                                              tmp + 2 * n3);
        c->launches++;
        CK(cudaMemcpyAsync(rz, tmp, n3 * 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(rqx, tmp + n3, n3 * 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(rqy, tmp + 2 * n3, n3 * 8, cudaMemcpyDeviceToHost, s));
        CK(cudaFreeAsync(tmp, s));
    }
    int r = read_clock(c);
    if (r) return r;
    if (max_lambda) *max_lambda = bits_to_double(c->h_clk[0].lam_bits[0]);
    return decode_err(c->h_clk[0].err, nullptr, nullptr, nullptr);
}

extern "C" int dgr_get_fhat(dgr_ctx *c, double *f1, double *f2, double *f3)
{
    if (!c || !f1 || !f2 || !f3 || c->nscen != 1) return DGR_ERR_INVALID;
    if (c->p.order != 1) return DGR_ERR_INVALID; /* p = 1 operators */
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
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    if (c->p.order != 1) return DGR_ERR_INVALID; /* p = 1 operators */
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const MeshDev m = mesh_dev(c);
    k_clock_set<<<1, 1, 0, s>>>(c->clk, 0.0, 0.0);
    k_avg<<<blocks(c->ne, 256), 256, 0, s>>>(m, c->U, c->avg);
    k_node_bounds<<<blocks(c->nn, DGR_NODE_BS), DGR_NODE_BS, 0, s>>>(m, c->avg, c->bounds);
    int *dl = c->p.record_decisions ? c->dec : nullptr;
    k_limit<true, false, false, 128><<<blocks(c->ne, 128), 128, 0, s>>>(m, c->U, c->bounds, c->wdA, c->wdA, c->clk,
                                                                         c->p.H0, c->p.VELZERO, 0, dl, nullptr);
    launch_limit_redo<true, false, false>(c, c->U, c->wdA, c->wdA, 0, dl, nullptr);
    c->launches += 4;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    c->wd_fresh = 0;
    return DGR_OK;
}

extern "C" int dgr_pdop(dgr_ctx *c)
{
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    if (c->p.order != 1) return DGR_ERR_INVALID; /* p = 1 operators */
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    k_clock_set<<<1, 1, 0, s>>>(c->clk, 0.0, 0.0);
    int *dp = c->p.record_decisions ? c->dec + c->ne : nullptr;
    k_limit<false, true, false, 128><<<blocks(c->ne, 128), 128, 0, s>>>(mesh_dev(c), c->U, c->bounds, c->wdA,
                                                                         c->wdA, c->clk, c->p.H0, c->p.VELZERO, 1,
                                                                         nullptr, dp);
    launch_limit_redo<false, true, false>(c, c->U, c->wdA, c->wdA, 1, nullptr, dp);
    c->launches += 2;
    CK(cudaGetLastError());
    int r = read_clock(c);
    if (r) return r;
    c->wd_fresh = 0;
    return decode_err(c->h_clk[0].err, nullptr, nullptr, nullptr);
}

extern "C" int dgr_wet_dry_status(dgr_ctx *c)
{
    if (!c || c->nscen != 1) return DGR_ERR_INVALID;
    if (c->p.order != 1) return DGR_ERR_INVALID; /* p = 1 operators */
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    int *wd = c->wd_stepped ? wd_after_step(c) : c->wdA;
    k_clock_set<<<1, 1, 0, s>>>(c->clk, 0.0, 0.0);
    k_wd_status<<<blocks(c->ne, 256), 256, 0, s>>>(mesh_dev(c), c->U, wd, c->clk, c->p.H0);
    c->launches += 2;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    c->wd_fresh = 0;
    return DGR_OK;
}

/* ---------------------------------------------------------- device loop ---- */

/* Capture one step with the current schedule into a graph (eager launches when the
 * schedule cannot be captured). */
static int build_graph(dgr_ctx *c)
{
    drop_graph(c);
    cudaStream_t s = c->stream;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const long long l0 = c->launches; /* captured launches are counted when they run */
    cudaError_t e = launch_step(c);
    c->launches = l0;
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return DGR_OK; /* run eagerly */
    }
    c->graph = g;
    if (cudaGraphInstantiate(&c->graph_exec, c->graph, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(c->graph);
        c->graph = nullptr;
        c->graph_exec = nullptr;
    }
    return DGR_OK;
}

/* Device loop for all scenarios: per scenario start clock (time_io[s] < 0 starts at t = 0
 * with dt0), final time, and the common step limit. */
static int run_impl(dgr_ctx *c, int nsteps, const double *final_time, double *time_io, double *dt_io,
                    int *steps_done)
{
    NvtxRange nv("dgr_run");
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    int r = read_clock(c);
    if (r) return r;
    for (int k = 0; k < c->nscen; ++k) {
        DevClock &h = c->h_clk[k];
        double t0 = time_io[k], dt = dt_io[k];
        if (t0 < 0) {
            t0 = 0.0;
            dt = c->p.dt0;
        }
        h.time = t0;
        h.dt = dt;
        h.final_time = final_time[k];
        h.step = 0;
        h.nsteps = nsteps;
        h.done = 0;
        h.dt_pending = 0;
    }
    r = write_clock(c);
    if (r) return r;
    if (!c->graph_exec) {
        r = build_graph(c);
        if (r) return r;
    }
    if (c->fusion) CK(cudaMemsetAsync(c->bar + 2, 0, 4, s)); /* no barrier time-out yet */
    CK(cudaEventRecord(c->ev0, s));
    launch_wd_refresh(c);
    for (int i = 0; i < nsteps; ++i) {
        if (c->graph_exec)
            CK(cudaGraphLaunch(c->graph_exec, s));
        else
            CK(launch_step(c));
    }
    c->launches += (long long)nsteps * kernels_per_step(c);
    k_clock_finish<<<blocks(c->nscen, 256), 256, 0, s>>>(c->clk, c->nscen, phys(c));
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, s));
    r = read_clock(c);
    if (r) return r;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    int any_step = 0;
    for (int k = 0; k < c->nscen; ++k) {
        time_io[k] = c->h_clk[k].time;
        dt_io[k] = c->h_clk[k].dt;
        if (steps_done) steps_done[k] = c->h_clk[k].step;
        any_step |= c->h_clk[k].step > 0;
    }
    if (c->p.wet_dry && any_step) {
        c->wd_fresh = 1;
        c->wd_stepped = 1;
    }
    r = check_barrier(c);
    if (r) return r;
    return first_error(c);
}

extern "C" int dgr_run(dgr_ctx *c, int nsteps, double final_time, double *time_io, double *dt_io, int *steps_done)
{
    if (!c || !time_io || !dt_io || nsteps < 0 || c->nscen != 1) return DGR_ERR_INVALID;
    return run_impl(c, nsteps, &final_time, time_io, dt_io, steps_done);
}

extern "C" int dgr_ensemble_run(dgr_ctx *c, int nsteps, const double *final_time, double *time_io, double *dt_io,
                                int *steps_done)
{
    if (!c || !final_time || !time_io || !dt_io || nsteps < 0) return DGR_ERR_INVALID;
    return run_impl(c, nsteps, final_time, time_io, dt_io, steps_done);
}

extern "C" int dgr_ensemble_last_error(dgr_ctx *c, int scenario, int *code, int *index, int *step)
{
    if (!c || scenario < 0 || scenario >= c->nscen) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    int r = read_clock(c);
    if (r) return r;
    decode_err(c->h_clk[scenario].err, code, index, step);
    const unsigned long long bad = bad_index(c);
    if (bad != ~0ull) { /* checked build: the item and, in place of the step, the kernel */
        if (code) *code = DGR_ERR_BAD_INDEX;
        if (index) *index = (int)(bad & 0xffffffffu);
        if (step) *step = (int)(bad >> 32);
    }
    return DGR_OK;
}

extern "C" int dgr_last_error(dgr_ctx *c, int *code, int *index, int *step)
{
    return dgr_ensemble_last_error(c, 0, code, index, step);
}

extern "C" int dgr_set_barrier_wait(dgr_ctx *c, unsigned max_polls, unsigned phantom_blocks)
{
    if (!c || max_polls == 0 || phantom_blocks > 1) return DGR_ERR_INVALID;
    c->bar_polls = max_polls;
    c->bar_phantom = phantom_blocks;
    drop_graph(c); /* the captured launches hold the old values */
    return DGR_OK;
}

extern "C" int dgr_set_schedule(dgr_ctx *c, int block_size, int fusion)
{
    if (!c || (block_size != 64 && block_size != 128 && block_size != 256) || fusion < 0 || fusion > 2)
        return DGR_ERR_INVALID;
    if (c->p.order == 2 && fusion != 0) return DGR_ERR_INVALID; /* the p = 2 step has no fused kernel */
    c->bs = block_size;
    c->fusion = fusion;
    drop_graph(c);
    return DGR_OK;
}

extern "C" int dgr_get_schedule(const dgr_ctx *c, int *block_size, int *fusion)
{
    if (!c) return DGR_ERR_INVALID;
    if (block_size) *block_size = c->bs;
    if (fusion) *fusion = c->fusion;
    return DGR_OK;
}

/*
 * Autotuner: times trial_steps steps of the device loop for every schedule (block size
 * 64/128/256 x fusion depth 0/1/2) from the current state, restoring state, flags and
 * clocks after each trial, and keeps the fastest.  Results do not depend on the schedule
 * (same items, same arithmetic); only the time does.  ms_out (9 entries, or NULL)
 * receives the ms per step of each trial at index 3*b + f (b: 64, 128, 256; f: fusion),
 * -1 where the schedule could not run.
 */
/* The trials of dgr_autotune, with the state saved in saveU/saveWD (owned by the caller,
 * which frees them on every return path). */
static int autotune_trials(dgr_ctx *c, int trial_steps, double *saveU, int *saveWD, int *best_bs_out,
                           int *best_f_out, double *ms_out)
{
    cudaStream_t s = c->stream;
    const size_t nU = 3 * (size_t)c->nm * c->ldE;
    CK(cudaMemcpyAsync(saveU, c->U, nU * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(saveWD, c->wdA, (size_t)c->ne * 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(saveWD + c->ne, c->wdB, (size_t)c->ne * 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(saveWD + 2 * (size_t)c->ne, c->wdC, (size_t)c->ne * 4, cudaMemcpyDeviceToDevice, s));
    int r = read_clock(c);
    if (r) return r;
    const std::vector<DevClock> clk0(c->h_clk, c->h_clk + c->nscen);
    const int fresh0 = c->wd_fresh, curB0 = c->wd_stepped;
    const int bss[3] = {64, 128, 256};
    double best = 1e300;
    int best_bs = c->bs, best_f = c->fusion;
    std::vector<double> t(c->nscen), d(c->nscen), fin(c->nscen, 1e300);
    for (int b = 0; b < 3; ++b)
        for (int f = 0; f < (c->p.order == 2 ? 1 : 3); ++f) {
            c->bs = bss[b];
            c->fusion = f;
            drop_graph(c);
            for (int k = 0; k < c->nscen; ++k) {
                t[k] = clk0[k].time;
                d[k] = clk0[k].dt > 0 ? clk0[k].dt : c->p.dt0;
            }
            /* one untimed step builds the graph and warms the caches */
            int rc = run_impl(c, 1, fin.data(), t.data(), d.data(), nullptr);
            double ms = -1.0;
            if (rc == DGR_OK) {
                rc = run_impl(c, trial_steps, fin.data(), t.data(), d.data(), nullptr);
                if (rc == DGR_OK) ms = c->last_ms / trial_steps;
            }
            cudaGetLastError();
            if (ms_out) ms_out[3 * b + f] = ms;
            if (ms > 0 && ms < best) {
                best = ms;
                best_bs = bss[b];
                best_f = f;
            }
            /* restore */
            CK(cudaMemcpyAsync(c->U, saveU, nU * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(c->wdA, saveWD, (size_t)c->ne * 4, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(c->wdB, saveWD + c->ne, (size_t)c->ne * 4, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(c->wdC, saveWD + 2 * (size_t)c->ne, (size_t)c->ne * 4, cudaMemcpyDeviceToDevice, s));
            std::copy(clk0.begin(), clk0.end(), c->h_clk);
            r = write_clock(c);
            if (r) return r;
            CK(cudaMemsetAsync(c->bar, 0, 16, s));
            c->wd_fresh = fresh0;
            c->wd_stepped = curB0;
        }
    *best_bs_out = best_bs;
    *best_f_out = best_f;
    return best < 1e300 ? DGR_OK : DGR_ERR_CUDA;
}

extern "C" int dgr_autotune(dgr_ctx *c, int trial_steps, int *block_size, int *fusion, double *ms_out)
{
    NvtxRange nv("dgr_autotune");
    if (!c || trial_steps <= 0) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const size_t nU = 3 * (size_t)c->nm * c->ldE;
    double *saveU = nullptr;
    int *saveWD = nullptr;
    CK(cudaMallocAsync((void **)&saveU, nU * 8, s));
    if (cudaMallocAsync((void **)&saveWD, 3 * (size_t)c->ne * 4, s) != cudaSuccess) {
        cudaFreeAsync(saveU, s);
        return DGR_ERR_CUDA;
    }
    int best_bs = c->bs, best_f = c->fusion;
    const int rc = autotune_trials(c, trial_steps, saveU, saveWD, &best_bs, &best_f, ms_out);
    const cudaError_t e1 = cudaFreeAsync(saveU, s), e2 = cudaFreeAsync(saveWD, s);
    const cudaError_t e3 = cudaStreamSynchronize(s);
    c->bs = best_bs;
    c->fusion = best_f;
    drop_graph(c);
    if (rc) return rc;
    CK(e1);
    CK(e2);
    CK(e3);
    if (block_size) *block_size = best_bs;
    if (fusion) *fusion = best_f;
    return DGR_OK;
}

extern "C" int dgr_get_decisions(dgr_ctx *c, int stage, int *limit, int *pdop)
{
    if (!c || stage < 0 || stage >= c->p.rk_stages) return DGR_ERR_INVALID;
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
 * Per-kernel device timing of whole steps: CUDA events around every launch of nsteps
 * steps (dt of the last run, or dt0) with the four-kernel schedule.  kernel_ms[0..3]
 * receive the average ms of one launch of: edge flux, element RHS+RK, node bounds,
 * limiter+PDop.
 */
/* dgr_profile_step of the p = 2 step: kernel_ms[0] edge fluxes, [1] element update */
static int profile_p2(dgr_ctx *c, int nsteps, double *kernel_ms)
{
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    cudaEvent_t ev[3];
    for (int i = 0; i < 3; ++i) CK(cudaEventCreate(&ev[i]));
    double acc[2] = {0, 0};
    int r = read_clock(c);
    if (r) return r;
    for (int k = 0; k < c->nscen; ++k) {
        if (!(c->h_clk[k].dt > 0)) c->h_clk[k].dt = c->p.dt0;
        c->h_clk[k].done = 0;
    }
    r = write_clock(c);
    if (r) return r;
    const MeshDev m = mesh_dev(c);
    int rc = DGR_OK;
    for (int it = 0; it < nsteps && rc == DGR_OK; ++it)
        for (int stage = 0; stage < c->p.rk_stages; ++stage) {
            const StageIO io = stage_io(c, stage);
            cudaEventRecord(ev[0], s);
            launch_p2_edge(c, io.S, stage, 2 * stage);
            cudaEventRecord(ev[1], s);
            const unsigned nb = blocks(c->ne, 128);
            if (io.mode == MODE_STAGE1)
                k_p2_element<MODE_STAGE1, 128><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, c->U, c->flux, io.OUT,
                                                                  c->clk, c->p.g);
            else if (io.mode == MODE_STAGE2)
                k_p2_element<MODE_STAGE2, 128><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, c->U, c->flux, io.OUT,
                                                                  c->clk, c->p.g);
            else if (io.mode == MODE_RK3_2)
                k_p2_element<MODE_RK3_2, 128><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, c->U, c->flux, io.OUT,
                                                                 c->clk, c->p.g);
            else
                k_p2_element<MODE_RK3_3, 128><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, c->U, c->flux, io.OUT,
                                                                 c->clk, c->p.g);
            cudaEventRecord(ev[2], s);
            c->launches += 2;
            if (cudaEventSynchronize(ev[2]) != cudaSuccess) {
                rc = DGR_ERR_CUDA;
                break;
            }
            for (int k = 0; k < 2; ++k) {
                float ms = 0;
                cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
                acc[k] += ms;
            }
        }
    for (int i = 0; i < 3; ++i) cudaEventDestroy(ev[i]);
    if (rc) return rc;
    CK(cudaGetLastError());
    kernel_ms[0] = acc[0] / ((double)c->p.rk_stages * nsteps);
    kernel_ms[1] = acc[1] / ((double)c->p.rk_stages * nsteps);
    kernel_ms[2] = kernel_ms[3] = 0.0;
    return DGR_OK;
}

extern "C" int dgr_profile_step(dgr_ctx *c, int nsteps, double *kernel_ms, int n)
{
    if (!c || nsteps <= 0 || !kernel_ms || n < 4) return DGR_ERR_INVALID;
    if (c->p.order == 2) return profile_p2(c, nsteps, kernel_ms);
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const bool wd = c->p.wet_dry != 0;
    cudaEvent_t ev[5];
    for (int i = 0; i < 5; ++i) CK(cudaEventCreate(&ev[i]));
    double acc[4] = {0, 0, 0, 0};
    int r = read_clock(c);
    if (r) return r;
    for (int k = 0; k < c->nscen; ++k) {
        if (!(c->h_clk[k].dt > 0)) c->h_clk[k].dt = c->p.dt0;
        c->h_clk[k].done = 0;
    }
    r = write_clock(c);
    if (r) return r;
    int rc = DGR_OK;
    for (int it = 0; it < nsteps && rc == DGR_OK; ++it) {
        launch_wd_refresh(c);
        for (int stage = 0; stage < c->p.rk_stages; ++stage) {
            const StageIO io = stage_io(c, stage);
            const double *S = io.S;
            double *OUT = io.OUT;
            const int *wd_in = io.wd_in;
            int *wd_out = io.wd_out;
            cudaEventRecord(ev[0], s);
            launch_edge(c, S, wd_in, stage, 2 * stage);
            cudaEventRecord(ev[1], s);
            switch (io.mode) {
            case MODE_STAGE1: launch_element<MODE_STAGE1>(c, S, wd_in, OUT); break;
            case MODE_STAGE2: launch_element<MODE_STAGE2>(c, S, wd_in, OUT); break;
            case MODE_RK3_2: launch_element<MODE_RK3_2>(c, S, wd_in, OUT); break;
            default: launch_element<MODE_RK3_3>(c, S, wd_in, OUT);
            }
            cudaEventRecord(ev[2], s);
            k_node_bounds<<<blocks(c->nn, DGR_NODE_BS), DGR_NODE_BS, 0, s>>>(mesh_dev(c), c->avg, c->bounds);
            cudaEventRecord(ev[3], s);
            if (wd)
                launch_limit<true, true, true>(c, OUT, wd_in, wd_out, 2 * stage + 1, nullptr, nullptr);
            else
                launch_limit<true, false, false>(c, OUT, wd_in, wd_out, 2 * stage + 1, nullptr, nullptr);
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
            c->wd_stepped = 1;
        }
    }
    for (int i = 0; i < 5; ++i) cudaEventDestroy(ev[i]);
    if (rc) return rc;
    CK(cudaGetLastError());
    for (int k = 0; k < 4; ++k) kernel_ms[k] = acc[k] / ((double)c->p.rk_stages * nsteps);
    return DGR_OK;
}

extern "C" int dgr_p2_reference(double *t, int n)
{
    if (!t || n < 234) return DGR_ERR_INVALID;
    const P2Ref R = make_p2_ref();
    int i = 0;
    for (int q = 0; q < P2_NQ; ++q) t[i++] = R.wq[q];
    for (int q = 0; q < P2_NQ; ++q)
        for (int k = 0; k < 3; ++k) t[i++] = R.lam[q][k];
    for (int q = 0; q < P2_NQ; ++q)
        for (int m = 0; m < P2_NM; ++m) t[i++] = R.phi[q][m];
    for (int q = 0; q < P2_NQ; ++q)
        for (int m = 0; m < P2_NM; ++m) t[i++] = R.dr[q][m];
    for (int q = 0; q < P2_NQ; ++q)
        for (int m = 0; m < P2_NM; ++m) t[i++] = R.ds[q][m];
    for (int gp = 0; gp < P2_NGP; ++gp) t[i++] = R.te[gp];
    for (int gp = 0; gp < P2_NGP; ++gp) t[i++] = R.wg[gp];
    for (int k = 0; k < 3; ++k)
        for (int gp = 0; gp < P2_NGP; ++gp)
            for (int m = 0; m < P2_NM; ++m) t[i++] = R.phie[k][gp][m];
    for (int m = 0; m < P2_NM; ++m) t[i++] = R.mass[m];
    for (int q = 0; q < P2_NQ; ++q) {
        t[i++] = -R.lam[q][0] + R.lam[q][1] - R.lam[q][2];
        t[i++] = -R.lam[q][0] - R.lam[q][1] + R.lam[q][2];
    }
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
        snprintf(dgr_cuda_err_buffer(), 256, "pow43: %s", cudaGetErrorString(e));
        return DGR_ERR_CUDA;
    }
    return DGR_OK;
}

static __global__ void k_div_rcp(int n, const double *__restrict__ a, const double *__restrict__ b, double *q,
                                 int *valid)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool ok = rcp_divisor_ok(b[i]);
    q[i] = div_rcp(a[i], b[i], 1.0 / b[i], ok);
    valid[i] = ok ? 1 : 0;
}

extern "C" int dgr_div_rcp_batch(const double *a, const double *b, double *q, int *valid, int n, int device)
{
    if (!a || !b || !q || !valid || n < 0) return DGR_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return DGR_ERR_NO_DEVICE;
    CK(cudaSetDevice(device));
    const size_t m = n ? (size_t)n : 1;
    double *d = nullptr;
    CK(cudaMalloc((void **)&d, 3 * m * sizeof(double) + m * sizeof(int)));
    int *dv = (int *)(d + 3 * m);
    cudaError_t e = cudaMemcpy(d, a, (size_t)n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + m, b, (size_t)n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n) k_div_rcp<<<blocks(n, 256), 256>>>(n, d, d + m, d + 2 * m, dv);
    if (e == cudaSuccess) e = cudaMemcpy(q, d + 2 * m, (size_t)n * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(valid, dv, (size_t)n * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        snprintf(dgr_cuda_err_buffer(), 256, "div_rcp: %s", cudaGetErrorString(e));
        return DGR_ERR_CUDA;
    }
    return DGR_OK;
}

/* --------------------------------------------------------------- gauges ---- */

extern "C" int dgr_set_gauges(dgr_ctx *c, int ngauges, const int *gauge_el, const double *gauge_w, int capacity)
{
    if (!c || ngauges < 0 || (ngauges > 0 && (!gauge_el || !gauge_w || capacity <= 0))) return DGR_ERR_INVALID;
    for (int g = 0; g < ngauges; ++g)
        if (gauge_el[g] < 0 || gauge_el[g] >= c->ne) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    drop_graph(c); /* the step graph gains or loses the recording kernel */
    int *ptrs_i[2] = {c->gauge_el, c->gauge_sid};
    for (int *q : ptrs_i)
        if (q) cudaFree(q);
    if (c->gauge_w) cudaFree(c->gauge_w);
    if (c->gauge_series) cudaFree(c->gauge_series);
    c->gauge_el = c->gauge_sid = nullptr;
    c->gauge_w = c->gauge_series = nullptr;
    c->gauge_n = c->gauge_cap = 0;
    if (ngauges == 0) return DGR_OK;
    std::vector<int> sid(ngauges);
    for (int g = 0; g < ngauges; ++g) {
        int k = 0;
        while (k + 1 < c->nscen && gauge_el[g] >= c->el_off[k + 1]) ++k;
        sid[g] = k;
    }
    int r = 0;
    if ((r = dalloc(&c->gauge_el, ngauges)) || (r = dalloc(&c->gauge_sid, ngauges)) ||
        (r = dalloc(&c->gauge_w, (size_t)ngauges * c->nm)) ||
        (r = dalloc(&c->gauge_series, (size_t)ngauges * capacity)))
        return r;
    CK(cudaMemcpy(c->gauge_el, gauge_el, (size_t)ngauges * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->gauge_sid, sid.data(), (size_t)ngauges * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->gauge_w, gauge_w, (size_t)ngauges * c->nm * 8, cudaMemcpyHostToDevice));
    CK(cudaMemset(c->gauge_series, 0, (size_t)ngauges * capacity * 8));
    c->gauge_n = ngauges;
    c->gauge_cap = capacity;
    return DGR_OK;
}

extern "C" int dgr_get_gauge_series(dgr_ctx *c, double *values)
{
    if (!c || !values || !c->gauge_n) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaMemcpy(values, c->gauge_series, (size_t)c->gauge_n * c->gauge_cap * 8, cudaMemcpyDeviceToHost));
    return DGR_OK;
}
