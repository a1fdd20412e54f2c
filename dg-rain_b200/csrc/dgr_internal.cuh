/*
 * Context of the device step shared by the C-ABI translation units (dgr_capi.cu: forward
 * step, ensemble, schedules; dgr_adjoint.cu: discrete adjoint).  Internal: not part of the
 * public header.
 */
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/dgrain.h"
#include "dgr_kernels.cuh"
#include "dgr_p2.cuh"

namespace dgr {
struct AdjointState; /* dgr_adjoint.cu */
}

/* last CUDA error text, per host thread (dgr_last_cuda_error) */
char *dgr_cuda_err_buffer();

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            snprintf(dgr_cuda_err_buffer(), 256, "%s:%d %s: %s", __FILE__, __LINE__, #call,          \
                     cudaGetErrorString(e_));                                                        \
            return DGR_ERR_CUDA;                                                                     \
        }                                                                                            \
    } while (0)

static inline int pad32(int n) { return (n + 31) & ~31; }

static inline double bits_to_double(unsigned long long b)
{
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
}

static inline unsigned blocks(int n, int t) { return (unsigned)((n + t - 1) / t); }

template <class T>
static inline int dalloc(T **p, size_t n)
{
    *p = nullptr;
    CK(cudaMalloc((void **)p, (n ? n : 1) * sizeof(T)));
    return DGR_OK;
}

struct dgr_ctx {
    dgr_params p;
    int nm;   /* state coefficients per element and variable: 3 (p = 1) or 6 (p = 2) */
    int nfp;  /* flux planes per edge: 6 (p = 1: Fhat.n of both sides) or 9 (p = 2: 3 Gauss points) */
    double *p2g;         /* p = 2 element geometry planes [P2G_N][ldE] */
    dgr::P2Ref p2ref;    /* p = 2 reference-element tables */
    int device;
    int nscen;
    int ne, nn, nf, nbnd;
    int ldE, ldF, ldN;
    std::vector<int> el_off, nd_off, ed_off; /* [nscen + 1] */
    std::vector<int> h_bnd;                  /* prescribed edges (flattened ids) */
    cudaStream_t stream;
    cudaEvent_t ev0, ev1;
    int num_sms;
    /* mesh */
    double *x, *y, *zn, *nfric, *n_el;
    int *el2v_aos, *el2v, *elem_edge, *e_in, *e_ex, *e_info, *n2e_ptr, *n2e, *bnd_edges, *bnd_type, *bnd_sid;
    int *bdry, *el_sid, *ed_sid;
    double *e_geo, *geo;
    /* state and work */
    double *U, *W, *flux, *avg, *bounds, *bzeta, *bqn, *bstage;
    int *wdA, *wdB, *wdC; /* wet/dry flags: stage s reads buffer s, writes buffer (s+1) mod stages */
    int *dec; /* [6][ne]: limit and pdop decisions of stage 0, 1, 2 */
    unsigned *bar;
    int *redo; /* edge queue of k_edge_flux -> k_edge_redo, [2 + nf] */
    unsigned bar_polls;   /* bound of a grid-barrier wait (dgr_set_barrier_wait) */
    unsigned bar_phantom; /* phantom arrivals a barrier waits for (0 except in tests) */
    dgr::DevClock *clk;
    dgr::DevClock *h_clk; /* pinned mirror [nscen] */
    double *h_stage;
    int wd_fresh;    /* WA already holds the status for the next step */
    int wd_stepped;  /* reference-semantic WD lives in the last stage's input buffer (WB for
                        RK2, WC for RK3), not in WA */
    long long launches;
    double last_ms;
    /* schedule of the device loop */
    int bs;     /* block size of element/limiter work: 64, 128 or 256 */
    int fusion; /* 0, 1 or 2 */
    cudaGraph_t graph;
    cudaGraphExec_t graph_exec;
    cudaGraph_t stage_graph;          /* the RK stages of one dgr_step, without the clock */
    cudaGraphExec_t stage_graph_exec;
    int stage_graph_tried;            /* its capture was attempted since the last drop_graph */
    dgr::AdjointState *adj; /* discrete adjoint storage, created on first use */
    /* gauge series recorded by the device loop (dgr_set_gauges) */
    int gauge_n, gauge_cap;
    int *gauge_el, *gauge_sid;
    double *gauge_w, *gauge_series; /* weights [n][nm], series [cap][n] */
    /* channel ends coupled to prescribed boundary edges (dgr_set_channel_ends) */
    int cpl_nends, cpl_nedges;
    int *cpl_ptr, *cpl_out, *cpl_edge, *cpl_slot; /* [nends + 1], [nends], [nedges], [nedges] */
    double *cpl_geo;                              /* [4][nedges]: length, nx, ny, mid-edge depth */
    double *cpl_io, *h_cpl_io;                    /* [4][nends] in/out, and its pinned mirror */
};

/* NVTX range over a host-side phase or launch (a timeline tool shows it by name; with no
 * tool attached the calls return at once).  Kernels replayed from a CUDA graph are
 * covered by the range of the call that replays the graph. */
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

static inline dgr::MeshDev mesh_dev(const dgr_ctx *c)
{
    dgr::MeshDev m;
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
    m.el_sid = c->el_sid;
    m.ed_sid = c->ed_sid;
    m.flux = c->p.flux;
    m.bad_index = reinterpret_cast<unsigned long long *>(c->bar + 4);
    m.redo = c->redo;
    return m;
}

static inline dgr::PhysParams phys(const dgr_ctx *c)
{
    dgr::PhysParams q;
    q.g = c->p.g;
    q.h0 = c->p.H0;
    q.velzero = c->p.VELZERO;
    q.cfl = c->p.cfl;
    q.dt0 = c->p.dt0;
    q.stages = c->p.rk_stages;
    return q;
}

/* Buffers of RK stage `stage`: state in/out, wet/dry flags in/out, element mode.  RK2:
 * U -> W -> U; RK3: U -> W -> W (in place) -> U.  Flags: stage s reads buffer s and writes
 * buffer (s+1) mod stages, so WA holds the next step's status after the last stage. */
struct StageIO {
    const double *S;
    double *OUT;
    const int *wd_in;
    int *wd_out;
    int mode;
};

static inline StageIO stage_io(const dgr_ctx *c, int stage)
{
    const int ns = c->p.rk_stages;
    int *bufs[3] = {c->wdA, c->wdB, c->wdC};
    StageIO io;
    io.S = stage == 0 ? c->U : c->W;
    io.OUT = stage == ns - 1 ? c->U : c->W;
    io.wd_in = c->p.wet_dry ? bufs[stage] : c->wdA;
    io.wd_out = bufs[(stage + 1) % ns];
    io.mode = stage == 0 ? dgr::MODE_STAGE1
                         : (ns == 2 ? dgr::MODE_STAGE2 : (stage == 1 ? dgr::MODE_RK3_2 : dgr::MODE_RK3_3));
    return io;
}

/* flags the reference's WD array holds after a step: the last stage's input */
static inline int *wd_after_step(const dgr_ctx *c) { return c->p.rk_stages == 3 ? c->wdC : c->wdB; }


/* dgr_capi.cu */
void drop_graph(dgr_ctx *c);
int upload_geometry(dgr_ctx *c);                 /* element geometry planes from x, y, zn, n */
int upload_scenarios(dgr_ctx *c, int s0, int s1, const double *zeta, const double *Qx, const double *Qy,
                     const int *WD);             /* state of scenarios [s0, s1), reference layout */
int read_clock(dgr_ctx *c);                      /* device clocks -> h_clk (synchronises) */
int write_clock(dgr_ctx *c);                     /* h_clk -> device clocks (synchronises) */
void launch_stage(dgr_ctx *c, int stage, bool count); /* one RK stage, four kernels */
void launch_edge(dgr_ctx *c, const double *S, const int *wd, int lam_slot, int phase); /* p = 1 edge fluxes */
void launch_p2_edge(dgr_ctx *c, const double *S, int lam_slot, int phase);            /* p = 2 edge fluxes */
void launch_wd_refresh(dgr_ctx *c);              /* status for the next step when stale */
int decode_err(unsigned long long key, int *code, int *index, int *step);
int first_error(const dgr_ctx *c);               /* first scenario failure code in h_clk */

/* dgr_adjoint.cu */
void adjoint_release(dgr_ctx *c);
void coupling_release(dgr_ctx *c);
