/*
 * Discrete adjoint and tangent-linear model of the device time loop: one mesh or a batched
 * ensemble (every scenario runs the same number of steps, each with its own CFL dt), p = 1
 * or p = 2.
 *
 * Objective: J = sum over steps n and gauges g of (zeta_g(u^{n+1}) - target[n][g])^2, with
 * zeta_g a fixed linear functional of one element's elevation coefficients (the
 * Crouzeix-Raviart interpolation of the three midpoint values at p = 1, the six modes
 * evaluated at the gauge point at p = 2); gauges of an ensemble name flattened elements and
 * J sums over all scenarios.  Parameters: per-element Manning n, node depth z, and the
 * initial state.
 *
 * Forward (dgr_adjoint_forward): the plain step (same kernels, same bits as dgr_run), the
 * per-step CFL dt and boundary time recorded, gauge residuals stored, and a checkpoint
 * (state, wet/dry status, clock) every K steps.
 *
 * Backward (dgr_adjoint_backward), per segment of K steps from the last:
 *   1. recompute the segment from its checkpoint with the recorded dt, keeping per step and
 *      stage the stage inputs and, at p = 1, the pre-limiter outputs, element means, node
 *      bounds and the wet/dry flags (the decisions are recomputed bit for bit, i.e. frozen);
 *   2. reverse each step: misfit, then per stage from the last: at p = 1 limiter+PDop,
 *      node bounds, element and edge reverse kernels (dgr_tlm.cuh); at p = 2 element, edge
 *      and trace-gather reverse kernels (dgr_p2_adjoint.cuh).
 * Memory: checkpoints 24 nm B per element per K steps (nm = 3 or 6 coefficients); segment
 * store per element and step about 390 B (p = 1, RK2) or 144 B per stage (p = 2), times K.
 *
 * TLM (dgr_tlm): the same steps in dual numbers with the recorded dt (frozen), giving J and
 * its directional derivative; its primal part is the forward bit for bit.
 */
#include <algorithm>
#include <type_traits>

#include "dgr_internal.cuh"
#include "dgr_p2_adjoint.cuh"
#include "dgr_tlm.cuh"

using namespace dgr;

namespace dgr {

struct AdjointState {
    int nsteps = 0, K = 0, nseg = 0, ng = 0, nu = 0;
    int ns = 2;  /* RK stages the storage was laid out for */
    int nsc = 1; /* scenarios: histories are [step][nsc], checkpoint clocks [segment][nsc] */
    int nw = 3;  /* gauge weights per gauge: the element's elevation coefficients */
    int have_forward = 0;
    int *g_el = nullptr, *u_el = nullptr, *u_ptr = nullptr, *u_g = nullptr; /* gauges; per gauge element */
    double *g_w = nullptr, *target = nullptr, *resid = nullptr, *sums = nullptr;
    double *dt_hist = nullptr, *time_hist = nullptr; /* [nsteps][nsc] */
    double *ckU = nullptr;
    int *ckWd = nullptr;
    DevClock *ckClk = nullptr;
    /* segment store */
    double *segU = nullptr, *segW = nullptr, *segR = nullptr, *segAvg = nullptr, *segB = nullptr;
    int *segWd = nullptr;
    /* adjoint work */
    double *lamU = nullptr, *lamW = nullptr, *Rbar = nullptr, *bbar = nullptr, *bnode = nullptr, *fbar = nullptr;
    double *zvb = nullptr, *zeb = nullptr, *nbar = nullptr, *zbar = nullptr;
    int *barg = nullptr;
    /* tangent work */
    double *Ud = nullptr, *Wd = nullptr, *flux_d = nullptr, *avg_d = nullptr, *bounds_d = nullptr;
    double *zd = nullptr, *neld = nullptr, *rd = nullptr, *rt = nullptr;
    double fwd_ms = 0, bwd_ms = 0, tlm_ms = 0;
};

}  // namespace dgr

void adjoint_release(dgr_ctx *c)
{
    AdjointState *a = c->adj;
    if (!a) return;
    void *ptrs[] = {a->g_el, a->u_el, a->u_ptr, a->u_g, a->g_w, a->target, a->resid, a->sums, a->dt_hist, a->time_hist, a->ckU, a->ckWd,
                    a->ckClk, a->segU, a->segW, a->segR, a->segAvg, a->segB, a->segWd, a->lamU, a->lamW,
                    a->Rbar, a->bbar, a->bnode, a->fbar, a->zvb, a->zeb, a->nbar, a->zbar, a->barg, a->Ud,
                    a->Wd, a->flux_d, a->avg_d, a->bounds_d, a->zd, a->neld, a->rd, a->rt};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    delete a;
    c->adj = nullptr;
}

/* ------------------------------------------------------------- storage layout ---- */

/* state planes of one copy of the state: 3 variables x nm coefficients */
static size_t planes(const dgr_ctx *c) { return (size_t)3 * c->nm * c->ldE; }
/* segment store, per step slot j: the step input u^n (seg_U), the inputs of stages 1..ns-1
 * (seg_W(j, s-1)), and at p = 1 per stage s the pre-limiter output, element means, node
 * bounds and input wet/dry flags */
static double *seg_U(const dgr_ctx *c, int j) { return c->adj->segU + (size_t)j * planes(c); }
static double *seg_W(const dgr_ctx *c, int j, int s)
{
    return c->adj->segW + ((size_t)j * (c->adj->ns - 1) + s) * planes(c);
}
static size_t seg_slot(const dgr_ctx *c, int j, int s) { return (size_t)j * c->adj->ns + s; }
static double *seg_R(const dgr_ctx *c, int j, int s) { return c->adj->segR + seg_slot(c, j, s) * planes(c); }
static double *seg_avg(const dgr_ctx *c, int j, int s) { return c->adj->segAvg + seg_slot(c, j, s) * 3 * c->ldE; }
static double *seg_B(const dgr_ctx *c, int j, int s) { return c->adj->segB + seg_slot(c, j, s) * 6 * c->ldN; }
static int *seg_wd(const dgr_ctx *c, int j, int s) { return c->adj->segWd + seg_slot(c, j, s) * c->ne; }
/* adjoint of the input of stage s >= 1 */
static double *lam_stage(const dgr_ctx *c, int s) { return c->adj->lamW + (size_t)(s - 1) * planes(c); }
/* recorded dt of step n, per scenario */
static const double *dt_row(const dgr_ctx *c, int n) { return c->adj->dt_hist + (size_t)n * c->adj->nsc; }

extern "C" int dgr_adjoint_setup(dgr_ctx *c, int nsteps, int ckpt_every, int ngauges, const int *gauge_el,
                                 const double *gauge_w, const double *target)
{
    if (!c || nsteps <= 0 || ckpt_every <= 0 || ngauges <= 0 || !gauge_el || !gauge_w) return DGR_ERR_INVALID;
    for (int g = 0; g < ngauges; ++g)
        if (gauge_el[g] < 0 || gauge_el[g] >= c->ne) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    adjoint_release(c);
    AdjointState *a = new AdjointState();
    c->adj = a;
    a->nsteps = nsteps;
    a->K = std::min(ckpt_every, nsteps);
    a->nseg = (nsteps + a->K - 1) / a->K;
    a->ng = ngauges;
    a->nsc = c->nscen;
    a->nw = c->nm;
    const bool p1 = c->nm == 3;
    const size_t E = c->ldE, F = c->ldF, N = c->ldN, K = a->K, P = planes(c), nsc = a->nsc;
    const size_t ns = nsteps, ng = ngauges, nw = a->nw;
    int r = 0;
#define AL(p, n)                       \
    do {                               \
        r = dalloc(&(p), (n));         \
        if (r) {                       \
            adjoint_release(c);        \
            return r;                  \
        }                              \
    } while (0)
    /* gauges grouped by element, in gauge order within an element */
    std::vector<int> order(ngauges);
    for (int g = 0; g < ngauges; ++g) order[g] = g;
    std::stable_sort(order.begin(), order.end(), [&](int p, int q) { return gauge_el[p] < gauge_el[q]; });
    std::vector<int> uel, uptr;
    for (int j = 0; j < ngauges; ++j) {
        if (j == 0 || gauge_el[order[j]] != gauge_el[order[j - 1]]) {
            uel.push_back(gauge_el[order[j]]);
            uptr.push_back(j);
        }
    }
    uptr.push_back(ngauges);
    a->nu = (int)uel.size();
    AL(a->g_el, ng);
    AL(a->u_el, uel.size());
    AL(a->u_ptr, uptr.size());
    AL(a->u_g, ng);
    AL(a->g_w, nw * ng);
    AL(a->target, ns * ng);
    AL(a->resid, ns * ng);
    AL(a->rd, ns * ng);
    AL(a->rt, ns * ng);
    AL(a->sums, 2);
    AL(a->dt_hist, ns * nsc);
    AL(a->time_hist, ns * nsc);
    AL(a->ckU, (size_t)a->nseg * P);
    AL(a->ckWd, (size_t)a->nseg * c->ne);
    AL(a->ckClk, (size_t)a->nseg * nsc);
    const size_t S = a->ns = c->p.rk_stages;
    AL(a->segU, K * P);
    AL(a->segW, K * (S - 1) * P);
    if (p1) {
        AL(a->segR, K * S * P);
        AL(a->segAvg, K * S * 3 * E);
        AL(a->segB, K * S * 6 * N);
        AL(a->segWd, K * S * c->ne);
        AL(a->Rbar, P);
        AL(a->bbar, 18 * E);
        AL(a->bnode, 6 * N);
        AL(a->barg, 6 * N);
    }
    AL(a->lamU, P);
    AL(a->lamW, (S - 1) * P);
    AL(a->fbar, (p1 ? 6 : 18) * F);
    AL(a->zvb, 3 * E);
    AL(a->zeb, (p1 ? 1 : 2) * F);
    AL(a->nbar, E);
    AL(a->zbar, (size_t)c->nn);
#undef AL
    cudaStream_t s = c->stream;
    CK(cudaMemcpyAsync(a->g_el, gauge_el, ng * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(a->u_el, uel.data(), uel.size() * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(a->u_ptr, uptr.data(), uptr.size() * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(a->u_g, order.data(), ng * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(a->g_w, gauge_w, nw * ng * 8, cudaMemcpyHostToDevice, s));
    if (target)
        CK(cudaMemcpyAsync(a->target, target, ns * ng * 8, cudaMemcpyHostToDevice, s));
    else
        CK(cudaMemsetAsync(a->target, 0, ns * ng * 8, s));
    CK(cudaMemsetAsync(a->fbar, 0, (p1 ? 6 : 18) * F * 8, s));
    CK(cudaStreamSynchronize(s));
    return DGR_OK;
}

extern "C" int dgr_adjoint_set_target(dgr_ctx *c, const double *target)
{
    if (!c || !c->adj || !target) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->adj->nsteps * c->adj->ng;
    CK(cudaMemcpyAsync(c->adj->target, target, n * 8, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DGR_OK;
}

extern "C" int dgr_set_bathymetry(dgr_ctx *c, const double *z)
{
    if (!c || !z || c->nscen != 1) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    CK(cudaMemcpyAsync(c->zn, z, (size_t)c->nn * 8, cudaMemcpyHostToDevice, c->stream));
    k_edge_zsetup<<<blocks(c->nf, 256), 256, 0, c->stream>>>(mesh_dev(c), c->e_geo);
    c->launches++;
    int r = upload_geometry(c);
    if (r) return r;
    c->wd_fresh = 0; /* the status depends on the depths */
    CK(cudaStreamSynchronize(c->stream));
    return DGR_OK;
}

/* ------------------------------------------------------------------ forward ---- */

static void clock_begin_step(dgr_ctx *c, int n, int replay)
{
    AdjointState *a = c->adj;
    k_adj_clock_begin<<<1, 256, 0, c->stream>>>(c->clk, c->nscen, phys(c), c->bnd_edges, c->bnd_type,
                                                  c->nscen > 1 ? c->bnd_sid : nullptr, c->nbnd, c->bzeta, c->bqn,
                                                  a->dt_hist, a->time_hist, n, replay);
}

/* boundary values of step n at the recorded times */
static void replay_forcing(dgr_ctx *c, int n)
{
    if (!c->nbnd) return;
    k_adj_forcing<<<blocks(c->nbnd, 256), 256, 0, c->stream>>>(c->clk, c->adj->time_hist, n, c->nscen, c->bnd_edges,
                                                               c->bnd_type, c->nscen > 1 ? c->bnd_sid : nullptr,
                                                               c->nbnd, c->bzeta, c->bqn);
    c->launches++;
}

/* every scenario's clock starts at (time, dt) (time < 0: t = 0 with the first-step dt) */
static int start_clock(dgr_ctx *c, double time, double dt)
{
    int r = read_clock(c);
    if (r) return r;
    if (time < 0) {
        time = 0.0;
        dt = c->p.dt0;
    }
    for (int k = 0; k < c->nscen; ++k) {
        DevClock &h = c->h_clk[k];
        h.time = time;
        h.dt = dt;
        h.final_time = 1e300;
        h.step = 0;
        h.nsteps = c->adj->nsteps;
        h.done = 0;
        h.dt_pending = 0;
        h.err = ~0ull;
    }
    return write_clock(c);
}

extern "C" int dgr_adjoint_forward(dgr_ctx *c, const double *zeta, const double *Qx, const double *Qy, const int *WD,
                                   double time, double dt, int replay_dt, double *J, double *gauge_values)
{
    NvtxRange nv("dgr_adjoint_forward");
    if (!c || !c->adj || !zeta || !Qx || !Qy || !WD) return DGR_ERR_INVALID;
    AdjointState *a = c->adj;
    if (replay_dt && !a->have_forward) return DGR_ERR_INVALID;
    if (c->p.rk_stages != a->ns) return DGR_ERR_INVALID; /* storage laid out for another scheme */
    CK(cudaSetDevice(c->device));
    int r = upload_scenarios(c, 0, c->nscen, zeta, Qx, Qy, WD);
    if (r) return r;
    r = start_clock(c, time, dt);
    if (r) return r;
    cudaStream_t s = c->stream;
    const size_t E9 = planes(c);
    const int nsc = a->nsc;
    CK(cudaEventRecord(c->ev0, s));
    launch_wd_refresh(c);
    for (int n = 0; n < a->nsteps; ++n) {
        if (n % a->K == 0) {
            const int sg = n / a->K;
            CK(cudaMemcpyAsync(a->ckU + sg * E9, c->U, E9 * 8, cudaMemcpyDeviceToDevice, s));
            CK(cudaMemcpyAsync(a->ckWd + (size_t)sg * c->ne, c->wdA, (size_t)c->ne * 4, cudaMemcpyDeviceToDevice,
                               s));
            CK(cudaMemcpyAsync(a->ckClk + (size_t)sg * nsc, c->clk, nsc * sizeof(DevClock), cudaMemcpyDeviceToDevice,
                               s));
        }
        clock_begin_step(c, n, replay_dt);
        for (int st = 0; st < c->p.rk_stages; ++st) launch_stage(c, st, true);
        k_clock_end<<<blocks(nsc, 128), 128, 0, s>>>(c->clk, nsc);
        k_misfit<<<blocks(a->ng, 128), 128, 0, s>>>(c->U, c->ldE, a->nw, a->ng, a->g_el, a->g_w, a->target + (size_t)n * a->ng,
                                  a->resid + (size_t)n * a->ng);
        c->launches += 3;
    }
    k_misfit_sum<<<1, 32, 0, s>>>(a->resid, nullptr, (long long)a->nsteps * a->ng, 0, a->sums);
    k_clock_finish<<<blocks(nsc, 128), 128, 0, s>>>(c->clk, nsc, phys(c));
    c->launches += 2;
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, s));
    r = read_clock(c);
    if (r) return r;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    a->fwd_ms = ms;
    if (c->p.wet_dry) {
        c->wd_fresh = 1;
        c->wd_stepped = 1;
    }
    r = first_error(c);
    if (r) return r;
    for (int k = 0; k < nsc; ++k)
        if (c->h_clk[k].step != a->nsteps) return DGR_ERR_INVALID;
    double sums[2];
    CK(cudaMemcpy(sums, a->sums, 16, cudaMemcpyDeviceToHost));
    if (J) *J = sums[0];
    if (gauge_values) {
        const size_t cnt = (size_t)a->nsteps * a->ng;
        std::vector<double> rr(cnt), tt(cnt);
        CK(cudaMemcpy(rr.data(), a->resid, cnt * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(tt.data(), a->target, cnt * 8, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < cnt; ++i) gauge_values[i] = rr[i] + tt[i];
    }
    a->have_forward = 1;
    return DGR_OK;
}

extern "C" int dgr_adjoint_dt(dgr_ctx *c, double *dt_out, double *time_out)
{
    if (!c || !c->adj || !c->adj->have_forward) return DGR_ERR_INVALID;
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->adj->nsteps * c->adj->nsc;
    if (dt_out) CK(cudaMemcpy(dt_out, c->adj->dt_hist, n * 8, cudaMemcpyDeviceToHost));
    if (time_out) CK(cudaMemcpy(time_out, c->adj->time_hist, n * 8, cudaMemcpyDeviceToHost));
    return DGR_OK;
}

/* ----------------------------------------------------------------- backward ---- */

/* one recorded stage of step slot j: the stage kernels with (p = 1) the pre-limiter
 * output, means and bounds kept in the segment store; S -> OUT (OUT may be the next step's
 * input slot) */
static void recorded_stage(dgr_ctx *c, int j, int stage, const double *S, double *OUT, const int *wd_in,
                           int *wd_out)
{
    const MeshDev m = mesh_dev(c);
    cudaStream_t s = c->stream;
    const int mode = stage_io(c, stage).mode;
    const double *U = seg_U(c, j);
    const unsigned nb = blocks(c->ne, 128);
    if (c->p.order == 2) {
        launch_p2_edge(c, S, stage, 2 * stage);
#define P2_EL(MD) \
    k_p2_element<MD, 128><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, S, U, c->flux, OUT, c->clk, c->p.g)
        if (mode == MODE_STAGE1)
            P2_EL(MODE_STAGE1);
        else if (mode == MODE_STAGE2)
            P2_EL(MODE_STAGE2);
        else if (mode == MODE_RK3_2)
            P2_EL(MODE_RK3_2);
        else
            P2_EL(MODE_RK3_3);
#undef P2_EL
        c->launches += 2;
        return;
    }
    const bool wd = c->p.wet_dry != 0;
    double *R = seg_R(c, j, stage), *avg = seg_avg(c, j, stage), *bnd = seg_B(c, j, stage);
    launch_edge(c, S, wd_in, stage, 2 * stage);
    const unsigned ne64 = blocks(c->ne, 64); /* the element kernel in blocks of 64, as the plain step's default */
    if (mode == MODE_STAGE1)
        k_element<MODE_STAGE1, 64><<<ne64, 64, 0, s>>>(m, S, U, wd_in, c->flux, R, avg, c->clk, c->p.g);
    else if (mode == MODE_STAGE2)
        k_element<MODE_STAGE2, 64><<<ne64, 64, 0, s>>>(m, S, U, wd_in, c->flux, R, avg, c->clk, c->p.g);
    else if (mode == MODE_RK3_2)
        k_element<MODE_RK3_2, 64><<<ne64, 64, 0, s>>>(m, S, U, wd_in, c->flux, R, avg, c->clk, c->p.g);
    else
        k_element<MODE_RK3_3, 64><<<ne64, 64, 0, s>>>(m, S, U, wd_in, c->flux, R, avg, c->clk, c->p.g);
    k_node_bounds<<<blocks(c->nn, DGR_NODE_BS), DGR_NODE_BS, 0, s>>>(m, avg, bnd);
    if (wd)
        k_limit_to<true><<<nb, 128, 0, s>>>(m, R, OUT, bnd, wd_in, wd_out, c->clk, c->p.H0, c->p.VELZERO,
                                            2 * stage + 1);
    else
        k_limit_to<false><<<nb, 128, 0, s>>>(m, R, OUT, bnd, wd_in, wd_out, c->clk, c->p.H0, c->p.VELZERO,
                                             2 * stage + 1);
    c->launches += 4;
}

/* reverse of one p = 2 stage: element, edge, trace gather */
static void reverse_stage_p2(dgr_ctx *c, int j, int n, int stage)
{
    AdjointState *a = c->adj;
    const MeshDev m = mesh_dev(c);
    cudaStream_t s = c->stream;
    const int ns = a->ns;
    const int mode = stage_io(c, stage).mode;
    const double *S = stage == 0 ? seg_U(c, j) : seg_W(c, j, stage - 1);
    double *lamO = stage == ns - 1 ? a->lamU : lam_stage(c, stage + 1);
    double *lamS = stage == 0 ? a->lamU : lam_stage(c, stage);
    const int u_acc = stage < ns - 1 ? 1 : 0;
    const double g = c->p.g;
    const unsigned nb = blocks(c->ne, 128);
#define P2_ADJ_EL(MD)                                                                                                  \
    k_p2_adj_element<MD><<<nb, 128, 0, s>>>(c->p2ref, m, c->p2g, S, lamO, lamS, a->lamU, u_acc, a->fbar, a->zvb,    \
                                            a->nbar, c->n_el, g, dt_row(c, n))
    if (mode == MODE_STAGE1)
        P2_ADJ_EL(MODE_STAGE1);
    else if (mode == MODE_STAGE2)
        P2_ADJ_EL(MODE_STAGE2);
    else if (mode == MODE_RK3_2)
        P2_ADJ_EL(MODE_RK3_2);
    else
        P2_ADJ_EL(MODE_RK3_3);
#undef P2_ADJ_EL
    if (c->p.flux == 0)
        k_p2_adj_edge<0><<<blocks(c->nf, 128), 128, 0, s>>>(c->p2ref, m, c->p2g, S, c->bzeta, c->bqn, a->fbar, a->zeb,
                                                            g);
    else
        k_p2_adj_edge<-1><<<blocks(c->nf, 128), 128, 0, s>>>(c->p2ref, m, c->p2g, S, c->bzeta, c->bqn, a->fbar,
                                                             a->zeb, g);
    k_p2_adj_trace<<<nb, 128, 0, s>>>(c->p2ref, m, a->fbar, lamS);
    c->launches += 3;
}

/* reverse of one stage of step n (slot j).  The adjoint of the stage output is lamU for the
 * last stage, else the adjoint of the next stage's input; the stage input's adjoint goes to
 * lamU (stage 0) or lam_stage(stage). */
static void reverse_stage(dgr_ctx *c, int j, int n, int stage)
{
    if (c->p.order == 2) {
        reverse_stage_p2(c, j, n, stage);
        return;
    }
    AdjointState *a = c->adj;
    const MeshDev m = mesh_dev(c);
    cudaStream_t s = c->stream;
    const bool wd = c->p.wet_dry != 0;
    const int ns = a->ns;
    const int mode = stage_io(c, stage).mode;
    const double *S = stage == 0 ? seg_U(c, j) : seg_W(c, j, stage - 1);
    const int *wd_in = seg_wd(c, j, stage);
    double *lamO = stage == ns - 1 ? a->lamU : lam_stage(c, stage + 1);
    double *lamS = stage == 0 ? a->lamU : lam_stage(c, stage);
    const int u_acc = stage < ns - 1 ? 1 : 0;
    const double h0 = c->p.H0, vz = c->p.VELZERO, g = c->p.g;
    const unsigned nb = blocks(c->ne, 128);
    if (wd)
        k_adj_limit<true><<<nb, 128, 0, s>>>(m, seg_R(c, j, stage), seg_B(c, j, stage), lamO, a->Rbar, a->bbar, a->zvb,
                                             h0, vz);
    else
        k_adj_limit<false><<<nb, 128, 0, s>>>(m, seg_R(c, j, stage), seg_B(c, j, stage), lamO, a->Rbar, a->bbar,
                                              a->zvb, h0, vz);
    k_adj_node<<<blocks(c->nn, 256), 256, 0, s>>>(m, seg_avg(c, j, stage), a->bbar, a->bnode, a->barg);
#define ADJ_EL(MD)                                                                                                 \
    k_adj_element<MD><<<nb, 128, 0, s>>>(m, S, wd_in, a->Rbar, a->bnode, a->barg, lamS, a->lamU, u_acc, a->fbar,   \
                                         a->zvb, a->nbar, c->n_el, g, dt_row(c, n))
    if (mode == MODE_STAGE1)
        ADJ_EL(MODE_STAGE1);
    else if (mode == MODE_STAGE2)
        ADJ_EL(MODE_STAGE2);
    else if (mode == MODE_RK3_2)
        ADJ_EL(MODE_RK3_2);
    else
        ADJ_EL(MODE_RK3_3);
#undef ADJ_EL
#define ADJ_EDGE(W, F) \
    k_adj_edge<W, F><<<blocks(c->nf, DGR_ADJ_EDGE_BS), DGR_ADJ_EDGE_BS, 0, s>>>(m, S, wd_in, c->bzeta, c->bqn,   \
                                                                          a->fbar, lamS, a->zeb, g)
    if (c->p.flux == 0) { /* the reference's Roe flux, compiled alone */
        if (wd)
            ADJ_EDGE(true, 0);
        else
            ADJ_EDGE(false, 0);
    } else {
        if (wd)
            ADJ_EDGE(true, -1);
        else
            ADJ_EDGE(false, -1);
    }
#undef ADJ_EDGE
    c->launches += 4;
}

/* planar [3 nm][ldE] -> the reference layout zeta/Qx/Qy[nm*el+k] on the host */
static int to_reference_layout(dgr_ctx *c, const double *planar, double *zeta, double *Qx, double *Qy)
{
    if (!zeta && !Qx && !Qy) return DGR_OK;
    const size_t n3 = (size_t)c->nm * c->ne;
    double *tmp = nullptr;
    int r = dalloc(&tmp, 3 * n3);
    if (r) return r;
    k_planar_to_aos_nm<<<blocks(c->ne, 256), 256, 0, c->stream>>>(c->ne, c->ldE, c->nm, planar, tmp, tmp + n3,
                                                                   tmp + 2 * n3);
    c->launches++;
    std::vector<double> h(3 * n3);
    cudaError_t e = cudaMemcpyAsync(h.data(), tmp, 3 * n3 * 8, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    CK(e);
    if (zeta) memcpy(zeta, h.data(), n3 * 8);
    if (Qx) memcpy(Qx, h.data() + n3, n3 * 8);
    if (Qy) memcpy(Qy, h.data() + 2 * n3, n3 * 8);
    return DGR_OK;
}

extern "C" int dgr_adjoint_backward(dgr_ctx *c, double *grad_n_el, double *grad_z, double *grad_zeta0,
                                    double *grad_Qx0, double *grad_Qy0)
{
    NvtxRange nv("dgr_adjoint_backward");
    if (!c || !c->adj || !c->adj->have_forward) return DGR_ERR_INVALID;
    AdjointState *a = c->adj;
    CK(cudaSetDevice(c->device));
    cudaStream_t s = c->stream;
    const MeshDev m = mesh_dev(c);
    const size_t E9 = planes(c);
    const bool p1 = c->nm == 3;
    const int nsc = a->nsc;
    CK(cudaEventRecord(c->ev0, s));
    CK(cudaMemsetAsync(a->lamU, 0, E9 * 8, s));
    CK(cudaMemsetAsync(a->zvb, 0, (size_t)3 * c->ldE * 8, s));
    CK(cudaMemsetAsync(a->zeb, 0, (size_t)(p1 ? 1 : 2) * c->ldF * 8, s));
    CK(cudaMemsetAsync(a->nbar, 0, (size_t)c->ldE * 8, s));
    for (int sg = a->nseg - 1; sg >= 0; --sg) {
        const int n0 = sg * a->K, len = std::min(a->K, a->nsteps - n0);
        /* 1. recompute the segment, recording */
        CK(cudaMemcpyAsync(seg_U(c, 0), a->ckU + sg * E9, E9 * 8, cudaMemcpyDeviceToDevice, s));
        if (p1)
            CK(cudaMemcpyAsync(seg_wd(c, 0, 0), a->ckWd + (size_t)sg * c->ne, (size_t)c->ne * 4,
                               cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(c->clk, a->ckClk + (size_t)sg * nsc, nsc * sizeof(DevClock), cudaMemcpyDeviceToDevice, s));
        const int ns = a->ns;
        for (int j = 0; j < len; ++j) {
            clock_begin_step(c, n0 + j, 1);
            const bool last = j + 1 == len;
            for (int st = 0; st < ns; ++st) {
                const double *S = st == 0 ? seg_U(c, j) : seg_W(c, j, st - 1);
                double *OUT = st < ns - 1 ? seg_W(c, j, st) : (last ? c->U : seg_U(c, j + 1));
                if (p1) {
                    int *wd_out = st < ns - 1 ? seg_wd(c, j, st + 1) : (last ? c->wdA : seg_wd(c, j + 1, 0));
                    recorded_stage(c, j, st, S, OUT, seg_wd(c, j, st), wd_out);
                } else {
                    recorded_stage(c, j, st, S, OUT, nullptr, nullptr);
                }
            }
            k_clock_end<<<blocks(nsc, 128), 128, 0, s>>>(c->clk, nsc);
            c->launches += 2;
        }
        /* 2. reverse the segment */
        for (int j = len - 1; j >= 0; --j) {
            const int n = n0 + j;
            replay_forcing(c, n);
            k_misfit_rev<<<blocks(a->nu, 128), 128, 0, s>>>(a->lamU, c->ldE, a->nw, a->nu, a->u_el, a->u_ptr, a->u_g,
                                                            a->g_w, a->resid + (size_t)n * a->ng);
            c->launches++;
            for (int st = ns - 1; st >= 0; --st) reverse_stage(c, j, n, st);
        }
    }
    if (p1)
        k_adj_zfold<<<blocks(c->ne, 256), 256, 0, s>>>(m, a->zeb, a->zvb);
    else
        k_p2_adj_zfold<<<blocks(c->ne, 256), 256, 0, s>>>(m, a->zeb, a->zvb);
    k_adj_znode<<<blocks(c->nn, 256), 256, 0, s>>>(m, a->zvb, a->zbar);
    c->launches += 2;
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, s));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    a->bwd_ms = ms;
    int r = read_clock(c);
    if (r) return r;
    r = first_error(c);
    if (r) return r;
    if (grad_n_el) CK(cudaMemcpy(grad_n_el, a->nbar, (size_t)c->ne * 8, cudaMemcpyDeviceToHost));
    if (grad_z) CK(cudaMemcpy(grad_z, a->zbar, (size_t)c->nn * 8, cudaMemcpyDeviceToHost));
    r = to_reference_layout(c, a->lamU, grad_zeta0, grad_Qx0, grad_Qy0);
    if (r) return r;
    c->wd_fresh = 0; /* the context state is the last recomputed one */
    return DGR_OK;
}

/* ---------------------------------------------------------------------- TLM ---- */

static int ensure_tlm(dgr_ctx *c)
{
    AdjointState *a = c->adj;
    if (a->Ud) return DGR_OK;
    const size_t F = c->ldF, N = c->ldN, P = planes(c);
    int r = 0;
    if ((r = dalloc(&a->Ud, P)) || (r = dalloc(&a->Wd, P)) || (r = dalloc(&a->flux_d, (size_t)c->nfp * F)) ||
        (r = dalloc(&a->avg_d, (size_t)3 * c->ldE)) || (r = dalloc(&a->bounds_d, 6 * N)) ||
        (r = dalloc(&a->zd, (size_t)c->nn)) || (r = dalloc(&a->neld, (size_t)c->ne)))
        return r;
    return DGR_OK;
}

/* reference layout [nm*el+k] x 3 (host) -> planar [3 nm][ldE] (device) */
static int upload_planar(dgr_ctx *c, const double *z, const double *x, const double *y, double *dst)
{
    const size_t n3 = (size_t)c->nm * c->ne;
    std::vector<double> h(3 * n3, 0.0);
    if (z) memcpy(h.data(), z, n3 * 8);
    if (x) memcpy(h.data() + n3, x, n3 * 8);
    if (y) memcpy(h.data() + 2 * n3, y, n3 * 8);
    double *tmp = nullptr;
    int r = dalloc(&tmp, 3 * n3);
    if (r) return r;
    cudaError_t e = cudaMemcpyAsync(tmp, h.data(), 3 * n3 * 8, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        k_aos_to_planar_nm<<<blocks(c->ne, 256), 256, 0, c->stream>>>(c->ne, c->ldE, c->nm, tmp, tmp + n3,
                                                                       tmp + 2 * n3, dst);
        c->launches++;
        e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(tmp);
    CK(e);
    return DGR_OK;
}

/* one p = 1 stage in two-lane arithmetic */
template <class T>
static void lanes_stage_p1(dgr_ctx *c, int n, int stage)
{
    AdjointState *a = c->adj;
    cudaStream_t s = c->stream;
    const MeshDev m = mesh_dev(c);
    const bool wd = c->p.wet_dry != 0;
    const double g = c->p.g, h0 = c->p.H0, vz = c->p.VELZERO;
    const StageIO io = stage_io(c, stage);
    const double *S = io.S;
    double *OUT = io.OUT;
    const double *Sx = stage == 0 ? a->Ud : a->Wd;
    double *OUTx = stage == a->ns - 1 ? a->Ud : a->Wd;
    const int *wd_in = io.wd_in;
    int *wd_out = io.wd_out;
    if (wd)
        k_tlm_edge<true, T><<<blocks(c->nf, 256), 256, 0, s>>>(m, S, Sx, wd_in, c->bzeta, c->bqn, a->zd, c->flux,
                                                               a->flux_d, g);
    else
        k_tlm_edge<false, T><<<blocks(c->nf, 256), 256, 0, s>>>(m, S, Sx, wd_in, c->bzeta, c->bqn, a->zd, c->flux,
                                                                a->flux_d, g);
#define TLM_EL(MD)                                                                                                 \
    k_tlm_element<MD, T><<<blocks(c->ne, 128), 128, 0, s>>>(m, S, Sx, c->U, a->Ud, wd_in, c->flux, a->flux_d, a->zd,  \
                                                            c->n_el, a->neld, OUT, OUTx, c->avg, a->avg_d, c->clk, g, \
                                                            dt_row(c, n))
    if (io.mode == MODE_STAGE1)
        TLM_EL(MODE_STAGE1);
    else if (io.mode == MODE_STAGE2)
        TLM_EL(MODE_STAGE2);
    else if (io.mode == MODE_RK3_2)
        TLM_EL(MODE_RK3_2);
    else
        TLM_EL(MODE_RK3_3);
#undef TLM_EL
    k_tlm_node<<<blocks(c->nn, 256), 256, 0, s>>>(m, c->avg, a->avg_d, c->bounds, a->bounds_d);
    if (wd)
        k_tlm_limit<true, T><<<blocks(c->ne, 128), 128, 0, s>>>(m, OUT, OUTx, c->bounds, a->bounds_d, a->zd, wd_in,
                                                                wd_out, h0, vz);
    else
        k_tlm_limit<false, T><<<blocks(c->ne, 128), 128, 0, s>>>(m, OUT, OUTx, c->bounds, a->bounds_d, a->zd, wd_in,
                                                                 wd_out, h0, vz);
    c->launches += 4;
}

/* one p = 2 stage in two-lane arithmetic */
template <class T>
static void lanes_stage_p2(dgr_ctx *c, int n, int stage)
{
    AdjointState *a = c->adj;
    cudaStream_t s = c->stream;
    const MeshDev m = mesh_dev(c);
    const double g = c->p.g;
    const StageIO io = stage_io(c, stage);
    const double *Sx = stage == 0 ? a->Ud : a->Wd;
    double *OUTx = stage == a->ns - 1 ? a->Ud : a->Wd;
    k_p2_tlm_edge<T><<<blocks(c->nf, 128), 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, Sx, c->bzeta, c->bqn, a->zd,
                                                        c->flux, a->flux_d, g);
#define P2_TLM_EL(MD)                                                                                              \
    k_p2_tlm_element<MD, T><<<blocks(c->ne, 128), 128, 0, s>>>(c->p2ref, m, c->p2g, io.S, Sx, c->U, a->Ud, c->flux, \
                                                               a->flux_d, a->zd, c->n_el, a->neld, io.OUT, OUTx,    \
                                                               c->clk, g, dt_row(c, n))
    if (io.mode == MODE_STAGE1)
        P2_TLM_EL(MODE_STAGE1);
    else if (io.mode == MODE_STAGE2)
        P2_TLM_EL(MODE_STAGE2);
    else if (io.mode == MODE_RK3_2)
        P2_TLM_EL(MODE_RK3_2);
    else
        P2_TLM_EL(MODE_RK3_3);
#undef P2_TLM_EL
    c->launches += 2;
}

/*
 * The recorded run's steps in two-lane arithmetic over the recorded dt sequence: T = Dual
 * gives the tangent-linear model (second lanes = tangents), T = Pert the scheme at a
 * perturbed point with the base run's decisions frozen (second lanes = perturbed values).
 * The second lanes of the state, depths and element n are in a->Ud, a->zd, a->neld on
 * entry.  Returns J of the base lane and, in out2, dJ (Dual) or J of the perturbed lane.
 */
template <class T>
static int run_lanes(dgr_ctx *c, double *J, double *out2)
{
    AdjointState *a = c->adj;
    cudaStream_t s = c->stream;
    const bool pert = std::is_same<T, ad::Pert>::value;
    CK(cudaMemsetAsync(a->flux_d, 0, (size_t)c->nfp * c->ldF * 8, s));
    CK(cudaEventRecord(c->ev0, s));
    launch_wd_refresh(c);
    for (int n = 0; n < a->nsteps; ++n) {
        replay_forcing(c, n);
        for (int stage = 0; stage < a->ns; ++stage) {
            if (c->p.order == 2)
                lanes_stage_p2<T>(c, n, stage);
            else
                lanes_stage_p1<T>(c, n, stage);
        }
        /* residuals of the base lane and of the second lane (a tangent has target 0) */
        k_misfit<<<blocks(a->ng, 128), 128, 0, s>>>(c->U, c->ldE, a->nw, a->ng, a->g_el, a->g_w, a->target + (size_t)n * a->ng,
                                  a->rt + (size_t)n * a->ng);
        k_misfit<<<blocks(a->ng, 128), 128, 0, s>>>(a->Ud, c->ldE, a->nw, a->ng, a->g_el, a->g_w,
                                  pert ? a->target + (size_t)n * a->ng : nullptr, a->rd + (size_t)n * a->ng);
        c->launches += 2;
    }
    k_misfit_sum<<<1, 32, 0, s>>>(a->rt, a->rd, (long long)a->nsteps * a->ng, pert ? 1 : 0, a->sums);
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev1, s));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    a->tlm_ms = ms;
    double sums[2];
    CK(cudaMemcpy(sums, a->sums, 16, cudaMemcpyDeviceToHost));
    if (J) *J = sums[0];
    if (out2) *out2 = sums[1];
    if (c->p.wet_dry) {
        c->wd_fresh = 1;
        c->wd_stepped = 1;
    }
    return DGR_OK;
}

extern "C" int dgr_tlm(dgr_ctx *c, const double *zeta, const double *Qx, const double *Qy, const int *WD,
                       const double *dzeta0, const double *dQx0, const double *dQy0, const double *dn_el,
                       const double *dz, double *J, double *dJ)
{
    NvtxRange nv("dgr_tlm");
    if (!c || !c->adj || !c->adj->have_forward || !zeta || !Qx || !Qy || !WD) return DGR_ERR_INVALID;
    AdjointState *a = c->adj;
    CK(cudaSetDevice(c->device));
    int r = ensure_tlm(c);
    if (r) return r;
    r = upload_scenarios(c, 0, c->nscen, zeta, Qx, Qy, WD);
    if (r) return r;
    cudaStream_t s = c->stream;
    const size_t ne = c->ne;
    CK(cudaMemsetAsync(a->Ud, 0, planes(c) * 8, s));
    if (dzeta0 || dQx0 || dQy0) {
        r = upload_planar(c, dzeta0, dQx0, dQy0, a->Ud);
        if (r) return r;
    }
    if (dz)
        CK(cudaMemcpyAsync(a->zd, dz, (size_t)c->nn * 8, cudaMemcpyHostToDevice, s));
    else
        CK(cudaMemsetAsync(a->zd, 0, (size_t)c->nn * 8, s));
    if (dn_el)
        CK(cudaMemcpyAsync(a->neld, dn_el, ne * 8, cudaMemcpyHostToDevice, s));
    else
        CK(cudaMemsetAsync(a->neld, 0, ne * 8, s));
    return run_lanes<ad::Dual>(c, J, dJ);
}

extern "C" int dgr_fd_frozen(dgr_ctx *c, const double *zeta, const double *Qx, const double *Qy, const int *WD,
                             const double *zeta_p, const double *Qx_p, const double *Qy_p, const double *n_el_p,
                             const double *z_p, double *J, double *J_p)
{
    NvtxRange nv("dgr_fd_frozen");
    if (!c || !c->adj || !c->adj->have_forward || !zeta || !Qx || !Qy || !WD) return DGR_ERR_INVALID;
    AdjointState *a = c->adj;
    CK(cudaSetDevice(c->device));
    int r = ensure_tlm(c);
    if (r) return r;
    r = upload_scenarios(c, 0, c->nscen, zeta, Qx, Qy, WD);
    if (r) return r;
    cudaStream_t s = c->stream;
    const size_t ne = c->ne;
    r = upload_planar(c, zeta_p ? zeta_p : zeta, Qx_p ? Qx_p : Qx, Qy_p ? Qy_p : Qy, a->Ud);
    if (r) return r;
    if (z_p)
        CK(cudaMemcpyAsync(a->zd, z_p, (size_t)c->nn * 8, cudaMemcpyHostToDevice, s));
    else
        CK(cudaMemcpyAsync(a->zd, c->zn, (size_t)c->nn * 8, cudaMemcpyDeviceToDevice, s));
    if (n_el_p)
        CK(cudaMemcpyAsync(a->neld, n_el_p, ne * 8, cudaMemcpyHostToDevice, s));
    else if (c->n_el)
        CK(cudaMemcpyAsync(a->neld, c->n_el, ne * 8, cudaMemcpyDeviceToDevice, s));
    else
        CK(cudaMemsetAsync(a->neld, 0, ne * 8, s));
    return run_lanes<ad::Pert>(c, J, J_p);
}

extern "C" int dgr_adjoint_timing(const dgr_ctx *c, double *forward_ms, double *backward_ms, double *tlm_ms)
{
    if (!c || !c->adj) return DGR_ERR_INVALID;
    if (forward_ms) *forward_ms = c->adj->fwd_ms;
    if (backward_ms) *backward_ms = c->adj->bwd_ms;
    if (tlm_ms) *tlm_ms = c->adj->tlm_ms;
    return DGR_OK;
}
