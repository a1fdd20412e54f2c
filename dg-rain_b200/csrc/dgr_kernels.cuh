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
#include "dgr_scheme.cuh"

/* Threads per block of the edge kernel, and the minimum resident blocks per SM requested
 * from the compiler for it (register cap 65536 / (DGR_EDGE_BS x blocks) = 85, so 80);
 * chosen by measurement (4,000,000 triangles: 0.332 ms per launch in blocks of 128, 0.338
 * in blocks of 64, 0.352 in blocks of 256), overridable at build time.  The element
 * kernels are capped at 128 registers and the limiter kernels at 64
 * (DGR_ELEMENT_THREADS_PER_SM and DGR_LIMIT_THREADS_PER_SM below). */
#ifndef DGR_EDGE_BS
#define DGR_EDGE_BS 128
#endif
#ifndef DGR_MINB_EDGE
#define DGR_MINB_EDGE (768 / DGR_EDGE_BS)
#endif
/* 1: the edge and limiter kernels take their divisions through shared reciprocals
 * (div_rcp), queueing the items where that is not valid for a plain-division redo launch;
 * 0: plain divisions.  Chosen by measurement, overridable at build time. */
/* Resident threads per SM requested for the limiter kernel (register cap 65536 / this);
 * chosen by measurement (1024: 64 registers, 0.244 ms at 4M triangles; 768: 80 registers,
 * 0.271 ms; 512: 0.350 ms). */
#ifndef DGR_LIMIT_THREADS_PER_SM
#define DGR_LIMIT_THREADS_PER_SM 1024
#endif
/* Resident threads per SM requested for the element kernel (register cap 65536 / this:
 * 128 registers at 512). */
#ifndef DGR_ELEMENT_THREADS_PER_SM
#define DGR_ELEMENT_THREADS_PER_SM 512
#endif
#ifndef DGR_EDGE_RCP
#define DGR_EDGE_RCP 1
#endif
#ifndef DGR_LIMIT_RCP
#define DGR_LIMIT_RCP 1
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

/* Clock and forcing of one scenario (one mesh of an ensemble; a single mesh is an
 * ensemble of one).  Every scenario advances with its own CFL dt. */
struct DevClock {
    double time;        /* current time */
    double dt;          /* dt of the step in progress, then of the next step */
    double final_time;
    double bc2_zeta;    /* type-2 boundary elevation of the step in progress */
    unsigned long long lam_bits[3]; /* max wave speed per stage, bits of a double >= 0 */
    unsigned long long err;         /* first failure key; ~0 = none */
    int step;           /* steps done in the current run */
    int nsteps;         /* step limit of the current run */
    int done;           /* 1: the run has finished, later kernels do nothing */
    int dt_pending;     /* 1: dt of the next step is still to be derived from the last stage's lam_bits */
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
    int flux;             /* numerical flux: 0 Roe (2DCode), 1 local Lax-Friedrichs, 2 HLLC (DG-SWEM) */
    unsigned long long *bad_index; /* checked build: first out-of-range gather, (kernel << 32 | item) */
    int *redo;            /* edges left to k_edge_redo: [0] count, [1] blocks done, [2..] edges */
};

/* Checked build (compiled with -DDGR_CHECKED): every index a kernel gathers from the
 * connectivity arrays is tested against its range before it is used; one out of range is
 * recorded in the context's bad-index word (the least (kernel << 32 | item) wins) and the
 * item skips its work, so a broken array becomes DGR_ERR_BAD_INDEX instead of a read or
 * write outside an array.  Without DGR_CHECKED the test compiles to nothing. */
enum { KID_EDGE = 1, KID_ELEMENT = 2, KID_NODE = 3, KID_LIMIT = 4 };
#ifdef DGR_CHECKED
DGR_DEV bool index_ok(const MeshDev &m, int idx, int n, int kernel, int item)
{
    if ((unsigned)idx < (unsigned)n) return true;
    atomicMin(m.bad_index, ((unsigned long long)kernel << 32) | (unsigned)item);
    return false;
}
#else
DGR_DEV constexpr bool index_ok(const MeshDev &, int, int, int, int) { return true; }
#endif

struct PhysParams {
    double g, h0, velzero, cfl, dt0;
    int stages; /* RK stages per step (2 or 3); the CFL dt follows the last stage's wave speed */
};

/* L2 prefetch of one block's slice [base, base + n) of `planes` planes of stride ld
 * (elements of T): one bulk prefetch per plane, issued by threads 0..planes-1.  The size is
 * rounded down to the 16 bytes a bulk prefetch moves, so it never reaches past the slice;
 * base * sizeof(T) and ld * sizeof(T) must be multiples of 16. */
template <class T>
DGR_DEV void l2_prefetch_slice(const T *p0, int ld, int planes, int base, int n)
{
    const unsigned bytes = (unsigned)((size_t)n * sizeof(T)) & ~15u;
    if (bytes == 0) return;
    for (int j = threadIdx.x; j < planes; j += blockDim.x)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(__cvta_generic_to_global(p0 + (size_t)j * ld + base)),
                     "r"(bytes)
                     : "memory");
}

/* L2 prefetch of the geometry of elements [base, base + n) (whole tiles when tiled: the
 * allocation holds every tile in full), in chunks of 4 KB over the block's threads. */
DGR_DEV void prefetch_geometry(const MeshDev &m, int base, int n)
{
    if (!DGR_GEO_TILED) {
        l2_prefetch_slice(m.geo, m.ldE, NG, base, n);
        return;
    }
    if (n <= 0) return;
    const char *p0 = reinterpret_cast<const char *>(m.geo + geo_offset(base & ~31, m.ldE));
    const unsigned bytes = (unsigned)(((base + n + 31) >> 5) - (base >> 5)) * NG * 32 * 8;
    for (unsigned off = threadIdx.x * 4096u; off < bytes; off += blockDim.x * 4096u) {
        const unsigned len = min(4096u, bytes - off);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(__cvta_generic_to_global(p0 + off)), "r"(len)
                     : "memory");
    }
}

/* ------------------------------------------------------------------ edges ---- */

/* One edge (2DCode/compute2DL.c:17-331): traces, ghost state, Roe flux(es); stores Fhat.n
 * for both sides and returns the edge's max wave speed (0 for a finished scenario).
 * FT: the numerical flux as a compile-time constant (0 Roe, 1 LLF, 2 HLLC), or -1 to take
 * it from the mesh at run time.  With `redo` non-null the Roe flux's divisions share one
 * reciprocal per divisor (RcpDiv, the same bits); an edge where that is not valid reports
 * no error and no speed and sets *redo: the caller queues it for k_edge_redo, which
 * redoes it with plain divisions in a launch of its own and overwrites its fluxes. */
template <bool WD, bool COH = false, int FT = -1>
DGR_DEV double edge_flux_item(const MeshDev &m, const double *S, const int *wd, const double *bzeta,
                              const double *bqn, double *flux, DevClock *clk, int phase, double g, int i,
                              bool *redo = nullptr)
{
    double lam = 0.0;
    DevClock *ck = clk + (m.ed_sid ? m.ed_sid[i] : 0);
    if (!ldm<COH>(&ck->done)) {
        const int el_in = m.e_in[i], el_ex = m.e_ex[i], info = m.e_info[i];
        const int k_in = info & 3, k_ex = (info >> 2) & 3, bd = (info >> 4) & 7;
        if (!(index_ok(m, el_in, m.ne, KID_EDGE, i) && index_ok(m, el_ex, m.ne, KID_EDGE, i) &&
              index_ok(m, k_in, 3, KID_EDGE, i) && index_ok(m, k_ex, 3, KID_EDGE, i)))
            return 0.0;
        const double nx = m.e_geo[i], ny = m.e_geo[m.ldF + i], z_edge = m.e_geo[2 * m.ldF + i];
        const int ld = m.ldE;
        const double zi = ldm<COH>(&S[k_in * ld + el_in]), qxi = ldm<COH>(&S[(3 + k_in) * ld + el_in]),
                     qyi = ldm<COH>(&S[(6 + k_in) * ld + el_in]);
        double ze, qxe, qye;
        if (bd)
            ghost_state<double>(bd, nx, ny, zi, qxi, qyi, ldm<COH>(&bzeta[i]), ldm<COH>(&bqn[i]), 0.0, ze, qxe, qye);
        else if (el_in == el_ex)
            ghost_state<double>(0, nx, ny, zi, qxi, qyi, 0.0, 0.0, ldm<COH>(&S[k_ex * ld + el_ex]), ze, qxe, qye);
        else {
            ze = ldm<COH>(&S[k_ex * ld + el_ex]);
            qxe = ldm<COH>(&S[(3 + k_ex) * ld + el_ex]);
            qye = ldm<COH>(&S[(6 + k_ex) * ld + el_ex]);
        }
        const int wdi = WD ? ldm<COH>(&wd[el_in]) : 1, wde = WD ? ldm<COH>(&wd[el_ex]) : 1;
        double fin[3], fex[3];
        int code;
        if (redo) {
            RcpDiv dv;
            lam = flux_core<double, WD, RcpDiv>(zi, qxi, qyi, ze, qxe, qye, z_edge, nx, ny, wdi, wde, g, fin, fex,
                                                code, FT >= 0 ? FT : m.flux, &dv);
            if (!dv.ok) { /* k_edge_redo rewrites this edge's fluxes, error and speed */
                *redo = true;
                code = 0;
                lam = 0.0;
            }
        } else {
            lam = flux_core<double, WD>(zi, qxi, qyi, ze, qxe, qye, z_edge, nx, ny, wdi, wde, g, fin, fex, code,
                                        FT >= 0 ? FT : m.flux);
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

template <bool WD, int FT>
__global__ void __launch_bounds__(DGR_EDGE_BS, DGR_MINB_EDGE) k_edge_flux(const __grid_constant__ MeshDev m, const double *__restrict__ S,
                                                                  const int *__restrict__ wd,
                                                                  const double *__restrict__ bzeta,
                                                                  const double *__restrict__ bqn,
                                                                  double *__restrict__ flux, DevClock *clk,
                                                                  int lam_slot, int phase, double g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < m.nf;
    const int sid = (valid && m.ed_sid) ? m.ed_sid[i] : 0;
    bool redo = false;
    const double lam =
        valid ? edge_flux_item<WD, false, FT>(m, S, wd, bzeta, bqn, flux, clk, phase, g, i,
                                              DGR_EDGE_RCP ? &redo : nullptr)
              : 0.0;
    if (redo) m.redo[2 + atomicAdd(&m.redo[0], 1)] = i;
    block_max_speed(lam, sid, valid, clk, lam_slot);
}

/* The edges k_edge_flux queued (m.redo: [0] count, [1] blocks done, [2..] edges), with
 * plain divisions: fluxes, error and wave speed as k_edge_flux would have given them.
 * Launched after every k_edge_flux; with nothing queued each block returns at once.  The
 * last block to finish clears the queue for the next launch. */
template <bool WD, int FT>
__global__ void __launch_bounds__(256) k_edge_redo(const __grid_constant__ MeshDev m, const double *__restrict__ S,
                                                   const int *__restrict__ wd, const double *__restrict__ bzeta,
                                                   const double *__restrict__ bqn, double *__restrict__ flux,
                                                   DevClock *clk, int lam_slot, int phase, double g)
{
    const int n = *(volatile int *)&m.redo[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = m.redo[2 + k];
        const double lam = edge_flux_item<WD, false, FT>(m, S, wd, bzeta, bqn, flux, clk, phase, g, i);
        const int sid = m.ed_sid ? m.ed_sid[i] : 0;
        if (lam > 0.0) atomicMax(&clk[sid].lam_bits[lam_slot], (unsigned long long)__double_as_longlong(lam));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&m.redo[1], 1) == (int)gridDim.x - 1) {
            m.redo[0] = 0;
            m.redo[1] = 0;
        }
    }
}

/* ---------------------------------------------------------------- elements ---- */

/* Gathered numerical fluxes of one element's three edges, sign flipped on the "ex" side
 * (2DCode/2DInnerProducts.c:319-329).  F[variable][local edge]. */
template <bool COH>
DGR_DEV bool gather_flux(const MeshDev &m, const double *flux, int el, double F[3][3])
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int ee = m.elem_edge[k * m.ldE + el];
        const int e = ee >> 1;
        const int side = ee & 1;
        if (!index_ok(m, e, m.nf, KID_ELEMENT, el)) return false;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double f = ldm<COH>(&flux[(3 * side + v) * m.ldF + e]);
            F[v][k] = side ? -f : f;
        }
    }
    return true;
}

/* One element of the RHS / RK stage (element_core); S is the stage input, U the step
 * input (stage 2 only).  MODE_RHS writes the RHS.  RCP: the fits' divisions by their
 * determinant share one reciprocal (div_rcp, the same bits); an element where that is not
 * valid is redone by element_item_plain (plain divisions, kept out of line). */
template <int MODE, bool COH = false, bool RCP = true>
DGR_DEV void element_item(const MeshDev &m, const double *S, const double *U, const int *wd, const double *flux,
                          double *out, double *avg, const DevClock *clk, double g, int el);

template <int MODE, bool COH>
__device__ __noinline__ void element_item_plain(const MeshDev &m, const double *S, const double *U, const int *wd,
                                                const double *flux, double *out, double *avg, const DevClock *clk,
                                                double g, int el)
{
    element_item<MODE, COH, false>(m, S, U, wd, flux, out, avg, clk, g, el);
}

template <int MODE, bool COH, bool RCP>
DGR_DEV void element_item(const MeshDev &m, const double *S, const double *U, const int *wd, const double *flux,
                          double *out, double *avg, const DevClock *clk, double g, int el)
{
    const DevClock *ck = clk + (m.el_sid ? m.el_sid[el] : 0);
    if (ldm<COH>(&ck->done)) return;
    const double rain = ck->rain;
    const int ld = m.ldE;
    const double *G = m.geo + geo_offset(el, ld);
    const int gs = geo_stride(ld);
    double F[3][3];
    if (!gather_flux<COH>(m, flux, el, F)) return;
    double zr[3], qxr[3], qyr[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        zr[k] = ldm<COH>(&S[k * ld + el]);
        qxr[k] = ldm<COH>(&S[(3 + k) * ld + el]);
        qyr[k] = ldm<COH>(&S[(6 + k) * ld + el]);
    }
    const double local_g = (ldm<COH>(&wd[el]) == 0) ? 0.0 : g;
    const auto uin = [U, ld, el](int v, int k) { return ldm<COH>(&U[(3 * v + k) * ld + el]); };
    const double dt = (MODE == MODE_RHS) ? 0.0 : ldm<COH>(&ck->dt);
    double w[3][3], a[3];
    bool rcp_ok = true;
    const auto geo = [G, gs](int j) { return G[(size_t)j * gs]; };
    const PlaneZGeo zg{G, gs};
    element_core<MODE, double, decltype(geo), PlaneZGeo, decltype(uin), RCP>(F, zr, qxr, qyr, geo, zg, uin, local_g,
                                                                          rain, dt, w, a, &rcp_ok);
    if (RCP && !rcp_ok) {
        element_item_plain<MODE, COH>(m, S, U, wd, flux, out, avg, clk, g, el);
        return;
    }
#pragma unroll
    for (int v = 0; v < 3; ++v) {
#pragma unroll
        for (int k = 0; k < 3; ++k) out[(3 * v + k) * ld + el] = w[v][k];
        if (MODE != MODE_RHS) avg[v * ld + el] = a[v];
    }
}

template <int MODE, int BS>
__global__ void __launch_bounds__(BS, DGR_ELEMENT_THREADS_PER_SM / BS) k_element(const __grid_constant__ MeshDev m, const double *__restrict__ S,
                                                          const double *__restrict__ U, const int *__restrict__ wd,
                                                          const double *__restrict__ flux, double *__restrict__ out,
                                                          double *__restrict__ avg, const DevClock *clk, double g)
{
    /* the block's geometry planes are requested from DRAM at once instead of in the order
     * the element computation reaches them (measured: 4 % off this kernel) */
    prefetch_geometry(m, blockIdx.x * BS, min(BS, m.ne - blockIdx.x * BS));
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
    if (!(index_ok(m, b, 3 * m.ne + 1, KID_NODE, n) && index_ok(m, e, 3 * m.ne + 1, KID_NODE, n) &&
          index_ok(m, e - b, 3 * m.ne + 1, KID_NODE, n)))
        return;
    for (int j = b; j < e; ++j) {
        const int el = m.n2e[j];
        if (!index_ok(m, el, m.ne, KID_NODE, n)) return;
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

#ifndef DGR_NODE_BS /* threads per block of the node-bounds kernel */
#define DGR_NODE_BS 256
#endif
static __global__ void __launch_bounds__(DGR_NODE_BS) k_node_bounds(MeshDev m, const double *__restrict__ avg,
                                                     double *__restrict__ bounds)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < m.nn) node_item(m, avg, bounds, n);
}

/* Element means of a state (used by the stand-alone limiter call). */
static __global__ void __launch_bounds__(256) k_avg(MeshDev m, const double *__restrict__ S, double *__restrict__ avg)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= m.ne) return;
    const int ld = m.ldE;
#pragma unroll
    for (int v = 0; v < 3; ++v)
        avg[v * ld + el] = (S[(3 * v) * ld + el] + S[(3 * v + 1) * ld + el] + S[(3 * v + 2) * ld + el]) / 3;
}

/* --------------------------------------------------------------- wet/dry ---- */

static __global__ void __launch_bounds__(256) k_wd_status(MeshDev m, const double *__restrict__ S, int *wd,
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
 * One element: vertex-based limiter and positive-depth operator (limit_core), then the
 * wet/dry status (2DCode/wetDry2D.c:16-60) that the reference calls next.  wd_in is the
 * status the element had; the new status goes to wd_out.
 */
template <bool LIMIT, bool PDOP, bool STATUS, bool COH = false, bool RCP = false>
DGR_DEV void limit_item(const MeshDev &m, double *S, const double *bounds, const int *wd_in, int *wd_out,
                        DevClock *clk, double h0, double velzero, int phase, int *dec_limit, int *dec_pdop, int el)
{
    DevClock *ck = clk + (m.el_sid ? m.el_sid[el] : 0);
    if (ldm<COH>(&ck->done)) return;
    const int ld = m.ldE;
    const int nd[3] = {m.el2v[el], m.el2v[ld + el], m.el2v[2 * ld + el]};
    if (!(index_ok(m, nd[0], m.nn, KID_LIMIT, el) && index_ok(m, nd[1], m.nn, KID_LIMIT, el) &&
          index_ok(m, nd[2], m.nn, KID_LIMIT, el)))
        return;
    const double zn[3] = {m.zn[nd[0]], m.zn[nd[1]], m.zn[nd[2]]};
    double w[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) w[v][k] = ldm<COH>(&S[(3 * v + k) * ld + el]);
    const int lb = m.ldN;
    const auto bnd = [bounds, lb, &nd](int v, int k, int is_min) {
        return ldm<COH>(&bounds[(3 * is_min + v) * lb + nd[k]]);
    };
    LimitDecisions dec;
    RcpDiv dv;
    if constexpr (RCP) {
        limit_core<LIMIT, PDOP, double, decltype(bnd), false, RcpDiv>(w, bnd, zn, h0, velzero, dec, nullptr, &dv);
        if (!dv.ok) { /* k_limit_redo redoes it with plain divisions from the untouched state */
            m.redo[2 + atomicAdd(&m.redo[0], 1)] = el;
            return;
        }
    } else {
        limit_core<LIMIT, PDOP, double>(w, bnd, zn, h0, velzero, dec);
    }
    if (LIMIT && dec_limit) dec_limit[el] = dec.modify;
    if (PDOP) {
        if (dec.code) atomicMin(&ck->err, err_key(ldm<COH>(&ck->step), phase, dec.code, el - ck->el_off));
        if (dec_pdop) dec_pdop[el] = 4 * dec.mass_branch + dec.mom_branch;
    }
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) S[(3 * v + k) * ld + el] = w[v][k];
    if (STATUS) {
        if constexpr (RCP) {
            const int st = wd_status(w[0], zn, ldm<COH>(&wd_in[el]), h0, &dv);
            /* the element's state is written: a status that needs the plain division is
             * taken with it here (one division, so inline) */
            wd_out[el] = dv.ok ? st : wd_status(w[0], zn, ldm<COH>(&wd_in[el]), h0);
        } else {
            wd_out[el] = wd_status(w[0], zn, ldm<COH>(&wd_in[el]), h0);
        }
    }
}

template <bool LIMIT, bool PDOP, bool STATUS, int BS>
__global__ void __launch_bounds__(BS, DGR_LIMIT_THREADS_PER_SM / BS) k_limit(const __grid_constant__ MeshDev m, double *__restrict__ S,
                                                        const double *__restrict__ bounds,
                                                        const int *__restrict__ wd_in, int *__restrict__ wd_out,
                                                        DevClock *clk, double h0, double velzero, int phase,
                                                        int *__restrict__ dec_limit, int *__restrict__ dec_pdop)
{
    const int el = blockIdx.x * BS + threadIdx.x;
    if (el < m.ne)
        limit_item<LIMIT, PDOP, STATUS, false, DGR_LIMIT_RCP>(m, S, bounds, wd_in, wd_out, clk, h0, velzero, phase,
                                                             dec_limit, dec_pdop, el);
}

/* The elements k_limit queued (m.redo, as k_edge_redo), with plain divisions, from their
 * state as k_limit left it (untouched).  The last block to finish clears the queue. */
template <bool LIMIT, bool PDOP, bool STATUS>
__global__ void __launch_bounds__(128) k_limit_redo(const __grid_constant__ MeshDev m, double *__restrict__ S,
                                                    const double *__restrict__ bounds, const int *__restrict__ wd_in,
                                                    int *__restrict__ wd_out, DevClock *clk, double h0,
                                                    double velzero, int phase, int *__restrict__ dec_limit,
                                                    int *__restrict__ dec_pdop)
{
    const int n = *(volatile int *)&m.redo[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        limit_item<LIMIT, PDOP, STATUS>(m, S, bounds, wd_in, wd_out, clk, h0, velzero, phase, dec_limit, dec_pdop,
                                        m.redo[2 + k]);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&m.redo[1], 1) == (int)gridDim.x - 1) {
            m.redo[0] = 0;
            m.redo[1] = 0;
        }
    }
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
            const double lam = __longlong_as_double((long long)c->lam_bits[p.stages - 1]);
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
        c->lam_bits[2] = 0;
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

static __global__ void __launch_bounds__(256) k_clock_begin(DevClock *clk, int nscen, PhysParams p,
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

static __global__ void k_clock_end(DevClock *clk, int nscen)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nscen) clock_end_item(clk, s);
}

/* After a run: derive each scenario's next dt so the host sees it. */
static __global__ void k_clock_finish(DevClock *clk, int nscen, PhysParams p)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nscen) return;
    DevClock *c = clk + s;
    if (c->dt_pending) {
        const double lam = __longlong_as_double((long long)c->lam_bits[p.stages - 1]);
        double dt = p.cfl * c->min_edge / lam;
        if ((c->time + dt) > c->final_time) dt = c->final_time - c->time;
        c->dt = dt;
        c->dt_pending = 0;
    }
}

/* Gauge values after a step of the device loop: row (step - 1) of the series holds
 * zeta_g = sum_k w[nm g + k] zeta_k(el_g) for the step count of the gauge's scenario (a
 * finished scenario rewrites its last row with the same state). */
static __global__ void k_gauge_record(const double *__restrict__ S, int ld, int nm, int ng, const int *__restrict__ g_el,
                                      const int *__restrict__ g_sid, const double *__restrict__ g_w,
                                      const DevClock *clk, int cap, double *__restrict__ series)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng) return;
    const int step = clk[g_sid[g]].step;
    if (step < 1 || step > cap) return;
    const int el = g_el[g];
    double z = g_w[nm * g] * S[el];
    for (int k = 1; k < nm; ++k) z += g_w[nm * g + k] * S[(size_t)k * ld + el];
    series[(size_t)(step - 1) * ng + g] = z;
}

/* Host-driven step (oneTimeStep2D, single mesh): set the step's dt, clear per-step words. */
static __global__ void k_clock_set(DevClock *clk, double time, double dt)
{
    clk->time = time;
    clk->dt = dt;
    clk->done = 0;
    clk->lam_bits[0] = 0;
    clk->lam_bits[1] = 0;
    clk->lam_bits[2] = 0;
}

/* Device-side boundary_conditions() at time t for the stand-alone call. */
static __global__ void k_forcing(const DevClock *clk, double t, const int *__restrict__ bnd_edges,
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
    int *wdA, *wdB, *wdC;
    DevClock *clk;
    int nscen;
    const int *bnd_edges, *bnd_type, *bnd_sid;
    int nbnd;
    PhysParams p;
    int *dec;         /* [4][ne] decisions, or nullptr */
    unsigned *bar;    /* [0] arrivals, [1] generation, [2] time-out flag */
    unsigned bar_polls;   /* polls of a barrier wait before it gives up */
    unsigned bar_phantom; /* blocks a barrier also waits for that never arrive (0; tests of the time-out) */
};

/* Polls of a grid-barrier wait before it gives up (about a second with the 64 ns sleeps). */
constexpr unsigned kBarrierSpins = 1u << 24;

/* Grid-wide barrier of a cooperative launch (every block resident).  The wait is bounded:
 * a block that polls `polls` times records a time-out, and every block leaves the kernel
 * at its next barrier check, so a broken invariant ends the launch with an error flag
 * instead of hanging the GPU.  `phantom` extra arrivals are expected on top of the grid's
 * blocks: nonzero only to make the wait run out on purpose (a test of that path).
 * Returns false once a time-out is recorded. */
DGR_DEV bool grid_barrier(unsigned *bar, unsigned polls, unsigned phantom)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = bar + 1;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        if (arrived == gridDim.x - 1 + phantom) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned spins = 0;
            while (*vgen == gen) {
                if (++spins > polls) {
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
__global__ void __launch_bounds__(BS, 512 / BS) k_step_fused(const __grid_constant__ FusedArgs a, int stage_begin, int stage_end,
                                                             int with_clock)
{
    if (with_clock) {
        if (blockIdx.x == 0)
            clock_begin_body(a.clk, a.nscen, a.p, a.bnd_edges, a.bnd_type, a.bnd_sid, a.nbnd, a.bzeta, a.bqn);
        if (!grid_barrier(a.bar, a.bar_polls, a.bar_phantom)) return;
    }
    const int stride = gridDim.x * BS;
    const int ne = a.m.ne;
    const int ns = a.p.stages;
    int *bufs[3] = {a.wdA, a.wdB, a.wdC};
    for (int stage = stage_begin; stage < stage_end; ++stage) {
        /* the buffers of stage_io (dgr_internal.cuh) */
        const double *S = stage == 0 ? a.U : a.W;
        double *OUT = stage == ns - 1 ? a.U : a.W;
        const int *wd_in = WD ? bufs[stage] : a.wdA;
        int *wd_out = bufs[(stage + 1) % ns];
        const int mode = stage == 0 ? MODE_STAGE1 : (ns == 2 ? MODE_STAGE2 : (stage == 1 ? MODE_RK3_2 : MODE_RK3_3));
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
        if (!grid_barrier(a.bar, a.bar_polls, a.bar_phantom)) return;
        for (int el = blockIdx.x * BS + threadIdx.x; el < ne; el += stride) {
            if (mode == MODE_STAGE1)
                element_item<MODE_STAGE1, true>(a.m, S, a.U, wd_in, a.flux, OUT, a.avg, a.clk, a.p.g, el);
            else if (mode == MODE_STAGE2)
                element_item<MODE_STAGE2, true>(a.m, S, a.U, wd_in, a.flux, OUT, a.avg, a.clk, a.p.g, el);
            else if (mode == MODE_RK3_2)
                element_item<MODE_RK3_2, true>(a.m, S, a.U, wd_in, a.flux, OUT, a.avg, a.clk, a.p.g, el);
            else
                element_item<MODE_RK3_3, true>(a.m, S, a.U, wd_in, a.flux, OUT, a.avg, a.clk, a.p.g, el);
        }
        if (!grid_barrier(a.bar, a.bar_polls, a.bar_phantom)) return;
        for (int n = blockIdx.x * BS + threadIdx.x; n < a.m.nn; n += stride) node_item<true>(a.m, a.avg, a.bounds, n);
        if (!grid_barrier(a.bar, a.bar_polls, a.bar_phantom)) return;
        for (int el = blockIdx.x * BS + threadIdx.x; el < ne; el += stride)
            limit_item<true, WD, WD, true>(a.m, OUT, a.bounds, wd_in, wd_out, a.clk, a.p.h0, a.p.velzero,
                                           2 * stage + 1, dl, dp, el);
        if (stage + 1 < stage_end || with_clock)
            if (!grid_barrier(a.bar, a.bar_polls, a.bar_phantom)) return;
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
static __global__ void k_edge_setup(int nf, int ldE, int ldF, const int *__restrict__ ed2el, const int *__restrict__ ed2v,
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
    /* bit 7: the "ex" element's local edge runs in the same direction as the "in" one (the
     * p = 2 step pairs Gauss points by it; opposite for consistently oriented elements) */
    const int ex_start = el2v_aos[3 * el_ex + k_ex];
    const int same_dir = (el_ex != el_in && ex_start == p0) ? 1 : 0;
    e_in[i] = el_in;
    e_ex[i] = el_ex;
    e_info[i] = k_in | (k_ex << 2) | ((bdry[i] & 7) << 4) | (same_dir << 7);
    e_geo[i] = nx;
    e_geo[ldF + i] = ny;
    e_geo[2 * ldF + i] = (z[v0] + z[v1]) / 2;
    elem_edge[k_in * ldE + el_in] = i << 1;
    if (el_ex != el_in) elem_edge[k_ex * ldE + el_ex] = (i << 1) | 1;
}

/* Per-element state-independent factors (element_geometry) of every element. */
static __global__ void k_element_setup(int ne, int ldE, const int *__restrict__ el2v_aos, const double *__restrict__ x,
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
    const double xv[3] = {x[v0], x[v1], x[v2]}, yv[3] = {y[v0], y[v1], y[v2]}, zv[3] = {z[v0], z[v1], z[v2]};
    const double nfv[3] = {nfric[v0], nfric[v1], nfric[v2]};
    double *G = geo + geo_offset(i, ldE);
    const int gs = geo_stride(ldE);
    element_geometry(xv, yv, zv, nfv, n_el ? n_el[i] : -1.0, g,
                     [G, gs](int j, double val) { G[(size_t)j * gs] = val; });
}

/* the Manning power on n arguments (diagnostic entry point) */
static __global__ void k_pow43(int n, const double *__restrict__ x, double *__restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = pow43(x[i]);
}

/* reference layout [3*el+k] <-> planar [3*v+k][ld] */
static __global__ void k_aos_to_planar(int ne, int ld, const double *__restrict__ a0, const double *__restrict__ a1,
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

static __global__ void k_planar_to_aos(int ne, int ld, const double *__restrict__ S, double *__restrict__ a0,
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

/* the same transposes for nm coefficients per element and variable ([nm*el+k] <->
 * planar [nm*v+k][ld]; nm = 3 for p = 1, 6 for p = 2) */
static __global__ void __launch_bounds__(256) k_aos_to_planar_nm(int ne, int ld, int nm, const double *__restrict__ a0,
                                                                 const double *__restrict__ a1,
                                                                 const double *__restrict__ a2, double *__restrict__ S)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= ne) return;
    const double *src[3] = {a0, a1, a2};
    for (int v = 0; v < 3; ++v)
        for (int k = 0; k < nm; ++k) S[(size_t)(nm * v + k) * ld + el] = src[v][(size_t)nm * el + k];
}

static __global__ void __launch_bounds__(256) k_planar_to_aos_nm(int ne, int ld, int nm, const double *__restrict__ S,
                                                                 double *__restrict__ a0, double *__restrict__ a1,
                                                                 double *__restrict__ a2)
{
    const int el = blockIdx.x * blockDim.x + threadIdx.x;
    if (el >= ne) return;
    double *dst[3] = {a0, a1, a2};
    for (int v = 0; v < 3; ++v)
        for (int k = 0; k < nm; ++k) dst[v][(size_t)nm * el + k] = S[(size_t)(nm * v + k) * ld + el];
}

/* edge fluxes back into the reference's element slots Fhat[3*el+k] */
static __global__ void k_flux_to_slots(MeshDev m, const double *__restrict__ flux, double *f1, double *f2, double *f3)
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
