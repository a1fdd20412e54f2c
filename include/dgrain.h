/*
 * dgrain.h — C ABI of the B200 DG-RAIN 2D shallow-water step.
 *
 * The reference (evalseth/DG-RAIN, 2DCode/) has no library interface: its step is a set
 * of link-level C functions over process-wide globals (2DCode/MeshAttributes.h:5-42).
 * This header replaces those functions one for one, with an explicit context instead of
 * globals and an int status instead of exit():
 *
 *   reference (2DCode/)                                   this ABI
 *   store_mesh(char*)            extract_mesh_attributes.c:39    dgr_read_fort14()
 *   extract_mesh_attributes()    extract_mesh_attributes.c:143   dgr_build_connectivity()
 *   initialize()                 initialize.c:29                 dgr_initial_state()
 *   boundary_conditions()        boundary_conditions.c:9         dgr_set_boundary() / dgr_boundary_conditions()
 *   compute2DL(double)           compute2DL.c:12                 dgr_compute_L()
 *   SlopeLimiter()               SlopeLimiter2D.c:10             dgr_slope_limiter()
 *   wetDryStatus2D()             wetDry2D.c:16                   dgr_wet_dry_status()
 *   PDop2D()                     wetDry2D.c:63                   dgr_pdop()
 *   oneTimeStep2D(double,double) time_evolution.c:10             dgr_step()
 *   time_evolution(double)       time_evolution.c:248            dgr_run()
 *   .dat writer                  time_evolution.c:324-390        dgr_write_dat()
 *
 * Data layout at this boundary is the reference's: state arrays are double[3*NumEl]
 * indexed [3*el+k] with k the local edge (v_k, v_{(k+1)%3}); mesh arrays are the
 * reference's EltoVert[3*NumEl], EdgtoEls[2*NumEdges], EdgtoVert[2*NumEdges],
 * BdryPrescribed[NumEdges] with 0-based indices.  Ownership stays with the caller: every
 * array passed in is copied before the call returns.
 *
 * Errors: every function returns DGR_OK (0) or a DGR_ERR_* code.  The numerical failures
 * that make the reference print a message and exit (2DCode/compute2DL.c:245-302,
 * 2DCode/wetDry2D.c:142-146,233-237) are returned as codes 1-5, and dgr_last_error()
 * gives the edge or element index the reference would have printed.
 *
 * Threading: a context belongs to one host thread at a time and owns one CUDA stream.
 * Separate contexts may be used from separate threads.
 */
#ifndef DGRAIN_H
#define DGRAIN_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DGR_ABI_VERSION 1

/* Exported entry points keep default visibility in a library built with
 * -fvisibility=hidden. */
#if defined(__GNUC__)
#define DGR_API __attribute__((visibility("default")))
#else
#define DGR_API
#endif

enum dgr_status {
    DGR_OK = 0,
    DGR_ERR_NAN_FLUX = 1,     /* 2DCode/compute2DL.c:245-249 and :298-302 */
    DGR_ERR_NAN_FLUX_IN = 2,  /* 2DCode/compute2DL.c:262-266 */
    DGR_ERR_NAN_FLUX_EX = 3,  /* 2DCode/compute2DL.c:281-285 */
    DGR_ERR_NEG_DEPTH = 4,    /* 2DCode/wetDry2D.c:142-146 */
    DGR_ERR_NAN_VELOCITY = 5, /* 2DCode/wetDry2D.c:233-237 */
    DGR_ERR_EDGE_MATCH = 6,   /* 2DCode/compute2DL.c:51-67 */
    DGR_ERR_BAD_INDEX = 7,    /* library built with DGR_CHECKED: a kernel met an out-of-range index in the
                                 connectivity (dgr_last_error: the item, and the kernel in place of the step) */
    DGR_ERR_INVALID = 10,     /* bad argument */
    DGR_ERR_MESH = 11,        /* inconsistent mesh (edge count, uncovered element edge) */
    DGR_ERR_IO = 12,          /* file cannot be read or written */
    DGR_ERR_CUDA = 13,        /* a CUDA call failed; see dgr_last_cuda_error() */
    DGR_ERR_NO_DEVICE = 14,   /* no CUDA device: this library has no CPU fallback */
    DGR_ERR_TOO_LARGE = 15,   /* size beyond a documented limit */
    DGR_ERR_TIMEOUT = 16      /* a bounded device-side wait gave up (persistent kernel barrier) */
};

/* Run parameters.  dgr_params_default() fills the reference's constants. */
typedef struct dgr_params {
    double g;        /* 9.81   2DCode/initialize.c:22 */
    double H0;       /* 1e-3   2DCode/initialize.c:26 */
    double VELZERO;  /* 1e-2   2DCode/initialize.c:27 */
    double cfl;      /* 0.1    2DCode/time_evolution.c:399 */
    double dt0;      /* 1e-7   2DCode/time_evolution.c:255 */
    int wet_dry;     /* 1: wet/dry on — compute2DL's WDON flux branch plus wetDryStatus2D and
                        PDop2D in the order of ChanNet/time_evolution.c:218-427.
                        0: the step exactly as 2DCode ships it. Default 1. */
    int tide_on;     /* 1: type-2 (outflow-list) edges get zeta_b = tide_amp*sin(2*pi*t/tide_period)
                        instead of 0.296 (extension; the reference has no tide). Default 0. */
    double tide_amp;
    double tide_period;
    double rain;     /* m/s added to the elevation right-hand side (extension). Default 0. */
    int device;      /* CUDA device ordinal. Default 0. */
    int record_decisions; /* 1: keep per-element limiter/PDop decisions of the last step. */
    int rk_stages;   /* 2: SSP-RK2 of 2DCode/time_evolution.c:10-246 (default).  3: SSP(3,3),
                        the coefficients of DG-SWEM src/prep_DG.F:1253-1270 (extension: the
                        limiter, PDop and status follow every stage as in the RK2 order). */
    int order;       /* 1: 2DCode's p = 1 Crouzeix-Raviart step (default).  2: p = 2 modal DG with
                        DG-SWEM's orthogonal basis (src/orthobasis_area.F) - an extension for
                        flows that stay wet: wet_dry must be 0, there is no limiter, and the
                        state is 6 modal coefficients per element and variable,
                        zeta[6*el + m] etc. (see dgr_p2_reference). */
    int flux;        /* numerical flux at edges: 0 the Roe flux of 2DCode/numericalFlux2D.c:6-108
                        (default); 1 the local Lax-Friedrichs flux of DG-SWEM
                        src/numerical_flux.F:887-1141; 2 DG-SWEM's HLLC flux (:1154-1400)
                        (extensions, for flows that stay wet).  Fixed at creation. */
} dgr_params;

/* Mesh in the reference's arrays (2DCode/MeshAttributes.h:5-20), 0-based. */
typedef struct dgr_mesh_view {
    int num_el, num_nodes, num_edges;
    const double *x_coord, *y_coord; /* [num_nodes] */
    const double *z;                 /* [num_nodes] depth, positive down */
    const double *nFriction;         /* [num_nodes] Manning n */
    const int *EltoVert;             /* [3*num_el] */
    const int *EdgtoEls;             /* [2*num_edges]; boundary edges repeat the element */
    const int *EdgtoVert;            /* [2*num_edges] */
    const int *BdryPrescribed;       /* [num_edges] 0 land, 1 inflow, 2 outflow, 3 inflow-2 */
    double minEdgLength;             /* 2DCode/extract_mesh_attributes.c:303 */
} dgr_mesh_view;

/* A mesh as read from a fort.14 file of the 2DCode dialect
 * (2DCode/extract_mesh_attributes.c:39-141): node lines carry "id x y z n". */
typedef struct dgr_fort14 {
    int num_el, num_nodes;
    double *x_coord, *y_coord, *z, *nFriction;
    int *EltoVert;                        /* 0-based */
    int num_inflow1, num_inflow2, num_outflow;
    int *inflow1, *inflow2, *outflow;     /* node pairs, 0-based, 2 per edge */
} dgr_fort14;

/* Forcing of one ensemble scenario (extensions: the reference has one mesh and no
 * time-dependent forcing).  n_el: per-element Manning n ([num_el], copied), or NULL for
 * the node average of 2DCode/2DInnerProducts.c:272-274. */
typedef struct dgr_scenario_params {
    double tide_amp, tide_period, rain;
    int tide_on;
    const double *n_el;
} dgr_scenario_params;

typedef struct dgr_ctx dgr_ctx;

DGR_API const char *dgr_status_string(int code);
DGR_API int dgr_abi_version(void);

/* ---- host-side mesh ingest (C, no GPU needed) ---------------------------------- */

/* store_mesh (2DCode/extract_mesh_attributes.c:39-141).  *out is freed by
 * dgr_fort14_free. */
DGR_API int dgr_read_fort14(const char *path, dgr_fort14 **out);
DGR_API void dgr_fort14_free(dgr_fort14 *m);

/* extract_mesh_attributes (2DCode/extract_mesh_attributes.c:143-361) with hashing
 * instead of the O(E*N) search; the outputs are identical, edge order and element slot
 * order included.  Output arrays hold num_nodes+num_el-1 edges (Euler's relation, which
 * the reference also requires, :218-257); DGR_ERR_MESH if the mesh breaks it.
 * Boundary lists are node pairs, 0-based. */
DGR_API int dgr_count_edges(int num_el, int num_nodes, const int *EltoVert, int *num_edges);
DGR_API int dgr_build_connectivity(int num_el, int num_nodes, const int *EltoVert,
                           const double *x_coord, const double *y_coord,
                           int num_inflow1, const int *inflow1,
                           int num_inflow2, const int *inflow2,
                           int num_outflow, const int *outflow,
                           int *EdgtoVert, int *EdgtoEls, int *BdryPrescribed,
                           double *minEdgLength);
/* The same arrays, bit for bit, built on the current CUDA device by sorting (mesh ingest on
 * the GPU; same arguments, host arrays in and out).  Every element must have three
 * distinct vertices (else DGR_ERR_MESH) and 6 x num_el must stay below 2^31. */
DGR_API int dgr_build_connectivity_device(int num_el, int num_nodes, const int *EltoVert, const double *x,
                                          const double *y, int n_inflow1, const int *inflow1, int n_inflow2,
                                          const int *inflow2, int n_outflow, const int *outflow, int *EdgtoVert,
                                          int *EdgtoEls, int *BdryPrescribed, double *minEdgLength);

/* initialize (2DCode/initialize.c:117-126): nodal elevations averaged onto the edge
 * midpoints, zero discharge, WD = -1.  zeta_nodal == NULL gives the reference's 0.1. */
DGR_API int dgr_initial_state(int num_el, const int *EltoVert, const double *zeta_nodal,
                      double *zeta, double *Qx, double *Qy, int *WD);

/* Writes one .dat file in the reference format (time_evolution.c:284-306,363-386):
 * one element per line, its three values as "%1.15f\t\t". */
DGR_API int dgr_write_dat(const char *path, int num_el, const double *values);

/* Restart files (resume a run where it stopped; the reference has none: 2DCode writes .dat
 * snapshots at FinalTime only, time_evolution.c:324-390).  Text in the .dat row layout —
 * one element per line, tab-separated — with each value printed with 17 significant
 * digits, so that reading it back gives the same bits (signed zeros included), the
 * element's wet/dry flag last on its line, and a header with the sizes and the clock
 * (time, and the dt of the next step).  nm = values per variable and element (3 at p = 1,
 * 6 at p = 2).  dgr_read_restart returns DGR_ERR_MESH for a file of another mesh size or
 * order and DGR_ERR_IO for a malformed one. */
DGR_API int dgr_write_restart(const char *path, int num_el, int nm, const double *zeta, const double *Qx,
                              const double *Qy, const int *WD, double time, double dt);
DGR_API int dgr_read_restart(const char *path, int num_el, int nm, double *zeta, double *Qx, double *Qy, int *WD,
                             double *time, double *dt);
/* The context's state, wet/dry flags and the given clock written to a restart file, and
 * read back into a context of the same mesh: a run continued from a loaded file (dgr_run
 * with the returned time and dt) is bit-identical to the run that never stopped. */
DGR_API int dgr_save_restart(dgr_ctx *ctx, const char *path, double time, double dt);
DGR_API int dgr_load_restart(dgr_ctx *ctx, const char *path, double *time, double *dt);

/* The context's current state as .dat files in the same format, formatted on the device
 * (the reference's snapshot writer, time_evolution.c:324-390, runs printf on the host):
 * zeta_path / qx_path / qy_path (any may be NULL) receive one element per line, its values
 * as "%1.15f\t\t", byte-identical to dgr_write_dat of the downloaded arrays.  At p = 2 a
 * line holds the element's six modal coefficients.  A value of magnitude >= 2^63 is not
 * formatted: DGR_ERR_INVALID, and that file is removed. */
DGR_API int dgr_write_state_dat(dgr_ctx *ctx, const char *zeta_path, const char *qx_path, const char *qy_path);
DGR_API int dgr_ensemble_write_state_dat(dgr_ctx *ctx, int scenario, const char *zeta_path, const char *qx_path,
                                         const char *qy_path);

/* Gauge time series recorded by the device loop (dgr_run / dgr_ensemble_run): after each
 * step, for gauge g in element gauge_el[g] (flattened numbering on an ensemble),
 * zeta_g = sum_k gauge_w[nm*g + k] zeta_k (nm = 3 midpoint values at p = 1, 6 modes at
 * p = 2) is stored in row (step - 1) of a device series [capacity][ngauges], step being the
 * gauge's scenario's step count in the current run; steps past capacity are not recorded.
 * ngauges = 0 removes the gauges.  The state never leaves the device for them. */
DGR_API int dgr_set_gauges(dgr_ctx *ctx, int ngauges, const int *gauge_el, const double *gauge_w, int capacity);
/* The recorded series [capacity][ngauges]: rows below the steps each scenario took in the
 * last run are that run's values. */
DGR_API int dgr_get_gauge_series(dgr_ctx *ctx, double *values);

/* Page-locked host memory for fast copies (cudaHostAlloc); NULL on failure. */
DGR_API void *dgr_host_alloc(size_t bytes);
DGR_API void dgr_host_free(void *p);

/* ---- device context ------------------------------------------------------------- */

DGR_API int dgr_params_default(dgr_params *p);
DGR_API int dgr_create(const dgr_mesh_view *mesh, const dgr_params *params, dgr_ctx **out);
DGR_API int dgr_destroy(dgr_ctx *ctx);
DGR_API int dgr_get_params(const dgr_ctx *ctx, dgr_params *out);
/* Only rain, tide_on, tide_amp, tide_period, cfl, dt0, record_decisions and rk_stages may
 * change. */
DGR_API int dgr_set_params(dgr_ctx *ctx, const dgr_params *params);
/* Per-element Manning n (extension); NULL restores the node average of
 * 2DCode/2DInnerProducts.c:272-274. */
DGR_API int dgr_set_element_manning(dgr_ctx *ctx, const double *n_el);

/* State in the reference layout.  Upload clears the error word and marks the wet/dry
 * flags stale, so the next step starts with wetDryStatus2D as the reference does. */
DGR_API int dgr_upload_state(dgr_ctx *ctx, const double *zeta, const double *Qx, const double *Qy,
                     const int *WD);
DGR_API int dgr_download_state(dgr_ctx *ctx, double *zeta, double *Qx, double *Qy, int *WD);

/* boundary_conditions(): the caller's bzeta/bQn arrays ([NumEdges], only prescribed
 * edges are read) ... */
DGR_API int dgr_set_boundary(dgr_ctx *ctx, const double *bzeta, const double *bQn);
/* ... or the device fills them for time t from the reference constants and the tide. */
DGR_API int dgr_boundary_conditions(dgr_ctx *ctx, double time);

/* Single operators on the device state, for drop-in use and parity checks. */
DGR_API int dgr_compute_L(dgr_ctx *ctx, double time, double *RHSZeta, double *RHSQx, double *RHSQy,
                  double *max_lambda);
DGR_API int dgr_slope_limiter(dgr_ctx *ctx);
DGR_API int dgr_pdop(dgr_ctx *ctx);
DGR_API int dgr_wet_dry_status(dgr_ctx *ctx);

/* oneTimeStep2D(time, dt): one SSP-RK2 step of the device state with the current
 * boundary values; returns the max wave speed of the second stage (the reference's
 * max_lambda), from which the caller sets the next dt.  The step's kernels are replayed
 * from a CUDA graph that the first call (and the first after dgr_set_params or
 * dgr_set_schedule) captures on the context's own stream. */
DGR_API int dgr_step(dgr_ctx *ctx, double time, double dt, double *max_lambda);

/* time_evolution(): up to nsteps steps while time < final_time, entirely on the device
 * (CFL dt, boundary forcing and clock stay on the GPU; one host sync at the end).
 * *time_io < 0 starts a new run at t = 0 with dt = dt0; otherwise (*time_io, *dt_io)
 * continue a previous run.  The steps of one call are replayed from a CUDA graph. */
DGR_API int dgr_run(dgr_ctx *ctx, int nsteps, double final_time, double *time_io, double *dt_io,
            int *steps_done);

/* ---- batched ensemble: many meshes advanced together ---------------------------- */

/* One context over nscen scenarios of uneven size.  The meshes are flattened into one
 * (disjoint union); every kernel launch advances all of them, each scenario with its own
 * CFL dt, clock, forcing, error word and results (identical to running it alone).
 * Single-mesh calls (dgr_step, dgr_upload_state, ...) require nscen == 1. */
DGR_API int dgr_ensemble_create(int nscen, const dgr_mesh_view *meshes, const dgr_scenario_params *sp,
                                const dgr_params *common, dgr_ctx **out);
DGR_API int dgr_ensemble_size(const dgr_ctx *ctx);
DGR_API int dgr_ensemble_upload_state(dgr_ctx *ctx, int scenario, const double *zeta, const double *Qx,
                                      const double *Qy, const int *WD);
DGR_API int dgr_ensemble_download_state(dgr_ctx *ctx, int scenario, double *zeta, double *Qx, double *Qy,
                                        int *WD);
/* All scenarios advance up to nsteps steps; arrays are [nscen]; time_io[s] < 0 starts
 * scenario s at t = 0 with dt0.  Returns the first scenario's failure code, if any
 * (per-scenario detail: dgr_ensemble_last_error). */
DGR_API int dgr_ensemble_run(dgr_ctx *ctx, int nsteps, const double *final_time, double *time_io,
                             double *dt_io, int *steps_done);
DGR_API int dgr_ensemble_last_error(dgr_ctx *ctx, int scenario, int *code, int *index, int *step);

/* Schedule of the device loop: block size (elements per block of the element and limiter
 * work: 64, the default, 128 or 256) and fusion depth (0, the default: ten kernels per
 * step; 1: one persistent cooperative kernel per RK stage; 2: one per step, clock
 * included).  dgr_autotune times
 * trial_steps steps of every schedule from the current state (restored afterwards),
 * keeps the fastest and reports it; ms_out (9 entries or NULL) gets ms per step at index
 * 3*b + f, b = 0,1,2 for 64,128,256.  Results do not depend on the schedule. */
DGR_API int dgr_set_schedule(dgr_ctx *ctx, int block_size, int fusion);
DGR_API int dgr_get_schedule(const dgr_ctx *ctx, int *block_size, int *fusion);
/* Bound of the persistent kernels' grid-barrier wait (fusion 1 and 2): a block that polls
 * max_polls times (default 2^24, about a second) gives up, every block leaves the launch
 * and the call returns DGR_ERR_TIMEOUT; the context stays usable.  No counterpart in the
 * reference, which has no device waits; it replaces the hang such a wait could cause by a
 * status, as the reference's failures (2DCode/compute2DL.c:245-302) become statuses here.
 * phantom_blocks = 1 makes every barrier also wait for a block that never arrives, so the
 * wait runs out on purpose: a test of the time-out path that faults nothing (0: normal). */
DGR_API int dgr_set_barrier_wait(dgr_ctx *ctx, unsigned max_polls, unsigned phantom_blocks);
DGR_API int dgr_autotune(dgr_ctx *ctx, int trial_steps, int *block_size, int *fusion, double *ms_out);

/* First failure since the last upload: status code, edge or element index, step. */
DGR_API int dgr_last_error(dgr_ctx *ctx, int *code, int *index, int *step);
DGR_API const char *dgr_last_cuda_error(void);

/* Per-element decisions of the last step (needs record_decisions = 1).  stage 0 .. rk_stages-1.
 * limit[el] = 1 when the limiter rewrote the element; pdop[el] = 4*mass + momentum
 * branch (see oracle/dgr_oracle.h for the branch numbering). */
DGR_API int dgr_get_decisions(dgr_ctx *ctx, int stage, int *limit, int *pdop);
/* Numerical fluxes of the last L evaluation in the reference's Fhat{1,2,3}dotn layout. */
DGR_API int dgr_get_fhat(dgr_ctx *ctx, double *F1, double *F2, double *F3);

/* Number of kernels this context has launched since creation (all launches, graph
 * replays included). */
DGR_API long long dgr_kernel_launches(const dgr_ctx *ctx);
/* Device time of the last dgr_run/dgr_step call in ms (CUDA events on the context's
 * stream). */
DGR_API double dgr_last_device_ms(const dgr_ctx *ctx);
/* Runs nsteps steps with CUDA events around every launch; kernel_ms[0..3] (n >= 4)
 * receive the average ms of one launch of: edge flux, element RHS + RK update, node
 * bounds, limiter + PDop. */
DGR_API int dgr_profile_step(dgr_ctx *ctx, int nsteps, double *kernel_ms, int n);

/* Slope limiter without any device allocation.  This entry point has no counterpart in
 * the reference.  It is for callers that may not allocate device memory: code handed its
 * buffers by a host framework or memory pool, or code running where cudaMalloc/cudaFree
 * are not allowed (cudaFree synchronises the device; allocating inside a stream capture
 * is an error).  They pass their own device arrays in the reference layout —
 * EltoVert[3*num_el], node depth z[num_nodes], zeta/Qx/Qy[3*num_el] limited in place —
 * and a cudaStream_t (NULL = default stream).  Every array must be memory a kernel on the
 * current device may use (that device's own memory, managed, or mapped pinned host
 * memory); anything else is refused with DGR_ERR_INVALID before any launch.  The result
 * equals dgr_slope_limiter's bit for bit, signed zeros included.  Scratch is a static
 * device array for at most DGR_NOALLOC_MAX_NODES nodes (7.5 MiB, held on every GPU that
 * loads this library until the process exits); larger meshes get DGR_ERR_TOO_LARGE.
 * All calls share that array, so calls that overlap on the GPU race.  The first call on
 * a device looks up the array's address and should come before any stream capture; the
 * address is kept for the life of the process, so the entry point must not be used on a
 * device after a cudaDeviceReset.  The call only enqueues work on the stream. */
#define DGR_NOALLOC_MAX_NODES 131072
DGR_API int dgr_slope_limiter_noalloc(int num_el, int num_nodes, const int *d_EltoVert, const double *d_z,
                                      double *d_zeta, double *d_Qx, double *d_Qy, double H0, void *stream);

/* ---- discrete adjoint and tangent-linear model (one mesh or an ensemble) ----------
 * Extension: the reference has no derivatives.  Objective over a run of nsteps steps:
 *   J = sum_n sum_g (zeta_g(u^{n+1}) - target[n*ngauges + g])^2,
 *   zeta_g(u) = sum_k w[nm*g + k] zeta_k of element gauge_el[g]
 * with nm = 3 at p = 1 (midpoint values; the Crouzeix-Raviart interpolation at a point is
 * such a functional) and nm = 6 at p = 2 (modes; the basis at the point).
 * Derivatives are those of the discrete scheme with every decision (wet/dry flags,
 * limiter clamps and redistribution, PDop branches, entropy-fix selections, node max/min
 * elements) and the CFL dt sequence frozen at the recorded forward run.  Parameters: the
 * per-element Manning n (dgr_set_element_manning; required for its gradient), the node
 * depth z (dgr_set_bathymetry, single mesh) and the initial state.
 * On an ensemble context every scenario runs nsteps steps with its own dt; element and
 * node indices, states and gradients use the flattened numbering (scenario s's element i
 * is the sum of the earlier scenarios' element counts plus i; nodes likewise) and J sums
 * over all scenarios' gauges. */

/* Allocates the adjoint storage: a checkpoint every ckpt_every steps plus a recompute
 * store of ckpt_every steps (about 390 B per element and step at p = 1 with RK2, 144 B per
 * element and stage at p = 2); target may be NULL (0). */
DGR_API int dgr_adjoint_setup(dgr_ctx *ctx, int nsteps, int ckpt_every, int ngauges, const int *gauge_el,
                              const double *gauge_w, const double *target);
DGR_API int dgr_adjoint_set_target(dgr_ctx *ctx, const double *target);
/* Forward run from the given state (reference layout; time < 0 starts at t = 0 with dt0)
 * with checkpoints; its steps are dgr_run's bit for bit.  replay_dt = 1 reuses the dt
 * sequence of the previous forward run instead of the CFL dt (finite differences with
 * frozen dt).  J and the gauge values [nsteps*ngauges] (NULL to skip) on return. */
DGR_API int dgr_adjoint_forward(dgr_ctx *ctx, const double *zeta, const double *Qx, const double *Qy,
                                const int *WD, double time, double dt, int replay_dt, double *J,
                                double *gauge_values);
/* Gradient of J of the last forward run: per-element n [num_el], node depth [num_nodes],
 * initial state (reference layout); any output may be NULL.  The context's state is
 * unspecified afterwards. */
DGR_API int dgr_adjoint_backward(dgr_ctx *ctx, double *grad_n_el, double *grad_z, double *grad_zeta0,
                                 double *grad_Qx0, double *grad_Qy0);
/* Tangent-linear run over the recorded dt sequence: J and dJ = J'(p) . (dn_el, dz, d state)
 * for the given directions (any may be NULL = 0). */
DGR_API int dgr_tlm(dgr_ctx *ctx, const double *zeta, const double *Qx, const double *Qy, const int *WD,
                    const double *dzeta0, const double *dQx0, const double *dQy0, const double *dn_el,
                    const double *dz, double *J, double *dJ);
/* The recorded run at a perturbed point (state *_p, per-element n n_el_p, node depths z_p;
 * NULL = unperturbed) with every decision and the dt sequence frozen at the recorded run's:
 * J of the base point and J_p of the perturbed one.  Central differences of J_p are
 * "finite differences with frozen masks and dt", the derivative the adjoint computes. */
DGR_API int dgr_fd_frozen(dgr_ctx *ctx, const double *zeta, const double *Qx, const double *Qy, const int *WD,
                          const double *zeta_p, const double *Qx_p, const double *Qy_p, const double *n_el_p,
                          const double *z_p, double *J, double *J_p);
/* dt and boundary-value time of every step of the last forward run [nsteps][scenarios]. */
DGR_API int dgr_adjoint_dt(dgr_ctx *ctx, double *dt, double *time);
/* Device time in ms of the last forward, backward and tangent-linear runs. */
DGR_API int dgr_adjoint_timing(const dgr_ctx *ctx, double *forward_ms, double *backward_ms, double *tlm_ms);
/* Node depths z [num_nodes] (the fort.14 depth column): recomputes every depth-dependent
 * factor on the device. */
DGR_API int dgr_set_bathymetry(dgr_ctx *ctx, const double *z);

/* Reference-element tables of the p = 2 step, for projecting fields onto and evaluating
 * them from the modal coefficients (n >= 234 doubles; no GPU needed):
 *   [0..6]      area-rule weights (sum 1)      [7..27]     barycentric coordinates [7][3]
 *   [28..69]    basis at the area points [7][6] [70..111]   d/dr [7][6]   [112..153] d/ds [7][6]
 *   [154..156]  Gauss points on [-1, 1]        [157..159]  Gauss weights
 *   [160..213]  basis at the Gauss points of local edge k [3][3][6]   [214..219] int phi_m^2
 *   [220..233]  reference coordinates (r, s) of the 7 area points [7][2]. */
DGR_API int dgr_p2_reference(double *tables, int n);

/* ---- channel <-> junction coupling (ChanNet/internal_BC.c:17-218) ----------------
 * This context's mesh is a ChanNet junction; 1D channels attach to its prescribed boundary
 * edges.  A channel END is the first node of a channel (the reference's
 * InflowJunctionEdges list, end_outflow = 0) or its last node (OutflowJunctionEdges,
 * end_outflow = 1); end k owns the mesh edges end_edges[end_ptr[k] .. end_ptr[k+1]) in the
 * order of the reference's list.  Each edge must be a prescribed boundary edge
 * (BdryPrescribed != 0) and belong to one end; each end has at least one edge.  One
 * context (not an ensemble), order 1.  Replaces the channel lists of
 * ChanNet/ChannelsAndJunctions.h:47-66 (struct channel) for the junction's side. */
DGR_API int dgr_set_channel_ends(dgr_ctx *ctx, int nends, const int *end_ptr, const int *end_edges,
                                 const int *end_outflow);

/* One coupling pass, internal_BC() for this junction (host arrays of nends):
 *   in:  a_end[k], q_end[k]: the channel's own trace A, Q at the junction node (the
 *        reference's A[1], Q[1] for an inflow end; A[2N-2], Q[2N-2] for an outflow end);
 *   out: the ends' edges get bzeta = a_end / (n len) - z_mid and bQn = +-q_end / (n len)
 *        on the device (read by the next dgr_step, as the reference's junction step reads
 *        junc->bzeta / bQn), and a_ghost[k], q_ghost[k] = the junction's sums over the
 *        end's edges of len * (zeta + z_mid) and +-len * (Qx nx + Qy ny) from the current
 *        state (the reference's A[0], Q[0] or A[2N-1], Q[2N-1]).
 * The reference's loop calls it after the channels' step and again after the junction's
 * (ChanNet/time_evolution.c:552-578).  Results are those of internal_BC bit for bit.
 * A coupled junction is stepped with dgr_step: the device clock of dgr_run rewrites every
 * prescribed edge's values each step from its boundary type (boundary_conditions()). */
DGR_API int dgr_couple_channel_ends(dgr_ctx *ctx, const double *a_end, const double *q_end, double *a_ghost,
                                    double *q_ghost);

/* The same pass with the ends' traces and ghosts in DEVICE arrays (nends doubles each),
 * enqueued on the context's stream without synchronising: for channel states that stay on
 * the GPU.  The caller orders its own work on those arrays with that stream.  Device,
 * managed and pinned host memory are accepted; pageable host memory is refused
 * (DGR_ERR_INVALID) before anything is launched. */
DGR_API int dgr_couple_channel_ends_device(dgr_ctx *ctx, const double *d_a_end, const double *d_q_end,
                                           double *d_a_ghost, double *d_q_ghost);

/* The context's CUDA stream (a cudaStream_t), for callers that order their own device
 * work against the context's (e.g. around dgr_couple_channel_ends_device). */
DGR_API int dgr_get_stream(dgr_ctx *ctx, void **stream);

/* The device's prescribed boundary values bzeta[e], bQn[e] for every edge (reference edge
 * numbering; only prescribed edges are meaningful). */
DGR_API int dgr_get_boundary(dgr_ctx *ctx, double *bzeta, double *bQn);

/* Diagnostic: y[i] = x[i]^(4./3) as the kernels evaluate the Manning term of
 * 2DCode/2DInnerProducts.c:318 (correctly rounded; see dgr_device.cuh). */
DGR_API int dgr_pow43_batch(const double *x, double *y, int n, int device);
/* Diagnostic: q[i] = a[i] / b[i] as the element kernel takes its divisions by the fit
 * determinant (one reciprocal per divisor and Markstein's correction, dgr_device.cuh:
 * div_rcp), valid[i] = 1 where that path applies (elsewhere the kernel uses the plain
 * division).  Where valid, q equals the IEEE quotient bit for bit. */
DGR_API int dgr_div_rcp_batch(const double *a, const double *b, double *q, int *valid, int n, int device);

#ifdef __cplusplus
}
#endif

#endif
