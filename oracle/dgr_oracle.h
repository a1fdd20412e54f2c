/*
 * ORACLE — test infrastructure only.  A CPU restatement, in plain C, of the reference
 * DG-RAIN 2D shallow-water step (2DCode/).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it, and only as the checker.  The product never
 * calls it.
 *
 * Parity pin: tests/test_oracle_pin.py checks every function here bit for bit against
 * the UNMODIFIED reference sources compiled by oracle/Makefile (oracle/_ref), and
 * against golden vectors that the same reference build wrote (tests/golden/).
 *
 * Unlike the reference, which keeps one mesh in process-wide globals
 * (2DCode/MeshAttributes.h:5-42), the restatement works on a context, so a test can
 * hold several meshes.  It also returns failures as status codes instead of exit(),
 * and it records the per-element decisions (limiter gate, positive-depth branches) that
 * the reference keeps in local variables, so the GPU's decisions can be compared.
 *
 * Extensions with no reference counterpart (parity unpinned, they reduce to the
 * reference when switched off): rain added to the elevation right-hand side, a
 * per-element Manning n, and the tide on type-2 edges (dg-rain_b200/csrc/dgr_forcing.h).
 */
#ifndef DGR_ORACLE_H
#define DGR_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* Status codes, identical to the DGR_ERR_* codes of include/dgrain.h. */
enum {
    ORC_OK = 0,
    ORC_ERR_NAN_FLUX = 1,     /* wet (or WD-off) flux NaN: 2DCode/compute2DL.c:245-249, :298-302 */
    ORC_ERR_NAN_FLUX_IN = 2,  /* dry interior flux NaN: :262-266 */
    ORC_ERR_NAN_FLUX_EX = 3,  /* dry exterior flux NaN: :281-285 */
    ORC_ERR_NEG_DEPTH = 4,    /* PDop height NaN: 2DCode/wetDry2D.c:142-146 */
    ORC_ERR_NAN_VELOCITY = 5, /* PDop velocity NaN: 2DCode/wetDry2D.c:233-237 */
    ORC_ERR_EDGE_MATCH = 6    /* local edge not found: 2DCode/compute2DL.c:51-67 */
};

orc_ctx *orc_create(int num_el, int num_nodes, int num_edges, const double *x, const double *y,
                    const double *z, const double *nfric, const int *el2v, const int *ed2el,
                    const int *ed2v, const int *bdry, double min_edge_length);
void orc_destroy(orc_ctx *c);

/* g, H0, VELZERO (2DCode/initialize.c:22,26-27 by default). */
void orc_set_constants(orc_ctx *c, double g, double h0, double velzero);
/* Per-element Manning n (NULL restores the node average of 2DCode/2DInnerProducts.c:272-274). */
void orc_set_element_manning(orc_ctx *c, const double *n_el);

void orc_set_state(orc_ctx *c, const double *zeta, const double *qx, const double *qy, const int *wd);
void orc_get_state(const orc_ctx *c, double *zeta, double *qx, double *qy, int *wd);
void orc_set_bc(orc_ctx *c, const double *bzeta, const double *bqn);
void orc_get_bc(const orc_ctx *c, double *bzeta, double *bqn);
void orc_get_rhs(const orc_ctx *c, double *rz, double *rqx, double *rqy);
void orc_get_fhat(const orc_ctx *c, double *f1, double *f2, double *f3);
double orc_max_lambda(const orc_ctx *c);
void orc_last_error(const orc_ctx *c, int *code, int *index);

/* Reference initial state of 2DCode/initialize.c:117-126 from given nodal elevations
 * (zeta_nodal == NULL means the reference's constant 0.1). */
void orc_initial_state(orc_ctx *c, const double *zeta_nodal);

/* Per-element decisions of the last limiter / PDop call.
 * limit[el] = 1 when the limiter rewrote the element (the 'modify' gate of
 * 2DCode/SlopeLimiter2D.c:166-200,310-311).
 * pdop[el] = 4*mass_branch + momentum_branch; mass_branch 0 none, 1 flattened to the
 * mean, 2 lifted the lowest vertex (2DCode/wetDry2D.c:93-139); momentum_branch 0 none,
 * 1 zeroed, 2 redistributed (:170-253). */
void orc_get_decisions(const orc_ctx *c, int *limit, int *pdop);

/* Single operators (same names and meaning as the reference functions). */
int orc_boundary_conditions(orc_ctx *c, double t, int tide_on, double amp, double period);
int orc_compute_L(orc_ctx *c, int wet_dry, double rain);
int orc_slope_limiter(orc_ctx *c);
int orc_pdop(orc_ctx *c);
void orc_wd_status(orc_ctx *c);
double orc_roe_flux(double *fhat3, double zeta_in, double zeta_ex, double qx_in, double qx_ex,
                    double qy_in, double qy_ex, double z_edge, double nx, double ny, double local_g,
                    double g);
void orc_inner_products(const orc_ctx *c, int el, double si[9], double vi[21]);

/* One SSP-RK2 step (2DCode/time_evolution.c:10-246; wet/dry calls in the order of
 * ChanNet/time_evolution.c:218-427 when wet_dry != 0).  Decisions of stage s (0 or 1)
 * are written to limit_s/pdop_s when those pointers are given. */
int orc_step(orc_ctx *c, double time, double dt, int wet_dry, double rain, int *limit0,
             int *pdop0, int *limit1, int *pdop1);

/* One SSP(3,3) step (extension; DG-SWEM src/prep_DG.F:1253-1270 coefficients). */
int orc_step3(orc_ctx *c, double time, double dt, int wet_dry, double rain);

/* orc_run with stages = 2 (SSP-RK2) or 3 (SSP(3,3)). */
int orc_run_rk(orc_ctx *c, int nsteps, double final_time, double cfl, double dt0, int wet_dry,
               double rain, int tide_on, double amp, double period, double *time_io, double *dt_io,
               double *dt_hist, int *steps_done, int stages);

/* Time loop of 2DCode/time_evolution.c:248-402 (no file output); see ref_run in
 * oracle/ref_driver.c for the clock convention. */
int orc_run(orc_ctx *c, int nsteps, double final_time, double cfl, double dt0, int wet_dry,
            double rain, int tide_on, double amp, double period, double *time_io, double *dt_io,
            double *dt_hist, int *steps_done);

/* Channel <-> junction coupling of ChanNet/internal_BC.c:17-218 on one junction mesh
 * (reference arrays: el2v [3*ne], ed2v / ed2el [2*nf], state [3*el+k]).  Channel ch has
 * chan_nodes[ch] nodes and its A, Q traces at [2*chan_off[ch], 2*chan_off[ch] + 2*nodes);
 * its inflow-end edges are in_edges[in_ptr[ch] .. in_ptr[ch+1]), its outflow-end edges
 * out_edges[out_ptr[ch] ..].  Writes bzeta / bqn of those edges and the channels' ghost
 * traces A/Q[0] (inflow) and A/Q[2*nodes-1] (outflow).  -1 on a bad edge. */
int orc_internal_bc(int ne, int nf, const double *x, const double *y, const double *z, const int *el2v,
                    const int *ed2v, const int *ed2el, const double *zeta, const double *qx, const double *qy,
                    double *bzeta, double *bqn, int nchan, const int *in_ptr, const int *in_edges,
                    const int *out_ptr, const int *out_edges, const int *chan_nodes, const int *chan_off,
                    double *A, double *Q);

#ifdef __cplusplus
}
#endif

#endif
