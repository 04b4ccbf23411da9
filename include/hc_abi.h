/*
 * hc_abi.h -- C ABI of the B200-native HelioCubed per-box MHD update.
 *
 * Every entry point returns an int status (HC_OK or a negative HC_ERR_*),
 * never throws, and takes plain pointers and sizes.  Device buffers are
 * caller-owned CUDA device pointers; `stream` is a cudaStream_t passed as
 * void* (NULL = legacy default stream).  One host thread per context.
 *
 * Data layout (identical to Proto BoxData<double,8> as used by the
 * reference): component-major SoA, radial index fastest,
 *   offset(c,i,j,k) = c*N + (i-lo0) + n0*((j-lo1) + n1*(k-lo2)),
 * over the storage box of the array.  Components are
 *   conserved  JU : rho, m_x, m_y, m_z, E, B_x, B_y, B_z  (Cartesian, times J)
 *   primitive  W  : rho, v_x, v_y, v_z, p, B_x, B_y, B_z  (Cartesian)
 * exactly as src/BoxOp_EulerCubedSphere.H:39-51 and src/MHD_AMR.H:99-101.
 *
 * A "level" is the six-panel cubed-sphere shell with one box per panel
 * (nr radial x na x na angular cells); level arrays hold the six boxes
 * back to back (box b = panel b), valid cells only unless stated.
 */
#ifndef HC_ABI_H
#define HC_ABI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HC_NUMCOMPS 8
#define HC_NPANELS 6

enum {
  HC_OK = 0,
  HC_ERR_ARG = -1,          /* bad argument (size, pointer, option value) */
  HC_ERR_CUDA = -2,         /* a CUDA runtime call failed */
  HC_ERR_UNSUPPORTED = -3,  /* option combination not built */
  HC_ERR_INVALID_STATE = -4,/* non-finite or non-positive-density cell */
  HC_ERR_NOMEM = -5
};

/* Option semantics mirror src/Inputs_Parsing.H:43-178 (ParseInputs). */
typedef struct hc_params {
  int spatial_order;        /* 2: PLM operator (src/BoxOp_SecondOrder.H); 4: Berta WENOZ */
  int limiter;              /* 0 unlimited, 1|2 minmod, 3 MC (Inputs_Parsing.H:71) */
  int riemann_solver;       /* 1 Rusanov, 2 Roe 8-wave (Inputs_Parsing.H:79) */
  int divergence_cleaning;  /* 1: Powell source (Inputs_Parsing.H:118) */
  int sun_gravity;          /* 1: solar gravity source (Inputs_Parsing.H:175) */
  int init_condition_type;  /* radial BC family; 1 = analytic wind (BoxOp_PreStage.H:7-47) */
  int temporal_order;       /* 4: classical RK4 (MHD_AMRRungeKutta.H:10-12) */
  int nr, na;               /* level cells per panel: radial, angular */
  int spatial_operator;     /* at order 4: 2 = Berta WENOZ (Inputs_Parsing.H:78) */
  int berta_detector_type;  /* 0 Jameson (Inputs_Parsing.H:82-84) */
  int berta_fallback_type;  /* 0 WENO3, 1 PLM (theta = 1.5 minmod3) */
  int autotune;             /* 1: time the order-2 stage tiles on the first level step (hc_ctx_autotune) */
  /* A radial slab of a larger shell: the level holds global radial cells
   * [radial_offset, radial_offset + nr) of a shell of radial_cells cells;
   * radial metrics and spacing are the shell's (0 = the level is the whole
   * shell).  The reference spreads its boxes over ranks (Proto's
   * DisjointBoxLayout); here a rank owns a radial range of all six panels
   * and receives its halo layers from its neighbours every stage. */
  int radial_offset;
  int radial_cells;
  int reserved_i[1];
  double gamma;             /* ratio of specific heats */
  double entropy_fix_coeff; /* Roe entropy fix, default 0.3 */
  double cfl;               /* dt = cfl / max(inverse dt) */
  double inner_radius;      /* cm */
  double outer_radius;      /* cm */
  double radial_stretch;    /* C in r = r0 + R_t expm1(C eta) (BoxOp_Utilities.H:36-46) */
  double strength;          /* analytic-wind perturbation strength (percent) */
  double berta_eta_d;       /* Jameson threshold, default 0.02 */
  double reserved_d[6];
} hc_params;

/* One box of a panel in panel index space (inclusive bounds), the ghost
 * width of its primitive storage and the panel (Proto block) it lies on. */
typedef struct hc_box {
  int lo[3];
  int hi[3];
  int ghost;
  int block;
} hc_box;

/* Seeded synthetic initial states (the configs' own inputs; the reference
 * defines no such problem).  kind 1: Parker-like wind + Gaussian pressure
 * pulse.  With s = r_ref / r at the cell-centre radius and X the cell-centre
 * unit direction: rho = rho0 s^2, v = vr X, p = p0 s^(2 gamma) (1 + amp
 * exp(-d^2 / (2 w^2))), B = b0 s^2 sign(X_z) X; d^2 = (i - pulse_i)^2 +
 * (angle to the pulse cell's direction / angular cell width)^2.  JU = J U
 * with J = dVolr <det A> of the cell. */
typedef struct hc_init {
  int kind;
  int pulse_block, pulse_i, pulse_j, pulse_k;
  int reserved_i[3];
  double rho0, p0, vr, b0, r_ref;   /* r_ref: radius where rho0/p0/b0 hold (cm) */
  double pulse_amp, pulse_width;    /* delta p = amp*p*exp(-d^2/(2 w^2)), d in cells */
  double reserved_d[4];
} hc_init;

typedef struct hc_ctx hc_ctx;

/* Last error message of the calling thread ("" if none). */
const char* hc_last_error(void);

/* Create a context on CUDA device `device`: validates options, builds the
 * level geometry (the metric caches the reference keeps in statics,
 * src/BoxOp_EulerCubedSphere.H:348-368) and its stage workspace.
 * Replaces BoxOp_EulerCubedSphere::levelGeometry + ParseInputs. */
int hc_ctx_create(const hc_params* params, int device, hc_ctx** out);
int hc_ctx_destroy(hc_ctx* ctx);

/* Number of doubles in one level array of valid cells (6*8*nr*na*na) and of
 * one ghosted level primitive array (6*8*(nr+4)*(na+4)^2). */
size_t hc_level_state_size(const hc_ctx* ctx);
size_t hc_level_primitive_size(const hc_ctx* ctx);

/* Per-box operator, second-order path with Cartesian primitives.
 * Replaces BoxOp_EulerCubedSphere::operator()(rhs, fluxes, W, dt, scale,
 * counter, cartesianPrimitives=true) (src/BoxOp_EulerCubedSphere.H:412-421,
 * body src/BoxOp_SecondOrder.H:155-370):
 *   rhs[valid]      += -scale * sum_d (F_d(i+1)-F_d(i))/dxi_d + Powell source
 *   flux[d][faces]   = F_d on valid.extrude(d) (overwritten; may be NULL)
 * w: primitives on valid.grow(ghost) (ghost >= 2).  panel_states[2d+side]
 * (d in {1,2}, may be NULL): reconstructed adjacent-panel states on the
 * seam face slab valid.extrude(d).face(d,side), 8 comps SoA, replacing the
 * local left (side 0) / right (side 1) state there
 * (src/BoxOp_SecondOrder.H:252-281). */
int hc_box_rhs(hc_ctx* ctx, const hc_box* box, const double* w,
               const double* const* panel_states, double scale,
               double* rhs, double* const* flux, void* stream);

/* Per-box fourth-order Berta pointwise-WENOZ operator (context created with
 * spatial_order 4, spatial_operator 2).  Replaces
 * BoxOp_EulerCubedSphere::operator() -> BertaOperator
 * (src/BoxOp_BertaCubedSphereImplem.H:1737-2076):
 *   rhs[valid]    += -scale * sum_d (F_d(i+1)-F_d(i))/dxi_d + Powell source
 *   flux[d][faces] = F_d on valid.extrude(d) (overwritten; may be NULL)
 * usph: native-basis conserved cell averages on valid.grow(ghost), ghost >= 5
 * (NGHOST, src/BoxOp_EulerCubedSphere.H:386-389).  Uses context scratch that
 * grows on first use of a larger box (a cudaMalloc: not inside a capture). */
int hc_box_rhs_o4(hc_ctx* ctx, const hc_box* box, const double* usph,
                  double scale, double* rhs, double* const* flux,
                  void* stream);

/* Solar gravity on second-order primitives, rhs[valid] += source.
 * Replaces gravitySecondOrderPrimitives (src/BoxOp_Gravity.H:3-82). */
int hc_box_gravity(hc_ctx* ctx, const hc_box* box, const double* w,
                   double* rhs, void* stream);

/* One box of a fourth-order operator batch: the box (ghost >= 5), its
 * native averages on valid.grow(ghost), its rhs on valid (accumulated) and
 * optional face fluxes on valid.extrude(d) (overwritten; NULL to skip). */
typedef struct hc_box_work {
  hc_box box;
  const double* usph;
  double* rhs;
  double* flux[3];
} hc_box_work;

typedef struct hc_o4_batch hc_o4_batch;

/* A batch of boxes of any sizes on this context's level (spatial_order 4):
 * allocates every box's operator scratch and builds the per-box kernel
 * contexts in device memory, once.  The arrays of `boxes` must stay
 * allocated while the batch lives.  Replaces the per-patch loop of the AMR
 * level evaluation (GridLevel::evaluate, src/MHD_AMR.H:1417-1499), which
 * calls the operator once per patch. */
int hc_o4_batch_create(hc_ctx* ctx, const hc_box_work* boxes, int nbox,
                       double scale, hc_o4_batch** out);

/* Evaluate every box of the batch: gravity (Gravity_Euler, when the context
 * has sun_gravity) and the Berta operator, each operator kernel one launch
 * over all boxes.  No allocation, no host synchronisation: may be captured
 * in a CUDA graph. */
int hc_o4_batch_rhs(hc_ctx* ctx, hc_o4_batch* batch, void* stream);

int hc_o4_batch_destroy(hc_o4_batch* batch);

/* An ensemble: several fourth-order levels (contexts of any sizes sharing
 * the Riemann solver, Powell, gravity and WENO fallback settings) advanced
 * together, one CFL step each per call step.  Each level keeps its own
 * state, dt, model time, insertion schedule and seam register; the stage
 * operator of all levels' panels is one batch, so every operator kernel is
 * one launch for the ensemble.  The results equal those of
 * hc_level_advance_cfl on each level alone, bit for bit.  The member
 * contexts must outlive the ensemble and must not step on their own while
 * it runs (they share their stage buffers with it).  Replaces running the
 * reference's per-solve step loop (exec/main.cpp:369-497) once per served
 * request; the reference has no ensemble batching. */
typedef struct hc_ensemble hc_ensemble;

int hc_ensemble_create(hc_ctx* const* members, int m, hc_ensemble** out);

/* nsteps steps of every member: ju[q] is member q's state; time_dev[q] and
 * dt_dev[q] as in hc_level_advance_cfl (time_dev and dt_dev may be NULL,
 * or hold NULL entries).  No host synchronisation, no allocation: may be
 * captured in a CUDA graph. */
int hc_ensemble_advance_cfl(hc_ensemble* ens, double* const* ju, int nsteps,
                            double* const* time_dev, double* const* dt_dev,
                            void* stream);

int hc_ensemble_destroy(hc_ensemble* ens);

/* Solar gravity at fourth order on native averages, rhs[valid] += source
 * (fourth-order cell and face products of dr/dxi, <rho>, <rho V_r> and the
 * averaged metrics; context created with spatial_order 4).  usph lives on
 * valid.grow(ghost), ghost >= 1.  Replaces Gravity_Euler
 * (src/BoxOp_Gravity.H:84-164). */
int hc_box_gravity_o4(hc_ctx* ctx, const hc_box* box, const double* usph,
                      double* rhs, void* stream);

/* Stage preparation of a level at time t; w holds hc_level_primitive_size
 * doubles.  Order 2: JU (valid) -> ghosted Cartesian primitives [6][8]
 * [na+4][na+4][nr+4] with panel-seam ghosts, floors and radial boundary
 * ghosts; replaces preStageLevel -> prepareSecondOrderPrimitives
 * (src/BoxOp_PreStage.H:434-501, src/BoxOp_SecondOrderPreStage.H:7-218).
 * Order 4: JU -> native conserved averages USph [6][8][na+10][na+10][nr+10]
 * by the Cartesian state conversion with seam ghosts (panel corners
 * included) and radial boundary ghosts; replaces preStageLevel ->
 * consToSphInterpEulerCartesian + fillRadialBoundaries
 * (src/MHD_StateConversion.H:153-316, src/BoxOp_SeamPressure.H:5-34). */
int hc_level_prepare(hc_ctx* ctx, const double* ju, double* w, double t,
                     void* stream);

/* Stage right-hand side of a level: k = gravity + L(w) (order 2: with
 * shared panel seam states; order 4: the Berta operator on each panel,
 * Gravity_Euler when sun_gravity).  Replaces the zero/gravity part of
 * preStageLevel plus StageLevel (src/BoxOp_EulerCubedSphereImplem.H:961-1012). */
int hc_level_rhs(hc_ctx* ctx, const double* w, double* k, void* stream);

/* The AMR form of a fourth-order level's stage preparation and evaluation
 * (CubedSphereAMR::prepare and evaluate on a level that covers the shell,
 * src/MHD_AMR.H:1417-1499):
 *
 * hc_level_prepare_cartesian is hc_level_prepare that also keeps the
 * level's fourth-order Cartesian averages (with their panel-seam ghosts) in
 * the caller's cart, hc_level_cartesian_size doubles: [6][8][na+12][na+12]
 * [nr], panel b's box (0, -6, -6) .. (nr-1, na+5, na+5), the coarse data a
 * finer level interpolates its ghosts from.
 *
 * hc_level_rhs_fluxes is hc_level_rhs evaluated as the AMR level
 * evaluation does it: every panel-seam face of k takes the mean of both
 * panels' fluxes at once (the per-stage panel flux register reflux), and
 * flux[d] (each may be NULL), [6][8][faces of valid.extrude(d)], receives
 * every panel's own face fluxes for the coarse-fine registers. */
size_t hc_level_cartesian_size(const hc_ctx* ctx);
int hc_level_prepare_cartesian(hc_ctx* ctx, const double* ju, double* w,
                               double* cart, double t, void* stream);
int hc_level_rhs_fluxes(hc_ctx* ctx, const double* w, double* k,
                        double* const* flux, void* stream);

/* One classical RK4 step of the level in place, with dt from host.
 * Replaces MBLevelRK::advance(order 4) (src/MHD_LevelRK.H:22-61, tableau
 * src/MHD_AMRRungeKutta.H:10-12).  At spatial order 4 the panel-seam
 * fluxes are reconciled after the step from the time-integrated flux
 * register: each side takes the mean of both sides (src/MHD_AMR.H:1478-1497). */
int hc_level_rk4_step(hc_ctx* ctx, double* ju, double dt, double t,
                      void* stream);

/* Stage `stage` (0..3) of hc_level_rk4_step, for callers that act between
 * stages: a radial slab receives its halo layers from the ranks next to it
 * there, where each stage's preparation exchanges the ghost cells of the
 * stage primitives between boxes and ranks (src/BoxOp_SecondOrderPreStage.H:55).
 * Stages 0, 1, 2, 3 called in order with the same
 * ju, dt and t launch exactly the kernels of hc_level_rk4_step; stage 3
 * writes the new state into ju (and at order 4 reconciles the panel seams).
 * With inv_dt_max (device) dt = cfl / *inv_dt_max; with time_dev (device)
 * the stage time is t + *time_dev + c_s dt.
 * hc_level_stage_state returns the buffer that stage `stage` reads and may
 * be overwritten between stages: `rows` rows of `row_length` doubles, radial
 * index fastest, the level's radial cell i at row offset first + i.  Stage
 * 0 reads ju itself; later stages read the context's stage state (order 4,
 * level layout) or stage primitives (order 2, ghosted layout; their ghosts
 * are refilled by the stage). */
int hc_level_rk4_stage(hc_ctx* ctx, double* ju, int stage, double dt, double t,
                       const double* inv_dt_max, const double* time_dev,
                       void* stream);
int hc_level_stage_state(hc_ctx* ctx, double* ju, int stage, double** data,
                         long* rows, int* row_length, int* first);

/* Order 4: the RK4 stages of this context (hc_level_rk4_step,
 * hc_level_rk4_stage, hc_level_advance_cfl) evaluate the operator on the
 * radial cells [lo, hi) only; every other cell's stage rhs is zero.  The
 * stage preparation still covers the whole level, so a slab whose halo
 * layers hold its neighbours' cells computes its own cells exactly and
 * spends no operator work on the halo.  (0, 0) restores the whole level.
 * Changing the window waits for the device (it rebuilds the operator's
 * work lists): not inside a stream capture. */
int hc_level_set_radial_window(hc_ctx* ctx, int lo, int hi);

/* hc_level_rk4_step without any device allocation by the library: for
 * callers that cannot call cudaMalloc while they step (inside a stream
 * capture, under a host framework that owns all device memory, in a serving
 * loop that must not wait on the allocator).  Its stage workspace is one
 * fixed 16 MiB device array inside the library (levels up to 6 x 21 x 21^2
 * cells; larger levels return HC_ERR_ARG with the sizes), held by every GPU
 * that loads the library until the process exits, shared by all calls on
 * that device: calls that overlap on the GPU race, so serialise them.  The
 * first call on a device looks up the array's device address; make that
 * first call before any stream capture, with the context's device current.
 * This entry point has no counterpart in the reference. */
int hc_level_rk4_step_noalloc(hc_ctx* ctx, double* ju, double dt, double t,
                              void* stream);

/* nsteps RK4 steps with dt = cfl/max(inverse dt) computed on the device
 * before every step (exec/main.cpp:377-383).  *time_dev (device double) is
 * advanced in place; dt_dev (device double, may be NULL) receives the
 * last dt.  No host synchronisation inside. */
int hc_level_advance_cfl(hc_ctx* ctx, double* ju, int nsteps,
                         double* time_dev, double* dt_dev, void* stream);

/* Maximum over valid cells of the CFL rate, written to the device double
 * *inv_dt_max.  Replaces dtCFLSecondOrderHost (src/BoxOp_SecondOrderCFL.H:
 * 99-210) and, at order 4, dtCFL/dtInv (src/BoxOp_EulerCubedSphereImplem.H:
 * 878-954,1013-1131), whose results are 1/max; the two use the same
 * arithmetic on JU. */
int hc_level_dt_cfl(hc_ctx* ctx, const double* ju, double* inv_dt_max,
                    void* stream);

/* *ok (device int) = 1 if every component of every valid cell is finite
 * and density is positive, else 0.  Replaces validConservedState
 * (src/BoxOp_EulerCubedSphereImplem.H:817-876). */
int hc_level_valid(hc_ctx* ctx, const double* ju, int* ok, void* stream);

/* ---------------------------------------------------------------------------
 * AMR Runge-Kutta stage logic on uneven boxes (advanceRungeKuttaSynchronous,
 * src/MHD_AMRRungeKutta.H:5-41, and restrictTo, src/MHD_AMR.H:597-609).
 * The hierarchy itself (layouts, regrid, coarse-fine ghosts, flux
 * registers) stays with the caller; these entries do the per-box arithmetic
 * of every box of every level in one launch each.
 * ------------------------------------------------------------------------- */

/* One box: its valid cells (arrays of 8 x ncells doubles, component-major,
 * the caller's cell order), the state U^n, the stage state and the four
 * stage right-hand sides (device pointers). */
typedef struct hc_rk_box {
  long long ncells;
  double* state;
  double* stage;
  double* rk[4];
} hc_rk_box;

/* One restriction: the coarse cells lo..hi (inclusive, coarse index space)
 * of `coarse` (stored over coarse_lo + [0, coarse_n)) become the mean of
 * the ratio[0] x ratio[1] x ratio[2] cells of `fine` (stored over fine_lo +
 * [0, fine_n), fine index space) they cover: Stencil::AvgDown(ratio). */
typedef struct hc_restrict_box {
  const double* fine;
  double* coarse;
  int fine_lo[3], fine_n[3];
  int coarse_lo[3], coarse_n[3];
  int lo[3], hi[3];
  int ratio[3];
  int reserved;
} hc_restrict_box;

/* One coarse-fine interface patch of the reflux (the flux-register
 * correction of src/MHD_AMR.H:651-665,916-931): the coarse faces lo..hi
 * (inclusive, coarse index space; faces of direction dir, face I between
 * cells I-1 and I) are covered by the fine level on side `fine_side` (1:
 * the fine cells are at and above the face, the coarse cell corrected is
 * I-1, whose high face it is; 0: the fine cells are below, the corrected
 * cell is I).  For each face, Fbar = mean of the ratio x ratio fine faces
 * covering it (fine face index ratio[dir] * I along dir), and
 *   rhs(C) += coef * (Fbar - F_coarse)   (fine_side 1: coef = -scale,
 *                                          fine_side 0: coef = +scale),
 * scale being the operator's scale / dxi[dir] of the coarse level.  Arrays
 * are 8 components, component-major over their storage boxes: fine_flux
 * and coarse_flux over face boxes (lo, n), rhs over a cell box. */
typedef struct hc_reflux_box {
  const double* fine_flux;
  const double* coarse_flux;
  double* rhs;
  int fine_lo[3], fine_n[3];
  int coarse_lo[3], coarse_n[3];
  int rhs_lo[3], rhs_n[3];
  int lo[3], hi[3];
  int ratio[3];
  int dir, fine_side;
  int reserved;
  double scale;
} hc_reflux_box;

typedef struct hc_amr_plan hc_amr_plan;

/* Validate the boxes, restrictions and reflux patches (host arrays; every
 * restriction and patch must read and write inside its arrays' boxes) and
 * keep a device copy of each list. */
int hc_amr_plan_create(hc_ctx* ctx, const hc_rk_box* boxes, int nbox, const hc_restrict_box* restricts,
                       int nrestrict, hc_amr_plan** out);
int hc_amr_plan_set_reflux(hc_amr_plan* plan, const hc_reflux_box* patches, int npatch);

/* Reflux patches first .. first+count-1 of the plan in one launch (patches
 * of one launch must not correct the same coarse cell). */
int hc_amr_reflux(hc_ctx* ctx, const hc_amr_plan* plan, int first, int count, void* stream);
int hc_amr_plan_destroy(hc_amr_plan* plan);

/* The tableau (order 3: Kutta RK3, 4: classical RK4, src/MHD_AMRRungeKutta.H:
 * 9-12) on every box of the plan.  stage s < order: stage = state, then
 * stage += (dt a[s][p]) rk[p] for each p < s with a[s][p] != 0 (amrCopyValid
 * + increment, :22-27); stage = order: state += (dt b[p]) rk[p] for p < order
 * in order (:37).  Each increment rounds the product, then the sum. */
int hc_amr_rk_stage(hc_ctx* ctx, const hc_amr_plan* plan, int order, int stage, double dt, void* stream);

/* Restrictions first .. first+count-1 of the plan in one launch.  The
 * reference restricts the finest level first (:26); give each level's
 * restrictions their own call, finest first, when levels chain. */
int hc_amr_restrict(hc_ctx* ctx, const hc_amr_plan* plan, int first, int count, void* stream);

/* Coarse-fine ghost interpolation of one fine box (the fourth-order
 * interpolation of src/MHD_AMRInterpolation.H:39-155 as
 * src/MHD_AMRFourthOrder.H:27-39 applies it to the donor data): every cell
 * p of the fine storage region fine_lo .. fine_lo + fine_n - 1 (fine index
 * space) outside the valid region valid_lo .. valid_hi gets, in each of its
 * ncomp components, the average over the cell of the tensor-product quartic
 * that matches the 5 x 5 x 5 coarse cell averages around its parent.  The
 * parent is q = floor(p / ratio) per direction and the weights of direction
 * d are those of hc_amr_cf_weights(ratio[d], p[d] - q[d] ratio[d]) (ratio
 * 1: the parent alone).  The sums run direction by direction as the
 * reference's passes do: first along i (coarse points q0-2 .. q0+2), then
 * along j over those results, then along k, each in increasing index and
 * skipping points of weight zero; products and sums are rounded as
 * written.  A first-pass point of nonzero weight outside the coarse array's
 * box (coarse_lo, coarse_n) makes its partial sum NaN.  A cell whose result
 * is not finite in every component is left unchanged (the reference leaves
 * its donor at zero for the exchange to fill).  Arrays are [ncomp][k][j][i]
 * SoA over their boxes (device); ratio 1..8, ncomp 1..16. */
typedef struct hc_cf_box {
  const double* coarse;
  double* fine;
  int coarse_lo[3], coarse_n[3];
  int fine_lo[3], fine_n[3];
  int valid_lo[3], valid_hi[3];
  int ratio[3];
  int ncomp;
} hc_cf_box;

/* Weights w[0..4] (coarse cells q-2 .. q+2 along one direction) of child
 * `child` (0 .. ratio-1) of a coarse cell: the average over the child of
 * the quartic whose averages over the five coarse cells are the data, from
 * the exact inverse of the five cells' moment matrix and the child's
 * moments (ratio 1: {0, 0, 1, 0, 0}).  Host arithmetic, no device needed. */
int hc_amr_cf_weights(int ratio, int child, double* w);

/* Validate and keep a device copy of the plan's interpolation boxes. */
int hc_amr_plan_set_cf_interp(hc_amr_plan* plan, const hc_cf_box* boxes, int nbox);

/* Interpolation boxes first .. first+count-1 of the plan in one launch
 * (boxes of one launch must not write the same fine array region). */
int hc_amr_cf_interpolate(hc_ctx* ctx, const hc_amr_plan* plan, int first, int count, void* stream);

/* The fourth-order <JU> and <U> of a fine box around the caller's
 * same-level exchange (src/MHD_AMRFourthOrder.H:41-80), two launches:
 *
 * hc_amr_cf_mapped, on every cell p of the mapped region (mapped_lo,
 * mapped_n; the reference's valid.grow(2)): valid cells copy the box's
 * state <JU>; the others get
 *   <JU>(p) = J(p) U(p) + sum_d (J(p+e_d) - J(p-e_d)) (U(p+e_d) - U(p-e_d)) / 48
 * from the donor Cartesian averages U (after hc_amr_cf_interpolate).
 *
 * hc_amr_cf_quotient, on every valid cell (after the caller's exchange of
 * the mapped ghosts): with Q = <JU> / J,
 *   out(p) = Q(p) - (sum_d 0.5 (J(p+e_d) - J(p-e_d)) D_d Q(p)) / (12 J(p)),
 * D_d the undivided derivative along d: centred, and second-order one-sided
 * on the block's (the panel's domain box at this level) first and last
 * cells (weights -3/2, 2, -1/2 and 1/2, -2, 3/2, summed over three cells
 * in increasing index).  Every product, sum and quotient is rounded as
 * written, the terms in the order shown, directions in order.
 *
 * Arrays are SoA over their own boxes: jac 1 component (its box must
 * contain valid.grow(3)), donor, state, mapped, out 8 components (donor:
 * valid.grow(3); state and out: valid; mapped: valid.grow(2)); the block
 * contains valid and is at least 3 cells wide in each direction. */
typedef struct hc_cf_fine_box {
  const double* jac;
  const double* donor;
  const double* state;
  double* mapped;
  double* out;
  int jac_lo[3], jac_n[3];
  int donor_lo[3], donor_n[3];
  int state_lo[3], state_n[3];
  int mapped_lo[3], mapped_n[3];
  int out_lo[3], out_n[3];
  int valid_lo[3], valid_hi[3];
  int block_lo[3], block_hi[3];
} hc_cf_fine_box;

/* One region copy between two SoA arrays: the same-level exchanges and
 * the coarse-to-fine source copies of the AMR prepare
 * (src/MHD_AMRFourthOrder.H:19-24,58,83-85).  For every point x of the
 * region lo .. hi (source index space) and every component c,
 *   dst(y, c) = src(x, c),   y[d] = sign[d] * x[perm[d]] + shift[d],
 * perm a permutation of {0, 1, 2} and sign[d] = +1 or -1: the index map
 * between two panels of the cubed sphere is a signed permutation; within
 * a panel perm = {0, 1, 2}, sign = {1, 1, 1}.  The region must lie in the
 * source box and its image in the destination box; ncomp 1..16. */
typedef struct hc_copy_box {
  const double* src;
  double* dst;
  int src_lo[3], src_n[3];
  int dst_lo[3], dst_n[3];
  int lo[3], hi[3];
  int perm[3], sign[3], shift[3];
  int ncomp;
} hc_copy_box;

/* Validate and keep a device copy of the plan's copies. */
int hc_amr_plan_set_copies(hc_amr_plan* plan, const hc_copy_box* copies, int ncopy);

/* Copies first .. first+count-1 of the plan in one launch.  Within one
 * launch no written region may overlap another copy's written or read
 * region of the same array (an exchange writes ghosts and reads valid
 * cells, so a level's exchange is one launch), and arrays given by
 * different base pointers must not share memory where one is written
 * (HC_ERR_ARG otherwise). */
int hc_amr_copy(hc_ctx* ctx, const hc_amr_plan* plan, int first, int count, void* stream);

int hc_amr_plan_set_cf_fine(hc_amr_plan* plan, const hc_cf_fine_box* boxes, int nbox);
int hc_amr_cf_mapped(hc_ctx* ctx, const hc_amr_plan* plan, int first, int count, void* stream);
int hc_amr_cf_quotient(hc_ctx* ctx, const hc_amr_plan* plan, int first, int count, void* stream);

/* The last step of a fine box's fourth-order preparation: its native
 * averages USph on the operator's input box (usph_lo, usph_n; valid.grow(5)
 * for the Berta operator) from its Cartesian averages U (after the
 * exchanges and the coarse-fine fill), and its radial boundary ghosts.
 * Replaces cachedNativeConversion + fillRadialBoundaries on the fine
 * boxes (src/MHD_AMRFourthOrder.H:86-100; conversion
 * src/MHD_CachedCartesianConversion.H:65-124, ghosts
 * src/BoxOp_PreStage.H:57-228), with the same arithmetic as the level's
 * stage preparation: cells with 0 <= i < nr take the fourth-order matrix
 * quotient of U at (i, j, k) and its angular neighbours; i < 0 the analytic
 * inner wind at time t; i >= nr the native value at nr - 1 scaled by
 * (r_last / r)^2 (B_t by r_last / r).  The context is the level's (its
 * geometry); the usph box's angular cells lie within [-5, na + 5), radial
 * within [-5, nr + 5); the cart box (8 components SoA) holds every
 * (i, j +- 1, k +- 1) the conversion reads; cart cells beyond the panel
 * must already hold the seam-interpolated averages (this library fills
 * those for whole levels only, so AMR boxes whose cart box crosses a panel
 * edge are the caller's). */
typedef struct hc_native_box {
  const double* cart;
  double* usph;
  int cart_lo[3], cart_n[3];
  int usph_lo[3], usph_n[3];
  int block;
} hc_native_box;

int hc_amr_plan_set_native(hc_amr_plan* plan, const hc_native_box* boxes, int nbox);
int hc_amr_native(hc_ctx* ctx, const hc_amr_plan* plan, int first, int count, double t, void* stream);

/* ---------------------------------------------------------------------------
 * Autotuner (no reference counterpart: the reference runs its face loops on
 * the host).  Order 2: the stage kernel runs one CTA per cell tile; the
 * tiles differ in shape and in the register cap (resident CTAs per SM), and
 * the fastest depends on the limiter / solver pair and the level size.
 * Order 4: the reconstruction, Roe point and final-flux kernels each come
 * in register-cap variants.  Order-2 results do not depend on the tile.  The
 * order-4 variants agree to round-off only: the code generator may contract
 * a multiply and an add into one fused operation differently under each
 * register cap.  Contexts that take the process-wide choice all use the same
 * variants.
 * ------------------------------------------------------------------------- */

/* Number of candidate tiles; with shapes non-null, shapes[5 t .. 5 t + 4] =
 * {cells x, y, z, min CTAs per SM with Rusanov, with Roe} for t < capacity. */
int hc_stage_tiles(int* shapes, int capacity);

/* Order 2: time every tile on this context's level with the state ju
 * (device, not modified): the fused RK stage (its first stage, into the
 * context's workspace) and the operator alone (hc_level_rhs), a few launches
 * each on `stream`, and keep the fastest of each for the context.  tiles
 * (host, nullable, 2 ints) gets {RK stage tile, operator tile}; ms (host,
 * nullable, 2 x count doubles) the median launch times, RK stage first.
 * Order 4: time the level operator (after the stage preparation of ju) for
 * each register-cap variant of the reconstruction, Roe point dissipation
 * and final-flux kernels in turn, keeping the best of each; tiles (3 ints)
 * gets the variants, ms (3 x hc_o4_variants() doubles) the operator times.
 * Blocks the host until the timing is done: call it outside stream capture.
 * The choice is also kept process-wide for contexts of the same device,
 * level size and scheme, which then skip the timing when created with
 * hc_params.autotune = 1. */
int hc_ctx_autotune(hc_ctx* ctx, const double* ju, int* tiles, double* ms, void* stream);

/* Number of register-cap variants per tuned fourth-order kernel; with
 * min_blocks non-null, min_blocks[3 q + v] = minimum resident CTAs per SM of
 * variant v of kernel q (0 reconstruction, 1 Roe point, 2 fused face chain). */
int hc_o4_variants(int* min_blocks, int capacity);

/* Use the given variants (3 ints, -1 keeps the current one). */
int hc_ctx_set_o4_variants(hc_ctx* ctx, const int* variants);

/* Use the given tiles (0 .. count-1) for the RK stage and the operator
 * alone; -1 keeps the current one. */
int hc_ctx_set_tiles(hc_ctx* ctx, int tile_rk, int tile_rhs);

/* Seeded synthetic initial state (valid cells) of the level. */
int hc_level_init(hc_ctx* ctx, const hc_init* init, double* ju, void* stream);

/* ---------------------------------------------------------------------------
 * Cone CME, finite spherical cloud (CME field model 4, the analytic cone of
 * src/MHD_ImportedCME.H:415-420 prepared by src/MHD_CME.H:1111-1136).
 * ------------------------------------------------------------------------- */

/* Fitted cone parameters (the reference's CMEParameters fields for a
 * finite cone: lat, lon, halfangle, apex_speed, windSpeed, dragGamma, r1
 * (r0 = 0), referenceTime, density, temperature). */
typedef struct hc_cone_spec {
  double lat_deg, lon_deg;   /* axis = orientation(lat, lon, 0) (0,0,1): (cos lat cos lon, cos lat sin lon, sin lat) */
  double half_angle_deg;     /* cloud radius a = r_inner sin(half angle) */
  double apex_speed;         /* km/s at reference_time */
  double wind_speed;         /* km/s, drag-based model ambient speed */
  double drag_gamma;         /* 1/km, drag-based model coefficient (0: ballistic), >= 0 */
  double reference_height;   /* leading-edge height at reference_time, solar radii (6.96e10 cm) */
  double reference_time;     /* s */
  double density;            /* total cloud density, g/cm^3 */
  double temperature;        /* K (equal proton and electron temperature) */
  double reserved[6];
} hc_cone_spec;

/* The prepared cloud: a sphere of radius `radius` whose centre moves along
 * `axis` at `speed`, its centre at distance entry_shift + speed (t -
 * entry_time) from the origin.  It touches the inner boundary first at
 * entry_time; the inner boundary feeds it while insertion_time <= t <
 * end_time (src/MHD_CME.H:968). */
typedef struct hc_cone {
  double axis[3];
  double radius;             /* cm */
  double entry_shift;        /* cm: r_inner - radius */
  double entry_time;         /* s */
  double speed;              /* km/s, the drag-based speed at entry_time */
  double end_time;           /* s: entry_time + 2 radius / speed */
  double insertion_time;     /* s: volume insertion time (reference height reached) */
  double density, temperature;
  double reserved[6];
} hc_cone;

/* Host function (no device work): prepareConeCloud with the drag-based
 * trajectory and boundary-contact bisection (src/MHD_CME.H:1069-1136) for
 * the level's inner radius (cm).  HC_ERR_ARG where the reference throws
 * (no outward trajectory to the inner boundary). */
int hc_cone_prepare(const hc_cone_spec* spec, double inner_radius, hc_cone* cone);

/* Volume insertion of the cloud at `time` into the level state JU (valid
 * cells, device): every cell whose centre lies inside the cloud takes the
 * cloud's density, radial velocity `speed` and pressure 2 k T rho / m_p,
 * keeping its magnetic field (Insert_CME for cones,
 * src/BoxOp_EulerCubedSphereImplem.H:1236-1300, at either order).
 * stats (device, nullable): [0] cells changed, [1] mass added (g), summed
 * in a fixed order. */
int hc_level_insert_cone(hc_ctx* ctx, const hc_cone* cone, double time, double* ju, double* stats, void* stream);

/* One inserted CME source of the insertion schedule (src/MHD_CME.H:
 * 1243-1334, CMEInsertionSchedule): its insertion time, whether it feeds
 * through the inner boundary, and when that feeding ends. */
typedef struct hc_cme_event {
  double insertion_time;
  double feeding_end;
  int boundary;
  int reserved;
} hc_cme_event;

/* The schedule event of a prepared cone cloud: a boundary source while the
 * cloud still crosses the inner boundary after insertion (:1251-1253). */
int hc_cone_event(const hc_cone* cone, hc_cme_event* event);

/* The driver's stabilisation after CME insertions (exec/main.cpp:374-420),
 * applied by hc_level_advance_cfl on the device with no host sync.  Each
 * step's dt uses CFL x fraction(time): the minimum over the sources inserted
 * by then (time >= insertion_time) of 0.2 + 0.8 early for a volume source,
 * or 0.2 + (f - 0.2) early + (1 - f) recovery for a boundary source, with
 * early = clamp((time - t - 600) / 1800, 0, 1), recovery = clamp((time -
 * end) / 1800, 0, 1), f = 0.5 with Roe and 1 with Rusanov, and end the
 * source's stabilisation end (t + 600, or max(feeding_end + 600, t + 2400)
 * for a boundary source) (src/MHD_CME.H:1275-1297, 1329-1332).  A Roe
 * context uses Rusanov dissipation while time is before the
 * latest stabilisation end, with dt shortened to land on it (the reference's
 * Rusanov window; at order 2 the device picks between the Roe and the
 * Rusanov stage kernels, both launched, each returning at once unless it
 * is the one wanted).  n = 0
 * clears; at most 8 events, ordered by insertion time.  The schedule is
 * copied to the device in order on `stream`.  After the first call every
 * hc_level_advance_cfl step runs the schedule (with no events it changes
 * nothing), so a graph captured after a call with n = 0 takes later
 * schedules. */
int hc_level_set_cme_schedule(hc_ctx* ctx, const hc_cme_event* events, int n, void* stream);

/* Feed prepared cone clouds through the inner boundary of an order-2 level
 * while they cross it (insertion_time <= t < end_time; the reference's
 * boundary source of a finite cloud).  Each stage's inner radial ghosts
 * whose point on the boundary sphere lies in a cloud take the cloud's
 * density, radial speed and pressure over the analytic wind, keeping its
 * field (src/BoxOp_PreStage.H:329-400).  In hc_level_rk4_step and
 * hc_level_advance_cfl the inner faces such a cloud covers take their
 * interior state from owned cells only and share that state's normal field
 * (src/BoxOp_SecondOrder.H:175-181, 282-311); hc_level_rhs and hc_box_rhs,
 * which take no time, do not.  hc_level_advance_cfl adds each crossing
 * cloud's (speed + sound speed) / first radial cell width to the step's
 * CFL rate (src/MHD_CME.H:1165-1191), and its rate takes the Alfven speeds
 * with density min(rho, the lightest crossing cloud's density)
 * (src/BoxOp_SecondOrderCFL.H:196-200); hc_level_dt_cfl, which takes no
 * time, does not.  At most 8 cones; n = 0 stops the
 * inlet.  The cones are copied on `stream`; launches captured in a graph
 * keep the inlet set when they were captured. */
int hc_level_set_inlet(hc_ctx* ctx, const hc_cone* cones, int n, void* stream);

/* Host copies of the level geometry used by the kernels, for tests:
 * what = 0 radial line [nr+1][4]: rlow^2, (rhigh^2-rlow^2)/(2dxi0),
 *          (rhigh-rlow)/dxi0, dVolr (last row: face only)
 * what = 1+d face normals adjA for direction d: [6][na+e1][na+e2][3]
 * what = 4 cell detA [6][na][na];  what = 5 cell detA_A [6][na][na][3][3]
 * Returns the number of doubles written (or needed if out is NULL). */
long hc_geometry_export(const hc_ctx* ctx, int what, double* out);

#ifdef __cplusplus
}
#endif
#endif /* HC_ABI_H */
