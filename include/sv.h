/*
 * sv.h -- C-ABI of the B200 Saint-Venant time step (libsv_b200.so).
 *
 * Drop-in boundary for the hot path of oojimaflib/mfcm: the 2-D Saint-Venant explicit
 * Runge-Kutta time step (face fluxes with wet/dry handling, bed slope, Manning friction,
 * rainfall = discharge boundary, outflow = head boundary, RK stage combination and the CFL
 * control number). Plain C types only; no exceptions cross this boundary; every function
 * returns 0 on success or a negative SV_E* code, with a message in sv_last_error().
 *
 * Ownership: an sv_ctx owns all device memory and one CUDA stream; host pointers are
 * borrowed for the duration of the call; sv_get_field is synchronous on the ctx stream.
 * Threading: one ctx is used by one host thread at a time (like the reference's single
 * sycl::queue); separate ctxs are independent.
 *
 * Each entry point names the reference interface it replaces (paths are relative to the
 * reference project's root).
 */
#ifndef SV_B200_H
#define SV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ------------------------------------------------------------------- */
#define SV_OK 0
#define SV_E_ARG (-1)       /* invalid argument (null pointer, size mismatch, bad id)      */
#define SV_E_CUDA (-2)      /* CUDA runtime error                                          */
#define SV_E_NOMEM (-3)     /* device allocation failed                                    */
#define SV_E_STATE (-4)     /* call not valid in the current state                         */
#define SV_E_NONFINITE (-5) /* the control number became NaN (state is no longer finite)    */
#define SV_E_TIMEOUT (-6)   /* a bounded device-side wait gave up                          */
#define SV_E_LIMIT (-7)     /* size beyond a documented maximum                            */

/* ---- precision --------------------------------------------------------------------- */
typedef enum {
  SV_F32 = 1,         /* FP32 state and arithmetic, FP64 reductions                   */
  SV_F64 = 2,         /* plain FP64: bit-for-bit the reference arithmetic at T=double */
  SV_F32_DATUM64 = 3  /* FP32 state, bed stored as FP32 offsets from FP64 tile datums   */
} sv_precision;

/* Mirrors the Cartesian2DMesh configuration (src/Mesh/Cartesian2DMesh.cpp:24-61):
 * "cell count" = (nx, ny), "cell size" = (dx, dy), "origin"; rotation angle 0 only. */
typedef struct {
  uint64_t nx, ny;
  double dx, dy;
  double origin_x, origin_y;
} sv_mesh_desc;

/* Mirrors the scheme configuration read by create_scheme (src/mfcm.cpp:19-36),
 * RungeKuttaTimeParameters (src/Config/TimeParameters.cpp:21-38) and the solver's
 * source-term/boundary lists (src/SaintVenant/Solver.cpp:61-67). */
typedef struct {
  int precision;        /* sv_precision                                                 */
  int rk_method;        /* named tableau index, see SV_RK_* (RungeKutta.cpp:54-115)      */
  double cn_target;     /* control-number target; the reference hard-codes 1.0
                           (src/TemporalScheme/RungeKutta.cpp:154)                      */
  double step_duration; /* "step duration seconds" L (TimeParameters.cpp:29-32)         */
  double initial_dt;    /* "initial timestep seconds" (TimeParameters.cpp:34)           */
  double max_dt;        /* 0 = no clamp (reference behaviour); > 0 clamps each new dt   */
  int rain_mode;        /* 0 = reference discharge clamp, 1 = physical clamp            */
  int manning;          /* 1 = "manning roughness" source term present                  */
  int head_first;       /* 1 = head boundary listed before discharge in the config      */
  int flags;            /* SV_FLAG_*                                                     */
} sv_params;

#define SV_FLAG_NO_TALLIES 1u /* skip the rain/outflow tally partials                    */
#define SV_FLAG_ELOSS_FIRST 2u /* energy loss listed before Manning roughness in the config:
                                  both add to du/dt and dv/dt, so their order sets the
                                  rounding; infiltration (dh/dt only) commutes with both   */

/* named Runge-Kutta tableaux, in the order of runge_kutta_named_coefficient_sets_ */
#define SV_RK_EULER 0
#define SV_RK_MIDPOINT 1
#define SV_RK_HEUN2 2
#define SV_RK_RALSTON2 3
#define SV_RK_KUTTA3 4
#define SV_RK_HEUN3 5
#define SV_RK_WRAY3 6
#define SV_RK_RALSTON3 7
#define SV_RK_SSPRK3 8
#define SV_RK_CLASSIC 9
#define SV_RK_RALSTON4 10
#define SV_RK_38RULE 11

/* field ids for sv_set_field / sv_get_field (cell fields are nx*ny, row-major i = y*nx+x;
 * face fields are (nx+1)*ny vertical faces followed by (ny+1)*nx horizontal faces) */
#define SV_FIELD_Z 0            /* bed elevation z_bed (Constants.hpp:39)                 */
#define SV_FIELD_H 1            /* depth h of U_[0] (State.hpp:40)                       */
#define SV_FIELD_U 2            /* x velocity u of U_[0]                                  */
#define SV_FIELD_V 3            /* y velocity v of U_[0]                                  */
#define SV_FIELD_N_SHALLOW 4    /* Manning n_shallow (ManningRoughnessSourceTerm.hpp:111) */
#define SV_FIELD_N_DEEP 5
#define SV_FIELD_D_SHALLOW 6
#define SV_FIELD_D_DEEP 7
#define SV_FIELD_QBDY0 8        /* discharge xbdy0 (BoundarySourceTerm.hpp:44), m/s       */
#define SV_FIELD_QBDY1 9        /* discharge xbdy1                                        */
#define SV_FIELD_HBDY0 10       /* head xbdy0 (NaN = not selected)                        */
#define SV_FIELD_HBDY1 11
#define SV_FIELD_RAIN_PATTERN 12 /* per-cell rain pattern P for SV_RAIN_PATTERN            */
#define SV_FIELD_INFIL_RATE 13  /* infiltration rate, m/s (InfiltrationSourceTerm.hpp:106)   */
#define SV_FIELD_INFIL_CAP 14   /* remaining infiltration capacity, m; consumed at every
                                   stage evaluation as in InfiltrationSourceTerm.cpp:61      */
#define SV_FIELD_ELOSS_FX 15    /* energy-loss coefficient fx/m (EnergyLossSourceTerm.hpp:199)*/
#define SV_FIELD_ELOSS_FY 16    /* energy-loss coefficient fy/m                              */
#define SV_FIELD_H_COMP 17      /* FP32 solvers: compensation carried by the depth update
                                   (part of the state for a bit-exact restart; zeroed
                                   whenever SV_FIELD_H is set)                              */
#define SV_FIELD_EDDY_MU 18     /* eddy viscosity: per-cell constant coefficient mu, m^2/s */
#define SV_FIELD_DHDT 20        /* dUdt_[0] of the last sv_eval_dudt(0, ...)              */
#define SV_FIELD_DUDT 21
#define SV_FIELD_DVDT 22
#define SV_FIELD_DHDX 23        /* dUdx_ / dUdy_ of the last sv_eval_dudt (State.cpp:176) */
#define SV_FIELD_DUDX 24
#define SV_FIELD_DVDX 25
#define SV_FIELD_DHDY 26
#define SV_FIELD_DUDY 27
#define SV_FIELD_DVDY 28
#define SV_FIELD_DZDX 29        /* bed slopes (Constants.cpp:39-40)                       */
#define SV_FIELD_DZDY 30
#define SV_FIELD_FLUX_H 40      /* face fluxes of the last sv_eval_dudt (Fluxes.hpp:43-49)*/
#define SV_FIELD_FLUX_U 41
#define SV_FIELD_FLUX_V 42
#define SV_FIELD_FLUX_Z 43
#define SV_FIELD_FLUX_BRANCH 44 /* wet/dry branch per face: 0,1,2.25,2.75,3,4             */
#define SV_FIELD_STATE_BASE 100 /* 100 + 3*s + {0,1,2}: h,u,v of U_[s]                    */
#define SV_FIELD_K_BASE 200     /* 200 + 3*s + {0,1,2}: h,u,v of dUdt_[s]                 */

/* ---- per-step boundary values (DischargeBoundarySourceTerm.hpp:114-146,
 *      HeadBoundarySourceTerm.hpp:114-146): values at the start (0) and end (1) of the step,
 *      varying linearly within it. --------------------------------------------------- */
#define SV_RAIN_NONE 0
#define SV_RAIN_UNIFORM 1  /* every cell: q0 = rain_q0, q1 = rain_q1 (m/s)                 */
#define SV_RAIN_FIELDS 2   /* per-cell SV_FIELD_QBDY0/QBDY1, uploaded by the caller        */
#define SV_RAIN_PATTERN 3  /* q0 = P * rain_q0, q1 = P * rain_q1 with P = RAIN_PATTERN     */
#define SV_HEAD_NONE 0
#define SV_HEAD_EDGES 1    /* one-cell strips along the edges in head_edges               */
#define SV_HEAD_FIELDS 2   /* per-cell SV_FIELD_HBDY0/HBDY1 (NaN = not selected)          */
/* stage boundary (StageBoundarySourceTerm.cpp:39-69): targets are water levels, the depth
 * target being level - bed; it takes the head boundary's place in the boundary order */
#define SV_STAGE_EDGES 3   /* one-cell strips along head_edges, levels head_h0/head_h1     */
#define SV_STAGE_FIELDS 4  /* per-cell levels in SV_FIELD_HBDY0/HBDY1 (NaN = not selected)*/
#define SV_EDGE_XMIN 1u
#define SV_EDGE_XMAX 2u
#define SV_EDGE_YMIN 4u
#define SV_EDGE_YMAX 8u

typedef struct {
  int rain_kind;
  double rain_q0, rain_q1;
  int head_kind;
  unsigned head_edges;
  double head_h0, head_h1;
} sv_forcing;

typedef struct {
  uint64_t accepted;  /* accepted timesteps                                              */
  uint64_t repeated;  /* rejected (repeated) timesteps                                   */
  double volume;      /* FP64 sum of h * cell area of U_[0]                              */
  double rain_in;     /* FP64 volume added by the discharge (rain) term                  */
  double outflow;     /* FP64 volume removed by the head (outflow) assignment            */
  double wall_in;     /* FP64 volume that entered through the mesh-edge faces (negative:
                         left); the reference's walls pass flow through their one-sided
                         flux branches, so volume = initial + rain_in - outflow + wall_in  */
} sv_stats;

typedef struct sv_ctx sv_ctx;

/* SaintVenantSolver constructor (src/SaintVenant/Solver.cpp:32-71) + RungeKuttaSolver
 * (src/TemporalScheme/RungeKutta.hpp:319-331): allocates U_[0..N], the k stages and the
 * bed constants on device `device`. The state U_[0] (h, u, v) and the bed start at zero.
 * Later calls on the solver launch work on that device's streams: make `device` the current
 * CUDA device before each call (one process per GPU, as the replicas run, satisfies this once
 * and for all). */
int sv_create(const sv_mesh_desc* mesh, const sv_params* params, int device, sv_ctx** out);
/* ~SaintVenantSolver */
void sv_destroy(sv_ctx* ctx);
/* Field<T,Mesh,C> host->device upload (src/Field/Field.hpp:36-251, DataArray.cpp:21-116);
 * SV_FIELD_Z recomputes dz/dx, dz/dy (Constants.cpp:39-40). Values are converted to the
 * ctx precision. */
int sv_set_field(sv_ctx* ctx, int field_id, const double* host, uint64_t n);
/* Field device->host read (DataArray::move_to_host, DataArray.cpp:95-116) */
int sv_get_field(sv_ctx* ctx, int field_id, double* host, uint64_t n);
/* ManningRoughnessSourceTerm "default shallow/deep n/depth" (ManningRoughnessSourceTerm.cpp:99-102);
 * uniform values (a later sv_set_field of that id makes it per-cell). */
int sv_set_manning(sv_ctx* ctx, double n_shallow, double n_deep, double d_shallow, double d_deep);
/* EddyViscositySourceTerm (EddyViscositySourceTerm.cpp:43-137): du/dt -= mu (u_xx + u_yy),
 * dv/dt -= mu (v_xx + v_yy) on cells deeper than 1e-6 m, capped like the roughness term, the
 * second derivatives being Minmod3 slopes of the stage's slopes. SV_EDDY_CONSTANT: mu is the
 * field SV_FIELD_EDDY_MU when set, else `mu` ("default mu"); SV_EDDY_SMAGORINSKY: mu =
 * mu_const + mu_smag * cell area * sqrt(u_x^2 + v_y^2 + 0.5 (|u_y| + |v_x|)^2) per cell and
 * stage ("constant coefficient", "dynamic coefficient"). */
#define SV_EDDY_OFF 0
#define SV_EDDY_CONSTANT 1
#define SV_EDDY_SMAGORINSKY 2
int sv_set_eddy_viscosity(sv_ctx* ctx, int mode, double mu, double mu_const, double mu_smag);
/* Configuration order of the momentum source terms (Solver.cpp:98-104): each adds to du/dt and
 * dv/dt, so the order sets the rounding. `terms` lists SV_TERM_* at most once each; terms not
 * listed follow in the default order (roughness, energy loss, eddy viscosity). Replaces
 * SV_FLAG_ELOSS_FIRST. */
#define SV_TERM_MANNING 1
#define SV_TERM_ELOSS 2
#define SV_TERM_EDDY 3
int sv_set_source_order(sv_ctx* ctx, const int* terms, int n);
/* SaintVenantSolver::start_new_step (Solver.cpp:116-129): boundary values for [t, t + L]. */
int sv_set_forcing(sv_ctx* ctx, const sv_forcing* forcing);
/* TypedTemporalScheme::dt_ (TemporalScheme.hpp:78) */
int sv_set_dt(sv_ctx* ctx, double dt);
int sv_get_dt(sv_ctx* ctx, double* dt);
/* SaintVenantSolver::update_dUdt (Solver.cpp:73-114): k = dU/dt of U_[state_no] into
 * dUdt_[state_no], with slopes and face fluxes kept for inspection (debug/parity path). */
int sv_eval_dudt(sv_ctx* ctx, int state_no, double t_sub, double dt);
/* RungeKuttaTemporalScheme::do_timestep (RungeKutta.cpp:141-167): all stages, the control
 * number and the accept/repeat decision; does not accept. */
int sv_do_timestep(sv_ctx* ctx, double t_local, double dt, double* cn, int* repeat, double* new_dt);
/* RungeKuttaSolver::accept_timestep (RungeKutta.hpp:428-431) */
int sv_accept(sv_ctx* ctx);
/* TypedTemporalScheme::step (TemporalScheme.hpp:112-149): the whole adaptive-dt loop of one
 * step of length L, run on the device (dt control included) with no host round trip per
 * timestep. `out` receives this step's counts and the running tallies. */
int sv_advance(sv_ctx* ctx, sv_stats* out);
/* SaintVenantVolumeMeasure::get_volume (src/SaintVenant/Measure.hpp:137-156) plus the
 * running rain/outflow tallies; FP64. */
int sv_get_stats(sv_ctx* ctx, sv_stats* out);
/* restore the running counters and FP64 tallies of sv_get_stats (accepted, repeated,
 * rain_in, outflow; volume is recomputed from the state) -- used to resume from a checkpoint
 * of the state, dt and stats; no reference counterpart (the reference has no restart) */
int sv_set_stats(sv_ctx* ctx, const sv_stats* stats);
/* device time (ms) of the last sv_advance, or -1 if not recorded */
int sv_last_advance_ms(sv_ctx* ctx, double* ms);

typedef struct {
  double total_ms;        /* device time of the whole call (CUDA events on the ctx stream)  */
  double stage_ms;        /* summed device time of the stage kernels                       */
  double finalize_ms;     /* summed device time of the reduction + dt-controller kernel    */
  uint64_t stage_launches;
  uint64_t finalize_launches;
} sv_timing;

/* Part of TypedTemporalScheme::step (TemporalScheme.hpp:119-146): at most `max_timesteps`
 * device-controlled timesteps (accepted or repeated) of the current step, stopping early when
 * the step completes (then `*step_done` = 1). `begin` = 1 starts a new step (t_local = 0).
 * With `timing` != NULL every kernel is bracketed by CUDA events on the ctx stream. */
int sv_run_timesteps(sv_ctx* ctx, uint64_t max_timesteps, int begin, sv_stats* out, int* step_done,
                     sv_timing* timing);
/* Stage-kernel variant (no reference counterpart: a launch-shape and schedule choice of this
 * library). Fused schedule, one pass per RK stage: 0-3 tiled shared-memory kernel (32x8, 32x8
 * at 3 CTAs/SM, 32x4 at 4 CTAs/SM, 64x4 at 3 CTAs/SM), 4-10 column-sweep kernel (16/32/64 rows
 * per warp, then 32 rows capped for 3, 4, 5 and 6 CTAs/SM; strips away from the mesh edge and
 * from coded-out cells run an interior form of it), 12-13 (FP32 solvers only) the 32-row
 * column sweep whose pairs of adjacent interior strips run two cells per lane with 8-byte
 * loads (capped for 3 and 4 CTAs/SM; meshes with an odd row length have no pairs), 14-15
 * (FP32 solvers only) the one-cell 32-row sweep capped for 7 and 8 CTAs/SM. Split
 * schedule, two passes per RK stage: 11 a slopes pass, then the tiled 32x8 kernel reading
 * those slopes. Every variant computes bit-identical FP64 results; FP32 results are
 * reproducible per variant. SV_F32_DATUM64 solvers take the column-sweep variants only. */
int sv_set_kernel_variant(sv_ctx* ctx, int variant);
int sv_get_kernel_variant(sv_ctx* ctx, int* variant);
/* Autotune: times every variant's stage kernel (both schedules) on the current state and keeps
 * the fastest;
 * `best_out` (may be NULL) receives the chosen variant. The state U_[0] is not modified. */
int sv_autotune(sv_ctx* ctx, int* best_out);
/* per-variant stage-kernel times (ms) measured by the last sv_autotune; ms[v] for v < n */
int sv_get_autotune_ms(sv_ctx* ctx, float* ms, int n);

/* ---- batches of independent catchments (no reference counterpart: the reference runs one
 *      catchment per process). Members are ordinary sv_ctx solvers; per timestep one batched
 *      launch per RK stage covers every member's tiles and one batched launch runs every
 *      member's reductions and dt controller, so each member keeps its own dt, step clock and
 *      tallies and its results are bit-identical to running it alone. All members share the
 *      batch's precision and a tableau whose stages use only the previous stage. ---------- */
typedef struct sv_batch sv_batch;
int sv_batch_create(int precision, int rk_method, int device, sv_batch** out);
void sv_batch_destroy(sv_batch* batch);
/* add a catchment (allocates its device memory); *id is its slot, reused after removal */
int sv_batch_add(sv_batch* batch, const sv_mesh_desc* mesh, const sv_params* params, int* id);
/* a solver made by sv_create and filled on its own (bed, state, roughness; its uploads run on
 * its own stream, so a server can prepare an arriving request while the batch advances)
 * joins the batch as a member: *id is its slot. Its precision, tableau and device must be the
 * batch's. The batch takes ownership: from now on the context is the member's
 * (sv_batch_member) and is freed by sv_batch_remove or sv_batch_destroy, not sv_destroy. Not to
 * be called while an advance of the same batch runs on another thread. */
int sv_batch_adopt(sv_batch* batch, sv_ctx* solver, int* id);
/* remove a catchment and free its device memory */
int sv_batch_remove(sv_batch* batch, int id);
/* the member's context, for sv_set_field / sv_get_field / sv_set_forcing / sv_get_stats
 * (owned by the batch: do not sv_destroy it); NULL for an empty slot */
sv_ctx* sv_batch_member(sv_batch* batch, int id);
/* TypedTemporalScheme::step for every member at once; out[id] (for id < n_out) receives each
 * member's step counts and running tallies. A member that fails does not stop the others:
 * every member still completes (or fails) its own step, out[] is filled for all of them, and
 * the call returns SV_E_NONFINITE (some member's time became NaN) or SV_E_LIMIT (some member
 * reached the step limit) -- sv_batch_status says which. */
int sv_batch_advance(sv_batch* batch, sv_stats* out, int n_out);
/* Several steps per call (TypedTemporalScheme::solve over up to SV_BATCH_MAX_STEPS steps):
 * member `id` (for id < n) runs nsteps[id] steps back to back, step s with the boundary values
 * forcing[id * max_steps + s]; members with id >= n or nsteps[id] = 0 sit the call out. Each
 * member moves to its next step on the device as soon as its current one ends, so members
 * with long timesteps do not wait for the slowest member at every step; results are
 * bit-identical to nsteps[id] calls of sv_batch_advance. out[id * max_steps + s] receives
 * step s's counts and the running tallies at its end (zeros for steps not run). A member
 * that fails stops alone (status via sv_batch_status, return code as sv_batch_advance).
 * SV_RAIN_FIELDS and SV_HEAD_FIELDS steps use the member's fields as they stand. */
#define SV_BATCH_MAX_STEPS 16
int sv_batch_advance_steps(sv_batch* batch, int max_steps, const int* nsteps, const sv_forcing* forcing,
                           sv_stats* out, int n);
/* Cap on the timesteps one member may take within one step (0, the default: no cap). The
 * reference's velocity formulation can blow up in thin films on steep beds, where dt shrinks
 * without bound and the step never ends; the cap turns that member into an SV_E_LIMIT
 * status, part-way through its step, instead of stalling the whole batch. */
int sv_batch_set_step_limit(sv_batch* batch, long long max_timesteps);
/* status[id] (for id < n) receives each slot's outcome of the last sv_batch_advance: SV_OK,
 * SV_E_NONFINITE (its state is no longer usable) or SV_E_LIMIT (left part-way through the
 * step); SV_OK for empty slots */
int sv_batch_status(sv_batch* batch, int* status, int n);
/* Persistent mode (no reference counterpart; the reference advances one catchment per
 * process, TemporalScheme.hpp:112-149): each sv_batch_advance / sv_batch_advance_steps runs as
 * ONE cooperative launch that fills the device. Every member advances through its queued
 * steps at its own dt; a member's timestep is its stage phases (column-sweep strips, 32 rows)
 * and a finalize phase (reductions, dt controller, step queue), and idle warps take work from
 * whichever member has some. on = 0 returns to one launch per stage. Two bounds end a launch
 * with SV_E_TIMEOUT: spin_limit polls of a waiting warp during which no warp completes a work
 * item (0: the default, 2^22 polls, about a second), and max_seconds of wall clock for the
 * whole launch (<= 0: the default, 120 s; queue fewer steps per call for longer runs). After a
 * timeout every member keeps the state of its last completed timestep. FP64 results are bit
 * for bit those of the other modes; FP32 results are reproducible for this mode. */
int sv_batch_set_persistent(sv_batch* batch, int on, uint64_t spin_limit, double max_seconds);
/* the stage-kernel variant every member of the batch runs (FP32 results are reproducible
 * per variant: a solo run with this variant gives a member's bits) */
int sv_batch_kernel_variant(sv_batch* batch, int* variant);
/* number of members and their total device memory in bytes */
int sv_batch_size(sv_batch* batch, int* n_members, uint64_t* device_bytes);

/* One FP64 Runge-Kutta timestep -- the stages of do_timestep followed by the control number
 * -- on device buffers the caller owns, without allocating any device memory. It has no
 * counterpart in the reference. It is for callers that must not allocate after start-up: a
 * host framework that owns every device allocation through its own pool and hands the solver
 * only pre-allocated buffers, or a real-time loop in which a cudaMalloc would synchronise the
 * device. Working memory is a fixed array inside this library (about 5.2 MB, held by every
 * GPU that loads the library until the process exits), which limits the mesh to 65536 cells
 * (256 x 256); larger meshes return SV_E_LIMIT.
 *   inputs  (device, FP64, nx*ny each): z, h, u, v = U_[0]
 *   outputs (device, FP64, nx*ny each): h_out, u_out, v_out = U_[N]; they must not overlap
 *           the inputs or each other (SV_E_ARG). result (device, 3 doubles): control number,
 *           suggested next dt, 1.0 if the timestep must be repeated else 0.0.
 *   manning: uniform n_shallow, n_deep, d_shallow, d_deep (host array of 4).
 *   forcing: SV_RAIN_NONE/UNIFORM and SV_HEAD_NONE/EDGES only (there is no field storage).
 *   params:  precision SV_F64 and a tableau whose stages use only the previous stage (euler,
 *            midpoint, heun2, ralston2, heun3, ralston3, classic).
 *   stream:  cudaStream_t to launch on (NULL = legacy default stream); nothing is synchronised.
 * The first call on each device looks up the array's device address (cudaGetSymbolAddress),
 * so make that first call before any stream capture; later calls outside capture look it up
 * again, so a device reset between calls is safe. Every call uses the same array and it
 * keeps the previous call's contents (each call rewrites all of it before reading): calls
 * that overlap on the GPU -- on different streams, or from different host threads -- race. */
int sv_timestep_noalloc(const sv_mesh_desc* mesh, const sv_params* params, const double manning[4],
                        const sv_forcing* forcing, const double* z, const double* h, const double* u,
                        const double* v, double* h_out, double* u_out, double* v_out, double t_local,
                        double dt, double* result, void* stream);

/* message of the last failing call on ctx (or, for ctx NULL, of the last failing sv_create or
 * sv_timestep_noalloc on this thread) */
const char* sv_last_error(const sv_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* SV_B200_H */
