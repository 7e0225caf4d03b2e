/* bowshock_b200 — C ABI of the B200 finite-volume backend.
 *
 * Drop-in boundary: these entry points are the reference's GPU solver interface `GpuSolver`
 * (crates/bowshock-cfd/src/gpu/mod.rs:233-414), which the engine's `GpuRunner` (crates/bowshock-core/src/engine/gpu.rs:28-169)
 * and the facade's `GpuBackend` runner (crates/bowshock-core/src/analysis.rs:1186-1253) drive, restated as plain C so a
 * Rust `B200Backend` can bind them with `extern "C"`. Each declaration names the reference method it replaces.
 * Plus the batched case arena (many uneven cases per launch), which has no counterpart in the reference.
 *
 * Conventions
 *  - Every call returns a status (BOWSHOCK_OK = 0) and never aborts the process; the message of the last failure of a
 *    handle is returned by bowshock_solver_last_error / bowshock_arena_last_error (reference: GpuError, gpu/mod.rs:29-56).
 *  - Arrays are row-major with i fastest: cell (i, j) at j*ni + i, node (i, j) at j*(ni+1) + i (reference grid.rs:1-4).
 *    Conserved state u = (rho, rho u, rho v, E) per cell, 4 doubles; turbulence (k, omega) per cell, 2 doubles.
 *  - Units are the reference's: rho_inf = c_inf = 1, p_inf = 1/gamma, lengths in nose diameters (gas.rs:41-43).
 *  - The handle owns all device memory; the caller owns host arrays, which are copied in and out; no pointer is kept
 *    past a call. Handles are not thread-safe; distinct handles may be used from distinct threads.
 *  - There is no CPU fallback: without a usable CUDA device, creation fails with BOWSHOCK_CUDA_ERROR.
 */
#ifndef BOWSHOCK_B200_H
#define BOWSHOCK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (reference error convention: gpu/mod.rs:29-56, bowshock-core error.rs:7-45) */
#define BOWSHOCK_OK 0
#define BOWSHOCK_UNSUPPORTED 1
#define BOWSHOCK_INVALID 2
#define BOWSHOCK_CUDA_ERROR 3
#define BOWSHOCK_NONFINITE 4
#define BOWSHOCK_TIMEOUT 5
#define BOWSHOCK_CANCELLED 6

/* limiter (flux.rs:5-13) */
#define BOWSHOCK_LIM_FIRST_ORDER 0
#define BOWSHOCK_LIM_MINMOD 1
#define BOWSHOCK_LIM_VAN_ALBADA 2
#define BOWSHOCK_LIM_VENKATAKRISHNAN 3
/* boundary conditions [imin, imax, jmin, jmax] (solver.rs:21-37) */
#define BOWSHOCK_BC_FREESTREAM 0
#define BOWSHOCK_BC_EXTRAPOLATE 1
#define BOWSHOCK_BC_SLIPWALL 2
#define BOWSHOCK_BC_CHARACTERISTIC 3
#define BOWSHOCK_BC_PRESSURE_OUTFLOW 4
/* scheme kinds (solver.rs:143-153) */
#define BOWSHOCK_SCHEME_EXPLICIT 0
#define BOWSHOCK_SCHEME_SMOOTHED 1
#define BOWSHOCK_SCHEME_MULTIGRID 2
#define BOWSHOCK_SCHEME_IMPLICIT 3
#define BOWSHOCK_DT_SUM 0
#define BOWSHOCK_DT_MIN_DIRECTION 1
#define BOWSHOCK_TURB_LAMINAR 0
#define BOWSHOCK_TURB_SST 1

/* solver.rs:40-48 `Config` */
typedef struct {
  double cfl;
  int32_t limiter;
  double freestream[4]; /* primitive (rho, u, v, p) */
  int32_t bc[4];
  uint64_t first_order_iters;
} bowshock_config;

/* implicit.rs:59-84 `ImplicitParams` (kind = BOWSHOCK_SCHEME_IMPLICIT), the explicit SSP-RK3 scheme, SSP-RK3 with implicit
 * residual smoothing (kind = BOWSHOCK_SCHEME_SMOOTHED, solver.rs:104-120 `Irs`: cfl_star > 0 is the per-direction CFL
 * limit above which a direction is smoothed, <= 0 none), or FAS multigrid with the SSP-RK3 smoother, solver.rs:123-140
 * `MgParams` (kind = BOWSHOCK_SCHEME_MULTIGRID, the smoother's residual smoothing in mg_cfl_star; Euler only, as the
 * reference) */
typedef struct {
  int32_t kind;
  double cfl0, cfl_max, growth;
  int32_t dt_mode, lines, implicit_bc;
  uint64_t sub_iters;
  int32_t roe;
  double eps_fix;
  uint64_t mg_levels, mg_pre, mg_post, mg_gamma, mg_coarsest;
  double cfl_star, mg_cfl_star;
  /* multigrid with the line-implicit smoother (no counterpart in the reference, whose FAS smoother is SSP-RK3,
   * multigrid.rs:87-112): each smoothing step one implicit iteration with the parameters above (cfl0 .. eps_fix) of the
   * active level, from that level's own CFL ramp; the same FAS transfers */
  int32_t mg_implicit;
  /* multigrid options (0 = the default 1): the fraction of the prolongated correction applied, and the factor of the
   * implicit smoother's CFL numbers per level (level l runs cfl0 and cfl_max times mg_cfl_scale^l) */
  double mg_relax, mg_cfl_scale;
} bowshock_scheme;

/* solver.rs:59-102 `Block` */
typedef struct {
  uint64_t i_end, j_end, j_sting;
} bowshock_block;

/* solver.rs:164-176 `Viscous`: roughness = equivalent sand grain of the body surface in nose diameters (0: smooth walls;
 * > 0 with SST: the Aupoix rough-wall state, turbulence.rs:292-320) */
typedef struct {
  double re_c, sutherland;
  int32_t turbulence;
  uint64_t wall_i_start;
  double roughness;
} bowshock_viscous;

/* solver.rs:186-193 `Nozzle` */
typedef struct {
  uint64_t j_end;
  double state[4];
  double turb[2];
} bowshock_nozzle;

typedef struct bowshock_solver bowshock_solver;

/* GpuSolver::new (gpu/mod.rs:243-249): grid from node coordinates (ni+1)*(nj+1), state at the free stream, iteration 0.
 * `device` is the CUDA device ordinal. Metrics are computed in FP64 on the host (grid.rs:65-119) and stored as FP32. */
int bowshock_solver_create(uint64_t ni, uint64_t nj, const double* x, const double* r, const bowshock_config* cfg, int device,
                           bowshock_solver** out);
/* drop (gpu/mod.rs, Drop of LazySolver) */
void bowshock_solver_destroy(bowshock_solver* s);
/* GpuError text of the last failed call on this handle */
const char* bowshock_solver_last_error(const bowshock_solver* s);
/* GpuSolver::ni / nj fields (gpu/mod.rs:237-238) */
int bowshock_solver_dims(const bowshock_solver* s, uint64_t* ni, uint64_t* nj);
/* GpuSolver::set_config (gpu/mod.rs:279-285): a boundary-condition change on a viscous run is refused (UNSUPPORTED) */
int bowshock_solver_set_config(bowshock_solver* s, const bowshock_config* cfg);
/* GpuSolver::set_low_mach (gpu/mod.rs:297-299) */
int bowshock_solver_set_low_mach(bowshock_solver* s, int on);
/* GpuSolver::set_block (gpu/mod.rs:302-308): NULL = no block; refused after set_viscous */
int bowshock_solver_set_block(bowshock_solver* s, const bowshock_block* block);
/* GpuSolver::set_nozzle (gpu/mod.rs:316-322): NULL = none; must follow set_block and precede set_viscous */
int bowshock_solver_set_nozzle(bowshock_solver* s, const bowshock_nozzle* nozzle);
/* GpuSolver::set_scheme (gpu/mod.rs:331-337): explicit or implicit; the CFL ramp restarts */
int bowshock_solver_set_scheme(bowshock_solver* s, const bowshock_scheme* scheme);
/* GpuSolver::set_viscous (gpu/mod.rs:351-357): NULL = Euler; the turbulence state restarts at the free stream, the wall
 * distance is computed on the device; roughness must be finite and >= 0 (INVALID otherwise) */
int bowshock_solver_set_viscous(bowshock_solver* s, const bowshock_viscous* v);
/* GpuSolver::set_state (gpu/mod.rs:378-381): overwrite the conserved state, restart the iteration counter and the ramp */
int bowshock_solver_set_state(bowshock_solver* s, const double* u);
/* GpuSolver::reset (gpu/mod.rs:384-387) */
int bowshock_solver_reset(bowshock_solver* s);
/* GpuSolver::state_f64 (gpu/mod.rs:390-392) */
int bowshock_solver_state(const bowshock_solver* s, double* u);
/* GpuSolver::turb_state (gpu/mod.rs:365-370): (k, omega) per cell and mu_t per cell; UNSUPPORTED without SST */
int bowshock_solver_turb_state(const bowshock_solver* s, double* turb, double* mu_t);
/* LazySolver::from_host's copy of the host turbulence state (gpu/mod.rs:251-263): set (k, omega) and mu_t */
int bowshock_solver_set_turb(bowshock_solver* s, const double* turb, const double* mu_t);
/* GpuSolver::iter / set_iter / restart_ramp (gpu/mod.rs:288-294, 344-347) */
int bowshock_solver_iter(const bowshock_solver* s, uint64_t* iter);
int bowshock_solver_set_iter(bowshock_solver* s, uint64_t iter);
int bowshock_solver_restart_ramp(bowshock_solver* s);
/* No counterpart in the reference (whose ramp only restarts): continue the CFL ramp from `ramp_k` iterations, for a
 * state handed over mid-run from another solver (implicit.rs:602). */
int bowshock_solver_set_ramp(bowshock_solver* s, uint64_t ramp_k);
/* GpuSolver::run (gpu/mod.rs:396-398): n iterations; residual[k] = density residual (L2 of d rho/dt over sqrt(n_active))
 * at the start of iteration k, accumulated in FP64 on the device. residual may be NULL. */
int bowshock_solver_run(bowshock_solver* s, uint64_t n, double* residual);
/* Solver::eval_residual + density_residual (solver.rs:474-654) of the current state without advancing it: the per-cell
 * residual (ni*nj*4) and local time step (ni*nj; explicit definition when compute_dt = 1), either output may be NULL */
int bowshock_solver_eval_residual(bowshock_solver* s, int compute_dt, double* res, double* dt, double* density_residual);
/* GpuSolver::turb_residual (gpu/mod.rs:373-375) */
int bowshock_solver_turb_residual(const bowshock_solver* s, double* r);
/* GpuSolver::read_boundary_into (gpu/mod.rs:401-404): the wall / base stencil cells (rows col_start(i), col_start(i)+1
 * and the two columns behind the base) of the conserved state into u (ni*nj*4); other cells are left untouched */
int bowshock_solver_read_boundary(const bowshock_solver* s, double* u);
/* GpuSolver::base_cells (gpu/mod.rs:408-413): [(i_end, j), (i_end+1, j)] conserved states for j in j_sting..j_end */
int bowshock_solver_base_cells(const bowshock_solver* s, double* out);

/* ---------------------------------------------------------------------------------------------- bodies and forces */
#define BOWSHOCK_NOSE_TANGENT_OGIVE 0
#define BOWSHOCK_NOSE_CONE 1
#define BOWSHOCK_NOSE_POWER 2
#define BOWSHOCK_NOSE_PARABOLIC 3
#define BOWSHOCK_NOSE_HAACK 4
#define BOWSHOCK_MAX_SEGMENTS 8

/* body_grid.rs:31-43, 233-251 `Nose`, `Segment`, `BaseBody` (lengths in nose diameters; param = power n, parabolic K or
 * Haack C) */
typedef struct {
  int32_t nose_kind;
  double fineness, half_angle, param;
  int32_t nseg;
  double seg_length[BOWSHOCK_MAX_SEGMENTS], seg_slope[BOWSHOCK_MAX_SEGMENTS];
  double sting_radius;
} bowshock_body;

/* Force integration of the current state (engine/run.rs:188-313), computed in FP64 on the device. */
typedef struct {
  double cd_nose, cd_nose_cell, cd_base, cp_base, cp_base_cell, cd_friction, y_plus_max;
  double cd_aft[BOWSHOCK_MAX_SEGMENTS];
  double cd_total; /* nose + aft segments + friction + base */
} bowshock_forces;

/* engine/run.rs:188-313 (wall_distribution, aft_drag, base_state, friction) on the device, in FP64 */
int bowshock_solver_forces(bowshock_solver* s, const bowshock_body* body, bowshock_forces* out);

/* ---------------------------------------------------------------------------------------------- run to a stop rule */
#define BOWSHOCK_WAKE_STING 0
#define BOWSHOCK_WAKE_BASE 1
#define BOWSHOCK_STOP_MAX_ITERATIONS 0
#define BOWSHOCK_STOP_RESIDUAL_DROP 1
#define BOWSHOCK_STOP_CD_STATIONARY 2
#define BOWSHOCK_STOP_BASE_PRESSURE_STATIONARY 3
#define BOWSHOCK_STOP_MEAN_STATIONARY 4
#define BOWSHOCK_STOP_NON_FINITE 5
#define BOWSHOCK_STOP_CANCELLED 6

/* The stop-rule part of numerics.rs:261-287 `Numerics` and the arguments of engine/run.rs:44 `run_on`. */
typedef struct {
  uint64_t max_iter, min_iter;
  double drop_orders;
  uint64_t monitor_window;
  int32_t has_monitor_tol;
  double monitor_tol;
  int32_t has_mean_window;
  uint64_t mean_window;
  int32_t has_drag_rel_tol;
  double drag_rel_tol;
  int32_t wake;    /* BOWSHOCK_WAKE_* */
  int32_t warm;    /* keep the state; no first-order start-up (run.rs:54-63) */
  double r_ref;    /* residual reference of the drop rule; < 0: the run's own peak */
} bowshock_run_params;

/* engine/result.rs `PointResult` (the scalar fields) */
typedef struct {
  uint64_t iters;
  double residual_peak, drop_orders;
  int32_t stop_reason;
  bowshock_forces forces;
  double last_monitor;
  /* a run stopped on a limit cycle (mean stationary): the mean of the monitored CD over the last window the rule compared
   * (6,000 iterations on the cycle); otherwise the final total CD. Not in the reference: the instantaneous CD of a limit
   * cycle depends on the phase, and a mean that reaches back to the start-up transient on the chunk the rule holds. */
  double cd_window;
} bowshock_point_result;

/* Progress callback, called between chunks of 50 iterations (progress.rs:1-8); return non-zero to cancel. */
typedef int (*bowshock_progress_fn)(void* user, uint64_t case_index, uint64_t iteration, double residual, double monitor);

/* engine/gpu.rs:86-169 `GpuRunner::run_on`: iterate in chunks of 50 to the stop rules of engine/run.rs:105-170 (stop
 * iteration CPU-equivalent inside a chunk), the monitor sampled every 50 iterations by the FP64 force pass, then the
 * forces of the final state. residual (cap entries) may be NULL. */
int bowshock_solver_run_to_stop(bowshock_solver* s, const bowshock_body* body, const bowshock_run_params* p, bowshock_point_result* out,
                                double* residual, uint64_t cap, bowshock_progress_fn progress, void* user);

/* ---------------------------------------------------------------------------------------------- mesher */
/* body_grid.rs:330-355 `BaseGridParams` (power-off) and body_grid.rs:112-131 `LargeGridParams` */
typedef struct {
  double x_up, x_down, r_far;
  uint64_t n_up, n_nose, n_seg[BOWSHOCK_MAX_SEGMENTS], n_wake, n_sting, n_gap, nj_out;
  double dx_tip, dr_wall;
  int32_t gap_one_sided;
} bowshock_base_grid;
typedef struct {
  double x_up, x_down, r_far;
  uint64_t n_up, n_nose, n_seg[BOWSHOCK_MAX_SEGMENTS], n_ext, nj;
  double dx_tip, dr_wall;
} bowshock_sting_grid;

/* body_grid.rs:360-452 `base_domain_grid`: node coordinates and the solid block. Call with x = r = NULL to get ni, nj. */
int bowshock_base_domain_grid(const bowshock_body* body, const bowshock_base_grid* p, uint64_t* ni, uint64_t* nj, double* x, double* r,
                              bowshock_block* block);
/* body_grid.rs:213-231 `large_domain_grid` (sting wake). Call with x = r = NULL to get ni, nj. */
int bowshock_large_domain_grid(const bowshock_body* body, const bowshock_sting_grid* p, uint64_t* ni, uint64_t* nj, double* x, double* r);

/* ---------------------------------------------------------------------------------------------- device mesher
 * No counterpart in the reference (its mesher is host code, one case at a time): the grids of many cases built on the
 * GPU — the 1D node distributions with their bisections (one warp per case), the nodes (a thread per node) and the FP64
 * metrics of every face and cell (a thread per face or cell, grid.rs:65-119). The arithmetic follows the host mesher
 * above operation by operation without multiply-add contraction; nodes and metrics differ from it only where the
 * device's tanh, tan, pow, acos, sin and hypot round differently from the host C library (an ulp or two). */
typedef struct {
  int32_t wake;               /* BOWSHOCK_WAKE_BASE: base_domain_grid; BOWSHOCK_WAKE_STING: large_domain_grid */
  bowshock_body body;
  bowshock_base_grid base;    /* read when wake = BOWSHOCK_WAKE_BASE */
  bowshock_sting_grid sting;  /* read when wake = BOWSHOCK_WAKE_STING */
} bowshock_mesh_request;
/* FP64 words of one case's metrics: i faces [nx, nr, len, r_mid] ((ni+1) nj each), j faces [nx, nr, len, r_mid]
 * (ni (nj+1) each), cells [area, volume per radian, xc, rc] (ni nj each), every array row-major (j, i). */
#define BOWSHOCK_MESH_METRIC_WORDS(ni, nj) (4 * (((ni) + 1) * (nj) + (ni) * ((nj) + 1) + (ni) * (nj)))
/* ni, nj and the solid block (zero for a sting grid) of a request, after the host mesher's argument checks (INVALID
 * where it would refuse the request); host arithmetic only. */
int bowshock_mesh_dims(const bowshock_mesh_request* q, uint64_t* ni, uint64_t* nj, bowshock_block* block);
/* The grids of n requests built on the device: x, r (host, case k's (ni+1)(nj+1) nodes after those of the cases before
 * it) and, if metrics is not NULL, BOWSHOCK_MESH_METRIC_WORDS per case in the same order; device_ms (may be NULL): the
 * device time of the three launches. INVALID for a refused request or a non-positive cell area. */
int bowshock_mesh_batch(uint64_t n, const bowshock_mesh_request* q, int device, double* x, double* r, double* metrics, double* device_ms);

/* ---------------------------------------------------------------------------------------------- batched case arena
 * No counterpart in the reference (it runs Mach points one at a time, analysis.rs:727-797): many cases with uneven grids
 * packed into one structure-of-arrays arena, every kernel launched once per iteration for all of them, per-case
 * convergence masks. The per-case numerics are those of the single-case solver. */
typedef struct {
  uint64_t ni, nj;
  const double *x, *r;
  bowshock_config cfg;
  int32_t low_mach;
  int32_t has_block;
  bowshock_block block;
  bowshock_scheme scheme; /* implicit for every case of an arena */
  int32_t has_viscous;
  bowshock_viscous viscous;
  bowshock_body body;
  bowshock_run_params run;
} bowshock_case_desc;
/* Distance of every cell centroid of one arena case to the nearest no-slip wall face, FP64 (turbulence.rs:91-125,
 * `wall_distance`), computed on the host with no device: the minimum over every wall segment of the clamped projection
 * distance, segments skipped only where their bounding box lies beyond the current minimum by a margin far above
 * rounding (the result is bit for bit that of the full search). The SST cases of an arena use it (computed once per
 * case). out: ni * nj values (row j, column i at j * ni + i); +inf for solid cells and where the case has no wall.
 * INVALID for a descriptor the arena would refuse. */
int bowshock_case_wall_distance(const bowshock_case_desc* d, double* out);

typedef struct bowshock_arena bowshock_arena;
int bowshock_arena_create(uint64_t ncases, const bowshock_case_desc* cases, int device, bowshock_arena** out);
/* bowshock_arena_create with every case's grid built on the device from meshes[k] (body -> nodes -> metrics, the device
 * mesher above) instead of from host nodes: cases[k].x and .r are ignored (may be NULL), cases[k].ni, .nj and the block
 * must be those of meshes[k] (bowshock_mesh_dims). */
int bowshock_arena_create_meshed(uint64_t ncases, const bowshock_case_desc* cases, const bowshock_mesh_request* meshes, int device,
                                 bowshock_arena** out);
void bowshock_arena_destroy(bowshock_arena* a);
const char* bowshock_arena_last_error(const bowshock_arena* a);
/* cells of all cases */
int bowshock_arena_cells(const bowshock_arena* a, uint64_t* ncells);
/* n iterations of every active case; residual (n x ncases, iteration-major) may be NULL */
int bowshock_arena_run(bowshock_arena* a, uint64_t n, double* residual);
/* Capture and instantiate the CUDA graph that bowshock_arena_run(a, n, ...) launches first (a chunk of min(n, 256)
 * iterations), without running anything: a following run of n iterations then spends no host time on graph
 * construction (the graph is rebuilt after a change of the active cases or the launch shapes). No counterpart in the
 * reference. */
int bowshock_arena_prepare(bowshock_arena* a, uint64_t n);
/* cold-start every case and iterate each to its stop rule, masking converged cases out; results per case */
int bowshock_arena_solve(bowshock_arena* a, bowshock_point_result* results, bowshock_progress_fn progress, void* user);
/* FP64 forces of every case's current state (ncases entries) */
int bowshock_arena_forces(bowshock_arena* a, bowshock_forces* out);
int bowshock_arena_state(const bowshock_arena* a, uint64_t k, double* u);
int bowshock_arena_set_state(bowshock_arena* a, uint64_t k, const double* u);
/* Per-case run parameters for the next bowshock_arena_solve (replacing the descriptor's): a warm start (warm = 1 keeps
 * the state and turbulence set through bowshock_arena_set_state / bowshock_arena_set_turb, no first-order start-up, drop
 * measured from r_ref; run.rs:54-63). No counterpart in the reference (its runs are one solver each). */
int bowshock_arena_set_run(bowshock_arena* a, uint64_t k, const bowshock_run_params* p);
/* (k, omega) and mu_t of SST case k (ni*nj*2 and ni*nj doubles; either may be NULL); UNSUPPORTED for other cases */
int bowshock_arena_turb_state(const bowshock_arena* a, uint64_t k, double* turb, double* mu_t);
int bowshock_arena_set_turb(bowshock_arena* a, uint64_t k, const double* turb, const double* mu_t);
/* The density residual every case's run would see first from its current state (FP64): with warm[k] != 0 as a warm run
 * (second-order reconstruction from the first iteration), else as a cold run's first iteration (first order); warm may
 * be NULL (all cold). The iteration counters are left as a run would start them. */
int bowshock_arena_first_residuals(bowshock_arena* a, const int32_t* warm, double* out);
/* The density residual of every iteration of case k in the last bowshock_arena_solve (n entries; at most cap copied into
 * out, which may be NULL to query n): the history GpuRunner::run_on keeps per run (engine/gpu.rs:143-158). */
int bowshock_arena_residual_history(const bowshock_arena* a, uint64_t k, double* out, uint64_t cap, uint64_t* n);
/* Where bowshock_arena_solve evaluates the stop rules (engine/run.rs:105-170): on the device after every 50-iteration
 * chunk (1, the default: one thread per case restates the rules, the host reads back each case's status), or on the
 * host from the read-back residuals and monitor (0, as engine/gpu.rs:123-164 does). The decisions are the same; a
 * mean window beyond 6,400 iterations always runs on the host. No counterpart in the reference. */
int bowshock_arena_set_run_control(bowshock_arena* a, int on_device);
/* per-case activity mask (1 = iterate), ncases entries */
int bowshock_arena_set_active(bowshock_arena* a, const int32_t* active);
/* mean device time of one arena iteration over the last bowshock_arena_run, in milliseconds (CUDA events) */
int bowshock_arena_last_ms_per_iter(const bowshock_arena* a, double* ms);
/* device time of the last bowshock_arena_solve in milliseconds: every iteration chunk and FP64 force pass, CUDA events
 * around each (host-side stop-rule checks between chunks excluded) */
int bowshock_arena_last_solve_ms(const bowshock_arena* a, double* ms);

/* Per-kernel profile (the reference's Profile of gpu/mod.rs:533-542): n iterations launched one kernel at a time with CUDA
 * events around each launch; per kernel group (prims, viscous, residual, i-lines, j-lines (the factorising first pass),
 * defect, turbulence, stage (and residual smoothing), i- and j-substitution passes, block assembly, SST line systems,
 * multigrid transfers) the total milliseconds and launch counts (BOWSHOCK_PROFILE_GROUPS entries each). */
#define BOWSHOCK_PROFILE_GROUPS 13
int bowshock_arena_profile(bowshock_arena* a, uint64_t n, double* ms, uint64_t* launches);
/* bowshock_arena_set_run_control for bowshock_solver_run_to_stop */
int bowshock_solver_set_run_control(bowshock_solver* s, int on_device);
/* the same profile of a single-case solver (any scheme, multigrid levels included) */
int bowshock_solver_profile(bowshock_solver* s, uint64_t n, double* ms, uint64_t* launches);
/* Launch shapes of the arena's kernels. At creation (arenas of 100,000 cells or more; otherwise 4 lines per block, no
 * prefetching) the autotuner picks, each the fastest in one timed iteration of the arena's own cases per
 * candidate (the state restored afterwards): per direction, lines per block (1, 2 or 4) of the block line solves' first
 * pass and how its walks fetch the cells' records (0: one cell at a time, 1: the next cell's ahead; 2, staged through
 * shared memory three cells ahead with one line per block, only when pinned), lines per block (1, 2, 4 or 8) of their
 * substitution passes and how those walks fetch their records (0 / 1 / 2 likewise), lines per block of the SST line
 * kernel; the residual kernel's variant (0: 256 threads per 32 x 8 tile, 1: 288) stays 1 unless pinned (the two round
 * differently). A direction with at most
 * staged_lines lines left in the launch (set at creation to two waves of the staged substitution kernel: 1,184 lines on
 * a 148-SM B200; >= 0, 0 never) runs both passes staged whatever prefetch / subst_prefetch say: with few lines the
 * walks wait on memory latency. Every candidate compiles to the same arithmetic (checked bit for bit), so none of these
 * changes a result. The smallest segment a lane eliminates per direction (segment_i / segment_j: 2, 4 or 8 cells;
 * fewer separators on short lines) is 2 unless pinned: it changes the rounding of the line solves. No counterpart in
 * the reference (its line solves run in Luma, gpu/implicit.rs:731-732). */
typedef struct {
  int32_t lines_i, lines_j, prefetch_i, prefetch_j, subst_i, subst_j, turb_lines, segment_i, segment_j, residual, subst_prefetch_i,
      subst_prefetch_j, staged_lines;
} bowshock_line_tuning;
int bowshock_arena_tuning(const bowshock_arena* a, bowshock_line_tuning* out);
/* Pin the launch shapes instead of the autotuner's (for reproducible runs: the segment lengths change the order of
 * rounding in the line solves, not their fixed point; the other fields change nothing in the results). Values out of
 * their ranges above give INVALID. No counterpart in the reference. */
int bowshock_arena_set_tuning(bowshock_arena* a, const bowshock_line_tuning* t);
/* No counterpart in the reference. groups (1 to 4, default 1): the active cases are split into that many groups of
 * about equal cells and each group's iterations form an independent chain in the chunk's CUDA graph, so the groups'
 * kernels run side by side; the states are those of one group bit for bit (every kernel touches only its own cases),
 * what changes is how many warps are in flight when few cases are left. */
int bowshock_arena_set_case_groups(bowshock_arena* a, int groups);
/* SST line systems (the reference couples k and omega loosely, turbulence.rs:542-611).
 * coupled = 0 (default): the reference's scheme, the mean flow's 4x4 lines and then the two scalar line systems of k and
 * omega. coupled = 1: the 6x6 block lines of (dU, dk, domega). The mean-flow operator freezes mu_t, so each 6x6 block
 * is lower block-triangular and the system is solved exactly by the 4x4 lines followed by the scalar lines with the
 * turbulence rows' coupling to dU (face mass fluxes, density in the sources) on their right-hand side. The residuals are
 * the reference's, so the converged state is the same; the iteration path is not. Takes effect from the next chunk. */
int bowshock_arena_set_sst_coupling(bowshock_arena* a, int coupled);
int bowshock_solver_set_sst_coupling(bowshock_solver* s, int coupled);
/* No counterpart in the reference. FAS multigrid transfers (multigrid.rs:115-171): on (default 1) the restriction of the
 * state is folded into the coarse level's primitives kernel and the forcing into its residual kernel; 0
 * launches the separate transfer kernels in the reference's order. The states are the same bit for bit. */
int bowshock_solver_set_mg_fusion(bowshock_solver* s, int on);

/* ---------------------------------------------------------------------------------------------- 3D Euler
 * The stability path (crates/bowshock-cfd/src/solver3.rs + implicit3.rs behind `GpuSolver3`, gpu/mod.rs:442-560, driven
 * by engine/run3.rs): a batch of cases (Mach number, incidence) on one shared 3D grid. Nodes (ni+1)(nj+1)(nk+1), index
 * (k*(nj+1)+j)*(ni+1)+i; j = 0 is the axis for i < axis_cells and the body wall beyond, j = nj and the i ends the far
 * field, k = 0 and k = nk symmetry planes (a half body revolved over [0, pi]). Fins are solid boxes of cells
 * (bowshock3_set_solid). */
typedef struct {
  double mach, alpha;       /* incidence [rad]: the air moves towards +z (gas3.rs:42-44) */
  double cfl;               /* CFL of the explicit scheme */
  int32_t limiter, low_mach;
  uint64_t first_order_iters;
  bowshock_scheme scheme;   /* BOWSHOCK_SCHEME_EXPLICIT or BOWSHOCK_SCHEME_IMPLICIT (three-factor, 5x5 blocks) */
} bowshock3_config;
typedef struct {            /* run3.rs:220-330 stop rules */
  uint64_t max_iter;
  double rel_tol;           /* CN stationary: range over the window below rel_tol |mean| */
  uint64_t window;          /* iterations, a multiple of 50 */
  double x_max;             /* wall faces with centroid x <= x_max carry the forces (the base station) */
} bowshock3_run_params;
typedef struct {            /* run3.rs `PointResult3` (scalars) */
  double cn, ca, x_cp;
  uint64_t iterations;
  int32_t stop_reason;      /* 0 max iterations, 1 residual drop, 2 CN stationary, 5 non-finite */
  double drop_orders;
} bowshock3_result;
typedef struct bowshock3_batch bowshock3_batch;
int bowshock3_create(uint64_t ni, uint64_t nj, uint64_t nk, const double* x, const double* y, const double* z, uint64_t axis_cells,
                     uint64_t ncases, const bowshock3_config* cfg, int device, bowshock3_batch** out);
void bowshock3_destroy(bowshock3_batch* b);
const char* bowshock3_last_error(const bowshock3_batch* b);
/* every case back to its free stream at iteration 0 (GpuSolver3::reset) */
int bowshock3_reset(bowshock3_batch* b);
/* GpuSolver3::set_config (gpu/mod.rs:482-487) for case k: free stream (Mach, incidence), CFL, limiter, first-order
 * iterations and the low-Mach flag may change between runs without touching the state; a changed scheme restarts the
 * case's CFL ramp. The batch runs one scheme: the explicit / implicit kind changes only for a batch of one case
 * (UNSUPPORTED otherwise). */
int bowshock3_set_config(bowshock3_batch* b, uint64_t k, const bowshock3_config* cfg);
/* Per-kernel profile (GpuSolver3::profile_step / profile_replay, gpu/mod.rs:525-535): n iterations launched one kernel
 * at a time with CUDA events around each; per group (primitives and ghosts, face fluxes, residual, assembly, first line
 * pass, substitution passes, defect, RK3 stage) the total milliseconds and launch counts, BOWSHOCK3_PROFILE_GROUPS each. */
#define BOWSHOCK3_PROFILE_GROUPS 8
int bowshock3_profile(bowshock3_batch* b, uint64_t n, double* ms, uint64_t* launches);
/* Solid boxes of the shared grid (crates/bowshock-cfd/src/grid3.rs:17-24 `SolidBox`, the fins; `Grid3::solid`, read by
 * Solver3::new, solver3.rs:84-97): 6 per box, i0 i1 j0 j1 k0 k1, half-open cell ranges; nbox 0 removes them. Solid cells
 * are never updated and act as slip walls (solver3.rs:362-405, implicit3.rs:14-16); the density norm runs over the fluid
 * cells; the forces add every face between a fluid and a solid cell (run3.rs:130-212). Resets every case to its free
 * stream. INVALID for an empty box or one outside the grid. */
int bowshock3_set_solid(bowshock3_batch* b, uint64_t nbox, const uint64_t* boxes);
/* No counterpart in the reference. on (default 1): the first line pass stages its walk through shared memory where a
 * warp's 32 lines are adjacent (i lines: nj a multiple of 32; j and k lines: ni a multiple of 32); 0 pins the unstaged
 * walk. The results are the same bit for bit; only the speed differs. */
int bowshock3_set_staging(bowshock3_batch* b, int on);
/* No counterpart in the reference. groups (1 to 4, at most the case count; default 1): the cases split into that many
 * groups of consecutive cases whose iterations run on streams of their own, so one group's kernels fill the SMs while
 * another's last wave runs. The states are the same bit for bit. INVALID out of range. */
int bowshock3_set_groups(bowshock3_batch* b, int groups);
/* iteration counter (first-order start-up) and CFL-ramp counter of every case */
int bowshock3_set_iter(bowshock3_batch* b, uint64_t iter, uint64_t ramp);
/* conserved state of case k, ni*nj*nk x 5 (Solver3::u layout) */
int bowshock3_set_state(bowshock3_batch* b, uint64_t k, const double* u);
int bowshock3_state(bowshock3_batch* b, uint64_t k, double* u);
/* GpuSolver3::read_boundary_into (gpu/mod.rs:519-523): only the cells the force integration reads (the first fluid cell
 * of every wall and fin face and the one behind it) of case k into u (ncell x 5, the layout of bowshock3_state); the
 * other entries of u are left as they are */
int bowshock3_read_boundary(bowshock3_batch* b, uint64_t k, double* u);
/* n iterations of every active case; residual (n x ncases, iteration-major) may be NULL (GpuSolver3::run) */
int bowshock3_run(bowshock3_batch* b, uint64_t n, double* residual);
/* residual (ncell x 5) and time step of case k for the current state (no update); density residual of case k */
int bowshock3_eval_residual(bowshock3_batch* b, uint64_t k, double* res, double* dt, double* density_residual);
/* run3.rs:85-127 `breakdown_on` / `LiftBreakdown`: the same forces split into 5 parts, nose (body wall with centroid
 * x <= x_nose), afterbody, fin sides (k faces of the solid boxes), fin edges (i faces) and fin tips (j faces); out:
 * (cn, ca, x_cp) x 5 parts x ncases, x_cp NaN where a part's normal force is below 1e-12 */
int bowshock3_forces_parts(bowshock3_batch* b, double x_max, double x_nose, double* out);
/* FP64 pressure forces of every case: (cn, ca, x_cp) x ncases (run3.rs `forces_on`: body wall and fin faces) */
int bowshock3_forces(bowshock3_batch* b, double x_max, double* out);
/* cold start of every case, iterated to the stop rules with per-case masks (run3.rs:220-330) */
int bowshock3_solve(bowshock3_batch* b, const bowshock3_run_params* p, bowshock3_result* out);
int bowshock3_last_ms_per_iter(const bowshock3_batch* b, double* ms);

/* ---------------------------------------------------------------------------------------------- learned warm start
 * No counterpart in the reference (its only warm start is the previous Mach point's field, crates/bowshock-core/src/engine/
 * run.rs:54-63, analysis.rs:744-748). A conv decoder (about 1.84 M parameters) maps BOWSHOCK_NET_IN inputs (12 geometry
 * parameters, the Mach number and log10 of the Reynolds number, zero-padded to 16) to BOWSHOCK_NET_OUT channels on the
 * 64 x 32 coarse level of the normalized 128 x 64 body-fitted grid (BOWSHOCK_NET_CELLS cells, row j = 0..31 of 64 columns
 * i, channel fastest). Layers: fully connected 16 -> 256 -> 4 x 8 x 128, then 3x3 convolutions with leaky ReLU (slope
 * 0.1) at 4 x 8 (128 -> 128, twice), 8 x 16 (nearest 2x upsampling, 128 -> 128, twice), 16 x 32 (up, 128 -> 64, 64 -> 64),
 * 32 x 64 (up, 64 -> 64, twice) and a linear 3x3 output convolution 64 -> 16 of which the first 6 channels are the
 * prediction. Every contraction, forward and backward, is a BF16 tcgen05 GEMM with FP32 accumulation in TMEM; weights are
 * FP32 masters trained by Adam (lr given, betas 0.9 / 0.999, eps 1e-8) on the masked mean squared error. The parameter
 * vector is, per layer in order, W [cout][kin] (kin = cin for a fully connected layer, 9 cin for a convolution with
 * column (ky*3 + kx)*cin + c) then b [cout], each layer's block padded to a multiple of 8 floats (bowshock_net_layout). */
#define BOWSHOCK_NET_IN 16
#define BOWSHOCK_NET_OUT 6
#define BOWSHOCK_NET_OUT_PAD 16
#define BOWSHOCK_NET_CELLS 2048
#define BOWSHOCK_NET_SLOPE 0.1f
typedef struct bowshock_net bowshock_net;
/* max_batch: a multiple of 8 (at most 4096); the buffers of every layer are sized for it */
int bowshock_net_create(int device, uint64_t max_batch, bowshock_net** out);
void bowshock_net_destroy(bowshock_net* n);
const char* bowshock_net_last_error(const bowshock_net* n);
int bowshock_net_num_params(const bowshock_net* n, uint64_t* nparams);
/* 9 integers per layer (fully connected, cin, cout, H, W, upsampled, activated, W offset, b offset) into out (cap entries) */
int bowshock_net_layout(const bowshock_net* n, int64_t* out, uint64_t cap, uint64_t* nlayers);
int bowshock_net_set_params(bowshock_net* n, const float* params);
int bowshock_net_get_params(bowshock_net* n, float* params);
/* fluid mask of the coarse cells (BOWSHOCK_NET_CELLS bytes, nonzero = fluid): the loss counts only these */
int bowshock_net_set_mask(bowshock_net* n, const uint8_t* mask);
/* y [batch][BOWSHOCK_NET_CELLS][BOWSHOCK_NET_OUT] from x [batch][BOWSHOCK_NET_IN] (host arrays) */
int bowshock_net_forward(bowshock_net* n, uint64_t batch, const float* x, float* y);
/* loss and its gradient with respect to every parameter (grad: num_params floats, may be NULL) for one batch (a multiple
 * of 8, at most max_batch) of inputs x and targets [batch][BOWSHOCK_NET_CELLS][BOWSHOCK_NET_OUT]; no update */
int bowshock_net_gradients(bowshock_net* n, uint64_t batch, const float* x, const float* target, float* grad, double* loss);
/* the training set, kept on the device: x [n][BOWSHOCK_NET_IN], target [n][BOWSHOCK_NET_CELLS][BOWSHOCK_NET_OUT] */
int bowshock_net_set_dataset(bowshock_net* n, uint64_t n_samples, const float* x, const float* target);
int bowshock_net_reset_optimizer(bowshock_net* n);
/* `steps` Adam steps on batches from epochs of a seeded shuffle of the dataset; loss (steps entries, may be NULL) */
int bowshock_net_train(bowshock_net* n, uint64_t steps, uint64_t batch, double lr, uint64_t seed, double* loss);
/* device time of the last bowshock_net_train (CUDA events), milliseconds */
int bowshock_net_last_train_ms(const bowshock_net* n, double* ms);
/* How the network runs its 3x3 convolutions with a multiple of 64 input channels (forward and input gradient): 2 (the
 * default) implicit GEMMs whose A tiles are 4D TMA boxes of the NHWC activations shifted by the tap (zeros outside the
 * image; an upsampling layer's input is upsampled into a buffer first), 1 implicit GEMMs whose A tiles are gathered by
 * cp.async into the swizzled layout, 0 an im2col matrix + the TMA-fed GEMM. All three feed the tensor cores the same K
 * blocks in the same order (the same sums). */
int bowshock_net_set_conv_mode(bowshock_net* n, int mode);
/* The network's implicit-GEMM convolution on caller-owned device memory: d[p][o] (FP32, p over batch x H x W output
 * pixels, H = h_in << up, W = w_in << up) = sum over the 3x3 taps and c channels of x[pixel shifted by the tap][ch]
 * w[o][tap * c + ch], x NHWC BF16 [batch][h_in][w_in][c] (c a multiple of 64, read through a nearest 2x upsampling when
 * up = 1, zeros outside the image), w BF16 [n][9 c]. mode 1: A gathered by cp.async; mode 2: A by TMA boxes (up = 0, and
 * W dividing 128 with H W a multiple or a divisor of 128). */
int bowshock_conv3x3_bf16(const void* x, int64_t batch, int64_t h_in, int64_t w_in, int64_t c, int64_t up, const void* w, int64_t n, float* d,
                          int32_t mode, void* stream, int* err_flag);
/* 1 (the default): GEMMs without a K split (the network's forward and input-gradient GEMMs, bowshock_gemm_bf16 with
 * splits = 1) run the persistent kernel (at most SMs x resident CTAs, each looping over tiles with two TMEM
 * accumulators so that one tile's epilogue overlaps the next tile's MMAs); 0: one CTA per tile. Same results.
 * Process-wide; returns the previous setting. */
int bowshock_gemm_set_persistent(int on);
/* The network's tensor-core GEMM on caller-owned device memory: d[m][n] = sum_k a[m][k] b[n][k], a and b BF16 row-major
 * (lda, ldb multiples of 8 elements, 16-byte aligned), d FP32 (ldd >= n); splits > 1 adds K slices atomically into d
 * (zeroed by the caller). stream: a cudaStream_t or NULL; err_flag: a device int set to 1 if a bounded wait gave up. */
int bowshock_gemm_bf16(const void* a, int64_t lda, const void* b, int64_t ldb, float* d, int64_t ldd, int64_t m, int64_t n, int64_t k,
                       int64_t splits, void* stream, int* err_flag);

/* bowshock_solver_run without any device allocation. No counterpart in the reference. For hosts that create their solvers
 * up front and then step them from code that may not allocate device memory: the GPU's free memory belongs to the host's
 * own pool (another framework's caching allocator on the same device), or the stepping loop cannot take the device-wide
 * synchronisation an allocation may cause. bowshock_solver_run allocates on its first call (CUDA graph instantiation,
 * timing events); this variant launches the same kernels directly on the solver's stream and takes the line solves'
 * records (blocks, factors, reduction multipliers) from a static 64 MiB device array of the library. A solver needs
 * BOWSHOCK_NOALLOC_BYTES(cells, lines) of it, cells and i + j lines of all multigrid levels counted (about 60,000 cells
 * for a single-level grid of aspect 2); a larger one gets BOWSHOCK_INVALID with a message and nothing is launched. Same residual
 * semantics and results as bowshock_solver_run (bit for bit), and bowshock_solver_turb_residual afterwards returns the
 * turbulence residual of its last iteration; the device time per iteration is not measured (no timing events).
 * The first call on a device looks the array's device address up (cudaGetSymbolAddress with that device current; a failed
 * lookup is retried by the next call); make that first call before any stream capture. Every call on a device shares the
 * array (nothing in it needs to start at zero); calls that overlap on one GPU, from solvers on other streams or threads,
 * race on it and must be serialised. As for every entry point, one solver must not be used from two host threads at once:
 * during this call the solver's launches point at the static array. */
#define BOWSHOCK_NOALLOC_SCRATCH_BYTES (64u << 20)
#define BOWSHOCK_NOALLOC_BYTES(cells, lines) (928ull * (unsigned long long)(cells) + 128ull + 22528ull * (unsigned long long)(lines))
int bowshock_solver_run_noalloc(bowshock_solver* s, uint64_t n, double* residual);

#ifdef __cplusplus
}
#endif
#endif /* BOWSHOCK_B200_H */
