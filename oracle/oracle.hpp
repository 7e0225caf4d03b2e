// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// f64 CPU restatement of the reference's axisymmetric finite-volume solver (crates/bowshock-cfd/src/{gas,grid,flux,bc,
// solver,implicit,multigrid,viscous,turbulence}.rs) and of the engine layer that drives it (crates/bowshock-core/src/
// engine/{body_grid,case,numerics,run}.rs, atmosphere.rs). It is the correctness oracle of the CUDA backend and the timed
// CPU baseline. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
//
// The reference is Rust and cannot be compiled in this environment (no rustc / cargo), so this is a restatement, written
// expression by expression in the reference's evaluation order; each function cites the reference file:line it follows.
// Parity of this restatement is pinned by ports of the reference's own unit tests (tests/test_oracle_*.py) and by the
// reference's published converged values of its G3 body (crates/bowshock-cfd/README.md:795-797).
#pragma once
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

namespace orc {

using Cons = std::array<double, 4>;
using Prim = std::array<double, 4>;
using M4 = std::array<double, 16>;

constexpr double GAMMA = 1.4;  // gas.rs:6
constexpr int NG = 2;          // solver.rs:195

// ---------------------------------------------------------------- gas.rs
Cons prim_to_cons(const Prim& w);                                    // gas.rs:12-16
Prim cons_to_prim(const Cons& q);                                    // gas.rs:18-24
double sound_speed(const Prim& w);                                   // gas.rs:27-29
Cons physical_flux(const Prim& w, double nx, double nr);             // gas.rs:33-38
Prim freestream(double mach);                                        // gas.rs:41-43
Prim reflect(const Prim& w, double nx, double nr);                   // gas.rs:47-50

// ---------------------------------------------------------------- grid.rs
struct Face {  // grid.rs:22-37
  double nx = 0, nr = 0, len = 0, rm = 0;
  double w() const { return len * rm; }
};

struct Grid {  // grid.rs:39-56
  size_t ni = 0, nj = 0;
  std::vector<double> x, r;
  std::vector<Face> iface, jface;
  std::vector<double> area, vol, xc, rc;
  std::pair<double, double> node(size_t i, size_t j) const {
    size_t k = j * (ni + 1) + i;
    return {x[k], r[k]};
  }
};
// grid.rs:65-119; returns false (and a message) on a non-positive cell area.
bool grid_from_nodes(size_t ni, size_t nj, std::vector<double> x, std::vector<double> r, Grid& out, std::string* err);
Grid grid_from_nodes_or_throw(size_t ni, size_t nj, std::vector<double> x, std::vector<double> r);
bool grid_coarsen(const Grid& g, Grid& out);                                // grid.rs:129-144
std::vector<double> geometric_offsets(double first, double length, size_t n);  // grid.rs:199-228

// ---------------------------------------------------------------- flux.rs
enum Limiter { FIRST_ORDER = 0, MINMOD = 1, VAN_ALBADA = 2, VENKATAKRISHNAN = 3 };
double limited_slope(double a, double b, int lim);                                            // flux.rs:18-50
void reconstruct(const Prim& m2, const Prim& m1, const Prim& p0, const Prim& p1, int lim, Prim& l, Prim& r);  // flux.rs:56-72
Cons hllc(const Prim& wl, const Prim& wr, double nx, double nr);                               // flux.rs:79-126
Cons rusanov(const Prim& wl, const Prim& wr, double nx, double nr);                            // flux.rs:132-147
constexpr double SHOCK_SENSOR_LO = 0.002, SHOCK_SENSOR_HI = 0.02;                               // flux.rs:151-152
double shock_weight(double pl, double pr);                                                     // flux.rs:158-162
Cons face_flux(const Prim& m2, const Prim& m1, const Prim& p0, const Prim& p1, int lim, double nx, double nr);  // flux.rs:173-186
constexpr double LOW_MACH_FLOOR = 0.05;                                                        // flux.rs:189
void low_mach_states(const Prim& l, const Prim& r, double nx, double nr, Prim& lo, Prim& ro);  // flux.rs:206-219
Cons face_flux_lm(const Prim& m2, const Prim& m1, const Prim& p0, const Prim& p1, int lim, double nx, double nr, bool low_mach);  // flux.rs:224-241

// ---------------------------------------------------------------- bc.rs
enum Regime { SUPERSONIC_INFLOW = 0, SUBSONIC_INFLOW = 1, SUBSONIC_OUTFLOW = 2, SUPERSONIC_OUTFLOW = 3 };
double normal_mach(const Prim& w, double nx, double nr);                                       // bc.rs:48-50
int regime(const Prim& interior, double nx, double nr);                                        // bc.rs:54-65
Prim characteristic_ghost(const Prim& fs, const Prim& interior, double nx, double nr, int* reg);  // bc.rs:69-93
Prim pressure_outflow_ghost(double p_back, const Prim& interior, double nx, double nr);        // bc.rs:97-103

// ---------------------------------------------------------------- solver.rs types
enum Bc { BC_FREESTREAM = 0, BC_EXTRAPOLATE = 1, BC_SLIPWALL = 2, BC_CHARACTERISTIC = 3, BC_PRESSURE_OUTFLOW = 4 };

struct Config {  // solver.rs:40-48
  double cfl = 0.5;
  int limiter = MINMOD;
  Prim freestream{1, 0, 0, 1.0 / GAMMA};
  int bc[4] = {BC_CHARACTERISTIC, BC_CHARACTERISTIC, BC_SLIPWALL, BC_CHARACTERISTIC};
  size_t first_order_iters = 0;
};

struct Block {  // solver.rs:59-102
  size_t i_end = 0, j_end = 0, j_sting = 0;
  bool solid(size_t i, size_t j) const { return i < i_end ? j < j_end : j < j_sting; }
  // row_start: SIZE_MAX when the whole row is solid
  size_t row_start(size_t j) const { return j < j_sting ? SIZE_MAX : (j < j_end ? i_end : 0); }
  size_t col_start(size_t i) const { return i < i_end ? j_end : j_sting; }
  bool coarsen(Block& out) const {
    if (i_end % 2 || j_end % 2 || j_sting % 2) return false;
    out = Block{i_end / 2, j_end / 2, j_sting / 2};
    return true;
  }
};

struct Irs {  // solver.rs:109-120
  double cfl_star = 0.0;
  bool on() const { return cfl_star > 0.0; }
};

struct MgParams {  // solver.rs:123-140
  size_t levels = 6, pre = 1, post = 1, gamma = 1, coarsest = 4;
  Irs irs{};
};

enum DtMode { DT_SUM = 0, DT_MIN_DIRECTION = 1 };
struct ImplicitParams {  // implicit.rs:59-84
  double cfl0 = 1.0, cfl_max = 30.0, growth = 1.02;
  int dt_mode = DT_SUM;
  bool lines = true, implicit_bc = true;
  size_t sub_iters = 2;
  bool roe = true;
  double eps_fix = 0.1;
};
ImplicitParams implicit_default();   // implicit.rs:79-80
ImplicitParams implicit_viscous();   // implicit.rs:83

enum SchemeKind { SCHEME_EXPLICIT = 0, SCHEME_SMOOTHED = 1, SCHEME_MULTIGRID = 2, SCHEME_IMPLICIT = 3 };
struct Scheme {  // solver.rs:143-153
  int kind = SCHEME_EXPLICIT;
  Irs irs{};
  MgParams mg{};
  ImplicitParams imp{};
};
bool scheme_eq(const Scheme& a, const Scheme& b);

enum Turbulence { TURB_LAMINAR = 0, TURB_SST = 1 };
struct Viscous {  // solver.rs:164-176, viscous.rs:45-57
  double re_c = 1e6, sutherland = 0.368;
  int turbulence = TURB_LAMINAR;
  size_t wall_i_start = 0;
  double roughness = 0.0;
  double mu(double t) const { return std::pow(t, 1.5) * (1.0 + sutherland) / (t + sutherland) / re_c; }
  bool rough() const { return turbulence == TURB_SST && roughness > 0.0; }
};
constexpr double PRANDTL = 0.72, PRANDTL_T = 0.9;  // solver.rs:179-181

struct Nozzle {  // solver.rs:186-193
  size_t j_end = 0;
  Prim state{};
  std::array<double, 2> turb{};
};

// ---------------------------------------------------------------- viscous.rs helpers
double temperature(const Prim& w);                                // viscous.rs:61-63
Prim wall_ghost(const Prim& w, const Face& f, bool noslip);       // viscous.rs:67-73

struct Walls {  // viscous.rs:83-128
  bool has_visc = false;
  Viscous visc{};
  bool jmin_slip = false;
  bool has_blk = false;
  Block blk{};
  bool has_nozzle = false;
  Nozzle nozzle{};
  bool noslip_jface(size_t i, size_t j) const;
  bool noslip_iface(size_t i, size_t j) const;
  bool rough_jface(size_t i, size_t j) const;
  bool jet_iface(size_t i, size_t j) const;
};

struct Side {  // viscous.rs:133-139
  Prim w{};
  size_t cell = 0;
  bool ghost = false;
  bool has_fixed = false;
  double fixed_mu = 0, fixed_mut = 0;
};
struct FaceSides {  // viscous.rs:143-147
  Side l, r;
  bool noslip = false;
};

// ---------------------------------------------------------------- the solver
struct Factor {  // implicit.rs:371-376
  std::vector<M4> lo, d, up;
};

struct Solver {  // solver.rs:197-255
  Grid grid;
  Config cfg;
  std::vector<Cons> u;
  std::vector<Prim> w;
  std::vector<Cons> fi, fj, res;
  std::vector<double> dt;
  std::vector<Cons> u0;
  size_t iter = 0;
  bool low_mach = false;
  bool has_block = false;
  Block block{};
  bool has_nozzle = false;
  Nozzle nozzle{};
  Scheme scheme{};
  Irs irs{};
  std::vector<Cons> forcing, mg_u0;
  std::vector<Solver> coarse;
  std::vector<double> irs_ei, irs_ej;
  size_t n_active = 0;
  size_t ramp_k = 0;
  bool has_viscous = false;
  Viscous viscous{};
  std::vector<std::array<double, 6>> grad;
  std::vector<double> mu, mu_t;
  std::vector<std::array<double, 3>> rough_wall;
  std::vector<Cons> fvi, fvj;
  std::vector<std::array<double, 2>> turb;
  std::vector<double> dwall;
  double turb_rnorm = 0.0;
  // implicit workspace (implicit.rs:497-525)
  Factor ws_fi, ws_fj;
  std::vector<Cons> ws_b, ws_du, ws_ai, ws_aj, ws_r, ws_corr;

  Solver() = default;
  Solver(Grid g, const Config& c);                       // solver.rs:263-304
  void set_block(const Block* b);                        // solver.rs:307-328
  void set_nozzle(const Nozzle* n);                      // solver.rs:333-344
  void set_viscous(const Viscous* v);                    // solver.rs:359-384
  size_t set_scheme(const Scheme& s);                    // multigrid.rs:29-64
  Walls walls() const;                                   // solver.rs:392-394
  bool sst() const { return has_viscous && viscous.turbulence == TURB_SST; }
  size_t pidx(long i, long j) const { return (size_t)(j + NG) * (grid.ni + 2 * NG) + (size_t)(i + NG); }
  Prim prim(size_t i, size_t j) const { return w[pidx((long)i, (long)j)]; }
  void fill_ghosts();                                    // solver.rs:423-452
  void fill_block_ghosts(const Block& b);                // solver.rs:457-471
  void eval_residual(bool compute_dt);                   // solver.rs:474-648
  double density_residual() const;                       // solver.rs:651-654
  double step();                                         // solver.rs:658-676
  double rk3_step();                                     // solver.rs:694-710
  void stage(double a, double b);                        // solver.rs:713-720
  void smooth_residual();                                // solver.rs:726-774
  double pressure(size_t i, size_t j) const { return cons_to_prim(u[j * grid.ni + i])[3]; }
  void restart_ramp() { ramp_k = 0; }                     // implicit.rs:88-90
};

Prim ghost_state(int bc, const Prim& fs, const Prim& edge, const Prim& mirror, const Face& f, double outward);  // solver.rs:413-421

// ---------------------------------------------------------------- implicit.rs
M4 flux_jacobian(const Prim& w, double nx, double nr);                                             // implicit.rs:95-108
M4 mm(const M4& a, const M4& b);                                                                   // implicit.rs:111-122
Cons mv(const M4& a, const Cons& x);                                                               // implicit.rs:125-131
M4 inv4(const M4& m);                                                                              // implicit.rs:141-175
void block_thomas(size_t n, size_t base, size_t stride, const std::vector<M4>& lo, const std::vector<M4>& d,
                  const std::vector<M4>& up, Cons* rhs, M4* y);                                    // implicit.rs:179-204
M4 abs_jacobian(const Prim& wl, const Prim& wr, double nx, double nr, double eps_fix);              // implicit.rs:209-241
M4 ghost_jacobian(int bc, const Prim& fs, const Prim& edge, const Face& f, double outward);        // implicit.rs:257-279
void cell_blocks(const Prim& wk, const Prim& wm, const Prim& wp, const Face& fl, const Face& fr, double vol, double dt,
                 bool lines, double src, bool roe, double eps_fix, double visc_l, double visc_r, M4& lo, M4& d, M4& up);  // implicit.rs:284-367
void assemble_into(const Solver& s, const ImplicitParams& p, bool dir_i, Factor& fac);            // implicit.rs:379-467
void solve_lines(const Solver& s, const Factor& fac, bool dir_i, std::vector<Cons>& x);           // implicit.rs:528-563
void apply_factor_into(const Solver& s, const Factor& fac, bool dir_i, const std::vector<Cons>& x, std::vector<Cons>& out);  // implicit.rs:566-594
double implicit_step(Solver& s, const ImplicitParams& p);                                         // implicit.rs:601-663
void compute_dt(Solver& s, double cfl, int mode);                                                  // implicit.rs:666-695

// ---------------------------------------------------------------- multigrid.rs
double mg_cycle(Solver& fine, const MgParams& p);                                                  // multigrid.rs:73-85

// ---------------------------------------------------------------- viscous.rs passes
bool iface_sides(const Grid& g, const std::vector<Prim>& w, const Walls& walls, size_t i, size_t j, FaceSides& out);  // viscous.rs:150-188
bool jface_sides(const Grid& g, const std::vector<Prim>& w, const Walls& walls, size_t i, size_t j, FaceSides& out);  // viscous.rs:191-215
std::pair<double, double> iface_centre(const Grid& g, size_t i, size_t j);
std::pair<double, double> jface_centre(const Grid& g, size_t i, size_t j);
void stencil(const Grid& g, const FaceSides& s, double xf, double rf, double& dd, double& ex, double& er);  // viscous.rs:244-250
void face_mu(const std::vector<double>& mu, const std::vector<double>& mu_t, const std::vector<std::array<double, 3>>& rough,
             const FaceSides& s, double& mu_f, double& mut_f);                                      // viscous.rs:256-270
double hoop_stress(double mue, const std::array<double, 6>& g, double v_c, double r_c);            // viscous.rs:413-416
double diffusion_rate(double mu_c, double mu_t_c, double rho_c, double len, double area);          // viscous.rs:421-424

// ---------------------------------------------------------------- turbulence.rs
constexpr double K_INF = 9e-9;
inline double omega_inf(double re_c) { return 1e-6 * re_c; }
constexpr double A1 = 0.31, BETA_STAR = 0.09, SIGMA_K1 = 0.85, SIGMA_K2 = 1.0, SIGMA_W1 = 0.5, SIGMA_W2 = 0.856,
                 BETA1 = 0.075, BETA2 = 0.0828, GAMMA1 = 5.0 / 9.0, GAMMA2 = 0.44;
constexpr size_t AUPOIX_ITERATIONS = 16;
constexpr double NU_T_WALL_MAX = 1e5;
constexpr size_t ROUGH_RAMP_CELLS = 8;
std::vector<double> wall_distance(const Grid& g, const Walls& walls);                               // turbulence.rs:91-125
void turb_init(Solver& s, double re_c);                                                            // turbulence.rs:128-138
double rough_ramp(size_t i, size_t wall_i_start);                                                  // turbulence.rs:288-290
std::array<double, 3> aupoix_wall(double nu, double speed, double d, double ks);                   // turbulence.rs:304-320
void turb_update(Solver& s);                                                                       // turbulence.rs:542-611

// ---------------------------------------------------------------- engine: body_grid.rs
enum NoseKind { NOSE_TANGENT_OGIVE = 0, NOSE_CONE = 1, NOSE_POWER = 2, NOSE_PARABOLIC = 3, NOSE_HAACK = 4 };
struct Nose {  // body_grid.rs:31-43
  int kind = NOSE_TANGENT_OGIVE;
  double fineness = 3.0;   // ogive / power / parabolic / haack
  double half_angle = 0.0; // cone
  double param = 0.0;      // power n, parabolic k, haack c
};
struct Body {  // body_grid.rs:54-109
  Nose nose{};
  double radius() const { return 0.5; }
  double nose_length() const;
  double r(double x) const;
  double slope(double x) const;
};
struct Segment {
  double length = 0, slope = 0;
};
struct BaseBody {  // body_grid.rs:246-319
  Body body{};
  std::vector<Segment> segments;
  double sting_radius = 0.0;
  std::pair<double, double> station(size_t k) const;
  double aft_length() const;
  double x_base() const { return station(segments.size()).first; }
  double base_radius() const { return station(segments.size()).second; }
  double r(double x) const;
};
struct LargeGridParams {  // body_grid.rs:112-131
  BaseBody body;
  double x_up = 0, x_down = 0, r_far = 0;
  size_t n_up = 0, n_nose = 0;
  std::vector<size_t> n_seg;
  size_t n_ext = 0, nj = 0;
  double dx_tip = 0, dr_wall = 0;
};
struct BaseGridParams {  // body_grid.rs:330-355 (power-off: no nozzle rows)
  BaseBody body;
  double x_up = 0, x_down = 0, r_far = 0;
  size_t n_up = 0, n_nose = 0;
  std::vector<size_t> n_seg;
  size_t n_wake = 0, n_sting = 0, n_gap = 0, nj_out = 0;
  double dx_tip = 0, dr_wall = 0;
  bool gap_one_sided = false;
};
std::vector<double> two_sided_nodes(double len, size_t n, double dx);                 // body_grid.rs:134-157
bool axial_nodes(const LargeGridParams& p, std::vector<double>& xs, std::string* err); // body_grid.rs:160-205
std::vector<double> radial_fractions(double dr_wall, double r_far, size_t nj);         // body_grid.rs:208-210
bool large_domain_grid(const LargeGridParams& p, Grid& out, std::string* err);         // body_grid.rs:213-231
bool base_domain_grid(const BaseGridParams& p, Grid& out, Block& blk, std::string* err);  // body_grid.rs:360-452

// ---------------------------------------------------------------- engine: numerics.rs / case.rs / run.rs
enum Wake { WAKE_STING = 0, WAKE_BASE = 1 };
struct Numerics {  // numerics.rs:261-287
  double cfl = 0.5;
  int limiter = VAN_ALBADA;
  bool low_mach = true;
  Scheme scheme{};
  size_t first_order_iters = 100, max_iter = 10000, min_iter = 0;
  double drop_orders = 6.0;
  int outflow = BC_CHARACTERISTIC;
  size_t monitor_window = 2000;
  bool has_monitor_tol = false;
  double monitor_tol = 0;
  bool has_mean_window = false;
  size_t mean_window = 0;
  bool has_drag_rel_tol = false;
  double drag_rel_tol = 0;
};
constexpr size_t MONITOR_EVERY = 50, DRAG_REL_WINDOW = 500;
constexpr double REGIME_SPLIT_MACH = 0.85, MONITOR_LIMIT = 1e3;
Numerics numerics_subsonic(unsigned level, int wake);   // numerics.rs:291-310
Numerics numerics_transonic();                          // numerics.rs:313-329
Numerics numerics_auto(double mach, unsigned level, int wake);  // numerics.rs:332-339
Numerics numerics_viscous(double mach, unsigned level);        // numerics.rs:345-362

struct Case {  // case.rs:33-46 (power-off)
  double mach = 0.5;
  BaseBody body;
  int wake = WAKE_STING;
  BaseGridParams grid_base;
  LargeGridParams grid_sting;
  Numerics numerics;
  bool has_viscous = false;
  Viscous viscous{};
};
Case case_new(double mach, const BaseBody& body, unsigned level, int wake, const Numerics& n);  // case.rs:51-78
Case case_viscous(double mach, const BaseBody& body, unsigned level, int wake, double re_c, double sutherland, double mach_max);  // case.rs:84-102
bool case_build_solver(const Case& c, Solver& s, std::string* err);  // case.rs:147-176
size_t layer_count(double h, double y1);                            // case.rs:185-187

// atmosphere.rs:84-112
struct AirState {
  double temperature_k, pressure_pa, density, sound_speed, viscosity;
};
bool isa_state(double altitude_m, AirState& out);
constexpr double SUTHERLAND_S = 110.4;

enum StopReason { STOP_MAX_ITERATIONS = 0, STOP_RESIDUAL_DROP = 1, STOP_CD_STATIONARY = 2, STOP_BASE_PRESSURE_STATIONARY = 3,
                  STOP_MEAN_STATIONARY = 4, STOP_NON_FINITE = 5, STOP_CANCELLED = 6 };

struct PointResult {  // engine/result.rs (the fields this build reports)
  size_t iters = 0;
  std::vector<double> residual;
  double residual_peak = 0, drop_orders = 0;
  int stop_reason = STOP_MAX_ITERATIONS;
  double cd_nose = 0, cd_nose_cell = 0;
  std::vector<double> cd_aft;
  double cd_base = 0, cd_friction = 0, cd_total = 0;
  double cp_base = NAN, cp_base_cell = NAN;
  double y_plus_max = NAN, farfield_dp = 0, min_rho = 0, min_p = 0, m_max = 0, m_wall_max = 0;
  std::vector<std::pair<size_t, double>> monitor_history;
};

struct WallPoint {
  double x, r, s0, s1, cp, cp_cell;
};
void wall_distribution(const BaseBody& body, const Solver& s, std::vector<WallPoint>& wall, double& cd, double& cd_cell);  // run.rs:252-282
void friction(const Case& c, const Solver& s, double& cd, double& y_plus_max);                                           // run.rs:207-248
void base_state(const Solver& s, double rb2, double& cd, double& mean, double& mean_cell);                               // run.rs:286-313
double monitor(const Case& c, const Solver& s);                                                                         // run.rs:174-185
bool stop_reason(const Case& c, size_t it, double r, double reference, size_t skip, const std::vector<std::pair<size_t, double>>& hist, int& why);  // run.rs:105-150
bool mean_stationary(const std::vector<std::pair<size_t, double>>& hist, size_t k);                                       // run.rs:157-170
PointResult run_on(const Case& c, Solver& s, bool warm, const double* r_ref);                                           // run.rs:44-89
PointResult finish(const Case& c, const Solver& s, std::vector<double> residual, double rmax,
                   std::vector<std::pair<size_t, double>> hist, int reason);                                            // run.rs:316-419

}  // namespace orc
