// TEST INFRASTRUCTURE — C entry points of the oracle, loaded through ctypes by oracle/oracle_ffi.py (tests and the CPU
// baseline only). Plain pointers and sizes; every call that can fail returns 0 on success and writes a message.
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "oracle.hpp"

using namespace orc;

extern "C" {

typedef struct {
  double cfl;
  int limiter;
  double fs[4];
  int bc[4];
  size_t first_order_iters;
} OrcConfig;

typedef struct {
  int kind;
  double cfl_star;
  size_t mg_levels, mg_pre, mg_post, mg_gamma, mg_coarsest;
  double mg_cfl_star;
  double cfl0, cfl_max, growth;
  int dt_mode, lines, implicit_bc;
  size_t sub_iters;
  int roe;
  double eps_fix;
} OrcScheme;

typedef struct {
  int nose_kind;
  double fineness, half_angle, param;
  int nseg;
  double seg_length[8], seg_slope[8];
  double sting_radius;
} OrcBody;

typedef struct {
  double x_up, x_down, r_far;
  size_t n_up, n_nose, n_seg[8], n_wake, n_sting, n_gap, nj_out;
  double dx_tip, dr_wall;
  int gap_one_sided;
} OrcBaseGrid;

typedef struct {
  double x_up, x_down, r_far;
  size_t n_up, n_nose, n_seg[8], n_ext, nj;
  double dx_tip, dr_wall;
} OrcStingGrid;

typedef struct {
  double cfl;
  int limiter, low_mach;
  OrcScheme scheme;
  size_t first_order_iters, max_iter, min_iter;
  double drop_orders;
  int outflow;
  size_t monitor_window;
  int has_monitor_tol;
  double monitor_tol;
  int has_mean_window;
  size_t mean_window;
  int has_drag_rel_tol;
  double drag_rel_tol;
} OrcNumerics;

typedef struct {
  double mach;
  OrcBody body;
  int wake;
  OrcBaseGrid grid_base;
  OrcStingGrid grid_sting;
  OrcNumerics numerics;
  int has_viscous;
  double re_c, sutherland;
  int turbulence;
  size_t wall_i_start;
  double roughness;
} OrcCase;

typedef struct {
  size_t iters;
  double residual_peak, drop_orders;
  int stop_reason;
  double cd_nose, cd_nose_cell, cd_aft[8], cd_base, cd_friction, cd_total, cp_base, cp_base_cell, y_plus_max, farfield_dp, min_rho, min_p,
      m_max, m_wall_max;
  double cd_window;  // mean stationary: mean monitored CD over the last compared window; otherwise cd_total
} OrcPointResult;

}  // extern "C"

static void put_err(char* buf, size_t len, const std::string& m) {
  if (buf && len) {
    std::snprintf(buf, len, "%s", m.c_str());
  }
}

static Scheme to_scheme(const OrcScheme& s) {
  Scheme o;
  o.kind = s.kind;
  o.irs.cfl_star = s.cfl_star;
  o.mg.levels = s.mg_levels;
  o.mg.pre = s.mg_pre;
  o.mg.post = s.mg_post;
  o.mg.gamma = s.mg_gamma;
  o.mg.coarsest = s.mg_coarsest;
  o.mg.irs.cfl_star = s.mg_cfl_star;
  o.imp.cfl0 = s.cfl0;
  o.imp.cfl_max = s.cfl_max;
  o.imp.growth = s.growth;
  o.imp.dt_mode = s.dt_mode;
  o.imp.lines = s.lines != 0;
  o.imp.implicit_bc = s.implicit_bc != 0;
  o.imp.sub_iters = s.sub_iters;
  o.imp.roe = s.roe != 0;
  o.imp.eps_fix = s.eps_fix;
  return o;
}
static OrcScheme from_scheme(const Scheme& s) {
  OrcScheme o{};
  o.kind = s.kind;
  o.cfl_star = s.irs.cfl_star;
  o.mg_levels = s.mg.levels;
  o.mg_pre = s.mg.pre;
  o.mg_post = s.mg.post;
  o.mg_gamma = s.mg.gamma;
  o.mg_coarsest = s.mg.coarsest;
  o.mg_cfl_star = s.mg.irs.cfl_star;
  o.cfl0 = s.imp.cfl0;
  o.cfl_max = s.imp.cfl_max;
  o.growth = s.imp.growth;
  o.dt_mode = s.imp.dt_mode;
  o.lines = s.imp.lines;
  o.implicit_bc = s.imp.implicit_bc;
  o.sub_iters = s.imp.sub_iters;
  o.roe = s.imp.roe;
  o.eps_fix = s.imp.eps_fix;
  return o;
}
static BaseBody to_body(const OrcBody& b) {
  BaseBody o;
  o.body.nose.kind = b.nose_kind;
  o.body.nose.fineness = b.fineness;
  o.body.nose.half_angle = b.half_angle;
  o.body.nose.param = b.param;
  for (int k = 0; k < b.nseg && k < 8; ++k) o.segments.push_back(Segment{b.seg_length[k], b.seg_slope[k]});
  o.sting_radius = b.sting_radius;
  return o;
}
static OrcBody from_body(const BaseBody& b) {
  OrcBody o{};
  o.nose_kind = b.body.nose.kind;
  o.fineness = b.body.nose.fineness;
  o.half_angle = b.body.nose.half_angle;
  o.param = b.body.nose.param;
  o.nseg = (int)b.segments.size();
  for (size_t k = 0; k < b.segments.size() && k < 8; ++k) {
    o.seg_length[k] = b.segments[k].length;
    o.seg_slope[k] = b.segments[k].slope;
  }
  o.sting_radius = b.sting_radius;
  return o;
}
static Numerics to_numerics(const OrcNumerics& n) {
  Numerics o;
  o.cfl = n.cfl;
  o.limiter = n.limiter;
  o.low_mach = n.low_mach != 0;
  o.scheme = to_scheme(n.scheme);
  o.first_order_iters = n.first_order_iters;
  o.max_iter = n.max_iter;
  o.min_iter = n.min_iter;
  o.drop_orders = n.drop_orders;
  o.outflow = n.outflow;
  o.monitor_window = n.monitor_window;
  o.has_monitor_tol = n.has_monitor_tol != 0;
  o.monitor_tol = n.monitor_tol;
  o.has_mean_window = n.has_mean_window != 0;
  o.mean_window = n.mean_window;
  o.has_drag_rel_tol = n.has_drag_rel_tol != 0;
  o.drag_rel_tol = n.drag_rel_tol;
  return o;
}
static OrcNumerics from_numerics(const Numerics& n) {
  OrcNumerics o{};
  o.cfl = n.cfl;
  o.limiter = n.limiter;
  o.low_mach = n.low_mach;
  o.scheme = from_scheme(n.scheme);
  o.first_order_iters = n.first_order_iters;
  o.max_iter = n.max_iter;
  o.min_iter = n.min_iter;
  o.drop_orders = n.drop_orders;
  o.outflow = n.outflow;
  o.monitor_window = n.monitor_window;
  o.has_monitor_tol = n.has_monitor_tol;
  o.monitor_tol = n.monitor_tol;
  o.has_mean_window = n.has_mean_window;
  o.mean_window = n.mean_window;
  o.has_drag_rel_tol = n.has_drag_rel_tol;
  o.drag_rel_tol = n.drag_rel_tol;
  return o;
}
static Case to_case(const OrcCase& c) {
  Case o;
  o.mach = c.mach;
  o.body = to_body(c.body);
  o.wake = c.wake;
  const OrcBaseGrid& gb = c.grid_base;
  o.grid_base.body = o.body;
  o.grid_base.x_up = gb.x_up;
  o.grid_base.x_down = gb.x_down;
  o.grid_base.r_far = gb.r_far;
  o.grid_base.n_up = gb.n_up;
  o.grid_base.n_nose = gb.n_nose;
  for (int k = 0; k < c.body.nseg; ++k) o.grid_base.n_seg.push_back(gb.n_seg[k]);
  o.grid_base.n_wake = gb.n_wake;
  o.grid_base.n_sting = gb.n_sting;
  o.grid_base.n_gap = gb.n_gap;
  o.grid_base.nj_out = gb.nj_out;
  o.grid_base.dx_tip = gb.dx_tip;
  o.grid_base.dr_wall = gb.dr_wall;
  o.grid_base.gap_one_sided = gb.gap_one_sided != 0;
  const OrcStingGrid& gs = c.grid_sting;
  o.grid_sting.body = o.body;
  o.grid_sting.x_up = gs.x_up;
  o.grid_sting.x_down = gs.x_down;
  o.grid_sting.r_far = gs.r_far;
  o.grid_sting.n_up = gs.n_up;
  o.grid_sting.n_nose = gs.n_nose;
  for (int k = 0; k < c.body.nseg; ++k) o.grid_sting.n_seg.push_back(gs.n_seg[k]);
  o.grid_sting.n_ext = gs.n_ext;
  o.grid_sting.nj = gs.nj;
  o.grid_sting.dx_tip = gs.dx_tip;
  o.grid_sting.dr_wall = gs.dr_wall;
  o.numerics = to_numerics(c.numerics);
  o.has_viscous = c.has_viscous != 0;
  o.viscous = Viscous{c.re_c, c.sutherland, c.turbulence, c.wall_i_start, c.roughness};
  return o;
}
static OrcCase from_case(const Case& c) {
  OrcCase o{};
  o.mach = c.mach;
  o.body = from_body(c.body);
  o.wake = c.wake;
  OrcBaseGrid& gb = o.grid_base;
  gb.x_up = c.grid_base.x_up;
  gb.x_down = c.grid_base.x_down;
  gb.r_far = c.grid_base.r_far;
  gb.n_up = c.grid_base.n_up;
  gb.n_nose = c.grid_base.n_nose;
  for (size_t k = 0; k < c.grid_base.n_seg.size() && k < 8; ++k) gb.n_seg[k] = c.grid_base.n_seg[k];
  gb.n_wake = c.grid_base.n_wake;
  gb.n_sting = c.grid_base.n_sting;
  gb.n_gap = c.grid_base.n_gap;
  gb.nj_out = c.grid_base.nj_out;
  gb.dx_tip = c.grid_base.dx_tip;
  gb.dr_wall = c.grid_base.dr_wall;
  gb.gap_one_sided = c.grid_base.gap_one_sided;
  OrcStingGrid& gs = o.grid_sting;
  gs.x_up = c.grid_sting.x_up;
  gs.x_down = c.grid_sting.x_down;
  gs.r_far = c.grid_sting.r_far;
  gs.n_up = c.grid_sting.n_up;
  gs.n_nose = c.grid_sting.n_nose;
  for (size_t k = 0; k < c.grid_sting.n_seg.size() && k < 8; ++k) gs.n_seg[k] = c.grid_sting.n_seg[k];
  gs.n_ext = c.grid_sting.n_ext;
  gs.nj = c.grid_sting.nj;
  gs.dx_tip = c.grid_sting.dx_tip;
  gs.dr_wall = c.grid_sting.dr_wall;
  o.numerics = from_numerics(c.numerics);
  o.has_viscous = c.has_viscous;
  o.re_c = c.viscous.re_c;
  o.sutherland = c.viscous.sutherland;
  o.turbulence = c.viscous.turbulence;
  o.wall_i_start = c.viscous.wall_i_start;
  o.roughness = c.viscous.roughness;
  return o;
}
static void fill_result(const PointResult& p, OrcPointResult* out) {
  std::memset(out, 0, sizeof(*out));
  out->iters = p.iters;
  out->residual_peak = p.residual_peak;
  out->drop_orders = p.drop_orders;
  out->stop_reason = p.stop_reason;
  out->cd_nose = p.cd_nose;
  out->cd_nose_cell = p.cd_nose_cell;
  for (size_t k = 0; k < p.cd_aft.size() && k < 8; ++k) out->cd_aft[k] = p.cd_aft[k];
  out->cd_base = p.cd_base;
  out->cd_friction = p.cd_friction;
  out->cd_total = p.cd_total;
  out->cp_base = p.cp_base;
  out->cp_base_cell = p.cp_base_cell;
  out->y_plus_max = p.y_plus_max;
  out->farfield_dp = p.farfield_dp;
  out->min_rho = p.min_rho;
  out->min_p = p.min_p;
  out->m_max = p.m_max;
  out->m_wall_max = p.m_wall_max;
}

template <class V>
static void copy_out(const V& v, double* out) {
  std::memcpy(out, v.data(), v.size() * sizeof(v[0]));
}

static Prim P4(const double* a) { return {a[0], a[1], a[2], a[3]}; }
static void W4(const std::array<double, 4>& v, double* o) {
  for (int k = 0; k < 4; ++k) o[k] = v[k];
}

extern "C" {

// ---------------------------------------------------------------- point kernels
void orc_physical_flux(const double* w, double nx, double nr, double* out) { W4(physical_flux(P4(w), nx, nr), out); }
void orc_hllc(const double* wl, const double* wr, double nx, double nr, double* out) { W4(hllc(P4(wl), P4(wr), nx, nr), out); }
void orc_rusanov(const double* wl, const double* wr, double nx, double nr, double* out) { W4(rusanov(P4(wl), P4(wr), nx, nr), out); }
double orc_shock_weight(double pl, double pr) { return shock_weight(pl, pr); }
double orc_limited_slope(double a, double b, int lim) { return limited_slope(a, b, lim); }
void orc_face_flux_lm(const double* m2, const double* m1, const double* p0, const double* p1, int lim, double nx, double nr, int low_mach,
                      double* out) {
  W4(face_flux_lm(P4(m2), P4(m1), P4(p0), P4(p1), lim, nx, nr, low_mach != 0), out);
}
void orc_face_flux(const double* m2, const double* m1, const double* p0, const double* p1, int lim, double nx, double nr, double* out) {
  W4(face_flux(P4(m2), P4(m1), P4(p0), P4(p1), lim, nx, nr), out);
}
void orc_low_mach_states(const double* l, const double* r, double nx, double nr, double* lo, double* ro) {
  Prim a, b;
  low_mach_states(P4(l), P4(r), nx, nr, a, b);
  W4(a, lo);
  W4(b, ro);
}
int orc_regime(const double* w, double nx, double nr) { return regime(P4(w), nx, nr); }
int orc_characteristic_ghost(const double* fs, const double* interior, double nx, double nr, double* out) {
  int reg = 0;
  W4(characteristic_ghost(P4(fs), P4(interior), nx, nr, &reg), out);
  return reg;
}
void orc_pressure_outflow_ghost(double p_back, const double* interior, double nx, double nr, double* out) {
  W4(pressure_outflow_ghost(p_back, P4(interior), nx, nr), out);
}
void orc_flux_jacobian(const double* w, double nx, double nr, double* out) {
  M4 a = flux_jacobian(P4(w), nx, nr);
  std::memcpy(out, a.data(), 16 * sizeof(double));
}
void orc_abs_jacobian(const double* wl, const double* wr, double nx, double nr, double eps_fix, double* out) {
  M4 a = abs_jacobian(P4(wl), P4(wr), nx, nr, eps_fix);
  std::memcpy(out, a.data(), 16 * sizeof(double));
}
void orc_inv4(const double* m, double* out) {
  M4 a;
  std::memcpy(a.data(), m, 16 * sizeof(double));
  M4 b = inv4(a);
  std::memcpy(out, b.data(), 16 * sizeof(double));
}
void orc_mm4(const double* a, const double* b, double* out) {
  M4 x, y;
  std::memcpy(x.data(), a, 16 * sizeof(double));
  std::memcpy(y.data(), b, 16 * sizeof(double));
  M4 c = mm(x, y);
  std::memcpy(out, c.data(), 16 * sizeof(double));
}
// lo, d, up: n blocks of 16 (row-major); rhs: n x 4, solved in place
void orc_block_thomas(size_t n, const double* lo, const double* d, const double* up, double* rhs) {
  std::vector<M4> L(n), D(n), U(n);
  for (size_t k = 0; k < n; ++k) {
    std::memcpy(L[k].data(), lo + 16 * k, 128);
    std::memcpy(D[k].data(), d + 16 * k, 128);
    std::memcpy(U[k].data(), up + 16 * k, 128);
  }
  std::vector<Cons> r(n);
  for (size_t k = 0; k < n; ++k) r[k] = {rhs[4 * k], rhs[4 * k + 1], rhs[4 * k + 2], rhs[4 * k + 3]};
  std::vector<M4> y(n);
  block_thomas(n, 0, 1, L, D, U, r.data(), y.data());
  for (size_t k = 0; k < n; ++k)
    for (int q = 0; q < 4; ++q) rhs[4 * k + q] = r[k][q];
}
void orc_aupoix_wall(double nu, double speed, double d, double ks, double* out) {
  auto a = aupoix_wall(nu, speed, d, ks);
  out[0] = a[0];
  out[1] = a[1];
  out[2] = a[2];
}
void orc_geometric_offsets(double first, double length, size_t n, double* out) {
  auto v = geometric_offsets(first, length, n);
  std::memcpy(out, v.data(), (n + 1) * sizeof(double));
}
void orc_two_sided_nodes(double len, size_t n, double dx, double* out) {
  auto v = two_sided_nodes(len, n, dx);
  std::memcpy(out, v.data(), (n + 1) * sizeof(double));
}
int orc_isa(double altitude_m, double* out5) {
  AirState a;
  if (!isa_state(altitude_m, a)) return 1;
  out5[0] = a.temperature_k;
  out5[1] = a.pressure_pa;
  out5[2] = a.density;
  out5[3] = a.sound_speed;
  out5[4] = a.viscosity;
  return 0;
}

// ---------------------------------------------------------------- solver handle
void* orc_solver_new(size_t ni, size_t nj, const double* x, const double* r, const OrcConfig* c, char* err, size_t errlen) {
  std::vector<double> X(x, x + (ni + 1) * (nj + 1)), R(r, r + (ni + 1) * (nj + 1));
  Grid g;
  std::string e;
  if (!grid_from_nodes(ni, nj, std::move(X), std::move(R), g, &e)) {
    put_err(err, errlen, e);
    return nullptr;
  }
  Config cfg;
  cfg.cfl = c->cfl;
  cfg.limiter = c->limiter;
  cfg.freestream = P4(c->fs);
  for (int k = 0; k < 4; ++k) cfg.bc[k] = c->bc[k];
  cfg.first_order_iters = c->first_order_iters;
  return new Solver(std::move(g), cfg);
}
void orc_solver_free(void* h) { delete static_cast<Solver*>(h); }
void orc_solver_get_config(void* h, OrcConfig* c) {
  Solver* s = static_cast<Solver*>(h);
  c->cfl = s->cfg.cfl;
  c->limiter = s->cfg.limiter;
  for (int k = 0; k < 4; ++k) {
    c->fs[k] = s->cfg.freestream[k];
    c->bc[k] = s->cfg.bc[k];
  }
  c->first_order_iters = s->cfg.first_order_iters;
}
void orc_solver_set_config(void* h, const OrcConfig* c) {
  Solver* s = static_cast<Solver*>(h);
  s->cfg.cfl = c->cfl;
  s->cfg.limiter = c->limiter;
  s->cfg.freestream = P4(c->fs);
  for (int k = 0; k < 4; ++k) s->cfg.bc[k] = c->bc[k];
  s->cfg.first_order_iters = c->first_order_iters;
}
int orc_solver_set_block(void* h, int has, size_t i_end, size_t j_end, size_t j_sting, char* err, size_t errlen) {
  try {
    Block b{i_end, j_end, j_sting};
    static_cast<Solver*>(h)->set_block(has ? &b : nullptr);
    return 0;
  } catch (const std::exception& e) {
    put_err(err, errlen, e.what());
    return 1;
  }
}
int orc_solver_get_block(void* h, size_t* out3) {
  Solver* s = static_cast<Solver*>(h);
  out3[0] = s->block.i_end;
  out3[1] = s->block.j_end;
  out3[2] = s->block.j_sting;
  return s->has_block ? 1 : 0;
}
void orc_solver_set_low_mach(void* h, int on) { static_cast<Solver*>(h)->low_mach = on != 0; }
int orc_solver_set_scheme(void* h, const OrcScheme* sc, char* err, size_t errlen) {
  try {
    return (int)static_cast<Solver*>(h)->set_scheme(to_scheme(*sc)) > 0 ? 0 : 1;
  } catch (const std::exception& e) {
    put_err(err, errlen, e.what());
    return -1;
  }
}
size_t orc_solver_mg_levels(void* h) { return static_cast<Solver*>(h)->coarse.size() + 1; }
int orc_solver_set_viscous(void* h, int has, double re_c, double sutherland, int turbulence, size_t wall_i_start, double roughness, char* err,
                           size_t errlen) {
  try {
    Viscous v{re_c, sutherland, turbulence, wall_i_start, roughness};
    static_cast<Solver*>(h)->set_viscous(has ? &v : nullptr);
    return 0;
  } catch (const std::exception& e) {
    put_err(err, errlen, e.what());
    return 1;
  }
}
int orc_solver_set_nozzle(void* h, int has, size_t j_end, const double* state, const double* turb2, char* err, size_t errlen) {
  try {
    Nozzle n;
    n.j_end = j_end;
    if (has) {
      n.state = P4(state);
      n.turb = {turb2[0], turb2[1]};
    }
    static_cast<Solver*>(h)->set_nozzle(has ? &n : nullptr);
    return 0;
  } catch (const std::exception& e) {
    put_err(err, errlen, e.what());
    return 1;
  }
}
double orc_solver_step(void* h) { return static_cast<Solver*>(h)->step(); }
void orc_solver_steps(void* h, size_t n, double* out) {
  Solver* s = static_cast<Solver*>(h);
  for (size_t k = 0; k < n; ++k) {
    double r = s->step();
    if (out) out[k] = r;
  }
}
void orc_solver_eval_residual(void* h, int compute_dt) { static_cast<Solver*>(h)->eval_residual(compute_dt != 0); }
double orc_solver_density_residual(void* h) { return static_cast<Solver*>(h)->density_residual(); }
void orc_solver_dims(void* h, size_t* ni, size_t* nj) {
  Solver* s = static_cast<Solver*>(h);
  *ni = s->grid.ni;
  *nj = s->grid.nj;
}
size_t orc_solver_iter(void* h) { return static_cast<Solver*>(h)->iter; }
void orc_solver_set_iter(void* h, size_t it) { static_cast<Solver*>(h)->iter = it; }
void orc_solver_restart_ramp(void* h) { static_cast<Solver*>(h)->restart_ramp(); }
size_t orc_solver_n_active(void* h) { return static_cast<Solver*>(h)->n_active; }
double orc_solver_turb_residual(void* h) { return static_cast<Solver*>(h)->turb_rnorm; }

enum {
  F_U = 0,
  F_RES = 1,
  F_DT = 2,
  F_W = 3,
  F_FI = 4,
  F_FJ = 5,
  F_TURB = 6,
  F_MUT = 7,
  F_DWALL = 8,
  F_MU = 9,
  F_GRAD = 10,
  F_X = 11,
  F_R = 12,
  F_VOL = 13,
  F_AREA = 14,
  F_XC = 15,
  F_RC = 16,
  F_FVI = 17,
  F_FJV = 18,
};
// Number of doubles of field `f`.
size_t orc_solver_field_len(void* h, int f) {
  Solver* s = static_cast<Solver*>(h);
  size_t ni = s->grid.ni, nj = s->grid.nj, n = ni * nj;
  switch (f) {
    case F_U:
    case F_RES:
      return 4 * n;
    case F_DT:
    case F_MUT:
    case F_DWALL:
    case F_MU:
    case F_VOL:
    case F_AREA:
    case F_XC:
    case F_RC:
      return f == F_MUT ? s->mu_t.size() : (f == F_DWALL ? s->dwall.size() : (f == F_MU ? s->mu.size() : n));
    case F_W:
      return 4 * s->w.size();
    case F_FI:
      return 4 * s->fi.size();
    case F_FJ:
      return 4 * s->fj.size();
    case F_TURB:
      return 2 * s->turb.size();
    case F_GRAD:
      return 6 * s->grad.size();
    case F_X:
    case F_R:
      return (ni + 1) * (nj + 1);
    case F_FVI:
      return 4 * s->fvi.size();
    case F_FJV:
      return 4 * s->fvj.size();
  }
  return 0;
}
void orc_solver_get(void* h, int f, double* out) {
  Solver* s = static_cast<Solver*>(h);
  switch (f) {
    case F_U:
      copy_out(s->u, out);
      break;
    case F_RES:
      copy_out(s->res, out);
      break;
    case F_DT:
      copy_out(s->dt, out);
      break;
    case F_W:
      copy_out(s->w, out);
      break;
    case F_FI:
      copy_out(s->fi, out);
      break;
    case F_FJ:
      copy_out(s->fj, out);
      break;
    case F_TURB:
      copy_out(s->turb, out);
      break;
    case F_MUT:
      copy_out(s->mu_t, out);
      break;
    case F_DWALL:
      copy_out(s->dwall, out);
      break;
    case F_MU:
      copy_out(s->mu, out);
      break;
    case F_GRAD:
      copy_out(s->grad, out);
      break;
    case F_X:
      copy_out(s->grid.x, out);
      break;
    case F_R:
      copy_out(s->grid.r, out);
      break;
    case F_VOL:
      copy_out(s->grid.vol, out);
      break;
    case F_AREA:
      copy_out(s->grid.area, out);
      break;
    case F_XC:
      copy_out(s->grid.xc, out);
      break;
    case F_RC:
      copy_out(s->grid.rc, out);
      break;
    case F_FVI:
      copy_out(s->fvi, out);
      break;
    case F_FJV:
      copy_out(s->fvj, out);
      break;
  }
}
void orc_solver_set(void* h, int f, const double* in) {
  Solver* s = static_cast<Solver*>(h);
  switch (f) {
    case F_U:
      std::memcpy(s->u.data(), in, s->u.size() * sizeof(Cons));
      break;
    case F_TURB:
      std::memcpy(s->turb.data(), in, s->turb.size() * sizeof(s->turb[0]));
      break;
    case F_MUT:
      std::memcpy(s->mu_t.data(), in, s->mu_t.size() * sizeof(double));
      break;
    case F_DT:
      std::memcpy(s->dt.data(), in, s->dt.size() * sizeof(double));
      break;
  }
}

// ---------------------------------------------------------------- case layer
int orc_case_new(double mach, const OrcBody* body, unsigned level, int wake, OrcCase* out) {
  BaseBody b = to_body(*body);
  Case c = case_new(mach, b, level, wake, numerics_auto(mach, level, wake));
  *out = from_case(c);
  return 0;
}
int orc_case_viscous(double mach, const OrcBody* body, unsigned level, int wake, double re_c, double sutherland, double mach_max,
                     OrcCase* out) {
  BaseBody b = to_body(*body);
  Case c = case_viscous(mach, b, level, wake, re_c, sutherland, mach_max);
  *out = from_case(c);
  return 0;
}
void orc_numerics_preset(int which, double mach, unsigned level, int wake, OrcNumerics* out) {
  Numerics n;
  switch (which) {
    case 0:
      n = numerics_subsonic(level, wake);
      break;
    case 1:
      n = numerics_transonic();
      break;
    case 2:
      n = numerics_auto(mach, level, wake);
      break;
    default:
      n = numerics_viscous(mach, level);
  }
  *out = from_numerics(n);
}
void* orc_case_build_solver(const OrcCase* c, char* err, size_t errlen) {
  try {
    Case cc = to_case(*c);
    Solver* s = new Solver();
    std::string e;
    if (!case_build_solver(cc, *s, &e)) {
      delete s;
      put_err(err, errlen, e);
      return nullptr;
    }
    return s;
  } catch (const std::exception& e) {
    put_err(err, errlen, e.what());
    return nullptr;
  }
}
// run_on (run.rs:44-89); r_ref < 0: none. The residual history goes to `residual` (up to cap entries).
int orc_run_on(const OrcCase* c, void* h, int warm, double r_ref, OrcPointResult* out, double* residual, size_t cap) {
  Case cc = to_case(*c);
  Solver* s = static_cast<Solver*>(h);
  PointResult p = run_on(cc, *s, warm != 0, r_ref >= 0 ? &r_ref : nullptr);
  fill_result(p, out);
  out->cd_window = p.cd_total;
  size_t k = cc.numerics.mean_window / MONITOR_EVERY;
  if (p.stop_reason == STOP_MEAN_STATIONARY && k > 0 && p.monitor_history.size() >= k) {
    double m = 0.0;
    for (size_t t = p.monitor_history.size() - k; t < p.monitor_history.size(); ++t) m += p.monitor_history[t].second;
    out->cd_window = m / (double)k;
  }
  if (residual)
    for (size_t k = 0; k < p.residual.size() && k < cap; ++k) residual[k] = p.residual[k];
  return 0;
}
// Post-processing of the current state (run.rs:316-419) with an empty history.
void orc_finish(const OrcCase* c, void* h, OrcPointResult* out) {
  Case cc = to_case(*c);
  PointResult p = finish(cc, *static_cast<Solver*>(h), {}, 0.0, {}, STOP_MAX_ITERATIONS);
  fill_result(p, out);
}
double orc_monitor(const OrcCase* c, void* h) { return monitor(to_case(*c), *static_cast<Solver*>(h)); }
size_t orc_sizeof_case() { return sizeof(OrcCase); }
size_t orc_sizeof_result() { return sizeof(OrcPointResult); }
}
