// TEST INFRASTRUCTURE — f64 restatement of crates/bowshock-core/src/engine/{body_grid,case,numerics,run}.rs and
// crates/bowshock-core/src/atmosphere.rs (power-off bodies; the nozzle grid rows and the fin correlations are out of scope).
#include <algorithm>
#include <stdexcept>

#include "oracle.hpp"

namespace orc {

// ======================================================================== Ogive (bowshock-reference shock_expansion.rs:42-82)
static double ogive_r(double fineness, double x) {
  double l = fineness, R = 0.5;
  if (x >= l) return R;
  x = std::fmax(x, 0.0);
  double rho = (l * l + R * R) / (2.0 * R);
  return std::sqrt(std::fmax(rho * rho - (l - x) * (l - x), 0.0)) - (rho - R);
}
static double ogive_slope(double fineness, double x) {
  double l = fineness, R = 0.5;
  if (x >= l) return 0.0;
  x = std::fmax(x, 0.0);
  double rho = (l * l + R * R) / (2.0 * R);
  return (l - x) / std::sqrt(std::fmax(rho * rho - (l - x) * (l - x), 1e-300));
}

// ======================================================================== body_grid.rs
double Body::nose_length() const {  // body_grid.rs:62-67
  if (nose.kind == NOSE_CONE) return radius() / std::tan(nose.half_angle);
  return nose.fineness;
}
double Body::r(double x) const {  // body_grid.rs:69-88
  if (x <= 0.0) return 0.0;
  double ln = nose_length(), rr = radius();
  if (x >= ln) return rr;
  double eta = x / ln;
  switch (nose.kind) {
    case NOSE_TANGENT_OGIVE:
      return ogive_r(nose.fineness, x);
    case NOSE_CONE:
      return x * std::tan(nose.half_angle);
    case NOSE_POWER:
      return rr * std::pow(eta, nose.param);
    case NOSE_PARABOLIC:
      return rr * (2.0 * eta - nose.param * eta * eta) / (2.0 - nose.param);
    default: {
      double t = 1.0 - 2.0 * eta;
      t = t < -1.0 ? -1.0 : (t > 1.0 ? 1.0 : t);
      double th = std::acos(t);
      double s = std::sin(th);
      return rr * std::sqrt(std::fmax((th - 0.5 * std::sin(2.0 * th) + nose.param * s * s * s) / M_PI, 0.0));
    }
  }
}
double Body::slope(double x) const {  // body_grid.rs:94-108
  double ln = nose_length();
  if (x >= ln) return 0.0;
  switch (nose.kind) {
    case NOSE_TANGENT_OGIVE:
      return ogive_slope(nose.fineness, x);
    case NOSE_CONE:
      return std::tan(nose.half_angle);
    default: {
      double h = 1e-6 * ln;
      double a = std::fmax(x - h, 0.0), b = std::fmin(x + h, ln);
      return (r(b) - r(a)) / (b - a);
    }
  }
}
std::pair<double, double> BaseBody::station(size_t k) const {  // body_grid.rs:269-276
  double x = body.nose_length(), r = body.radius();
  for (size_t t = 0; t < k; ++t) {
    x += segments[t].length;
    r += segments[t].length * segments[t].slope;
  }
  return {x, r};
}
double BaseBody::aft_length() const {  // body_grid.rs:278-280
  double a = 0.0;
  for (const auto& s : segments) a = a + s.length;
  return a;
}
double BaseBody::r(double x) const {  // body_grid.rs:290-311
  if (x <= body.nose_length()) return body.r(x);
  double x0 = body.nose_length(), r0 = body.radius();
  for (const auto& s : segments) {
    double x1 = x0 + s.length;
    if (x < x1) return r0 + (x - x0) * s.slope;
    x0 = x1;
    r0 += s.length * s.slope;
  }
  return base_radius();
}

std::vector<double> two_sided_nodes(double len, size_t n, double dx) {  // body_grid.rs:134-157
  auto node = [&](double delta, size_t k) {
    double t = (double)k / (double)n;
    if (delta < 1e-9) return len * t;
    return 0.5 * len * (1.0 + std::tanh(delta * (t - 0.5)) / std::tanh(0.5 * delta));
  };
  std::vector<double> out(n + 1);
  if (dx >= len / (double)n) {
    for (size_t k = 0; k <= n; ++k) out[k] = node(0.0, k);
    return out;
  }
  double lo = 0.0, hi = 40.0;
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (lo + hi);
    if (node(mid, 1) > dx)
      lo = mid;
    else
      hi = mid;
  }
  double delta = 0.5 * (lo + hi);
  for (size_t k = 0; k <= n; ++k) out[k] = node(delta, k);
  return out;
}

bool axial_nodes(const LargeGridParams& p, std::vector<double>& xs, std::string* err) {  // body_grid.rs:160-205
  const BaseBody& bb = p.body;
  size_t nseg = bb.segments.size();
  double ln = bb.body.nose_length();
  auto bad = [&](const char* m) {
    if (err) *err = m;
    return false;
  };
  if (!(p.x_up > 0.0 && p.x_down > bb.aft_length() && nseg >= 1 && ln > 0.0 && p.dx_tip > 0.0))
    return bad("x_up and dx_tip must be positive and x_down must exceed the aft length");
  if (p.n_seg.size() != nseg) return bad("n_seg needs one entry per body segment");
  for (const auto& s : bb.segments)
    if (!(s.length > 0.0)) return bad("segment lengths must be positive");
  if (!(p.n_up >= 1 && p.n_nose >= 2 && p.n_ext >= 1)) return bad("cell counts");
  for (size_t n : p.n_seg)
    if (n < 1) return bad("cell counts");
  std::vector<double> nose = two_sided_nodes(ln, p.n_nose, p.dx_tip);
  double d_tip = nose[1] - nose[0];
  double d_sh = nose[p.n_nose] - nose[p.n_nose - 1];
  xs.clear();
  std::vector<double> up = geometric_offsets(d_tip, p.x_up, p.n_up);
  for (size_t k = p.n_up; k >= 1; --k) xs.push_back(-up[k]);
  for (double v : nose) xs.push_back(v);
  double d_prev = d_sh;
  for (size_t k = 0; k < nseg; ++k) {
    const Segment& seg = bb.segments[k];
    size_t n = p.n_seg[k];
    double x0 = bb.station(k).first;
    bool geometric_fits = d_prev * (1.0 - std::pow(0.2, (int)n)) / 0.8 < seg.length;
    std::vector<double> offs = (k == nseg - 1 && seg.slope == 0.0 && geometric_fits) ? geometric_offsets(d_prev, seg.length, n)
                                                                                   : two_sided_nodes(seg.length, n, p.dx_tip);
    for (size_t i = 1; i <= n; ++i) xs.push_back(x0 + offs[i]);
    d_prev = offs[n] - offs[n - 1];
  }
  double x_base = bb.x_base();
  std::vector<double> ext = geometric_offsets(d_prev, p.x_down - bb.aft_length(), p.n_ext);
  for (size_t k = 1; k <= p.n_ext; ++k) xs.push_back(x_base + ext[k]);
  return true;
}

std::vector<double> radial_fractions(double dr_wall, double r_far, size_t nj) { return geometric_offsets(dr_wall / r_far, 1.0, nj); }  // body_grid.rs:208-210

bool large_domain_grid(const LargeGridParams& p, Grid& out, std::string* err) {  // body_grid.rs:213-231
  std::vector<double> xs;
  if (!axial_nodes(p, xs, err)) return false;
  if (!(p.nj >= 1 && p.dr_wall > 0.0 && p.r_far > 0.0)) {
    if (err) *err = "nj >= 1, dr_wall > 0 and r_far > 0 are required";
    return false;
  }
  size_t ni = xs.size() - 1, nj = p.nj;
  std::vector<double> sj = radial_fractions(p.dr_wall, p.r_far, nj);
  std::vector<double> x((ni + 1) * (nj + 1)), r((ni + 1) * (nj + 1));
  for (size_t i = 0; i <= ni; ++i) {
    double r_in = p.body.r(xs[i]);
    for (size_t j = 0; j <= nj; ++j) {
      x[j * (ni + 1) + i] = xs[i];
      r[j * (ni + 1) + i] = r_in + sj[j] * (p.r_far - r_in);
    }
  }
  return grid_from_nodes(ni, nj, std::move(x), std::move(r), out, err);
}

bool base_domain_grid(const BaseGridParams& p, Grid& out, Block& blk, std::string* err) {  // body_grid.rs:360-452
  const BaseBody& bb = p.body;
  double ln = bb.body.nose_length();
  auto bad = [&](const char* m) {
    if (err) *err = m;
    return false;
  };
  if (!(p.n_up >= 1 && p.n_nose >= 2 && p.n_wake >= 2 && p.n_gap >= 2 && p.nj_out >= 1)) return bad("cell counts");
  if (bb.segments.empty() || p.n_seg.size() != bb.segments.size()) return bad("n_seg needs one entry >= 1 per body segment");
  for (size_t n : p.n_seg)
    if (n < 1) return bad("n_seg needs one entry >= 1 per body segment");
  for (const auto& s : bb.segments)
    if (!(s.length > 0.0)) return bad("segment lengths must be positive");
  if (!(p.n_sting == 0 || p.n_sting >= 2)) return bad("n_sting must be 0 or >= 2");
  if (bb.sting_radius >= bb.base_radius()) return bad("sting thicker than the base");
  if (!(ln > 0.0 && p.x_up > 0.0 && p.x_down > 0.0 && p.dx_tip > 0.0 && p.dr_wall > 0.0 && p.r_far > bb.base_radius()))
    return bad("x_up, x_down, dx_tip, dr_wall must be positive, r_far must exceed the base radius");
  std::vector<double> nose = two_sided_nodes(ln, p.n_nose, p.dx_tip);
  double d_tip = nose[1] - nose[0];
  std::vector<double> xs;
  std::vector<double> up = geometric_offsets(d_tip, p.x_up, p.n_up);
  for (size_t k = p.n_up; k >= 1; --k) xs.push_back(-up[k]);
  for (double v : nose) xs.push_back(v);
  for (size_t k = 0; k < bb.segments.size(); ++k) {
    std::vector<double> seg_nodes = two_sided_nodes(bb.segments[k].length, p.n_seg[k], p.dx_tip);
    double x0 = bb.station(k).first;
    for (size_t i = 1; i <= p.n_seg[k]; ++i) xs.push_back(x0 + seg_nodes[i]);
  }
  size_t i_end = xs.size() - 1;
  double d_base = xs[i_end] - xs[i_end - 1];
  std::vector<double> wake = geometric_offsets(d_base, p.x_down, p.n_wake);
  double x_base = bb.x_base();
  for (size_t k = 1; k <= p.n_wake; ++k) xs.push_back(x_base + wake[k]);
  size_t ni = xs.size() - 1;
  size_t j_sting = p.n_sting, j_end = p.n_sting + p.n_gap;
  size_t nj = j_end + p.nj_out;
  double re = bb.base_radius(), rs = bb.sting_radius;
  std::vector<double> gap(p.n_gap + 1);
  if (p.gap_one_sided) {
    std::vector<double> off = geometric_offsets(p.dr_wall, re - rs, p.n_gap);
    for (size_t k = 0; k <= p.n_gap; ++k) gap[k] = (re - rs) - off[p.n_gap - k];
  } else {
    gap = two_sided_nodes(re - rs, p.n_gap, p.dr_wall);
  }
  std::vector<double> sj = radial_fractions(p.dr_wall, p.r_far - re, p.nj_out);
  std::vector<double> x((ni + 1) * (nj + 1)), r((ni + 1) * (nj + 1));
  for (size_t i = 0; i <= ni; ++i) {
    double rw = bb.r(xs[i]);
    for (size_t j = 0; j <= nj; ++j) {
      double rad;
      if (i >= i_end) {
        if (j <= j_sting)
          rad = rs - (double)(j_sting - j) * p.dr_wall;
        else if (j <= j_end)
          rad = rs + gap[j - j_sting];
        else
          rad = re + sj[j - j_end] * (p.r_far - re);
      } else if (j <= j_end) {
        rad = rw - (double)(j_end - j) * p.dr_wall;
      } else {
        rad = rw + sj[j - j_end] * (p.r_far - rw);
      }
      x[j * (ni + 1) + i] = xs[i];
      r[j * (ni + 1) + i] = rad;
    }
  }
  if (!grid_from_nodes(ni, nj, std::move(x), std::move(r), out, err)) return false;
  blk = Block{i_end, j_end, j_sting};
  return true;
}

// ======================================================================== numerics.rs
static ImplicitParams rans_implicit() {  // numerics.rs:245
  ImplicitParams p;
  p.dt_mode = DT_SUM;
  p.cfl_max = 50.0;
  p.sub_iters = 3;
  return p;
}
static ImplicitParams rans_implicit_supersonic() {  // numerics.rs:258
  ImplicitParams p = rans_implicit();
  p.cfl_max = 20.0;
  return p;
}
Numerics numerics_subsonic(unsigned level, int wake) {  // numerics.rs:291-310
  Numerics n;
  n.cfl = 0.5;
  n.limiter = VAN_ALBADA;
  n.low_mach = true;
  n.scheme.kind = SCHEME_IMPLICIT;
  n.scheme.imp = implicit_default();
  n.first_order_iters = 100;
  n.max_iter = (size_t)10000 << level;
  n.min_iter = 0;
  n.drop_orders = 6.0;
  n.outflow = BC_CHARACTERISTIC;
  n.monitor_window = 2000;
  n.has_monitor_tol = wake == WAKE_BASE;
  n.monitor_tol = 1e-3;
  return n;
}
Numerics numerics_transonic() {  // numerics.rs:313-329
  Numerics n;
  n.cfl = 0.5;
  n.limiter = MINMOD;
  n.low_mach = false;
  n.scheme.kind = SCHEME_EXPLICIT;
  n.first_order_iters = 300;
  n.max_iter = 60000;
  n.min_iter = 0;
  n.drop_orders = 6.0;
  n.outflow = BC_CHARACTERISTIC;
  n.monitor_window = 2000;
  n.has_monitor_tol = true;
  n.monitor_tol = 2e-4;
  return n;
}
Numerics numerics_auto(double mach, unsigned level, int wake) {  // numerics.rs:332-339
  Numerics n = mach < REGIME_SPLIT_MACH ? numerics_subsonic(level, wake) : numerics_transonic();
  n.has_monitor_tol = true;
  n.monitor_tol = wake == WAKE_BASE ? 1e-3 : 2e-4;
  return n;
}
Numerics numerics_viscous(double mach, unsigned level) {  // numerics.rs:345-362
  bool subsonic = mach < REGIME_SPLIT_MACH;
  Numerics n;
  n.cfl = 0.5;
  n.limiter = subsonic ? VAN_ALBADA : MINMOD;
  n.low_mach = subsonic;
  n.scheme.kind = SCHEME_IMPLICIT;
  n.scheme.imp = mach < 1.0 ? rans_implicit() : rans_implicit_supersonic();
  n.first_order_iters = 200;
  n.max_iter = (size_t)80000 << level;
  n.min_iter = 0;
  n.drop_orders = 5.0;
  n.outflow = BC_CHARACTERISTIC;
  n.monitor_window = 2000;
  n.has_monitor_tol = true;
  n.monitor_tol = 1e-4;
  n.has_mean_window = true;
  n.mean_window = 6000;
  return n;
}

// ======================================================================== case.rs
static size_t even_ceil(double x) {  // case.rs:179-182
  size_t n = (size_t)std::ceil(x);
  return n + n % 2;
}
size_t layer_count(double h, double y1) { return even_ceil(std::log(1.0 + 0.2 * h / y1) / std::log(1.2)); }  // case.rs:185-187

static LargeGridParams sting_grid(const BaseBody& body, unsigned level) {  // case.rs:190-227
  size_t f = (size_t)1 << level;
  double dx_tip = 0.03 / (double)f;
  double l_body = body.x_base();
  size_t nseg = body.segments.size();
  auto count = [&](size_t per, double length) { return std::max<size_t>(std::min(per, even_ceil(length / dx_tip)), 4); };
  LargeGridParams p;
  p.body = body;
  for (size_t k = 0; k < nseg; ++k) {
    const Segment& s = body.segments[k];
    size_t per = s.slope != 0.0 ? 24 * f : (k + 1 == nseg ? 36 * f : 40 * f);
    p.n_seg.push_back(count(per, s.length));
  }
  p.x_up = 10.0 * l_body;
  p.x_down = 5.0 * l_body;
  p.r_far = 10.0 * l_body;
  p.n_up = 30 * f;
  p.n_nose = 48 * f;
  p.n_ext = 30 * f;
  p.nj = 70 * f;
  p.dx_tip = dx_tip;
  p.dr_wall = 0.03 / (double)f;
  return p;
}

Case case_new(double mach, const BaseBody& body, unsigned level, int wake, const Numerics& n) {  // case.rs:51-78
  size_t f = (size_t)1 << level;
  double dx_tip = 0.03 / (double)f;
  double l_body = body.x_base();
  size_t n_sting = body.sting_radius > 0.0 ? 4 * f : 0;
  auto count = [&](size_t per, double length) { return std::max<size_t>(std::min(per, even_ceil(length / dx_tip)), 4); };
  Case c;
  c.mach = mach;
  c.body = body;
  c.wake = wake;
  BaseGridParams& g = c.grid_base;
  g.body = body;
  for (const auto& s : body.segments) g.n_seg.push_back(count(s.slope == 0.0 ? 40 * f : 24 * f, s.length));
  g.x_up = 10.0 * l_body;
  g.x_down = 5.0 * l_body;
  g.r_far = 10.0 * l_body;
  g.n_up = 28 * f;
  g.n_nose = 48 * f;
  g.n_wake = 40 * f;
  g.n_sting = n_sting;
  g.n_gap = 12 * f;
  g.nj_out = 64 * f;
  g.dx_tip = dx_tip;
  g.dr_wall = 0.03 / (double)f;
  g.gap_one_sided = false;
  c.grid_sting = sting_grid(body, level);
  c.numerics = n;
  return c;
}

Case case_viscous(double mach, const BaseBody& body, unsigned level, int wake, double re_c, double sutherland, double mach_max) {  // case.rs:84-102
  Case c = case_new(mach, body, level, wake, numerics_viscous(mach, level));
  double cf = 0.027 * std::pow(re_c * mach_max * c.body.x_base(), -1.0 / 7.0);
  double y1 = 1.0 / (re_c * mach_max * std::sqrt(0.5 * cf));
  double re = c.body.base_radius(), rs = c.body.sting_radius;
  c.grid_base.dr_wall = y1;
  c.grid_base.nj_out = layer_count(c.grid_base.r_far - re, y1);
  c.grid_base.n_gap = layer_count(re - rs, y1);
  c.grid_base.gap_one_sided = true;
  c.grid_sting.dr_wall = y1;
  c.grid_sting.nj = layer_count(c.grid_sting.r_far, y1);
  size_t wall_i_start = wake == WAKE_BASE ? c.grid_base.n_up : c.grid_sting.n_up;
  c.has_viscous = true;
  c.viscous = Viscous{re_c, sutherland, TURB_SST, wall_i_start, 0.0};
  return c;
}

bool case_build_solver(const Case& c, Solver& s, std::string* err) {  // case.rs:147-176
  const Numerics& n = c.numerics;
  Config cfg;
  cfg.cfl = n.cfl;
  cfg.limiter = n.limiter;
  cfg.freestream = freestream(c.mach);
  cfg.bc[0] = BC_CHARACTERISTIC;
  cfg.bc[1] = n.outflow;
  cfg.bc[2] = BC_SLIPWALL;
  cfg.bc[3] = BC_CHARACTERISTIC;
  cfg.first_order_iters = n.first_order_iters;
  Grid g;
  if (c.wake == WAKE_BASE) {
    Block b;
    if (!base_domain_grid(c.grid_base, g, b, err)) return false;
    s = Solver(std::move(g), cfg);
    s.set_block(&b);
  } else {
    if (!large_domain_grid(c.grid_sting, g, err)) return false;
    s = Solver(std::move(g), cfg);
  }
  s.low_mach = n.low_mach;
  s.set_scheme(n.scheme);
  s.set_viscous(c.has_viscous ? &c.viscous : nullptr);
  return true;
}

// ======================================================================== atmosphere.rs:84-112
bool isa_state(double h, AirState& out) {
  const double R = 287.05287, G = 1.4, T0 = 288.15, P0 = 101325.0, LAPSE = 0.0065, TROP = 11000.0, CEIL = 20000.0, TS = 216.65,
               PT = 22632.06, HS = 6341.62, PEXP = 5.255877, MU_REF = 1.716e-5, T_REF = 273.15;
  double t, p;
  if (h >= 0.0 && h <= TROP) {
    t = T0 - LAPSE * h;
    p = P0 * std::pow(t / T0, PEXP);
  } else if (h > TROP && h <= CEIL) {
    t = TS;
    p = PT * std::exp(-(h - TROP) / HS);
  } else {
    return false;
  }
  out.temperature_k = t;
  out.pressure_pa = p;
  out.density = p / (R * t);
  out.sound_speed = std::sqrt(G * R * t);
  out.viscosity = MU_REF * std::pow(t / T_REF, 1.5) * (T_REF + SUTHERLAND_S) / (t + SUTHERLAND_S);
  return true;
}

// ======================================================================== run.rs
void wall_distribution(const BaseBody& body, const Solver& s, std::vector<WallPoint>& wall, double& cd, double& cd_cell) {  // run.rs:252-282
  const Grid& g = s.grid;
  size_t ni = g.ni;
  const Prim fs = s.cfg.freestream;
  double p_inf = fs[3], q_inf = 0.5 * fs[0] * fs[1] * fs[1];
  auto cp = [&](double p) { return (p - p_inf) / q_inf; };
  double ln = body.body.nose_length(), rb2 = body.body.radius() * body.body.radius();
  wall.clear();
  cd = 0.0;
  cd_cell = 0.0;
  size_t i_wall_end = s.has_block ? s.block.i_end : ni;
  for (size_t i = 0; i < i_wall_end; ++i) {
    size_t j0 = s.has_block ? s.block.col_start(i) : 0;
    auto n0 = g.node(i, j0), n1 = g.node(i + 1, j0);
    double xm = 0.5 * (n0.first + n1.first), rm = 0.5 * (n0.second + n1.second);
    if (xm <= 0.0) continue;
    double p0 = s.pressure(i, j0), p1 = s.pressure(i, j0 + 1);
    double d0 = std::hypot(g.xc[j0 * ni + i] - xm, g.rc[j0 * ni + i] - rm);
    double d1 = std::hypot(g.xc[(j0 + 1) * ni + i] - xm, g.rc[(j0 + 1) * ni + i] - rm);
    double pw = p0 + (p0 - p1) * d0 / (d1 - d0);
    double s0 = n0.second * n0.second / rb2, s1 = n1.second * n1.second / rb2;
    if (n1.first <= ln + 1e-12) {
      cd += cp(pw) * (s1 - s0);
      cd_cell += cp(p0) * (s1 - s0);
    }
    wall.push_back(WallPoint{xm, rm, s0, s1, cp(pw), cp(p0)});
  }
}

static std::vector<double> aft_drag(const BaseBody& bb, const std::vector<WallPoint>& wall) {  // run.rs:188-199
  std::vector<double> cd_aft(bb.segments.size(), 0.0);
  std::vector<double> stations;
  for (size_t k = 0; k <= bb.segments.size(); ++k) stations.push_back(bb.station(k).first);
  for (const auto& w : wall)
    for (size_t k = 0; k < cd_aft.size(); ++k)
      if (w.x >= stations[k] && w.x < stations[k + 1]) {
        cd_aft[k] += w.cp * (w.s1 - w.s0);
        break;
      }
  return cd_aft;
}

void friction(const Case& c, const Solver& s, double& cd, double& y_plus_max) {  // run.rs:207-248
  if (!s.has_viscous) {
    cd = 0.0;
    y_plus_max = NAN;
    return;
  }
  const Viscous& v = s.viscous;
  const Grid& g = s.grid;
  size_t ni = g.ni;
  const Prim fs = s.cfg.freestream;
  double q_inf = 0.5 * fs[0] * fs[1] * fs[1];
  double r2 = c.body.body.radius() * c.body.body.radius();
  double x_base = c.body.x_base();
  std::vector<size_t> rows;
  if (!s.has_block)
    rows = {0};
  else
    rows = {s.block.j_end, s.block.j_sting};
  cd = 0.0;
  y_plus_max = 0.0;
  Walls wl = s.walls();
  for (size_t j : rows)
    for (size_t i = 0; i < ni; ++i) {
      if (!wl.noslip_jface(i, j)) continue;
      auto n0 = g.node(i, j), n1 = g.node(i + 1, j);
      double xm = 0.5 * (n0.first + n1.first);
      if (xm >= x_base) continue;
      const Face& f = g.jface[j * ni + i];
      size_t cc = j * ni + i;
      Prim w = cons_to_prim(s.u[cc]);
      double tx = f.nr, tr = -f.nx;
      double u_t = w[1] * tx + w[2] * tr;
      double d_n = std::fabs((g.xc[cc] - xm) * f.nx + (g.rc[cc] - f.rm) * f.nr);
      double mu = v.mu(temperature(w));
      double mu_tw = v.rough() ? w[0] * aupoix_wall(mu / w[0], std::hypot(w[1], w[2]), d_n, v.roughness)[2] : 0.0;
      double tau = (mu + mu_tw) * u_t / d_n;
      cd += 2.0 * tau * tx * f.rm * f.len / (q_inf * r2);
      y_plus_max = std::fmax(y_plus_max, d_n * std::sqrt(w[0] * std::fabs(tau)) / mu);
    }
}

void base_state(const Solver& s, double rb2, double& cd, double& mean, double& mean_cell) {  // run.rs:286-313
  cd = 0.0;
  if (!s.has_block) {
    mean = NAN;
    mean_cell = NAN;
    return;
  }
  const Grid& g = s.grid;
  size_t ni = g.ni;
  const Prim fs = s.cfg.freestream;
  double p_inf = fs[3], q_inf = 0.5 * fs[0] * fs[1] * fs[1];
  auto cp = [&](double p) { return (p - p_inf) / q_inf; };
  size_t ie = s.block.i_end;
  double m = 0.0, mc = 0.0, s_sum = 0.0;
  size_t j0 = s.has_nozzle ? s.nozzle.j_end : s.block.j_sting;
  for (size_t j = j0; j < s.block.j_end; ++j) {
    auto n0 = g.node(ie, j), n1 = g.node(ie, j + 1);
    double xm = n0.first, rm = 0.5 * (n0.second + n1.second);
    double p0 = s.pressure(ie, j), p1 = s.pressure(ie + 1, j);
    double d0 = std::hypot(g.xc[j * ni + ie] - xm, g.rc[j * ni + ie] - rm);
    double d1 = std::hypot(g.xc[j * ni + ie + 1] - xm, g.rc[j * ni + ie + 1] - rm);
    double pw = p0 + (p0 - p1) * d0 / (d1 - d0);
    double ds = (n1.second * n1.second - n0.second * n0.second) / rb2;
    cd -= cp(pw) * ds;
    m += cp(pw) * ds;
    mc += cp(p0) * ds;
    s_sum += ds;
  }
  mean = m / s_sum;
  mean_cell = mc / s_sum;
}

double monitor(const Case& c, const Solver& s) {  // run.rs:174-185
  const BaseBody& bb = c.body;
  double rb2 = bb.body.radius() * bb.body.radius();
  if (c.has_viscous) {
    std::vector<WallPoint> wall;
    double cd_nose, cd_cell;
    wall_distribution(bb, s, wall, cd_nose, cd_cell);
    double fore = cd_nose;
    for (double a : aft_drag(bb, wall)) fore = fore + a;
    double cf, yp;
    friction(c, s, cf, yp);
    double cb, mn, mc;
    base_state(s, rb2, cb, mn, mc);
    return fore + cf + cb;
  }
  if (c.wake == WAKE_STING) {
    std::vector<WallPoint> wall;
    double cd_nose, cd_cell;
    wall_distribution(bb, s, wall, cd_nose, cd_cell);
    return cd_nose;
  }
  double cb, mn, mc;
  base_state(s, rb2, cb, mn, mc);
  return mn;
}

bool mean_stationary(const std::vector<std::pair<size_t, double>>& hist, size_t k) {  // run.rs:157-170
  size_t from = 0;
  while (from < hist.size() && hist[from].first <= 2000) ++from;
  size_t hn = hist.size() - from;
  if (k == 0 || hn < 2 * k) return false;
  const auto* w = &hist[hist.size() - 2 * k];
  double m0 = 0, m1 = 0;
  for (size_t t = 0; t < k; ++t) m0 += w[t].second;
  for (size_t t = k; t < 2 * k; ++t) m1 += w[t].second;
  m0 /= (double)k;
  m1 /= (double)k;
  double m = 0.5 * (m0 + m1);
  double lo = INFINITY, hi = -INFINITY;
  for (size_t t = 0; t < 2 * k; ++t) {
    lo = std::fmin(lo, w[t].second);
    hi = std::fmax(hi, w[t].second);
  }
  double a = w[2 * k - 2].second - m, b = w[2 * k - 1].second - m;
  return std::fabs(m1 - m0) <= 2e-3 * std::fabs(m) && hi - lo <= 0.05 * std::fabs(m) && a * b < 0.0;
}

bool stop_reason(const Case& c, size_t it, double r, double reference, size_t skip, const std::vector<std::pair<size_t, double>>& hist,
                 int& why) {  // run.rs:105-150
  const Numerics& n = c.numerics;
  if (!std::isfinite(r) || (!hist.empty() && hist.back().first == it + 1 &&
                            (!std::isfinite(hist.back().second) || std::fabs(hist.back().second) > MONITOR_LIMIT))) {
    why = STOP_NON_FINITE;
    return true;
  }
  if (it + 1 < n.min_iter) return false;
  if (it > skip && reference / r >= std::pow(10.0, n.drop_orders)) {
    why = STOP_RESIDUAL_DROP;
    return true;
  }
  if (n.has_drag_rel_tol) {
    size_t k = DRAG_REL_WINDOW / MONITOR_EVERY;
    if (c.has_viscous && !hist.empty() && hist.back().first == it + 1 && it + 1 >= DRAG_REL_WINDOW && reference / r >= 100.0 &&
        hist.size() >= k) {
      double lo = INFINITY, hi = -INFINITY, mean = 0.0;
      for (size_t t = hist.size() - k; t < hist.size(); ++t) {
        lo = std::fmin(lo, hist[t].second);
        hi = std::fmax(hi, hist[t].second);
        mean += hist[t].second;
      }
      mean /= (double)k;
      if (hi - lo < n.drag_rel_tol * std::fabs(mean)) {
        why = STOP_CD_STATIONARY;
        return true;
      }
    }
  }
  if (n.has_monitor_tol) {
    if (it % 500 == 499 && it + 1 >= 2 * n.monitor_window && reference / r >= 100.0) {
      size_t k = n.monitor_window / MONITOR_EVERY;
      double lo = INFINITY, hi = -INFINITY;
      for (size_t t = hist.size() - k; t < hist.size(); ++t) {
        lo = std::fmin(lo, hist[t].second);
        hi = std::fmax(hi, hist[t].second);
      }
      if (hi - lo < n.monitor_tol) {
        why = (!c.has_viscous && c.wake == WAKE_BASE) ? STOP_BASE_PRESSURE_STATIONARY : STOP_CD_STATIONARY;
        return true;
      }
    }
  }
  if (c.has_viscous && n.has_mean_window && !hist.empty()) {
    if (hist.back().first == it + 1 && mean_stationary(hist, n.mean_window / MONITOR_EVERY)) {
      why = STOP_MEAN_STATIONARY;
      return true;
    }
  }
  return false;
}

PointResult run_on(const Case& c, Solver& s, bool warm, const double* r_ref) {  // run.rs:44-89
  const Numerics& n = c.numerics;
  s.cfg.freestream = freestream(c.mach);
  s.cfg.cfl = n.cfl;
  s.cfg.limiter = n.limiter;
  s.cfg.first_order_iters = n.first_order_iters;
  s.low_mach = n.low_mach;
  if (!scheme_eq(s.scheme, n.scheme)) s.set_scheme(n.scheme);
  if (!warm) {
    Cons q = prim_to_cons(freestream(c.mach));
    std::fill(s.u.begin(), s.u.end(), q);
    if (s.has_viscous) {
      Viscous v = s.viscous;
      s.set_viscous(&v);
    }
  }
  s.iter = warm ? n.first_order_iters : 0;
  s.restart_ramp();
  size_t skip = warm ? 0 : 20;
  bool sample = c.wake == WAKE_BASE || n.has_monitor_tol || n.has_drag_rel_tol;
  std::vector<double> residual;
  std::vector<std::pair<size_t, double>> hist;
  double rmax = 0.0;
  int reason = STOP_MAX_ITERATIONS;
  for (size_t it = 0; it < n.max_iter; ++it) {
    double r = s.step();
    residual.push_back(r);
    if (it >= skip) rmax = std::fmax(rmax, r);
    if (sample && it % MONITOR_EVERY == MONITOR_EVERY - 1) hist.emplace_back(it + 1, monitor(c, s));
    int why;
    if (stop_reason(c, it, r, r_ref ? *r_ref : rmax, skip, hist, why)) {
      reason = why;
      break;
    }
  }
  return finish(c, s, std::move(residual), rmax, std::move(hist), reason);
}

PointResult finish(const Case& c, const Solver& s, std::vector<double> residual, double rmax, std::vector<std::pair<size_t, double>> hist,
                   int reason) {  // run.rs:316-419 (the fields this build reports)
  const Grid& g = s.grid;
  size_t ni = g.ni, nj = g.nj;
  const Prim fs = s.cfg.freestream;
  double p_inf = fs[3];
  const BaseBody& bb = c.body;
  double rb2 = bb.body.radius() * bb.body.radius();
  PointResult pr;
  std::vector<WallPoint> wall;
  wall_distribution(bb, s, wall, pr.cd_nose, pr.cd_nose_cell);
  pr.cd_aft = aft_drag(bb, wall);
  base_state(s, rb2, pr.cd_base, pr.cp_base, pr.cp_base_cell);
  double m_wall_max = 0.0;
  size_t i_wall_end = s.has_block ? s.block.i_end : ni;
  for (size_t i = 0; i < i_wall_end; ++i) {
    size_t j0 = s.has_block ? s.block.col_start(i) : 0;
    if (g.xc[j0 * ni + i] > 0.0) {
      Prim w = cons_to_prim(s.u[j0 * ni + i]);
      m_wall_max = std::fmax(m_wall_max, std::hypot(w[1], w[2]) / sound_speed(w));
    }
  }
  auto dev = [&](size_t i, size_t j) { return std::fabs(s.pressure(i, j) / p_inf - 1.0); };
  double farfield_dp = 0.0;
  for (size_t i = 0; i < ni; ++i) farfield_dp = std::fmax(farfield_dp, dev(i, nj - 1));
  for (size_t j = 0; j < nj; ++j) farfield_dp = std::fmax(std::fmax(farfield_dp, dev(0, j)), dev(ni - 1, j));
  double min_rho = INFINITY, min_p = INFINITY, m_max = 0.0;
  for (size_t cc = 0; cc < s.u.size(); ++cc) {
    if (s.has_block && s.block.solid(cc % ni, cc / ni)) continue;
    Prim w = cons_to_prim(s.u[cc]);
    min_rho = std::fmin(min_rho, w[0]);
    min_p = std::fmin(min_p, w[3]);
    m_max = std::fmax(m_max, std::hypot(w[1], w[2]) / sound_speed(w));
  }
  double fore = pr.cd_nose;
  for (double a : pr.cd_aft) fore = fore + a;
  friction(c, s, pr.cd_friction, pr.y_plus_max);
  pr.cd_total = fore + pr.cd_friction + pr.cd_base;
  double last = residual.empty() ? rmax : residual.back();
  pr.drop_orders = (rmax > 0.0 && last > 0.0) ? std::log10(rmax / last) : 0.0;
  pr.iters = residual.size();
  pr.residual = std::move(residual);
  pr.residual_peak = rmax;
  pr.stop_reason = reason;
  pr.farfield_dp = farfield_dp;
  pr.min_rho = min_rho;
  pr.min_p = min_p;
  pr.m_max = m_max;
  pr.m_wall_max = m_wall_max;
  pr.monitor_history = std::move(hist);
  return pr;
}

}  // namespace orc
