// TEST INFRASTRUCTURE — f64 restatement of crates/bowshock-cfd/src/{gas,grid,flux,bc,solver,implicit,multigrid,viscous,
// turbulence}.rs. Every function names the reference lines it follows; the evaluation order of the reference is kept.
// OpenMP parallel-for loops over rows / lines stand where the reference uses rayon's par_chunks_mut (same granularity);
// every row is independent, so results do not depend on the thread count.
#include <algorithm>
#include <cstdint>
#include <stdexcept>

#include "oracle.hpp"

namespace orc {

static inline double fmax_rs(double a, double b) { return std::fmax(a, b); }  // Rust f64::max (NaN-ignoring)
static inline double fmin_rs(double a, double b) { return std::fmin(a, b); }
static inline double clamp_rs(double x, double lo, double hi) {  // Rust f64::clamp (NaN stays NaN)
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}

// ======================================================================== gas.rs
Cons prim_to_cons(const Prim& w) {  // gas.rs:12-16
  double rho = w[0], u = w[1], v = w[2], p = w[3];
  return {rho, rho * u, rho * v, p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v)};
}
Prim cons_to_prim(const Cons& q) {  // gas.rs:18-24
  double rho = q[0];
  double u = q[1] / rho;
  double v = q[2] / rho;
  double p = (GAMMA - 1.0) * (q[3] - 0.5 * rho * (u * u + v * v));
  return {rho, u, v, p};
}
double sound_speed(const Prim& w) { return std::sqrt(GAMMA * w[3] / w[0]); }  // gas.rs:27-29
Cons physical_flux(const Prim& w, double nx, double nr) {                     // gas.rs:33-38
  double rho = w[0], u = w[1], v = w[2], p = w[3];
  double un = u * nx + v * nr;
  double e = p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v);
  return {rho * un, rho * u * un + p * nx, rho * v * un + p * nr, (e + p) * un};
}
Prim freestream(double mach) { return {1.0, mach, 0.0, 1.0 / GAMMA}; }  // gas.rs:41-43
Prim reflect(const Prim& w, double nx, double nr) {                      // gas.rs:47-50
  double un = w[1] * nx + w[2] * nr;
  return {w[0], w[1] - 2.0 * un * nx, w[2] - 2.0 * un * nr, w[3]};
}

// ======================================================================== grid.rs
bool grid_from_nodes(size_t ni, size_t nj, std::vector<double> x, std::vector<double> r, Grid& out, std::string* err) {
  // grid.rs:65-119
  if (x.size() != (ni + 1) * (nj + 1) || r.size() != x.size()) {
    if (err) *err = "node array size mismatch";
    return false;
  }
  auto nn = [&](size_t i, size_t j) { return j * (ni + 1) + i; };
  Grid g;
  g.ni = ni;
  g.nj = nj;
  g.iface.assign((ni + 1) * nj, Face{});
  for (size_t j = 0; j < nj; ++j)
    for (size_t i = 0; i <= ni; ++i) {
      size_t a = nn(i, j), b = nn(i, j + 1);
      double dx = x[b] - x[a], dr = r[b] - r[a];
      double len = std::hypot(dx, dr);
      g.iface[j * (ni + 1) + i] = Face{dr / len, -dx / len, len, 0.5 * (r[a] + r[b])};
    }
  g.jface.assign(ni * (nj + 1), Face{});
  for (size_t j = 0; j <= nj; ++j)
    for (size_t i = 0; i < ni; ++i) {
      size_t a = nn(i, j), b = nn(i + 1, j);
      double dx = x[b] - x[a], dr = r[b] - r[a];
      double len = std::hypot(dx, dr);
      g.jface[j * ni + i] = Face{-dr / len, dx / len, len, 0.5 * (r[a] + r[b])};
    }
  g.area.assign(ni * nj, 0.0);
  g.vol.assign(ni * nj, 0.0);
  g.xc.assign(ni * nj, 0.0);
  g.rc.assign(ni * nj, 0.0);
  for (size_t j = 0; j < nj; ++j)
    for (size_t i = 0; i < ni; ++i) {
      size_t p[4] = {nn(i, j), nn(i + 1, j), nn(i + 1, j + 1), nn(i, j + 1)};
      double a = 0, v = 0, sx = 0, sr = 0;
      const int tris[2][3] = {{0, 1, 2}, {0, 2, 3}};
      for (auto& t : tris) {
        size_t k0 = p[t[0]], k1 = p[t[1]], k2 = p[t[2]];
        double at = 0.5 * ((x[k1] - x[k0]) * (r[k2] - r[k0]) - (x[k2] - x[k0]) * (r[k1] - r[k0]));
        double cx = (x[k0] + x[k1] + x[k2]) / 3.0;
        double cr = (r[k0] + r[k1] + r[k2]) / 3.0;
        a += at;
        v += at * cr;
        sx += at * cx;
        sr += at * cr;
      }
      if (a <= 0.0 || std::isnan(a)) {
        if (err) *err = "non-positive cell area at (" + std::to_string(i) + "," + std::to_string(j) + ")";
        return false;
      }
      size_t c = j * ni + i;
      g.area[c] = a;
      g.vol[c] = v;
      g.xc[c] = sx / a;
      g.rc[c] = sr / a;
    }
  g.x = std::move(x);
  g.r = std::move(r);
  out = std::move(g);
  return true;
}

Grid grid_from_nodes_or_throw(size_t ni, size_t nj, std::vector<double> x, std::vector<double> r) {
  Grid g;
  std::string e;
  if (!grid_from_nodes(ni, nj, std::move(x), std::move(r), g, &e)) throw std::runtime_error(e);
  return g;
}

bool grid_coarsen(const Grid& g, Grid& out) {  // grid.rs:129-144
  if (g.ni % 2 || g.nj % 2) return false;
  size_t ci = g.ni / 2, cj = g.nj / 2;
  std::vector<double> x, r;
  x.reserve((ci + 1) * (cj + 1));
  r.reserve((ci + 1) * (cj + 1));
  for (size_t j = 0; j <= cj; ++j)
    for (size_t i = 0; i <= ci; ++i) {
      size_t k = 2 * j * (g.ni + 1) + 2 * i;
      x.push_back(g.x[k]);
      r.push_back(g.r[k]);
    }
  out = grid_from_nodes_or_throw(ci, cj, std::move(x), std::move(r));
  return true;
}

std::vector<double> geometric_offsets(double first, double length, size_t n) {  // grid.rs:199-228
  auto sum = [&](double q) {
    double s = 0.0, d = first;
    for (size_t k = 0; k < n; ++k) {
      s += d;
      d *= q;
    }
    return s;
  };
  double lo = 0.2, hi = 4.0;
  for (int k = 0; k < 200; ++k) {
    double mid = 0.5 * (lo + hi);
    if (sum(mid) < length)
      lo = mid;
    else
      hi = mid;
  }
  double q = 0.5 * (lo + hi);
  std::vector<double> v;
  v.reserve(n + 1);
  double s = 0.0, d = first;
  for (size_t k = 0; k < n; ++k) {
    v.push_back(s);
    s += d;
    d *= q;
  }
  v.push_back(length);
  return v;
}

// ======================================================================== flux.rs
double limited_slope(double a, double b, int lim) {  // flux.rs:18-50
  switch (lim) {
    case FIRST_ORDER:
      return 0.0;
    case MINMOD:
      if (a * b <= 0.0) return 0.0;
      return std::fabs(a) < std::fabs(b) ? a : b;
    case VAN_ALBADA: {
      const double EPS = 1e-14;
      if (a * b <= 0.0) return 0.0;
      return (a * (b * b + EPS) + b * (a * a + EPS)) / (a * a + b * b + 2.0 * EPS);
    }
    default: {
      const double EPS = 1e-14;
      if (a * b <= 0.0) return 0.0;
      return 2.0 * b * (a * a + a * b + EPS) / (2.0 * a * a + a * b + b * b + 2.0 * EPS);
    }
  }
}

void reconstruct(const Prim& m2, const Prim& m1, const Prim& p0, const Prim& p1, int lim, Prim& l, Prim& r) {  // flux.rs:56-72
  l = m1;
  r = p0;
  for (int k = 0; k < 4; ++k) {
    double phi_l = limited_slope(m1[k] - m2[k], p0[k] - m1[k], lim);
    double phi_r = limited_slope(p0[k] - m1[k], p1[k] - p0[k], lim);
    l[k] = m1[k] + 0.5 * phi_l;
    r[k] = p0[k] - 0.5 * phi_r;
  }
  if (l[0] <= 0.0 || l[3] <= 0.0) l = m1;
  if (r[0] <= 0.0 || r[3] <= 0.0) r = p0;
}

Cons hllc(const Prim& wl, const Prim& wr, double nx, double nr) {  // flux.rs:79-126
  double rl = wl[0], ul = wl[1], vl = wl[2], pl = wl[3];
  double rr = wr[0], ur = wr[1], vr = wr[2], pr = wr[3];
  double unl = ul * nx + vl * nr;
  double unr = ur * nx + vr * nr;
  double cl = std::sqrt(GAMMA * pl / rl);
  double cr = std::sqrt(GAMMA * pr / rr);
  double el = pl / (GAMMA - 1.0) + 0.5 * rl * (ul * ul + vl * vl);
  double er = pr / (GAMMA - 1.0) + 0.5 * rr * (ur * ur + vr * vr);
  double sql = std::sqrt(rl), sqr = std::sqrt(rr);
  double inv = 1.0 / (sql + sqr);
  double uh = (sql * ul + sqr * ur) * inv;
  double vh = (sql * vl + sqr * vr) * inv;
  double hl = (el + pl) / rl;
  double hr = (er + pr) / rr;
  double hh = (sql * hl + sqr * hr) * inv;
  double ch2 = (GAMMA - 1.0) * (hh - 0.5 * (uh * uh + vh * vh));
  double ch = std::sqrt(fmax_rs(ch2, 1e-300));
  double unh = uh * nx + vh * nr;
  double sl = fmin_rs(unl - cl, unh - ch);
  double sr = fmax_rs(unr + cr, unh + ch);
  if (sl >= 0.0) return physical_flux(wl, nx, nr);
  if (sr <= 0.0) return physical_flux(wr, nx, nr);
  double sm = (pr - pl + rl * unl * (sl - unl) - rr * unr * (sr - unr)) / (rl * (sl - unl) - rr * (sr - unr));
  if (sm >= 0.0) {
    Cons f = physical_flux(wl, nx, nr);
    double fac = rl * (sl - unl) / (sl - sm);
    Cons us = {fac, fac * (ul + (sm - unl) * nx), fac * (vl + (sm - unl) * nr),
               fac * (el / rl + (sm - unl) * (sm + pl / (rl * (sl - unl))))};
    Cons q = {rl, rl * ul, rl * vl, el};
    return {f[0] + sl * (us[0] - q[0]), f[1] + sl * (us[1] - q[1]), f[2] + sl * (us[2] - q[2]), f[3] + sl * (us[3] - q[3])};
  } else {
    Cons f = physical_flux(wr, nx, nr);
    double fac = rr * (sr - unr) / (sr - sm);
    Cons us = {fac, fac * (ur + (sm - unr) * nx), fac * (vr + (sm - unr) * nr),
               fac * (er / rr + (sm - unr) * (sm + pr / (rr * (sr - unr))))};
    Cons q = {rr, rr * ur, rr * vr, er};
    return {f[0] + sr * (us[0] - q[0]), f[1] + sr * (us[1] - q[1]), f[2] + sr * (us[2] - q[2]), f[3] + sr * (us[3] - q[3])};
  }
}

Cons rusanov(const Prim& wl, const Prim& wr, double nx, double nr) {  // flux.rs:132-147
  double rl = wl[0], ul = wl[1], vl = wl[2], pl = wl[3];
  double rr = wr[0], ur = wr[1], vr = wr[2], pr = wr[3];
  double unl = ul * nx + vl * nr;
  double unr = ur * nx + vr * nr;
  double smax = fmax_rs(std::fabs(unl) + std::sqrt(GAMMA * pl / rl), std::fabs(unr) + std::sqrt(GAMMA * pr / rr));
  Cons fl = physical_flux(wl, nx, nr), fr = physical_flux(wr, nx, nr);
  Cons ql = {rl, rl * ul, rl * vl, pl / (GAMMA - 1.0) + 0.5 * rl * (ul * ul + vl * vl)};
  Cons qr = {rr, rr * ur, rr * vr, pr / (GAMMA - 1.0) + 0.5 * rr * (ur * ur + vr * vr)};
  Cons out{};
  for (int k = 0; k < 4; ++k) out[k] = 0.5 * (fl[k] + fr[k]) - 0.5 * smax * (qr[k] - ql[k]);
  return out;
}

double shock_weight(double pl, double pr) {  // flux.rs:158-162
  double s = std::fabs(pr - pl) / fmin_rs(pl, pr);
  double t = clamp_rs((s - SHOCK_SENSOR_LO) / (SHOCK_SENSOR_HI - SHOCK_SENSOR_LO), 0.0, 1.0);
  return t * t * (3.0 - 2.0 * t);
}

static Cons blend(const Cons& c, const Prim& l, const Prim& r, double t, double nx, double nr) {
  if (t == 0.0) return c;
  Cons f = rusanov(l, r, nx, nr);
  Cons out = c;
  for (int k = 0; k < 4; ++k) out[k] = (1.0 - t) * c[k] + t * f[k];
  return out;
}

Cons face_flux(const Prim& m2, const Prim& m1, const Prim& p0, const Prim& p1, int lim, double nx, double nr) {  // flux.rs:173-186
  Prim l, r;
  reconstruct(m2, m1, p0, p1, lim, l, r);
  Cons c = hllc(l, r, nx, nr);
  double t = shock_weight(m1[3], p0[3]);
  return blend(c, l, r, t, nx, nr);
}

void low_mach_states(const Prim& l, const Prim& r, double nx, double nr, Prim& lo, Prim& ro) {  // flux.rs:206-219
  double unl = l[1] * nx + l[2] * nr;
  double unr = r[1] * nx + r[2] * nr;
  double ml = std::sqrt(l[1] * l[1] + l[2] * l[2]) / std::sqrt(GAMMA * l[3] / l[0]);
  double mr = std::sqrt(r[1] * r[1] + r[2] * r[2]) / std::sqrt(GAMMA * r[3] / r[0]);
  double z = clamp_rs(fmax_rs(ml, mr), LOW_MACH_FLOOR, 1.0);
  if (z >= 1.0) {
    lo = l;
    ro = r;
    return;
  }
  double avg = 0.5 * (unl + unr);
  double dl = avg + z * (unl - avg) - unl;
  double dr = avg + z * (unr - avg) - unr;
  lo = {l[0], l[1] + dl * nx, l[2] + dl * nr, l[3]};
  ro = {r[0], r[1] + dr * nx, r[2] + dr * nr, r[3]};
}

Cons face_flux_lm(const Prim& m2, const Prim& m1, const Prim& p0, const Prim& p1, int lim, double nx, double nr, bool low_mach) {
  // flux.rs:224-241
  if (!low_mach) return face_flux(m2, m1, p0, p1, lim, nx, nr);
  Prim l0, r0, l, r;
  reconstruct(m2, m1, p0, p1, lim, l0, r0);
  low_mach_states(l0, r0, nx, nr, l, r);
  Cons c = hllc(l, r, nx, nr);
  double t = shock_weight(m1[3], p0[3]);
  return blend(c, l, r, t, nx, nr);
}

// ======================================================================== bc.rs
double normal_mach(const Prim& w, double nx, double nr) { return (w[1] * nx + w[2] * nr) / sound_speed(w); }  // bc.rs:48-50
int regime(const Prim& interior, double nx, double nr) {                                                       // bc.rs:54-65
  double m = normal_mach(interior, nx, nr);
  if (m <= -1.0) return SUPERSONIC_INFLOW;
  if (m < 0.0) return SUBSONIC_INFLOW;
  if (m < 1.0) return SUBSONIC_OUTFLOW;
  return SUPERSONIC_OUTFLOW;
}
Prim characteristic_ghost(const Prim& fs, const Prim& interior, double nx, double nr, int* reg_out) {  // bc.rs:69-93
  int reg = regime(interior, nx, nr);
  if (reg_out) *reg_out = reg;
  double g1 = GAMMA - 1.0;
  if (reg == SUPERSONIC_INFLOW) return fs;
  if (reg == SUPERSONIC_OUTFLOW) return interior;
  double ci = sound_speed(interior), ce = sound_speed(fs);
  double uni = interior[1] * nx + interior[2] * nr;
  double une = fs[1] * nx + fs[2] * nr;
  double r_out = uni + 2.0 * ci / g1;
  double r_in = une - 2.0 * ce / g1;
  double un_b = 0.5 * (r_out + r_in);
  double c_b = fmax_rs(0.25 * g1 * (r_out - r_in), 1e-8);
  const Prim& rf = un_b >= 0.0 ? interior : fs;
  double un_ref = un_b >= 0.0 ? uni : une;
  double s = rf[3] / std::pow(rf[0], GAMMA);
  double rho = std::pow(c_b * c_b / (GAMMA * s), 1.0 / g1);
  double p = rho * c_b * c_b / GAMMA;
  double dn = un_b - un_ref;
  return {rho, rf[1] + dn * nx, rf[2] + dn * nr, p};
}
Prim pressure_outflow_ghost(double p_back, const Prim& interior, double nx, double nr) {  // bc.rs:97-103
  if (normal_mach(interior, nx, nr) >= 1.0) return interior;
  return {interior[0], interior[1], interior[2], p_back};
}

// ======================================================================== viscous.rs helpers
double temperature(const Prim& w) { return GAMMA * w[3] / w[0]; }  // viscous.rs:61-63
Prim wall_ghost(const Prim& w, const Face& f, bool noslip) {       // viscous.rs:67-73
  if (noslip) return {w[0], -w[1], -w[2], w[3]};
  return reflect(w, f.nx, f.nr);
}
bool Walls::noslip_jface(size_t i, size_t j) const {  // viscous.rs:97-103
  if (!has_visc) return false;
  if (!has_blk) return j == 0 && jmin_slip && i >= visc.wall_i_start;
  return (j == blk.j_end && i >= visc.wall_i_start && i < blk.i_end) || (j == blk.j_sting && blk.j_sting > 0 && i >= blk.i_end);
}
bool Walls::noslip_iface(size_t i, size_t j) const {  // viscous.rs:107-109
  return has_visc && has_blk && (i == blk.i_end && j >= blk.j_sting && j < blk.j_end) && !(has_nozzle && j < nozzle.j_end);
}
bool Walls::rough_jface(size_t i, size_t j) const {  // viscous.rs:114-121
  if (!has_visc) return false;
  if (!visc.rough()) return false;
  if (!has_blk) return j == 0 && jmin_slip && i >= visc.wall_i_start;
  return j == blk.j_end && i >= visc.wall_i_start && i < blk.i_end;
}
bool Walls::jet_iface(size_t i, size_t j) const { return has_blk && i == blk.i_end && has_nozzle && j < nozzle.j_end; }  // viscous.rs:125-127

// ======================================================================== solver.rs
ImplicitParams implicit_default() { return ImplicitParams{}; }
ImplicitParams implicit_viscous() {
  ImplicitParams p;
  p.dt_mode = DT_MIN_DIRECTION;
  p.cfl_max = 10.0;
  p.sub_iters = 3;
  return p;
}
bool scheme_eq(const Scheme& a, const Scheme& b) {
  if (a.kind != b.kind) return false;
  switch (a.kind) {
    case SCHEME_EXPLICIT:
      return true;
    case SCHEME_SMOOTHED:
      return a.irs.cfl_star == b.irs.cfl_star;
    case SCHEME_MULTIGRID:
      return a.mg.levels == b.mg.levels && a.mg.pre == b.mg.pre && a.mg.post == b.mg.post && a.mg.gamma == b.mg.gamma &&
             a.mg.coarsest == b.mg.coarsest && a.mg.irs.cfl_star == b.mg.irs.cfl_star;
    default: {
      const ImplicitParams &p = a.imp, &q = b.imp;
      return p.cfl0 == q.cfl0 && p.cfl_max == q.cfl_max && p.growth == q.growth && p.dt_mode == q.dt_mode && p.lines == q.lines &&
             p.implicit_bc == q.implicit_bc && p.sub_iters == q.sub_iters && p.roe == q.roe && p.eps_fix == q.eps_fix;
    }
  }
}

Solver::Solver(Grid g, const Config& c) : grid(std::move(g)), cfg(c) {  // solver.rs:263-304
  size_t ni = grid.ni, nj = grid.nj;
  Cons q = prim_to_cons(cfg.freestream);
  u.assign(ni * nj, q);
  w.assign((ni + 2 * NG) * (nj + 2 * NG), cfg.freestream);
  fi.assign((ni + 1) * nj, Cons{});
  fj.assign(ni * (nj + 1), Cons{});
  res.assign(ni * nj, Cons{});
  dt.assign(ni * nj, 0.0);
  u0.assign(ni * nj, Cons{});
  irs_ei.assign(ni * nj, 0.0);
  irs_ej.assign(ni * nj, 0.0);
  n_active = ni * nj;
}

void Solver::set_block(const Block* b) {  // solver.rs:307-328
  if (b) {
    bool ok = b->i_end >= 1 && b->i_end + 2 <= grid.ni && b->j_end >= 2 && b->j_end + 2 <= grid.nj && b->j_end > b->j_sting &&
              (b->j_sting == 0 || b->j_sting >= 2);
    if (!ok) throw std::runtime_error("block out of range");
    has_block = true;
    block = *b;
  } else {
    has_block = false;
  }
  if (!turb.empty()) dwall = wall_distance(grid, walls());
  size_t ni = grid.ni;
  n_active = has_block ? ni * grid.nj - block.i_end * block.j_end - (ni - block.i_end) * block.j_sting : ni * grid.nj;
}

void Solver::set_nozzle(const Nozzle* n) {  // solver.rs:333-344
  if (n) {
    if (!has_block) throw std::runtime_error("a nozzle needs a block");
    if (!(block.j_sting == 0 && n->j_end >= 2 && n->j_end + 2 <= block.j_end && n->j_end % 2 == 0))
      throw std::runtime_error("nozzle out of range");
    if (!(n->state[0] > 0.0 && n->state[3] > 0.0 && n->state[1] >= sound_speed(n->state)))
      throw std::runtime_error("nozzle exit must be supersonic");
    if (scheme.kind == SCHEME_MULTIGRID) throw std::runtime_error("nozzle needs Scheme::Explicit or Scheme::Implicit");
    has_nozzle = true;
    nozzle = *n;
  } else {
    has_nozzle = false;
  }
  if (!turb.empty()) dwall = wall_distance(grid, walls());
}

void Solver::set_viscous(const Viscous* v) {  // solver.rs:359-384
  if (v && !(scheme.kind == SCHEME_EXPLICIT || scheme.kind == SCHEME_IMPLICIT))
    throw std::runtime_error("viscous terms need Scheme::Explicit or Scheme::Implicit");
  size_t ni = grid.ni, nj = grid.nj;
  if (v) {
    has_viscous = true;
    viscous = *v;
    grad.assign(ni * nj, std::array<double, 6>{});
    mu.assign(ni * nj, 0.0);
    mu_t.assign(ni * nj, 0.0);
    if (v->rough())
      rough_wall.assign(ni * nj, std::array<double, 3>{});
    else
      rough_wall.clear();
    fvi.assign((ni + 1) * nj, Cons{});
    fvj.assign(ni * (nj + 1), Cons{});
  } else {
    has_viscous = false;
    grad.clear();
    mu.clear();
    mu_t.clear();
    rough_wall.clear();
    fvi.clear();
    fvj.clear();
  }
  turb.clear();
  dwall.clear();
  turb_rnorm = 0.0;
  if (v && v->turbulence == TURB_SST) turb_init(*this, v->re_c);
}

Walls Solver::walls() const {  // solver.rs:392-394, viscous.rs:91-93
  Walls wl;
  wl.has_visc = has_viscous;
  wl.visc = viscous;
  wl.jmin_slip = cfg.bc[2] == BC_SLIPWALL;
  wl.has_blk = has_block;
  wl.blk = block;
  wl.has_nozzle = has_nozzle;
  wl.nozzle = nozzle;
  return wl;
}

Prim ghost_state(int bc, const Prim& fs, const Prim& edge, const Prim& mirror, const Face& f, double outward) {  // solver.rs:413-421
  switch (bc) {
    case BC_FREESTREAM:
      return fs;
    case BC_EXTRAPOLATE:
      return edge;
    case BC_SLIPWALL:
      return reflect(mirror, f.nx, f.nr);
    case BC_CHARACTERISTIC:
      return characteristic_ghost(fs, edge, outward * f.nx, outward * f.nr, nullptr);
    default:
      return pressure_outflow_ghost(fs[3], edge, outward * f.nx, outward * f.nr);
  }
}

void Solver::fill_ghosts() {  // solver.rs:423-452
  long ni = (long)grid.ni, nj = (long)grid.nj;
  const Prim fs = cfg.freestream;
  Walls wl = walls();
  for (long j = 0; j < nj; ++j)
    for (long k = 1; k <= NG; ++k) {
      const Face& f = grid.iface[(size_t)j * (ni + 1)];
      Prim edge = w[pidx(0, j)], mir = w[pidx(k - 1, j)];
      w[pidx(-k, j)] = ghost_state(cfg.bc[0], fs, edge, mir, f, -1.0);
      const Face& f2 = grid.iface[(size_t)j * (ni + 1) + ni];
      Prim edge2 = w[pidx(ni - 1, j)], mir2 = w[pidx(ni - k, j)];
      w[pidx(ni + k - 1, j)] = ghost_state(cfg.bc[1], fs, edge2, mir2, f2, 1.0);
    }
  for (long i = 0; i < ni; ++i)
    for (long k = 1; k <= NG; ++k) {
      const Face& f = grid.jface[(size_t)i];
      Prim edge = w[pidx(i, 0)], mir = w[pidx(i, k - 1)];
      w[pidx(i, -k)] = wl.noslip_jface((size_t)i, 0) ? wall_ghost(mir, f, true) : ghost_state(cfg.bc[2], fs, edge, mir, f, -1.0);
      const Face& f2 = grid.jface[(size_t)nj * ni + i];
      Prim edge2 = w[pidx(i, nj - 1)], mir2 = w[pidx(i, nj - k)];
      w[pidx(i, nj + k - 1)] = ghost_state(cfg.bc[3], fs, edge2, mir2, f2, 1.0);
    }
}

void Solver::fill_block_ghosts(const Block& b) {  // solver.rs:457-471
  size_t ni = grid.ni;
  Walls wl = walls();
  for (size_t i = 0; i < ni; ++i) {
    size_t j0 = b.col_start(i);
    if (j0 == 0) continue;
    Face f = grid.jface[j0 * ni + i];
    for (size_t k = 1; k <= (size_t)NG; ++k) {
      Prim src = w[pidx((long)i, (long)(j0 + k - 1))];
      w[pidx((long)i, (long)j0 - (long)k)] = wall_ghost(src, f, wl.noslip_jface(i, j0));
    }
  }
}

// viscous passes (defined below)
static void cell_pass(const Viscous& v, const Grid& g, const std::vector<Prim>& w, const Walls& walls,
                      std::vector<std::array<double, 6>>& grad, std::vector<double>& mu);
static void rough_pass(const Grid& g, const std::vector<Prim>& w, const Walls& walls, const std::vector<double>& dwall,
                       const std::vector<double>& mu, double ks, std::vector<std::array<double, 3>>& out);
static void visc_face_pass(const Grid& g, const std::vector<Prim>& w, const Walls& walls, const std::vector<std::array<double, 6>>& grad,
                           const std::vector<double>& mu, const std::vector<double>& mu_t, const std::vector<std::array<double, 3>>& rough,
                           std::vector<Cons>& fvi, std::vector<Cons>& fvj);

void Solver::eval_residual(bool compute_dt) {  // solver.rs:474-648
  const size_t ni = grid.ni, nj = grid.nj;
  const size_t nw = ni + 2 * NG;
  const int lim = iter < cfg.first_order_iters ? FIRST_ORDER : cfg.limiter;
  const double cfl = cfg.cfl;
  const bool lm = low_mach;
  const bool hb = has_block;
  const Block blk = block;
  const Irs irs_ = irs;
  const bool visc = has_viscous;
  const Walls wl = walls();
  (void)nw;
  // 1. primitives
#pragma omp parallel for schedule(static)
  for (long j = 0; j < (long)nj; ++j)
    for (size_t i = 0; i < ni; ++i) w[pidx((long)i, j)] = cons_to_prim(u[(size_t)j * ni + i]);
  fill_ghosts();
  if (hb) fill_block_ghosts(blk);

  // 2a. i-face fluxes
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    long jj = jl;
    for (size_t i = 0; i <= ni; ++i) {
      long ii = (long)i;
      const Face& f = grid.iface[j * (ni + 1) + i];
      Cons& out = fi[j * (ni + 1) + i];
      if (hb && j < blk.j_end) {
        if (j < blk.j_sting || i < blk.i_end) {
          out = Cons{};
          continue;
        }
        if (i <= blk.i_end + 1) {
          const Face& fb = grid.iface[j * (ni + 1) + blk.i_end];
          Prim m1 = w[pidx(ii - 1, jj)], p0 = w[pidx(ii, jj)], p1 = w[pidx(ii + 1, jj)];
          Prim m2;
          if (wl.jet_iface(blk.i_end, j)) {
            Prim jw = wl.nozzle.state;
            if (i == blk.i_end) {
              m2 = jw;
              m1 = jw;
            } else {
              m2 = jw;
            }
          } else if (i == blk.i_end) {
            bool ns = wl.noslip_iface(i, j);
            m2 = wall_ghost(p1, fb, ns);
            m1 = wall_ghost(p0, fb, ns);
          } else {
            m2 = wall_ghost(m1, fb, wl.noslip_iface(blk.i_end, j));
          }
          out = face_flux_lm(m2, m1, p0, p1, lim, f.nx, f.nr, lm);
          continue;
        }
      }
      out = face_flux_lm(w[pidx(ii - 2, jj)], w[pidx(ii - 1, jj)], w[pidx(ii, jj)], w[pidx(ii + 1, jj)], lim, f.nx, f.nr, lm);
    }
  }
  // 2b. j-face fluxes
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl <= (long)nj; ++jl) {
    size_t j = (size_t)jl;
    long jj = jl;
    for (size_t i = 0; i < ni; ++i) {
      long ii = (long)i;
      const Face& f = grid.jface[j * ni + i];
      Cons& out = fj[j * ni + i];
      if (hb && j < blk.col_start(i)) {
        out = Cons{};
        continue;
      }
      out = face_flux_lm(w[pidx(ii, jj - 2)], w[pidx(ii, jj - 1)], w[pidx(ii, jj)], w[pidx(ii, jj + 1)], lim, f.nx, f.nr, lm);
    }
  }
  // 2c. viscous
  if (visc) {
    cell_pass(viscous, grid, w, wl, grad, mu);
    if (viscous.rough()) rough_pass(grid, w, wl, dwall, mu, viscous.roughness, rough_wall);
    visc_face_pass(grid, w, wl, grad, mu, mu_t, rough_wall, fvi, fvj);
  }
  // 3. cell residuals
  const bool has_forcing = !forcing.empty();
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      if (hb && blk.solid(i, j)) {
        res[c] = Cons{};
        dt[c] = 0.0;
        irs_ei[c] = 0.0;
        irs_ej[c] = 0.0;
        continue;
      }
      const Face& fl = grid.iface[j * (ni + 1) + i];
      const Face& fr = grid.iface[j * (ni + 1) + i + 1];
      const Face& fb = grid.jface[j * ni + i];
      const Face& ft = grid.jface[(j + 1) * ni + i];
      const Cons& gl = fi[j * (ni + 1) + i];
      const Cons& gr = fi[j * (ni + 1) + i + 1];
      const Cons& gb = fj[j * ni + i];
      const Cons& gt = fj[(j + 1) * ni + i];
      double wl_ = fl.w(), wr_ = fr.w(), wb_ = fb.w(), wt_ = ft.w();
      const Prim& wc = w[pidx((long)i, (long)j)];
      double inv_v = 1.0 / grid.vol[c];
      Cons out{};
      if (visc) {
        const Cons& hl = fvi[j * (ni + 1) + i];
        const Cons& hr = fvi[j * (ni + 1) + i + 1];
        const Cons& hb_ = fvj[j * ni + i];
        const Cons& ht = fvj[(j + 1) * ni + i];
        for (int k = 0; k < 4; ++k)
          out[k] = -((gr[k] - hr[k]) * wr_ - (gl[k] - hl[k]) * wl_ + (gt[k] - ht[k]) * wt_ - (gb[k] - hb_[k]) * wb_) * inv_v;
        double t_tt = hoop_stress(mu[c] + mu_t[c], grad[c], wc[2], grid.rc[c]);
        out[2] += (wc[3] - t_tt) * grid.area[c] * inv_v;
      } else {
        for (int k = 0; k < 4; ++k) out[k] = -(gr[k] * wr_ - gl[k] * wl_ + gt[k] * wt_ - gb[k] * wb_) * inv_v;
        out[2] += wc[3] * grid.area[c] * inv_v;
      }
      if (has_forcing)
        for (int k = 0; k < 4; ++k) out[k] += forcing[c][k];
      res[c] = out;
      if (compute_dt) {
        double cs = sound_speed(wc);
        auto lam = [&](const Face& f) { return (std::fabs(wc[1] * f.nx + wc[2] * f.nr) + cs) * f.len; };
        double xi = 0.0, xj = 0.0;
        if (visc) {
          xi = diffusion_rate(mu[c], mu_t[c], wc[0], 0.5 * (fl.len + fr.len), grid.area[c]);
          xj = diffusion_rate(mu[c], mu_t[c], wc[0], 0.5 * (fb.len + ft.len), grid.area[c]);
        }
        if (irs_.on()) {
          double li = 0.5 * (lam(fl) + lam(fr)), lj = 0.5 * (lam(fb) + lam(ft));
          if (visc) {
            li += xi;
            lj += xj;
          }
          double d = cfl * grid.area[c] / (li + lj);
          dt[c] = d;
          auto coef = [&](double l) {
            double rr = d * l / grid.area[c] / irs_.cfl_star;
            return fmax_rs(0.25 * (rr * rr - 1.0), 0.0);
          };
          irs_ei[c] = coef(li);
          irs_ej[c] = coef(lj);
        } else {
          double sum = lam(fl) + lam(fr) + lam(fb) + lam(ft);
          dt[c] = visc ? cfl * grid.area[c] / (0.5 * sum + xi + xj) : cfl * grid.area[c] / (0.5 * sum);
        }
      }
    }
  }
}

double Solver::density_residual() const {  // solver.rs:651-654 (serial sum: deterministic)
  double s = 0.0;
  for (const Cons& r : res) s += r[0] * r[0];
  return std::sqrt(s / (double)n_active);
}

double Solver::step() {  // solver.rs:658-676
  double rn;
  switch (scheme.kind) {
    case SCHEME_EXPLICIT:
      irs = Irs{};
      rn = rk3_step();
      break;
    case SCHEME_SMOOTHED:
      irs = scheme.irs;
      rn = rk3_step();
      break;
    case SCHEME_MULTIGRID:
      rn = mg_cycle(*this, scheme.mg);
      break;
    default:
      rn = implicit_step(*this, scheme.imp);
  }
  if (sst()) turb_update(*this);
  iter += 1;
  return rn;
}

double Solver::rk3_step() {  // solver.rs:694-710
  eval_residual(true);
  double rn = density_residual();
  smooth_residual();
  u0 = u;
  stage(1.0, 0.0);
  eval_residual(false);
  smooth_residual();
  stage(0.25, 0.75);
  eval_residual(false);
  smooth_residual();
  stage(2.0 / 3.0, 1.0 / 3.0);
  return rn;
}

void Solver::stage(double a, double b) {  // solver.rs:713-720
#pragma omp parallel for schedule(static)
  for (long c = 0; c < (long)u.size(); ++c)
    for (int k = 0; k < 4; ++k) u[c][k] = a * (u[c][k] + dt[c] * res[c][k]) + b * u0[c][k];
}

// solver.rs:784-803
static void thomas_irs(size_t n, const std::vector<Cons>& rhs_v, size_t rbase, size_t rstride, const std::vector<double>& lo,
                       const std::vector<double>& up, std::vector<Cons>& x, std::vector<double>& cp) {
  Cons prev{};
  for (size_t k = 0; k < n; ++k) {
    double a = lo[k], c = up[k];
    double b = 1.0 + a + c;
    double m = b + a * (k > 0 ? cp[k - 1] : 0.0);
    cp[k] = -c / m;
    const Cons& r = rhs_v[rbase + k * rstride];
    for (int q = 0; q < 4; ++q) x[k][q] = (r[q] + a * prev[q]) / m;
    prev = x[k];
  }
  for (size_t kk = n > 0 ? n - 1 : 0; kk-- > 0;) {
    Cons nx = x[kk + 1];
    for (int q = 0; q < 4; ++q) x[kk][q] -= cp[kk] * nx[q];
  }
}

void Solver::smooth_residual() {  // solver.rs:726-774
  if (!irs.on()) return;
  size_t ni = grid.ni, nj = grid.nj;
  auto solid = [&](size_t i, size_t j) { return has_block && block.solid(i, j); };
  std::vector<Cons> x(ni * nj);
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    auto e = [&](size_t i) { return irs_ei[j * ni + i]; };
    auto face = [&](size_t i) { return (solid(i, j) || solid(i + 1, j)) ? 0.0 : 0.5 * (e(i) + e(i + 1)); };
    std::vector<double> lo(ni), up(ni), cp(ni);
    std::vector<Cons> xr(ni);
    for (size_t k = 0; k < ni; ++k) {
      lo[k] = k > 0 ? face(k - 1) : 0.0;
      up[k] = k + 1 < ni ? face(k) : 0.0;
    }
    thomas_irs(ni, res, j * ni, 1, lo, up, xr, cp);
    for (size_t k = 0; k < ni; ++k) x[j * ni + k] = xr[k];
  }
#pragma omp parallel for schedule(static)
  for (long il = 0; il < (long)ni; ++il) {
    size_t i = (size_t)il;
    auto e = [&](size_t j) { return irs_ej[j * ni + i]; };
    auto face = [&](size_t j) { return (solid(i, j) || solid(i, j + 1)) ? 0.0 : 0.5 * (e(j) + e(j + 1)); };
    std::vector<double> lo(nj), up(nj), cp(nj);
    std::vector<Cons> xr(nj);
    for (size_t k = 0; k < nj; ++k) {
      lo[k] = k > 0 ? face(k - 1) : 0.0;
      up[k] = k + 1 < nj ? face(k) : 0.0;
    }
    thomas_irs(nj, x, i, ni, lo, up, xr, cp);
    for (size_t k = 0; k < nj; ++k) res[k * ni + i] = xr[k];
  }
}

// ======================================================================== implicit.rs
static const M4 ZERO4 = {};
static const M4 EYE4 = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
static const M4 NOSLIP4 = {1, 0, 0, 0, 0, -1, 0, 0, 0, 0, -1, 0, 0, 0, 0, 1};  // implicit.rs:254

M4 flux_jacobian(const Prim& w, double nx, double nr) {  // implicit.rs:95-108
  double rho = w[0], u_ = w[1], v = w[2], p = w[3];
  double g1 = GAMMA - 1.0;
  double q2 = u_ * u_ + v * v;
  double th = u_ * nx + v * nr;
  double phi = 0.5 * g1 * q2;
  double h = GAMMA * p / (g1 * rho) + 0.5 * q2;
  return {0.0,
          nx,
          nr,
          0.0,
          phi * nx - u_ * th,
          th + (2.0 - GAMMA) * u_ * nx,
          u_ * nr - g1 * v * nx,
          g1 * nx,
          phi * nr - v * th,
          v * nx - g1 * u_ * nr,
          th + (2.0 - GAMMA) * v * nr,
          g1 * nr,
          th * (phi - h),
          h * nx - g1 * u_ * th,
          h * nr - g1 * v * th,
          GAMMA * th};
}
M4 mm(const M4& a, const M4& b) {  // implicit.rs:111-122
  M4 c{};
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 4; ++k) {
      double aik = a[4 * i + k];
      for (int j = 0; j < 4; ++j) c[4 * i + j] += aik * b[4 * k + j];
    }
  return c;
}
Cons mv(const M4& a, const Cons& x) {  // implicit.rs:125-131
  Cons y{};
  for (int i = 0; i < 4; ++i) y[i] = a[4 * i] * x[0] + a[4 * i + 1] * x[1] + a[4 * i + 2] * x[2] + a[4 * i + 3] * x[3];
  return y;
}
static inline void axpy(M4& a, double s, const M4& b) {  // implicit.rs:134-138
  for (int k = 0; k < 16; ++k) a[k] += s * b[k];
}
M4 inv4(const M4& m) {  // implicit.rs:141-175
  M4 a = m, inv = EYE4;
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(a[4 * r + c]) > std::fabs(a[4 * piv + c])) piv = r;
    if (piv != c)
      for (int k = 0; k < 4; ++k) {
        std::swap(a[4 * c + k], a[4 * piv + k]);
        std::swap(inv[4 * c + k], inv[4 * piv + k]);
      }
    double d = 1.0 / a[4 * c + c];
    for (int k = 0; k < 4; ++k) {
      a[4 * c + k] *= d;
      inv[4 * c + k] *= d;
    }
    for (int r = 0; r < 4; ++r)
      if (r != c) {
        double f = a[4 * r + c];
        if (f != 0.0)
          for (int k = 0; k < 4; ++k) {
            a[4 * r + k] -= f * a[4 * c + k];
            inv[4 * r + k] -= f * inv[4 * c + k];
          }
      }
  }
  return inv;
}
void block_thomas(size_t n, size_t base, size_t stride, const std::vector<M4>& lo, const std::vector<M4>& d, const std::vector<M4>& up,
                  Cons* rhs, M4* y) {  // implicit.rs:179-204
  for (size_t k = 0; k < n; ++k) {
    size_t c = base + k * stride;
    M4 m = d[c];
    Cons r = rhs[k];
    if (k > 0) {
      M4 t = mm(lo[c], y[k - 1]);
      axpy(m, -1.0, t);
      Cons lg = mv(lo[c], rhs[k - 1]);
      for (int q = 0; q < 4; ++q) r[q] -= lg[q];
    }
    M4 minv = inv4(m);
    rhs[k] = mv(minv, r);
    if (k + 1 < n) y[k] = mm(minv, up[c]);
  }
  for (size_t kk = n > 0 ? n - 1 : 0; kk-- > 0;) {
    Cons t = mv(y[kk], rhs[kk + 1]);
    for (int q = 0; q < 4; ++q) rhs[kk][q] -= t[q];
  }
}
M4 abs_jacobian(const Prim& wl, const Prim& wr, double nx, double nr, double eps_fix) {  // implicit.rs:209-241
  double sl = std::sqrt(wl[0]), sr = std::sqrt(wr[0]);
  double inv = 1.0 / (sl + sr);
  double u_ = (sl * wl[1] + sr * wr[1]) * inv, v = (sl * wl[2] + sr * wr[2]) * inv;
  double hl = GAMMA * wl[3] / ((GAMMA - 1.0) * wl[0]) + 0.5 * (wl[1] * wl[1] + wl[2] * wl[2]);
  double hr = GAMMA * wr[3] / ((GAMMA - 1.0) * wr[0]) + 0.5 * (wr[1] * wr[1] + wr[2] * wr[2]);
  double h = (sl * hl + sr * hr) * inv;
  double c = std::sqrt(fmax_rs((GAMMA - 1.0) * (h - 0.5 * (u_ * u_ + v * v)), 1e-300));
  double a = u_ * nx + v * nr;
  double eps = eps_fix * c;
  auto fix = [&](double l) { return std::fabs(l) >= eps ? std::fabs(l) : 0.5 * (l * l / eps + eps); };
  double e1 = fix(a), e2 = fix(a + c), e3 = fix(a - c);
  double d1 = (e2 - e1) / c;
  double d2 = (e2 + e3 - 2.0 * e1) / (2.0 * c * c);
  Prim wa = {1.0, u_, v, (GAMMA - 1.0) / GAMMA * (h - 0.5 * (u_ * u_ + v * v))};
  M4 am = flux_jacobian(wa, nx, nr);
  M4 b1 = am, b2 = am;
  for (int q = 0; q < 4; ++q) {
    b1[5 * q] -= a;
    b2[5 * q] -= a + c;
  }
  M4 prod = mm(b1, b2);
  M4 out{};
  for (int k = 0; k < 16; ++k) out[k] = d1 * b1[k] + d2 * prod[k];
  for (int q = 0; q < 4; ++q) out[5 * q] += e1;
  return out;
}
static inline double spectral(const Prim& w, double nx, double nr) { return std::fabs(w[1] * nx + w[2] * nr) + sound_speed(w); }  // implicit.rs:244-246
static M4 reflection(double nx, double nr) {  // implicit.rs:249-251
  return {1.0, 0.0, 0.0, 0.0, 0.0, 1.0 - 2.0 * nx * nx, -2.0 * nx * nr, 0.0, 0.0, -2.0 * nx * nr, 1.0 - 2.0 * nr * nr, 0.0, 0.0, 0.0, 0.0, 1.0};
}
M4 ghost_jacobian(int bc, const Prim& fs, const Prim& edge, const Face& f, double outward) {  // implicit.rs:257-279
  switch (bc) {
    case BC_FREESTREAM:
      return ZERO4;
    case BC_EXTRAPOLATE:
      return EYE4;
    case BC_SLIPWALL:
      return reflection(f.nx, f.nr);
    default: {
      Cons u0 = prim_to_cons(edge);
      Cons g0 = prim_to_cons(ghost_state(bc, fs, edge, edge, f, outward));
      M4 t = ZERO4;
      for (int q = 0; q < 4; ++q) {
        double h = 1e-7 * (1.0 + std::fabs(u0[q]));
        Cons up = u0;
        up[q] += h;
        Prim e = cons_to_prim(up);
        Cons g = prim_to_cons(ghost_state(bc, fs, e, e, f, outward));
        for (int r = 0; r < 4; ++r) t[4 * r + q] = (g[r] - g0[r]) / h;
      }
      return t;
    }
  }
}
void cell_blocks(const Prim& wk, const Prim& wm, const Prim& wp, const Face& fl, const Face& fr, double vol, double dt, bool lines, double src,
                 bool roe, double eps_fix, double visc_l, double visc_r, M4& lo, M4& d, M4& up) {  // implicit.rs:284-367
  double s = 0.5 * dt / vol;
  double wl = fl.w(), wr = fr.w();
  M4 dis_l, dis_r;
  if (roe) {
    M4 dl = abs_jacobian(wm, wk, fl.nx, fl.nr, eps_fix), dr = abs_jacobian(wk, wp, fr.nx, fr.nr, eps_fix);
    double tl = shock_weight(wm[3], wk[3]), tr = shock_weight(wk[3], wp[3]);
    if (tl > 0.0 || tr > 0.0) {
      double lam_l = fmax_rs(spectral(wk, fl.nx, fl.nr), spectral(wm, fl.nx, fl.nr));
      double lam_r = fmax_rs(spectral(wk, fr.nx, fr.nr), spectral(wp, fr.nx, fr.nr));
      for (auto& x : dl) x *= 1.0 - tl;
      for (auto& x : dr) x *= 1.0 - tr;
      for (int q = 0; q < 4; ++q) {
        dl[5 * q] += tl * lam_l;
        dr[5 * q] += tr * lam_r;
      }
    }
    dis_l = dl;
    dis_r = dr;
  } else {
    double lam_l = fmax_rs(spectral(wk, fl.nx, fl.nr), spectral(wm, fl.nx, fl.nr));
    double lam_r = fmax_rs(spectral(wk, fr.nx, fr.nr), spectral(wp, fr.nx, fr.nr));
    dis_l = ZERO4;
    dis_r = ZERO4;
    for (int q = 0; q < 4; ++q) {
      dis_l[5 * q] = lam_l;
      dis_r[5 * q] = lam_r;
    }
  }
  for (int q = 0; q < 4; ++q) {
    dis_l[5 * q] += 2.0 * visc_l;
    dis_r[5 * q] += 2.0 * visc_r;
  }
  d = EYE4;
  M4 ak_r = flux_jacobian(wk, fr.nx, fr.nr);
  M4 ak_l = flux_jacobian(wk, fl.nx, fl.nr);
  axpy(d, s * wr, ak_r);
  axpy(d, -s * wl, ak_l);
  axpy(d, s * wr, dis_r);
  axpy(d, s * wl, dis_l);
  if (src != 0.0) {
    double g1 = GAMMA - 1.0;
    double c = -dt * src * g1;
    d[8] += c * 0.5 * (wk[1] * wk[1] + wk[2] * wk[2]);
    d[9] += -c * wk[1];
    d[10] += -c * wk[2];
    d[11] += c;
  }
  if (!lines) {
    lo = ZERO4;
    up = ZERO4;
    return;
  }
  lo = flux_jacobian(wm, fl.nx, fl.nr);
  axpy(lo, 1.0, dis_l);
  for (auto& x : lo) x *= -s * wl;
  up = flux_jacobian(wp, fr.nx, fr.nr);
  axpy(up, -1.0, dis_r);
  for (auto& x : up) x *= s * wr;
}

static void face_lambdas(const Grid& g, const std::vector<Prim>& w, const Walls& walls, const std::vector<double>& mu,
                         const std::vector<double>& mu_t, const std::vector<std::array<double, 3>>& rough, bool dir_i, size_t i, size_t j,
                         double& lam_l, double& lam_r);

static inline void fit_factor(Factor& f, size_t n) {
  if (f.lo.size() != n) {
    f.lo.assign(n, ZERO4);
    f.d.assign(n, ZERO4);
    f.up.assign(n, ZERO4);
  }
}

void assemble_into(const Solver& s, const ImplicitParams& p, bool dir_i, Factor& fac) {  // implicit.rs:379-467
  const size_t ni = s.grid.ni, nj = s.grid.nj;
  const bool hb = s.has_block;
  const Block blk = s.block;
  const Prim fs = s.cfg.freestream;
  const Walls walls = s.walls();
  const bool viscous_on = s.has_viscous;
  auto ghost_t = [&](int bc, const Prim& edge, const Face& f, double outward, bool noslip) -> M4 {
    if (p.implicit_bc) {
      if (noslip && bc == BC_SLIPWALL) return NOSLIP4;
      return ghost_jacobian(bc, fs, edge, f, outward);
    }
    return ZERO4;
  };
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      if (hb && blk.solid(i, j)) {
        fac.lo[c] = ZERO4;
        fac.d[c] = EYE4;
        fac.up[c] = ZERO4;
        continue;
      }
      long ii = (long)i, jj = (long)j;
      const Prim& wk = s.w[s.pidx(ii, jj)];
      double src;
      size_t k, kn, k0;
      if (dir_i) {
        src = 0.0;
        k = i;
        kn = ni;
        k0 = hb ? (blk.row_start(j) == SIZE_MAX ? ni : blk.row_start(j)) : 0;
      } else {
        src = s.grid.area[c] / s.grid.vol[c];
        k = j;
        kn = nj;
        k0 = hb ? blk.col_start(i) : 0;
      }
      const Face& fl = dir_i ? s.grid.iface[j * (ni + 1) + i] : s.grid.jface[j * ni + i];
      const Face& fr = dir_i ? s.grid.iface[j * (ni + 1) + i + 1] : s.grid.jface[(j + 1) * ni + i];
      size_t wm_idx = dir_i ? s.pidx(ii - 1, jj) : s.pidx(ii, jj - 1);
      size_t wp_idx = dir_i ? s.pidx(ii + 1, jj) : s.pidx(ii, jj + 1);
      bool wall_lower = k == k0 && k0 > 0;
      bool jet = wall_lower && dir_i && walls.jet_iface(k0, j);
      Prim wm;
      if (jet)
        wm = walls.nozzle.state;
      else if (wall_lower && dir_i) {
        const Face& fb = s.grid.iface[j * (ni + 1) + k0];
        wm = wall_ghost(wk, fb, walls.noslip_iface(k0, j));
      } else
        wm = s.w[wm_idx];
      double lam_l = 0.0, lam_r = 0.0;
      if (viscous_on) face_lambdas(s.grid, s.w, walls, s.mu, s.mu_t, s.rough_wall, dir_i, i, j, lam_l, lam_r);
      M4 l, dd, uu;
      cell_blocks(wk, wm, s.w[wp_idx], fl, fr, s.grid.vol[c], s.dt[c], p.lines, src, p.roe, p.eps_fix, lam_l, lam_r, l, dd, uu);
      if (k == k0) {
        M4 t;
        if (jet)
          t = ZERO4;
        else if (wall_lower) {
          bool ns = dir_i ? walls.noslip_iface(k0, j) : walls.noslip_jface(i, k0);
          t = ns ? NOSLIP4 : reflection(fl.nx, fl.nr);
        } else
          t = ghost_t(dir_i ? s.cfg.bc[0] : s.cfg.bc[2], wk, fl, -1.0, !dir_i && walls.noslip_jface(i, 0));
        M4 lt = mm(l, t);
        axpy(dd, 1.0, lt);
        l = ZERO4;
      }
      if (k == kn - 1) {
        M4 t = ghost_t(dir_i ? s.cfg.bc[1] : s.cfg.bc[3], wk, fr, 1.0, false);
        M4 ut = mm(uu, t);
        axpy(dd, 1.0, ut);
        uu = ZERO4;
      }
      fac.lo[c] = l;
      fac.d[c] = dd;
      fac.up[c] = uu;
    }
  }
}

static inline size_t seg_start(bool hb, const Block& b, bool dir_i, size_t ni, size_t i, size_t j) {  // implicit.rs:471-477
  if (!hb) return 0;
  if (dir_i) {
    size_t rs = b.row_start(j);
    return rs == SIZE_MAX ? ni : rs;
  }
  return b.col_start(i);
}

void solve_lines(const Solver& s, const Factor& fac, bool dir_i, std::vector<Cons>& x) {  // implicit.rs:528-563
  const size_t ni = s.grid.ni, nj = s.grid.nj;
  if (dir_i) {
#pragma omp parallel for schedule(static)
    for (long jl = 0; jl < (long)nj; ++jl) {
      size_t j = (size_t)jl;
      size_t k0 = seg_start(s.has_block, s.block, true, ni, 0, j);
      size_t n = ni - k0;
      if (n == 0) continue;
      std::vector<M4> y(n);
      block_thomas(n, j * ni + k0, 1, fac.lo, fac.d, fac.up, &x[j * ni + k0], y.data());
    }
  } else {
#pragma omp parallel for schedule(static)
    for (long il = 0; il < (long)ni; ++il) {
      size_t i = (size_t)il;
      size_t k0 = seg_start(s.has_block, s.block, false, ni, i, 0);
      size_t n = nj - k0;
      std::vector<Cons> rhs(n);
      std::vector<M4> y(n);
      for (size_t k = 0; k < n; ++k) rhs[k] = x[(k0 + k) * ni + i];
      if (n > 0) block_thomas(n, k0 * ni + i, ni, fac.lo, fac.d, fac.up, rhs.data(), y.data());
      for (size_t k = 0; k < n; ++k) x[(k0 + k) * ni + i] = rhs[k];
    }
  }
}

void apply_factor_into(const Solver& s, const Factor& fac, bool dir_i, const std::vector<Cons>& x, std::vector<Cons>& out) {  // implicit.rs:566-594
  const size_t ni = s.grid.ni, nj = s.grid.nj;
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      if (s.has_block && s.block.solid(i, j)) {
        out[c] = Cons{};
        continue;
      }
      size_t k0 = seg_start(s.has_block, s.block, dir_i, ni, i, j);
      size_t k = dir_i ? i : j, kn = dir_i ? ni : nj, stride = dir_i ? 1 : ni;
      Cons v = mv(fac.d[c], x[c]);
      if (k > k0) {
        Cons a = mv(fac.lo[c], x[c - stride]);
        for (int q = 0; q < 4; ++q) v[q] += a[q];
      }
      if (k + 1 < kn) {
        Cons a = mv(fac.up[c], x[c + stride]);
        for (int q = 0; q < 4; ++q) v[q] += a[q];
      }
      out[c] = v;
    }
  }
}

double implicit_step(Solver& s, const ImplicitParams& p) {  // implicit.rs:601-663
  double cfl = fmin_rs(p.cfl0 * std::pow(p.growth, (int)std::min<size_t>(s.ramp_k, 10000)), p.cfl_max);
  s.ramp_k += 1;
  s.eval_residual(false);
  double rn = s.density_residual();
  compute_dt(s, cfl, p.dt_mode);
  const size_t ni = s.grid.ni, nj = s.grid.nj, n = ni * nj;
  fit_factor(s.ws_fi, n);
  fit_factor(s.ws_fj, n);
  s.ws_b.resize(n);
  s.ws_du.resize(n);
  if (p.sub_iters > 1) {
    s.ws_ai.resize(n);
    s.ws_aj.resize(n);
    s.ws_r.resize(n);
    s.ws_corr.resize(n);
  }
  assemble_into(s, p, true, s.ws_fi);
  assemble_into(s, p, false, s.ws_fj);
  for (size_t c = 0; c < n; ++c) {
    const Cons& r = s.res[c];
    double d = s.dt[c];
    s.ws_b[c] = {r[0] * d, r[1] * d, r[2] * d, r[3] * d};
  }
  s.ws_du = s.ws_b;
  solve_lines(s, s.ws_fi, true, s.ws_du);
  solve_lines(s, s.ws_fj, false, s.ws_du);
  for (size_t it = 1; it < std::max<size_t>(p.sub_iters, 1); ++it) {
    apply_factor_into(s, s.ws_fi, true, s.ws_du, s.ws_ai);
    apply_factor_into(s, s.ws_fj, false, s.ws_du, s.ws_aj);
    for (size_t c = 0; c < n; ++c)
      for (int q = 0; q < 4; ++q) s.ws_r[c][q] = s.ws_b[c][q] - (s.ws_ai[c][q] + s.ws_aj[c][q] - s.ws_du[c][q]);
    s.ws_corr = s.ws_r;
    solve_lines(s, s.ws_fi, true, s.ws_corr);
    solve_lines(s, s.ws_fj, false, s.ws_corr);
    for (size_t c = 0; c < n; ++c)
      for (int q = 0; q < 4; ++q) s.ws_du[c][q] += s.ws_corr[c][q];
  }
  // update with positivity damping
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      if (s.has_block && s.block.solid(i, j)) continue;
      size_t c = j * ni + i;
      const Cons& dq = s.ws_du[c];
      double alpha = 1.0;
      for (int t = 0; t < 8; ++t) {
        Cons q = {s.u[c][0] + alpha * dq[0], s.u[c][1] + alpha * dq[1], s.u[c][2] + alpha * dq[2], s.u[c][3] + alpha * dq[3]};
        Prim wq = cons_to_prim(q);
        if (wq[0] > 0.0 && wq[3] > 0.0 && std::isfinite(q[0]) && std::isfinite(q[1]) && std::isfinite(q[2]) && std::isfinite(q[3])) {
          s.u[c] = q;
          break;
        }
        alpha *= 0.5;
      }
    }
  }
  return rn;
}

void compute_dt(Solver& s, double cfl, int mode) {  // implicit.rs:666-695
  const size_t ni = s.grid.ni, nj = s.grid.nj;
  const bool viscous_on = s.has_viscous;
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      if (s.has_block && s.block.solid(i, j)) {
        s.dt[c] = 0.0;
        continue;
      }
      const Prim& wc = s.w[s.pidx((long)i, (long)j)];
      auto lam = [&](const Face& f) { return spectral(wc, f.nx, f.nr) * f.len; };
      double li = 0.5 * (lam(s.grid.iface[j * (ni + 1) + i]) + lam(s.grid.iface[j * (ni + 1) + i + 1]));
      double lj = 0.5 * (lam(s.grid.jface[j * ni + i]) + lam(s.grid.jface[(j + 1) * ni + i]));
      double a = s.grid.area[c];
      if (viscous_on) {
        const Face &fl = s.grid.iface[j * (ni + 1) + i], &fr = s.grid.iface[j * (ni + 1) + i + 1];
        const Face &fb = s.grid.jface[j * ni + i], &ft = s.grid.jface[(j + 1) * ni + i];
        li += diffusion_rate(s.mu[c], s.mu_t[c], wc[0], 0.5 * (fl.len + fr.len), a);
        lj += diffusion_rate(s.mu[c], s.mu_t[c], wc[0], 0.5 * (fb.len + ft.len), a);
      }
      s.dt[c] = mode == DT_SUM ? cfl * a / (li + lj) : cfl * a / (2.0 * fmin_rs(li, lj));
    }
  }
}

// ======================================================================== multigrid.rs
size_t Solver::set_scheme(const Scheme& sch) {  // multigrid.rs:29-64
  if (has_viscous && !(sch.kind == SCHEME_EXPLICIT || sch.kind == SCHEME_IMPLICIT))
    throw std::runtime_error("viscous terms need Scheme::Explicit or Scheme::Implicit");
  if (has_nozzle && sch.kind == SCHEME_MULTIGRID) throw std::runtime_error("nozzle needs Scheme::Explicit or Scheme::Implicit");
  scheme = sch;
  coarse.clear();
  if (sch.kind != SCHEME_MULTIGRID) return 1;
  const MgParams& p = sch.mg;
  std::vector<Solver> levels;
  while (levels.size() + 1 < p.levels) {
    const Solver& fine = levels.empty() ? *this : levels.back();
    Grid g;
    if (!grid_coarsen(fine.grid, g)) break;
    if (g.ni < 8 || g.nj < 8) break;
    bool has_b = false;
    Block b{};
    if (fine.has_block) {
      if (!fine.block.coarsen(b)) break;
      has_b = true;
    }
    Config c;
    c.cfl = cfg.cfl;
    c.limiter = FIRST_ORDER;
    c.freestream = cfg.freestream;
    for (int k = 0; k < 4; ++k) c.bc[k] = cfg.bc[k];
    c.first_order_iters = 0;
    size_t n = g.ni * g.nj;
    Solver s(std::move(g), c);
    s.low_mach = low_mach;
    s.set_block(has_b ? &b : nullptr);
    s.forcing.assign(n, Cons{});
    s.mg_u0.assign(n, Cons{});
    s.irs = p.irs;
    levels.push_back(std::move(s));
  }
  size_t n = levels.size() + 1;
  coarse = std::move(levels);
  return n;
}

static void mg_restrict(const Solver& fine, Solver& coarse) {  // multigrid.rs:115-173
  const size_t fni = fine.grid.ni, cni = coarse.grid.ni, cnj = coarse.grid.nj;
  auto solid = [&](size_t c) { return fine.has_block && fine.block.solid(c % fni, c / fni); };
  auto child = [&](size_t ci, size_t cj, size_t* out) {
    size_t c0 = 2 * cj * fni + 2 * ci;
    out[0] = c0;
    out[1] = c0 + 1;
    out[2] = c0 + fni;
    out[3] = c0 + fni + 1;
  };
#pragma omp parallel for schedule(static)
  for (long cjl = 0; cjl < (long)cnj; ++cjl) {
    size_t cj = (size_t)cjl;
    for (size_t ci = 0; ci < cni; ++ci) {
      Cons s{};
      double v = 0.0;
      size_t ch[4];
      child(ci, cj, ch);
      for (size_t c : ch) {
        if (solid(c)) continue;
        for (int k = 0; k < 4; ++k) s[k] += fine.grid.vol[c] * fine.u[c][k];
        v += fine.grid.vol[c];
      }
      if (v > 0.0)
        for (int k = 0; k < 4; ++k) coarse.u[cj * cni + ci][k] = s[k] / v;
    }
  }
  coarse.mg_u0 = coarse.u;
  for (auto& f : coarse.forcing) f = Cons{};
  coarse.eval_residual(false);
#pragma omp parallel for schedule(static)
  for (long cjl = 0; cjl < (long)cnj; ++cjl) {
    size_t cj = (size_t)cjl;
    for (size_t ci = 0; ci < cni; ++ci) {
      Cons s{};
      double v = 0.0;
      size_t ch[4];
      child(ci, cj, ch);
      for (size_t c : ch) {
        if (solid(c)) continue;
        for (int k = 0; k < 4; ++k) s[k] += fine.grid.vol[c] * fine.res[c][k];
        v += fine.grid.vol[c];
      }
      if (v > 0.0)
        for (int k = 0; k < 4; ++k) coarse.forcing[cj * cni + ci][k] = s[k] / v - coarse.res[cj * cni + ci][k];
    }
  }
}

static void mg_prolong_correct(const Solver& coarse, Solver& fine) {  // multigrid.rs:177-218
  const size_t fni = fine.grid.ni, fnj = fine.grid.nj, cni = coarse.grid.ni, cnj = coarse.grid.nj;
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)fnj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < fni; ++i) {
      if (fine.has_block && fine.block.solid(i, j)) continue;
      size_t ci = i / 2, cj = j / 2;
      size_t ci2 = i % 2 == 0 ? (ci > 0 ? ci - 1 : 0) : std::min(ci + 1, cni - 1);
      size_t cj2 = j % 2 == 0 ? (cj > 0 ? cj - 1 : 0) : std::min(cj + 1, cnj - 1);
      const size_t ca[4] = {ci, ci2, ci, ci2};
      const size_t cb[4] = {cj, cj, cj2, cj2};
      const double wt[4] = {9.0, 3.0, 3.0, 1.0};
      Cons d{};
      double wsum = 0.0;
      for (int t = 0; t < 4; ++t) {
        if (coarse.has_block && coarse.block.solid(ca[t], cb[t])) continue;
        size_t c = cb[t] * cni + ca[t];
        for (int k = 0; k < 4; ++k) d[k] += wt[t] * (coarse.u[c][k] - coarse.mg_u0[c][k]);
        wsum += wt[t];
      }
      for (int k = 0; k < 4; ++k) d[k] /= wsum;
      size_t c = j * fni + i;
      double alpha = 1.0;
      for (int t = 0; t < 6; ++t) {
        Cons q = {fine.u[c][0] + alpha * d[0], fine.u[c][1] + alpha * d[1], fine.u[c][2] + alpha * d[2], fine.u[c][3] + alpha * d[3]};
        Prim w = cons_to_prim(q);
        if (w[0] > 0.0 && w[3] > 0.0) {
          fine.u[c] = q;
          break;
        }
        alpha *= 0.5;
      }
    }
  }
}

static double mg_level(Solver& fine, Solver* coarse, size_t ncoarse, const MgParams& p) {  // multigrid.rs:87-112
  size_t n_pre = ncoarse == 0 ? p.coarsest : p.pre;
  double rn = NAN;
  for (size_t k = 0; k < n_pre; ++k) {
    double r = fine.rk3_step();
    if (k == 0) rn = r;
  }
  if (ncoarse == 0) return rn;
  Solver& next = coarse[0];
  fine.eval_residual(false);
  if (std::isnan(rn)) rn = fine.density_residual();
  mg_restrict(fine, next);
  for (size_t g = 0; g < std::max<size_t>(p.gamma, 1); ++g) mg_level(next, coarse + 1, ncoarse - 1, p);
  mg_prolong_correct(next, fine);
  for (size_t k = 0; k < p.post; ++k) fine.rk3_step();
  return rn;
}

double mg_cycle(Solver& fine, const MgParams& p) {  // multigrid.rs:73-85
  std::vector<Solver> coarse = std::move(fine.coarse);
  for (auto& c : coarse) {
    c.cfg.freestream = fine.cfg.freestream;
    c.cfg.cfl = fine.cfg.cfl;
    c.low_mach = fine.low_mach;
    c.irs = p.irs;
  }
  fine.irs = p.irs;
  double rn = mg_level(fine, coarse.data(), coarse.size(), p);
  fine.coarse = std::move(coarse);
  return rn;
}

// ======================================================================== viscous.rs
bool iface_sides(const Grid& g, const std::vector<Prim>& w, const Walls& walls, size_t i, size_t j, FaceSides& out) {  // viscous.rs:150-188
  const size_t ni = g.ni;
  auto P = [&](long ii, long jj) { return w[(size_t)(jj + NG) * (ni + 2 * NG) + (size_t)(ii + NG)]; };
  long ii = (long)i, jj = (long)j;
  if (walls.has_blk) {
    const Block& b = walls.blk;
    if (j < b.j_end) {
      if (j < b.j_sting || i < b.i_end) return false;
      if (i == b.i_end) {
        size_t c = j * ni + i;
        Prim wr = P(ii, jj);
        if (walls.has_nozzle && j < walls.nozzle.j_end) {
          Side l;
          l.w = walls.nozzle.state;
          l.cell = c;
          l.ghost = true;
          if (walls.has_visc) {
            const Nozzle& n = walls.nozzle;
            double mut = walls.visc.turbulence == TURB_SST ? n.state[0] * n.turb[0] / n.turb[1] : 0.0;
            l.has_fixed = true;
            l.fixed_mu = walls.visc.mu(temperature(n.state));
            l.fixed_mut = mut;
          }
          Side r;
          r.w = wr;
          r.cell = c;
          out = FaceSides{l, r, false};
          return true;
        }
        bool noslip = walls.noslip_iface(i, j);
        Prim wl = wall_ghost(wr, g.iface[j * (ni + 1) + i], noslip);
        Side l, r;
        l.w = wl;
        l.cell = c;
        l.ghost = true;
        r.w = wr;
        r.cell = c;
        out = FaceSides{l, r, noslip};
        return true;
      }
    }
  }
  Side l, r;
  if (i == 0) {
    size_t c = j * ni;
    l.w = P(-1, jj), l.cell = c, l.ghost = true;
    r.w = P(0, jj), r.cell = c;
  } else if (i == ni) {
    size_t c = j * ni + ni - 1;
    l.w = P(ii - 1, jj), l.cell = c;
    r.w = P(ii, jj), r.cell = c, r.ghost = true;
  } else {
    l.w = P(ii - 1, jj), l.cell = j * ni + i - 1;
    r.w = P(ii, jj), r.cell = j * ni + i;
  }
  out = FaceSides{l, r, false};
  return true;
}

bool jface_sides(const Grid& g, const std::vector<Prim>& w, const Walls& walls, size_t i, size_t j, FaceSides& out) {  // viscous.rs:191-215
  const size_t ni = g.ni, nj = g.nj;
  auto P = [&](long ii, long jj) { return w[(size_t)(jj + NG) * (ni + 2 * NG) + (size_t)(ii + NG)]; };
  long ii = (long)i, jj = (long)j;
  Side l, r;
  if (walls.has_blk) {
    size_t j0 = walls.blk.col_start(i);
    if (j < j0) return false;
    if (j == j0 && j0 > 0) {
      size_t c = j * ni + i;
      l.w = P(ii, jj - 1), l.cell = c, l.ghost = true;
      r.w = P(ii, jj), r.cell = c;
      out = FaceSides{l, r, walls.noslip_jface(i, j)};
      return true;
    }
  }
  if (j == 0) {
    size_t c = i;
    l.w = P(ii, -1), l.cell = c, l.ghost = true;
    r.w = P(ii, 0), r.cell = c;
    out = FaceSides{l, r, walls.noslip_jface(i, 0)};
  } else if (j == nj) {
    size_t c = (nj - 1) * ni + i;
    l.w = P(ii, jj - 1), l.cell = c;
    r.w = P(ii, jj), r.cell = c, r.ghost = true;
    out = FaceSides{l, r, false};
  } else {
    l.w = P(ii, jj - 1), l.cell = (j - 1) * ni + i;
    r.w = P(ii, jj), r.cell = j * ni + i;
    out = FaceSides{l, r, false};
  }
  return true;
}

std::pair<double, double> iface_centre(const Grid& g, size_t i, size_t j) {  // viscous.rs:219-222
  auto a = g.node(i, j), b = g.node(i, j + 1);
  return {0.5 * (a.first + b.first), 0.5 * (a.second + b.second)};
}
std::pair<double, double> jface_centre(const Grid& g, size_t i, size_t j) {  // viscous.rs:226-229
  auto a = g.node(i, j), b = g.node(i + 1, j);
  return {0.5 * (a.first + b.first), 0.5 * (a.second + b.second)};
}
static inline void side_pos(const Grid& g, const Side& s, double xf, double rf, double& x, double& r) {  // viscous.rs:233-240
  x = g.xc[s.cell];
  r = g.rc[s.cell];
  if (s.ghost) {
    x = 2.0 * xf - x;
    r = 2.0 * rf - r;
  }
}
void stencil(const Grid& g, const FaceSides& s, double xf, double rf, double& dd, double& ex, double& er) {  // viscous.rs:244-250
  double xl, rl, xr, rr;
  side_pos(g, s.l, xf, rf, xl, rl);
  side_pos(g, s.r, xf, rf, xr, rr);
  double dx = xr - xl, dr = rr - rl;
  dd = std::hypot(dx, dr);
  ex = dx / dd;
  er = dr / dd;
}
void face_mu(const std::vector<double>& mu, const std::vector<double>& mu_t, const std::vector<std::array<double, 3>>& rough,
             const FaceSides& s, double& mu_f, double& mut_f) {  // viscous.rs:256-270
  auto mu_side = [&](const Side& sd) { return sd.has_fixed ? sd.fixed_mu : mu[sd.cell]; };
  auto mut_side = [&](const Side& sd) {
    if (sd.has_fixed) return sd.fixed_mut;
    if (sd.ghost && s.noslip) return rough.empty() ? -mu_t[sd.cell] : 2.0 * rough[sd.cell][2] - mu_t[sd.cell];
    return mu_t[sd.cell];
  };
  mu_f = 0.5 * (mu_side(s.l) + mu_side(s.r));
  mut_f = 0.5 * (mut_side(s.l) + mut_side(s.r));
}
static inline std::array<double, 3> phi3(const Prim& w) { return {w[1], w[2], temperature(w)}; }  // viscous.rs:274-276

static void cell_pass(const Viscous& v, const Grid& g, const std::vector<Prim>& w, const Walls& walls,
                      std::vector<std::array<double, 6>>& grad, std::vector<double>& mu) {  // viscous.rs:280-316
  const size_t ni = g.ni, nj = g.nj;
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      if (walls.has_blk && walls.blk.solid(i, j)) {
        grad[c] = {};
        mu[c] = 0.0;
        continue;
      }
      const Prim& wc = w[(j + NG) * (ni + 2 * NG) + i + NG];
      mu[c] = v.mu(temperature(wc));
      auto pc = phi3(wc);
      const Face& fl = g.iface[j * (ni + 1) + i];
      const Face& fr = g.iface[j * (ni + 1) + i + 1];
      const Face& fb = g.jface[j * ni + i];
      const Face& ft = g.jface[(j + 1) * ni + i];
      FaceSides s;
      iface_sides(g, w, walls, i, j, s);
      Prim nb_l = s.l.w;
      iface_sides(g, w, walls, i + 1, j, s);
      Prim nb_r = s.r.w;
      jface_sides(g, w, walls, i, j, s);
      Prim nb_b = s.l.w;
      jface_sides(g, w, walls, i, j + 1, s);
      Prim nb_t = s.r.w;
      std::array<double, 6> gg{};
      const Face* fs[4] = {&fr, &fl, &ft, &fb};
      const double sg[4] = {1.0, -1.0, 1.0, -1.0};
      const Prim* nbs[4] = {&nb_r, &nb_l, &nb_t, &nb_b};
      for (int t = 0; t < 4; ++t) {
        auto pn = phi3(*nbs[t]);
        for (int m = 0; m < 3; ++m) {
          double pf = 0.5 * (pc[m] + pn[m]);
          gg[2 * m] += sg[t] * pf * fs[t]->nx * fs[t]->len;
          gg[2 * m + 1] += sg[t] * pf * fs[t]->nr * fs[t]->len;
        }
      }
      double inv_a = 1.0 / g.area[c];
      for (auto& x : gg) x *= inv_a;
      grad[c] = gg;
    }
  }
}

static Cons viscous_flux(const Grid& g, const std::vector<std::array<double, 6>>& grad, const std::vector<double>& mu,
                         const std::vector<double>& mu_t, const std::vector<std::array<double, 3>>& rough, const FaceSides& sides,
                         const Face& f, double xf, double rf) {  // viscous.rs:319-343
  if (f.rm == 0.0) return Cons{};
  double dd, ex, er;
  stencil(g, sides, xf, rf, dd, ex, er);
  const auto& gl = grad[sides.l.cell];
  const auto& gr = grad[sides.r.cell];
  auto pl = phi3(sides.l.w), pr = phi3(sides.r.w);
  double gf[6];
  for (int m = 0; m < 3; ++m) {
    double gbx = 0.5 * (gl[2 * m] + gr[2 * m]), gbr = 0.5 * (gl[2 * m + 1] + gr[2 * m + 1]);
    double corr = (pr[m] - pl[m]) / dd - (gbx * ex + gbr * er);
    gf[2 * m] = gbx + corr * ex;
    gf[2 * m + 1] = gbr + corr * er;
  }
  double mu_f, mut_f;
  face_mu(mu, mu_t, rough, sides, mu_f, mut_f);
  double uf = 0.5 * (sides.l.w[1] + sides.r.w[1]), vf = 0.5 * (sides.l.w[2] + sides.r.w[2]);
  double u_x = gf[0], u_r = gf[1], v_x = gf[2], v_r = gf[3], t_x = gf[4], t_r = gf[5];
  double div = u_x + v_r + vf / f.rm;
  double mue = mu_f + mut_f;
  double txx = mue * (2.0 * u_x - 2.0 / 3.0 * div);
  double trr = mue * (2.0 * v_r - 2.0 / 3.0 * div);
  double txr = mue * (u_r + v_x);
  double kappa = (mu_f / PRANDTL + mut_f / PRANDTL_T) / (GAMMA - 1.0);
  return {0.0, txx * f.nx + txr * f.nr, txr * f.nx + trr * f.nr, (uf * txx + vf * txr + kappa * t_x) * f.nx + (uf * txr + vf * trr + kappa * t_r) * f.nr};
}

static void visc_face_pass(const Grid& g, const std::vector<Prim>& w, const Walls& walls, const std::vector<std::array<double, 6>>& grad,
                           const std::vector<double>& mu, const std::vector<double>& mu_t, const std::vector<std::array<double, 3>>& rough,
                           std::vector<Cons>& fvi, std::vector<Cons>& fvj) {  // viscous.rs:347-381
  const size_t ni = g.ni, nj = g.nj;
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i <= ni; ++i) {
      FaceSides s;
      if (iface_sides(g, w, walls, i, j, s)) {
        auto c = iface_centre(g, i, j);
        fvi[j * (ni + 1) + i] = viscous_flux(g, grad, mu, mu_t, rough, s, g.iface[j * (ni + 1) + i], c.first, c.second);
      } else
        fvi[j * (ni + 1) + i] = Cons{};
    }
  }
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl <= (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      FaceSides s;
      if (jface_sides(g, w, walls, i, j, s)) {
        auto c = jface_centre(g, i, j);
        fvj[j * ni + i] = viscous_flux(g, grad, mu, mu_t, rough, s, g.jface[j * ni + i], c.first, c.second);
      } else
        fvj[j * ni + i] = Cons{};
    }
  }
}

static void rough_pass(const Grid& g, const std::vector<Prim>& w, const Walls& walls, const std::vector<double>& dwall,
                       const std::vector<double>& mu, double ks, std::vector<std::array<double, 3>>& out) {  // viscous.rs:387-409
  const size_t ni = g.ni, nj = g.nj;
  size_t wall_i_start = walls.has_visc ? walls.visc.wall_i_start : 0;
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      out[c] = {0.0, 0.0, 0.0};
      bool rough = walls.rough_jface(i, j);
      if ((walls.has_blk && walls.blk.solid(i, j)) || !(rough || walls.noslip_jface(i, j) || walls.noslip_iface(i, j))) continue;
      const Prim& wc = w[(j + NG) * (ni + 2 * NG) + i + NG];
      double nu = mu[c] / wc[0];
      if (rough) {
        double ks_eff = ks * rough_ramp(i, wall_i_start);
        auto a = aupoix_wall(nu, std::hypot(wc[1], wc[2]), dwall[c], ks_eff);
        out[c] = {a[0], a[1], wc[0] * a[2]};
      } else {
        out[c] = {0.0, 60.0 * nu / (BETA1 * dwall[c] * dwall[c]), 0.0};
      }
    }
  }
}

double hoop_stress(double mue, const std::array<double, 6>& g, double v_c, double r_c) {  // viscous.rs:413-416
  double div = g[0] + g[3] + v_c / r_c;
  return mue * (2.0 * v_c / r_c - 2.0 / 3.0 * div);
}
double diffusion_rate(double mu_c, double mu_t_c, double rho_c, double len, double area) {  // viscous.rs:421-424
  double lv = GAMMA * (mu_c / PRANDTL + mu_t_c / PRANDTL_T) / rho_c;
  return 2.0 * lv * len * len / area;
}
static void face_lambdas(const Grid& g, const std::vector<Prim>& w, const Walls& walls, const std::vector<double>& mu,
                         const std::vector<double>& mu_t, const std::vector<std::array<double, 3>>& rough, bool dir_i, size_t i, size_t j,
                         double& lam_l, double& lam_r) {  // viscous.rs:429-454
  auto lam = [&](bool ok, const FaceSides& s, std::pair<double, double> c) {
    if (!ok) return 0.0;
    double dd, ex, er;
    stencil(g, s, c.first, c.second, dd, ex, er);
    double mu_f, mut_f;
    face_mu(mu, mu_t, rough, s, mu_f, mut_f);
    double rho_f = 0.5 * (s.l.w[0] + s.r.w[0]);
    return GAMMA * (mu_f / PRANDTL + mut_f / PRANDTL_T) / (rho_f * dd);
  };
  FaceSides a, b;
  if (dir_i) {
    bool oa = iface_sides(g, w, walls, i, j, a);
    bool ob = iface_sides(g, w, walls, i + 1, j, b);
    lam_l = lam(oa, a, iface_centre(g, i, j));
    lam_r = lam(ob, b, iface_centre(g, i + 1, j));
  } else {
    bool oa = jface_sides(g, w, walls, i, j, a);
    bool ob = jface_sides(g, w, walls, i, j + 1, b);
    lam_l = lam(oa, a, jface_centre(g, i, j));
    lam_r = lam(ob, b, jface_centre(g, i, j + 1));
  }
}

// ======================================================================== turbulence.rs
std::vector<double> wall_distance(const Grid& g, const Walls& walls) {  // turbulence.rs:91-125
  const size_t ni = g.ni, nj = g.nj;
  std::vector<std::array<double, 4>> segs;
  for (size_t j = 0; j <= nj; ++j)
    for (size_t i = 0; i < ni; ++i)
      if (walls.noslip_jface(i, j)) {
        auto a = g.node(i, j), b = g.node(i + 1, j);
        segs.push_back({a.first, a.second, b.first, b.second});
      }
  for (size_t j = 0; j < nj; ++j)
    for (size_t i = 0; i <= ni; ++i)
      if (walls.noslip_iface(i, j)) {
        auto a = g.node(i, j), b = g.node(i, j + 1);
        segs.push_back({a.first, a.second, b.first, b.second});
      }
  std::vector<double> d(ni * nj, std::numeric_limits<double>::infinity());
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      if (walls.has_blk && walls.blk.solid(i, j)) continue;
      double px = g.xc[j * ni + i], pr = g.rc[j * ni + i];
      double& out = d[j * ni + i];
      for (const auto& s : segs) {
        double ex = s[2] - s[0], er = s[3] - s[1];
        double t = clamp_rs(((px - s[0]) * ex + (pr - s[1]) * er) / (ex * ex + er * er), 0.0, 1.0);
        out = fmin_rs(out, std::hypot(px - (s[0] + t * ex), pr - (s[1] + t * er)));
      }
    }
  }
  return d;
}

void turb_init(Solver& s, double re_c) {  // turbulence.rs:128-138
  size_t n = s.grid.ni * s.grid.nj;
  s.turb.assign(n, std::array<double, 2>{K_INF, omega_inf(re_c)});
  s.dwall = wall_distance(s.grid, s.walls());
  size_t ni = s.grid.ni;
  for (size_t c = 0; c < n; ++c)
    if (!(s.has_block && s.block.solid(c % ni, c / ni))) s.mu_t[c] = s.u[c][0] * K_INF / omega_inf(re_c);
}

enum KindTag { KIND_CELL = 0, KIND_INF = 1, KIND_FIXED = 2, KIND_WALL = 3 };
static inline int bc_kind(int bc) { return (bc == BC_FREESTREAM || bc == BC_CHARACTERISTIC || bc == BC_PRESSURE_OUTFLOW) ? KIND_INF : KIND_CELL; }

struct Ctx {  // turbulence.rs:161-246
  const std::vector<std::array<double, 3>>* rough;
  const Grid* grid;
  const std::vector<Prim>* w;
  Walls walls;
  int bc[4];
  const std::vector<double>* mu;
  const std::vector<double>* mu_t;
  const std::vector<std::array<double, 2>>* turb;
  const std::vector<double>* dwall;
  std::array<double, 2> inf;
  bool solid(size_t i, size_t j) const { return walls.has_blk && walls.blk.solid(i, j); }
  double rho(size_t c) const {
    size_t ni = grid->ni;
    return (*w)[(c / ni + NG) * (ni + 2 * NG) + c % ni + NG][0];
  }
  bool iface(size_t i, size_t j, FaceSides& s, int& kind) const {
    if (!iface_sides(*grid, *w, walls, i, j, s)) return false;
    if (i == 0)
      kind = bc_kind(bc[0]);
    else if (i == grid->ni)
      kind = bc_kind(bc[1]);
    else if (s.l.ghost && s.l.has_fixed && walls.has_nozzle)
      kind = KIND_FIXED;
    else if (s.l.ghost && s.noslip)
      kind = KIND_WALL;
    else
      kind = KIND_CELL;
    return true;
  }
  bool jface(size_t i, size_t j, FaceSides& s, int& kind) const {
    if (!jface_sides(*grid, *w, walls, i, j, s)) return false;
    if (s.l.ghost) {
      if (s.noslip)
        kind = KIND_WALL;
      else if (j == 0)
        kind = bc_kind(bc[2]);
      else
        kind = KIND_CELL;
    } else if (s.r.ghost)
      kind = bc_kind(bc[3]);
    else
      kind = KIND_CELL;
    return true;
  }
  std::array<double, 2> kw(const Side& s, int kind) const {
    size_t c = s.cell;
    if (!s.ghost) return (*turb)[c];
    switch (kind) {
      case KIND_CELL:
        return (*turb)[c];
      case KIND_INF:
        return inf;
      case KIND_FIXED:
        return walls.nozzle.turb;
      default: {
        double k = (*turb)[c][0], om = (*turb)[c][1];
        if (rough->empty()) {
          double nu = (*mu)[c] / rho(c);
          double d = (*dwall)[c];
          return {-k, 2.0 * (60.0 * nu / (BETA1 * d * d)) - om};
        }
        const auto& r = (*rough)[c];
        return {2.0 * r[0] - k, 2.0 * r[1] - om};
      }
    }
  }
};

static inline double strain2(const std::array<double, 6>& g, double v, double r) {  // turbulence.rs:250-255
  double vr = v / r;
  double div = g[0] + g[3] + vr;
  double shear = g[1] + g[2];
  return 2.0 * (g[0] * g[0] + g[3] * g[3] + vr * vr) + shear * shear - 2.0 / 3.0 * div * div;
}
static inline void blend_args(double nu, double k, double om, double d, double& t1, double& t2) {  // turbulence.rs:259-261
  t1 = std::sqrt(k) / (BETA_STAR * om * d);
  t2 = 500.0 * nu / (d * d * om);
}
static inline double f2_of(double nu, double k, double om, double d) {  // turbulence.rs:265-269
  double t1, t2;
  blend_args(nu, k, om, d, t1, t2);
  double b = fmax_rs(2.0 * t1, t2);
  return std::tanh(b * b);
}
double rough_ramp(size_t i, size_t wall_i_start) {  // turbulence.rs:288-290
  size_t a = (i + 1) > wall_i_start ? (i + 1) - wall_i_start : 0;
  return fmin_rs((double)a / (double)ROUGH_RAMP_CELLS, 1.0);
}
std::array<double, 3> aupoix_wall(double nu, double speed, double d, double ks) {  // turbulence.rs:304-320
  double smooth = 60.0 * nu / (BETA1 * d * d);
  auto at = [&](double u2) -> std::array<double, 3> {
    double u_tau = std::sqrt(u2);
    double ks_plus = fmax_rs(u_tau * ks / nu, 1e-30);
    double t = std::tanh(ks_plus / 125.0);
    double k_plus = fmax_rs(std::tanh((std::log10(ks_plus / 30.0) + 1.0 - t) * t), 0.0) / std::sqrt(BETA_STAR);
    double om_rough = 300.0 * nu / (ks * ks) / std::tanh(15.0 / (4.0 * ks_plus)) + 191.0 * u_tau / ks * (1.0 - std::exp(-ks_plus / 250.0));
    double k_w = k_plus * u2, om_w = fmin_rs(om_rough, smooth);
    return {k_w, om_w, fmin_rs(k_w / om_w, NU_T_WALL_MAX * nu)};
  };
  double u2 = nu * speed / d;
  for (size_t k = 0; k < AUPOIX_ITERATIONS; ++k) u2 = (nu + at(u2)[2]) * speed / d;
  return at(u2);
}
static inline double eddy_viscosity(double rho, double k, double om, double s, double f2, double re_c) {  // turbulence.rs:324-326
  return fmin_rs(rho * A1 * k / fmax_rs(A1 * om, s * f2), 1e5 / re_c);
}

struct Blend {
  double f1 = 0, x = 0;
};
struct TFace {  // turbulence.rs:401-410
  double m = 0;
  double g[2] = {0, 0};
  double flux[2] = {0, 0};
  std::array<double, 2> l{}, r{};
};
struct CellTerms {  // turbulence.rs:466-474
  double r[2] = {0, 0}, d0[2] = {0, 0};
  double lo[2][2] = {{0, 0}, {0, 0}}, dd[2][2] = {{0, 0}, {0, 0}}, up[2][2] = {{0, 0}, {0, 0}};
};

static TFace tface(const Ctx& cx, const std::vector<std::array<double, 4>>& tg, const std::vector<Blend>& blend, const FaceSides& sides,
                   int kind, const Face& f, double xf, double rf, double m) {  // turbulence.rs:413-435
  auto kl = cx.kw(sides.l, kind), kr = cx.kw(sides.r, kind);
  TFace out;
  out.m = m;
  out.l = kl;
  out.r = kr;
  if (f.rm == 0.0) return out;
  double w = f.w();
  double dd, ex, er;
  stencil(*cx.grid, sides, xf, rf, dd, ex, er);
  const auto& gl = tg[sides.l.cell];
  const auto& gr = tg[sides.r.cell];
  double mu_f, mut_f;
  face_mu(*cx.mu, *cx.mu_t, *cx.rough, sides, mu_f, mut_f);
  double f1l = blend[sides.l.cell].f1, f1r = blend[sides.r.cell].f1;
  for (int e = 0; e < 2; ++e) {
    double s1 = e == 0 ? SIGMA_K1 : SIGMA_W1, s2 = e == 0 ? SIGMA_K2 : SIGMA_W2;
    double sigma = 0.5 * (f1l * s1 + (1.0 - f1l) * s2 + f1r * s1 + (1.0 - f1r) * s2);
    double coef = mu_f + sigma * mut_f;
    double gbx = 0.5 * (gl[2 * e] + gr[2 * e]), gbr = 0.5 * (gl[2 * e + 1] + gr[2 * e + 1]);
    double corr = (kr[e] - kl[e]) / dd - (gbx * ex + gbr * er);
    double gn = (gbx + corr * ex) * f.nx + (gbr + corr * er) * f.nr;
    out.flux[e] = coef * gn * w;
    out.g[e] = coef * w / dd;
  }
  return out;
}

static inline M4 diag2(double a, double b) {
  M4 m = ZERO4;
  m[0] = a;
  m[5] = b;
  m[10] = 1.0;
  m[15] = 1.0;
  return m;
}
static inline M4 offdiag2(double a, double b) {
  M4 m = ZERO4;
  m[0] = a;
  m[5] = b;
  return m;
}

void turb_update(Solver& s) {  // turbulence.rs:542-611
  const Viscous v = s.viscous;
  const size_t ni = s.grid.ni, nj = s.grid.nj, n = ni * nj;
  const std::array<double, 2> inf = {K_INF, omega_inf(v.re_c)};
  Ctx cx;
  cx.rough = &s.rough_wall;
  cx.grid = &s.grid;
  cx.w = &s.w;
  cx.walls = s.walls();
  for (int k = 0; k < 4; ++k) cx.bc[k] = s.cfg.bc[k];
  cx.mu = &s.mu;
  cx.mu_t = &s.mu_t;
  cx.turb = &s.turb;
  cx.dwall = &s.dwall;
  cx.inf = inf;
  std::vector<std::array<double, 4>> tg(n);
  std::vector<Blend> blend(n);
  std::vector<TFace> ti((ni + 1) * nj), tj(ni * (nj + 1));
  std::vector<CellTerms> cells(n);
  // kernel 1: scalar gradients (turbulence.rs:337-372)
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      if (cx.solid(i, j)) {
        tg[c] = {};
        continue;
      }
      auto pc = s.turb[c];
      FaceSides sl, sr, sb, st;
      int kl, kr, kb, kt;
      cx.iface(i, j, sl, kl);
      cx.iface(i + 1, j, sr, kr);
      cx.jface(i, j, sb, kb);
      cx.jface(i, j + 1, st, kt);
      const Face* fs[4] = {&s.grid.iface[j * (ni + 1) + i + 1], &s.grid.iface[j * (ni + 1) + i], &s.grid.jface[(j + 1) * ni + i],
                           &s.grid.jface[j * ni + i]};
      const double sg[4] = {1.0, -1.0, 1.0, -1.0};
      std::array<double, 2> nb[4] = {cx.kw(sr.r, kr), cx.kw(sl.l, kl), cx.kw(st.r, kt), cx.kw(sb.l, kb)};
      std::array<double, 4> g{};
      for (int t = 0; t < 4; ++t)
        for (int m = 0; m < 2; ++m) {
          double pf = 0.5 * (pc[m] + nb[t][m]);
          g[2 * m] += sg[t] * pf * fs[t]->nx * fs[t]->len;
          g[2 * m + 1] += sg[t] * pf * fs[t]->nr * fs[t]->len;
        }
      double inv_a = 1.0 / s.grid.area[c];
      for (auto& x : g) x *= inv_a;
      tg[c] = g;
    }
  }
  // kernel 2: blends (turbulence.rs:375-397)
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      if (cx.solid(i, j)) {
        blend[c] = Blend{};
        continue;
      }
      double rho = cx.rho(c);
      double nu = s.mu[c] / rho;
      double k = s.turb[c][0], om = s.turb[c][1];
      double d = s.dwall[c];
      const auto& g = tg[c];
      double x = 2.0 * rho * SIGMA_W2 * (g[0] * g[2] + g[1] * g[3]) / om;
      double cd = fmax_rs(x, 1e-20);
      double t1, t2;
      blend_args(nu, k, om, d, t1, t2);
      double t3 = 4.0 * rho * SIGMA_W2 * k / (cd * d * d);
      double a = fmin_rs(fmax_rs(t1, t2), t3);
      blend[c] = Blend{std::tanh(std::pow(a, 4)), x};
    }
  }
  // kernel 3: face data (turbulence.rs:438-462)
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i <= ni; ++i) {
      FaceSides sd;
      int kind;
      if (cx.iface(i, j, sd, kind)) {
        const Face& f = s.grid.iface[j * (ni + 1) + i];
        auto c = iface_centre(s.grid, i, j);
        ti[j * (ni + 1) + i] = tface(cx, tg, blend, sd, kind, f, c.first, c.second, s.fi[j * (ni + 1) + i][0] * f.w());
      } else
        ti[j * (ni + 1) + i] = TFace{};
    }
  }
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl <= (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      FaceSides sd;
      int kind;
      if (cx.jface(i, j, sd, kind)) {
        const Face& f = s.grid.jface[j * ni + i];
        auto c = jface_centre(s.grid, i, j);
        tj[j * ni + i] = tface(cx, tg, blend, sd, kind, f, c.first, c.second, s.fj[j * ni + i][0] * f.w());
      } else
        tj[j * ni + i] = TFace{};
    }
  }
  // kernel 4: cell terms (turbulence.rs:477-519)
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      CellTerms& o = cells[c];
      if (cx.solid(i, j)) {
        o = CellTerms{};
        continue;
      }
      double vol = s.grid.vol[c];
      double rho = cx.rho(c);
      double k = s.turb[c][0], om = s.turb[c][1];
      double phi[2] = {k, om};
      const Blend& b = blend[c];
      const Prim& wc = s.w[s.pidx((long)i, (long)j)];
      double s2 = strain2(s.grad[c], wc[2], s.grid.rc[c]);
      double mut_c = s.mu_t[c];
      double prod = fmin_rs(mut_c * s2, 10.0 * BETA_STAR * rho * k * om);
      double beta = b.f1 * BETA1 + (1.0 - b.f1) * BETA2;
      double gamma = b.f1 * GAMMA1 + (1.0 - b.f1) * GAMMA2;
      double sources[2] = {prod - BETA_STAR * rho * om * k,
                           gamma * rho * prod / fmax_rs(mut_c, 1e-30) - beta * rho * om * om + (1.0 - b.f1) * b.x};
      double dest[2] = {BETA_STAR * om, 2.0 * beta * om};
      const TFace* lo_f[2] = {&ti[j * (ni + 1) + i], &tj[j * ni + i]};
      const TFace* up_f[2] = {&ti[j * (ni + 1) + i + 1], &tj[(j + 1) * ni + i]};
      size_t rs = s.has_block ? (s.block.row_start(j) == SIZE_MAX ? ni : s.block.row_start(j)) : 0;
      size_t cs = s.has_block ? s.block.col_start(i) : 0;
      bool ends_lo[2] = {i == rs, j == cs};
      bool ends_up[2] = {i == ni - 1, j == nj - 1};
      double rate[2] = {0.0, 0.0};
      for (int dir = 0; dir < 2; ++dir) {
        double a_lo = fmax_rs(lo_f[dir]->m, 0.0), a_up = fmax_rs(-up_f[dir]->m, 0.0);
        for (int e = 0; e < 2; ++e) {
          rate[e] += a_lo * (lo_f[dir]->l[e] - phi[e]) + a_up * (up_f[dir]->r[e] - phi[e]) + up_f[dir]->flux[e] - lo_f[dir]->flux[e];
          o.lo[dir][e] = ends_lo[dir] ? 0.0 : -(a_lo + lo_f[dir]->g[e]);
          o.up[dir][e] = ends_up[dir] ? 0.0 : -(a_up + up_f[dir]->g[e]);
          o.dd[dir][e] = a_lo + a_up + lo_f[dir]->g[e] + up_f[dir]->g[e];
        }
      }
      for (int e = 0; e < 2; ++e) {
        o.r[e] = rate[e] / vol + sources[e];
        o.d0[e] = rho * vol / s.dt[c] + rho * vol * dest[e];
      }
    }
  }
  // coefficients of the two linear systems (turbulence.rs:559-579)
  Factor fac_i, fac_j;
  fac_i.lo.assign(n, ZERO4);
  fac_i.d.assign(n, EYE4);
  fac_i.up.assign(n, ZERO4);
  fac_j = fac_i;
  std::vector<Cons> x(n, Cons{});
  for (size_t c = 0; c < n; ++c) {
    if (cx.solid(c % ni, c / ni)) continue;
    const CellTerms& t = cells[c];
    double vol = s.grid.vol[c];
    x[c] = {vol * t.r[0], vol * t.r[1], 0.0, 0.0};
    fac_i.lo[c] = offdiag2(t.lo[0][0], t.lo[0][1]);
    fac_i.up[c] = offdiag2(t.up[0][0], t.up[0][1]);
    fac_i.d[c] = diag2(t.d0[0] + t.dd[0][0], t.d0[1] + t.dd[0][1]);
    fac_j.lo[c] = offdiag2(t.lo[1][0] / t.d0[0], t.lo[1][1] / t.d0[1]);
    fac_j.up[c] = offdiag2(t.up[1][0] / t.d0[0], t.up[1][1] / t.d0[1]);
    fac_j.d[c] = diag2(1.0 + t.dd[1][0] / t.d0[0], 1.0 + t.dd[1][1] / t.d0[1]);
  }
  solve_lines(s, fac_i, true, x);
  solve_lines(s, fac_j, false, x);
  // clipped update and eddy viscosity (turbulence.rs:584-603)
  std::vector<std::array<double, 2>> turb_new(n);
  std::vector<double> mut_new(n);
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)nj; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < ni; ++i) {
      size_t c = j * ni + i;
      if (cx.solid(i, j)) {
        turb_new[c] = {0.0, 0.0};
        mut_new[c] = 0.0;
        continue;
      }
      double k0 = s.turb[c][0], w0 = s.turb[c][1];
      double k = fmax_rs(fmax_rs(k0 + x[c][0], 0.1 * k0), 1e-3 * inf[0]);
      double om = fmax_rs(fmax_rs(w0 + x[c][1], 0.1 * w0), 1e-3 * inf[1]);
      double rho = cx.rho(c);
      double nu = s.mu[c] / rho;
      double strain = std::sqrt(fmax_rs(strain2(s.grad[c], s.w[s.pidx((long)i, (long)j)][2], s.grid.rc[c]), 0.0));
      turb_new[c] = {k, om};
      mut_new[c] = eddy_viscosity(rho, k, om, strain, f2_of(nu, k, om, s.dwall[c]), v.re_c);
    }
  }
  double sum = 0.0;
  for (const auto& t : cells) sum += t.r[0] * t.r[0];
  s.turb.swap(turb_new);
  s.mu_t.swap(mut_new);
  s.turb_rnorm = std::sqrt(sum / (double)s.n_active);
}

}  // namespace orc
