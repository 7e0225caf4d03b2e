// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// f64 CPU restatement of the reference's 3D Euler path: crates/bowshock-cfd/src/{gas3,bc3,flux3,grid3,solver3,implicit3}.rs
// and the runner / forces of crates/bowshock-core/src/engine/run3.rs (pressure forces CN, CA and the centre of pressure).
// Solid boxes (fins, solver3.rs:13, grid3.rs:17-24) in the residual, time step, stages, implicit blocks and forces. The
// oracle of the CUDA 3D path; only tests/ load it.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "oracle.hpp"

namespace orc3 {

using C5 = std::array<double, 5>;
using M5 = std::array<double, 25>;
constexpr double G = orc::GAMMA;
constexpr int NG = 2;

static inline double fmax_rs(double a, double b) { return std::fmax(a, b); }
static inline double fmin_rs(double a, double b) { return std::fmin(a, b); }
static inline double clamp_rs(double x, double lo, double hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}

// ---------------------------------------------------------------- gas3.rs
C5 prim_to_cons3(const C5& w) {  // gas3.rs:14-17
  double rho = w[0], u = w[1], v = w[2], ww = w[3], p = w[4];
  return {rho, rho * u, rho * v, rho * ww, p / (G - 1.0) + 0.5 * rho * (u * u + v * v + ww * ww)};
}
C5 cons_to_prim3(const C5& q) {  // gas3.rs:20-25
  double rho = q[0];
  double u = q[1] / rho, v = q[2] / rho, w = q[3] / rho;
  double p = (G - 1.0) * (q[4] - 0.5 * rho * (u * u + v * v + w * w));
  return {rho, u, v, w, p};
}
double sound_speed3(const C5& w) { return std::sqrt(G * w[4] / w[0]); }  // gas3.rs:28-30
C5 physical_flux3(const C5& w, const double* n) {                          // gas3.rs:34-39
  double rho = w[0], u = w[1], v = w[2], ww = w[3], p = w[4];
  double un = u * n[0] + v * n[1] + ww * n[2];
  double e = p / (G - 1.0) + 0.5 * rho * (u * u + v * v + ww * ww);
  return {rho * un, rho * u * un + p * n[0], rho * v * un + p * n[1], rho * ww * un + p * n[2], (e + p) * un};
}
C5 freestream3(double mach, double alpha) { return {1.0, mach * std::cos(alpha), 0.0, mach * std::sin(alpha), 1.0 / G}; }  // gas3.rs:42-44
C5 reflect3(const C5& w, const double* n) {  // gas3.rs:48-51
  double un = w[1] * n[0] + w[2] * n[1] + w[3] * n[2];
  return {w[0], w[1] - 2.0 * un * n[0], w[2] - 2.0 * un * n[1], w[3] - 2.0 * un * n[2], w[4]};
}

// ---------------------------------------------------------------- bc3.rs
double normal_mach3(const C5& w, const double* n) { return (w[1] * n[0] + w[2] * n[1] + w[3] * n[2]) / sound_speed3(w); }  // bc3.rs:10-12
C5 characteristic_ghost3(const C5& fs, const C5& in, const double* n) {  // bc3.rs:30-56
  double m = normal_mach3(in, n);
  if (m <= -1.0) return fs;
  if (m >= 1.0) return in;
  double g1 = G - 1.0;
  double ci = sound_speed3(in), ce = sound_speed3(fs);
  double uni = in[1] * n[0] + in[2] * n[1] + in[3] * n[2];
  double une = fs[1] * n[0] + fs[2] * n[1] + fs[3] * n[2];
  double r_out = uni + 2.0 * ci / g1;
  double r_in = une - 2.0 * ce / g1;
  double un_b = 0.5 * (r_out + r_in);
  double c_b = fmax_rs(0.25 * g1 * (r_out - r_in), 1e-8);
  const C5& rf = un_b >= 0.0 ? in : fs;
  double un_ref = un_b >= 0.0 ? uni : une;
  double s = rf[4] / std::pow(rf[0], G);
  double rho = std::pow(c_b * c_b / (G * s), 1.0 / g1);
  double p = rho * c_b * c_b / G;
  double dn = un_b - un_ref;
  return {rho, rf[1] + dn * n[0], rf[2] + dn * n[1], rf[3] + dn * n[2], p};
}

// ---------------------------------------------------------------- flux3.rs
std::array<double, 2> face_rot(const double* c) {  // flux3.rs:11-19
  double r = std::hypot(c[1], c[2]);
  if (r < 1e-300) return {0.0, 1.0};
  return {c[1] / r, c[2] / r};
}
void reconstruct3(const C5& m2, const C5& m1, const C5& p0, const C5& p1, int lim, const std::array<double, 2>& rot, C5& lo,
                  C5& ro) {  // flux3.rs:27-54
  double s = rot[0], co = rot[1];
  auto fwd = [&](const C5& w) { return C5{w[0], w[1], w[2] * s + w[3] * co, w[2] * co - w[3] * s, w[4]}; };
  C5 a = fwd(m2), b = fwd(m1), c = fwd(p0), d = fwd(p1);
  C5 l = b, r = c;
  for (int k = 0; k < 5; ++k) {
    double phi_l = orc::limited_slope(b[k] - a[k], c[k] - b[k], lim);
    double phi_r = orc::limited_slope(c[k] - b[k], d[k] - c[k], lim);
    l[k] = b[k] + 0.5 * phi_l;
    r[k] = c[k] - 0.5 * phi_r;
  }
  if (l[0] <= 0.0 || l[4] <= 0.0) l = b;
  if (r[0] <= 0.0 || r[4] <= 0.0) r = c;
  auto back = [&](const C5& w, const C5& orig, bool fallback) {
    if (fallback) return orig;
    return C5{w[0], w[1], w[2] * s + w[3] * co, w[2] * co - w[3] * s, w[4]};
  };
  lo = back(l, m1, l == b);
  ro = back(r, p0, r == c);
}
C5 hllc3(const C5& wl, const C5& wr, const double* n) {  // flux3.rs:59-117
  double rl = wl[0], ul = wl[1], vl = wl[2], zl = wl[3], pl = wl[4];
  double rr = wr[0], ur = wr[1], vr = wr[2], zr = wr[3], pr = wr[4];
  double unl = ul * n[0] + vl * n[1] + zl * n[2];
  double unr = ur * n[0] + vr * n[1] + zr * n[2];
  double cl = std::sqrt(G * pl / rl), cr = std::sqrt(G * pr / rr);
  double el = pl / (G - 1.0) + 0.5 * rl * (ul * ul + vl * vl + zl * zl);
  double er = pr / (G - 1.0) + 0.5 * rr * (ur * ur + vr * vr + zr * zr);
  double sql = std::sqrt(rl), sqr = std::sqrt(rr);
  double inv = 1.0 / (sql + sqr);
  double uh = (sql * ul + sqr * ur) * inv, vh = (sql * vl + sqr * vr) * inv, wh = (sql * zl + sqr * zr) * inv;
  double hl = (el + pl) / rl, hr = (er + pr) / rr;
  double hh = (sql * hl + sqr * hr) * inv;
  double ch2 = (G - 1.0) * (hh - 0.5 * (uh * uh + vh * vh + wh * wh));
  double ch = std::sqrt(fmax_rs(ch2, 1e-300));
  double unh = uh * n[0] + vh * n[1] + wh * n[2];
  double sl = fmin_rs(unl - cl, unh - ch);
  double sr = fmax_rs(unr + cr, unh + ch);
  if (sl >= 0.0) return physical_flux3(wl, n);
  if (sr <= 0.0) return physical_flux3(wr, n);
  double sm = (pr - pl + rl * unl * (sl - unl) - rr * unr * (sr - unr)) / (rl * (sl - unl) - rr * (sr - unr));
  C5 out;
  if (sm >= 0.0) {
    C5 f = physical_flux3(wl, n);
    double fac = rl * (sl - unl) / (sl - sm);
    double d = sm - unl;
    C5 star = {fac, fac * (ul + d * n[0]), fac * (vl + d * n[1]), fac * (zl + d * n[2]), fac * (el / rl + d * (sm + pl / (rl * (sl - unl))))};
    C5 q = {rl, rl * ul, rl * vl, rl * zl, el};
    for (int k = 0; k < 5; ++k) out[k] = f[k] + sl * (star[k] - q[k]);
  } else {
    C5 f = physical_flux3(wr, n);
    double fac = rr * (sr - unr) / (sr - sm);
    double d = sm - unr;
    C5 star = {fac, fac * (ur + d * n[0]), fac * (vr + d * n[1]), fac * (zr + d * n[2]), fac * (er / rr + d * (sm + pr / (rr * (sr - unr))))};
    C5 q = {rr, rr * ur, rr * vr, rr * zr, er};
    for (int k = 0; k < 5; ++k) out[k] = f[k] + sr * (star[k] - q[k]);
  }
  return out;
}
C5 rusanov3(const C5& wl, const C5& wr, const double* n) {  // flux3.rs:121-135
  double rl = wl[0], ul = wl[1], vl = wl[2], zl = wl[3], pl = wl[4];
  double rr = wr[0], ur = wr[1], vr = wr[2], zr = wr[3], pr = wr[4];
  double unl = ul * n[0] + vl * n[1] + zl * n[2];
  double unr = ur * n[0] + vr * n[1] + zr * n[2];
  double smax = fmax_rs(std::fabs(unl) + std::sqrt(G * pl / rl), std::fabs(unr) + std::sqrt(G * pr / rr));
  C5 fl = physical_flux3(wl, n), fr = physical_flux3(wr, n);
  C5 ql = {rl, rl * ul, rl * vl, rl * zl, pl / (G - 1.0) + 0.5 * rl * (ul * ul + vl * vl + zl * zl)};
  C5 qr = {rr, rr * ur, rr * vr, rr * zr, pr / (G - 1.0) + 0.5 * rr * (ur * ur + vr * vr + zr * zr)};
  C5 out;
  for (int k = 0; k < 5; ++k) out[k] = 0.5 * (fl[k] + fr[k]) - 0.5 * smax * (qr[k] - ql[k]);
  return out;
}
static C5 blend3(const C5& l, const C5& r, double pl, double pr, const double* n) {  // flux3.rs:146-158
  C5 c = hllc3(l, r, n);
  double t = orc::shock_weight(pl, pr);
  if (t == 0.0) return c;
  C5 f = rusanov3(l, r, n);
  C5 out = c;
  for (int k = 0; k < 5; ++k) out[k] = (1.0 - t) * c[k] + t * f[k];
  return out;
}
void low_mach_states3(const C5& l, const C5& r, const double* n, C5& lo, C5& ro) {  // flux3.rs:163-176
  double unl = l[1] * n[0] + l[2] * n[1] + l[3] * n[2];
  double unr = r[1] * n[0] + r[2] * n[1] + r[3] * n[2];
  double ml = std::sqrt(l[1] * l[1] + l[2] * l[2] + l[3] * l[3]) / std::sqrt(G * l[4] / l[0]);
  double mr = std::sqrt(r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) / std::sqrt(G * r[4] / r[0]);
  double z = clamp_rs(fmax_rs(ml, mr), orc::LOW_MACH_FLOOR, 1.0);
  if (z >= 1.0) {
    lo = l;
    ro = r;
    return;
  }
  double avg = 0.5 * (unl + unr);
  double dl = avg + z * (unl - avg) - unl;
  double dr = avg + z * (unr - avg) - unr;
  lo = {l[0], l[1] + dl * n[0], l[2] + dl * n[1], l[3] + dl * n[2], l[4]};
  ro = {r[0], r[1] + dr * n[0], r[2] + dr * n[1], r[3] + dr * n[2], r[4]};
}
C5 face_flux_lm3(const C5& m2, const C5& m1, const C5& p0, const C5& p1, int lim, const double* n, const std::array<double, 2>& rot,
                 bool low_mach) {  // flux3.rs:140-143, 180-188
  C5 l, r;
  reconstruct3(m2, m1, p0, p1, lim, rot, l, r);
  if (low_mach) {
    C5 l2, r2;
    low_mach_states3(l, r, n, l2, r2);
    return blend3(l2, r2, m1[4], p0[4], n);
  }
  return blend3(l, r, m1[4], p0[4], n);
}

// ---------------------------------------------------------------- grid3.rs
struct Face3 {
  double n[3] = {0, 0, 0};
  double area = 0;
  double c[3] = {0, 0, 0};
};
struct Grid3 {
  size_t ni = 0, nj = 0, nk = 0;
  std::vector<double> x, y, z;
  std::vector<Face3> iface, jface, kface;
  std::vector<double> vol;
  std::vector<std::array<double, 3>> xc;
  size_t axis_cells = 0;
  size_t cell(size_t i, size_t j, size_t k) const { return (k * nj + j) * ni + i; }
};

static std::array<double, 3> cross(const std::array<double, 3>& a, const std::array<double, 3>& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
static std::array<double, 3> sub(const std::array<double, 3>& a, const std::array<double, 3>& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
static double dot3(const double* a, const std::array<double, 3>& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// grid3.rs:66-174: faces from their 4 corners (cyclic order right-handed for the +axis normal), volumes by the divergence
// theorem over the face centroids, one global handedness sign; false on a negative cell volume.
bool grid3_from_nodes(size_t ni, size_t nj, size_t nk, std::vector<double> x, std::vector<double> y, std::vector<double> z, Grid3& g,
                      std::string* err) {
  g = Grid3{};
  g.ni = ni, g.nj = nj, g.nk = nk;
  auto node = [&](size_t i, size_t j, size_t k) { return (k * (nj + 1) + j) * (ni + 1) + i; };
  auto pt = [&](size_t i, size_t j, size_t k) {
    size_t n = node(i, j, k);
    return std::array<double, 3>{x[n], y[n], z[n]};
  };
  using IJK = std::array<size_t, 3>;
  auto face = [&](const std::array<IJK, 4>& cn, Face3& f, std::array<double, 3>& s) {
    std::array<std::array<double, 3>, 4> p;
    for (int q = 0; q < 4; ++q) p[q] = pt(cn[q][0], cn[q][1], cn[q][2]);
    s = cross(sub(p[2], p[0]), sub(p[3], p[1]));
    s = {0.5 * s[0], 0.5 * s[1], 0.5 * s[2]};
    double area = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    if (area < 1e-300) {
      f.n[0] = f.n[1] = f.n[2] = 0.0;
      f.area = 0.0;
    } else {
      f.n[0] = s[0] / area, f.n[1] = s[1] / area, f.n[2] = s[2] / area;
      f.area = area;
    }
    for (int m = 0; m < 3; ++m) f.c[m] = 0.25 * (p[0][m] + p[1][m] + p[2][m] + p[3][m]);
  };
  g.iface.assign((ni + 1) * nj * nk, Face3{});
  g.jface.assign(ni * (nj + 1) * nk, Face3{});
  g.kface.assign(ni * nj * (nk + 1), Face3{});
  std::vector<std::array<double, 3>> si(g.iface.size()), sj(g.jface.size()), sk(g.kface.size());
  for (size_t k = 0; k < nk; ++k)
    for (size_t j = 0; j < nj; ++j)
      for (size_t i = 0; i <= ni; ++i) {
        size_t q = (k * nj + j) * (ni + 1) + i;
        face({IJK{i, j, k}, IJK{i, j + 1, k}, IJK{i, j + 1, k + 1}, IJK{i, j, k + 1}}, g.iface[q], si[q]);
      }
  for (size_t k = 0; k < nk; ++k)
    for (size_t j = 0; j <= nj; ++j)
      for (size_t i = 0; i < ni; ++i) {
        size_t q = (k * (nj + 1) + j) * ni + i;
        face({IJK{i, j, k}, IJK{i, j, k + 1}, IJK{i + 1, j, k + 1}, IJK{i + 1, j, k}}, g.jface[q], sj[q]);
      }
  for (size_t k = 0; k <= nk; ++k)
    for (size_t j = 0; j < nj; ++j)
      for (size_t i = 0; i < ni; ++i) {
        size_t q = (k * nj + j) * ni + i;
        face({IJK{i, j, k}, IJK{i + 1, j, k}, IJK{i + 1, j + 1, k}, IJK{i, j + 1, k}}, g.kface[q], sk[q]);
      }
  g.vol.assign(ni * nj * nk, 0.0);
  g.xc.assign(g.vol.size(), {0, 0, 0});
  for (size_t k = 0; k < nk; ++k)
    for (size_t j = 0; j < nj; ++j)
      for (size_t i = 0; i < ni; ++i) {
        auto qi = [&](size_t ii) { return (k * nj + j) * (ni + 1) + ii; };
        auto qj = [&](size_t jj) { return (k * (nj + 1) + jj) * ni + i; };
        auto qk = [&](size_t kk) { return (kk * nj + j) * ni + i; };
        double v = 0.0;
        v += 1.0 * dot3(g.iface[qi(i + 1)].c, si[qi(i + 1)]);
        v += -1.0 * dot3(g.iface[qi(i)].c, si[qi(i)]);
        v += 1.0 * dot3(g.jface[qj(j + 1)].c, sj[qj(j + 1)]);
        v += -1.0 * dot3(g.jface[qj(j)].c, sj[qj(j)]);
        v += 1.0 * dot3(g.kface[qk(k + 1)].c, sk[qk(k + 1)]);
        v += -1.0 * dot3(g.kface[qk(k)].c, sk[qk(k)]);
        size_t c = (k * nj + j) * ni + i;
        g.vol[c] = v / 3.0;
        std::array<double, 3> m = {0, 0, 0};
        for (int b = 0; b < 8; ++b) {
          size_t dk = b >> 2 & 1, dj = b >> 1 & 1, di = b & 1;
          auto p = pt(i + di, j + dj, k + dk);
          for (int a = 0; a < 3; ++a) m[a] += 0.125 * p[a];
        }
        g.xc[c] = m;
      }
  double tot = 0.0;
  for (double v : g.vol) tot += v;
  if (tot < 0.0) {
    for (auto* fam : {&g.iface, &g.jface, &g.kface})
      for (auto& f : *fam) f.n[0] = -f.n[0], f.n[1] = -f.n[1], f.n[2] = -f.n[2];
    for (auto& v : g.vol) v = -v;
  }
  double vmax = 0.0;
  for (double v : g.vol) vmax = fmax_rs(vmax, std::fabs(v));
  for (size_t k = 0; k < nk; ++k)
    for (size_t j = 0; j < nj; ++j)
      for (size_t i = 0; i < ni; ++i) {
        double v = g.vol[(k * nj + j) * ni + i];
        if (v < -1e-12 * vmax || std::isnan(v)) {
          if (err) *err = "negative cell volume at (" + std::to_string(i) + "," + std::to_string(j) + "," + std::to_string(k) + ")";
          return false;
        }
      }
  g.x = std::move(x), g.y = std::move(y), g.z = std::move(z);
  return true;
}

// grid3.rs:189-206: node (i, j, k) = (x, r sin theta_k, r cos theta_k)
bool revolve(size_t ni, size_t nj, const double* x2, const double* r2, size_t nk, const double* theta, Grid3& g, std::string* err) {
  size_t n2 = (ni + 1) * (nj + 1);
  std::vector<double> x, y, z;
  x.reserve(n2 * (nk + 1)), y.reserve(n2 * (nk + 1)), z.reserve(n2 * (nk + 1));
  for (size_t k = 0; k <= nk; ++k) {
    double s = std::sin(theta[k]), c = std::cos(theta[k]);
    for (size_t n = 0; n < n2; ++n) {
      x.push_back(x2[n]);
      y.push_back(r2[n] * s);
      z.push_back(r2[n] * c);
    }
  }
  return grid3_from_nodes(ni, nj, nk, std::move(x), std::move(y), std::move(z), g, err);
}

// ---------------------------------------------------------------- implicit3.rs (blocks)
M5 flux_jacobian3(const C5& w, const double* n) {  // implicit3.rs:44-60
  double rho = w[0], u = w[1], v = w[2], ww = w[3], p = w[4];
  double nx = n[0], ny = n[1], nz = n[2];
  double g1 = G - 1.0;
  double q2 = u * u + v * v + ww * ww;
  double th = u * nx + v * ny + ww * nz;
  double phi = 0.5 * g1 * q2;
  double h = G * p / (g1 * rho) + 0.5 * q2;
  return {0.0,
          nx,
          ny,
          nz,
          0.0,
          phi * nx - u * th,
          th + (2.0 - G) * u * nx,
          u * ny - g1 * v * nx,
          u * nz - g1 * ww * nx,
          g1 * nx,
          phi * ny - v * th,
          v * nx - g1 * u * ny,
          th + (2.0 - G) * v * ny,
          v * nz - g1 * ww * ny,
          g1 * ny,
          phi * nz - ww * th,
          ww * nx - g1 * u * nz,
          ww * ny - g1 * v * nz,
          th + (2.0 - G) * ww * nz,
          g1 * nz,
          th * (phi - h),
          h * nx - g1 * u * th,
          h * ny - g1 * v * th,
          h * nz - g1 * ww * th,
          G * th};
}
M5 mm5(const M5& a, const M5& b) {  // implicit3.rs:62-74
  M5 c{};
  for (int i = 0; i < 5; ++i)
    for (int k = 0; k < 5; ++k) {
      double aik = a[5 * i + k];
      for (int j = 0; j < 5; ++j) c[5 * i + j] += aik * b[5 * k + j];
    }
  return c;
}
C5 mv5(const M5& a, const C5& x) {  // implicit3.rs:77-83
  C5 y;
  for (int i = 0; i < 5; ++i) y[i] = a[5 * i] * x[0] + a[5 * i + 1] * x[1] + a[5 * i + 2] * x[2] + a[5 * i + 3] * x[3] + a[5 * i + 4] * x[4];
  return y;
}
static void axpy5(M5& a, double s, const M5& b) {
  for (int k = 0; k < 25; ++k) a[k] += s * b[k];
}
static M5 eye5() {
  M5 m{};
  for (int q = 0; q < 5; ++q) m[6 * q] = 1.0;
  return m;
}
M5 inv5(const M5& m) {  // implicit3.rs:94-125
  M5 a = m, inv = eye5();
  for (int c = 0; c < 5; ++c) {
    int piv = c;
    for (int r = c + 1; r < 5; ++r)
      if (std::fabs(a[5 * r + c]) > std::fabs(a[5 * piv + c])) piv = r;
    if (piv != c)
      for (int k = 0; k < 5; ++k) std::swap(a[5 * c + k], a[5 * piv + k]), std::swap(inv[5 * c + k], inv[5 * piv + k]);
    double d = 1.0 / a[5 * c + c];
    for (int k = 0; k < 5; ++k) a[5 * c + k] *= d, inv[5 * c + k] *= d;
    for (int r = 0; r < 5; ++r)
      if (r != c) {
        double f = a[5 * r + c];
        if (f != 0.0)
          for (int k = 0; k < 5; ++k) a[5 * r + k] -= f * a[5 * c + k], inv[5 * r + k] -= f * inv[5 * c + k];
      }
  }
  return inv;
}
M5 abs_jacobian3(const C5& wl, const C5& wr, const double* n, double eps_fix) {  // implicit3.rs:160-193
  double sl = std::sqrt(wl[0]), sr = std::sqrt(wr[0]);
  double inv = 1.0 / (sl + sr);
  double u = (sl * wl[1] + sr * wr[1]) * inv, v = (sl * wl[2] + sr * wr[2]) * inv, ww = (sl * wl[3] + sr * wr[3]) * inv;
  auto ke = [](const C5& w) { return 0.5 * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]); };
  double hl = G * wl[4] / ((G - 1.0) * wl[0]) + ke(wl);
  double hr = G * wr[4] / ((G - 1.0) * wr[0]) + ke(wr);
  double h = (sl * hl + sr * hr) * inv;
  double q2h = 0.5 * (u * u + v * v + ww * ww);
  double c = std::sqrt(fmax_rs((G - 1.0) * (h - q2h), 1e-300));
  double a = u * n[0] + v * n[1] + ww * n[2];
  double eps = eps_fix * c;
  auto fix = [&](double l) { return std::fabs(l) >= eps ? std::fabs(l) : 0.5 * (l * l / eps + eps); };
  double e1 = fix(a), e2 = fix(a + c), e3 = fix(a - c);
  double d1 = (e2 - e1) / c;
  double d2 = (e2 + e3 - 2.0 * e1) / (2.0 * c * c);
  C5 wa = {1.0, u, v, ww, (G - 1.0) / G * (h - q2h)};
  M5 am = flux_jacobian3(wa, n);
  M5 b1 = am, b2 = am;
  for (int q = 0; q < 5; ++q) b1[6 * q] -= a, b2[6 * q] -= a + c;
  M5 prod = mm5(b1, b2);
  M5 out;
  for (int k = 0; k < 25; ++k) out[k] = d1 * b1[k] + d2 * prod[k];
  for (int q = 0; q < 5; ++q) out[6 * q] += e1;
  return out;
}
static double spectral3(const C5& w, const double* n) { return std::fabs(w[1] * n[0] + w[2] * n[1] + w[3] * n[2]) + sound_speed3(w); }
M5 reflection3(const double* n) {  // implicit3.rs:202-210
  M5 m = eye5();
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) m[5 * (1 + a) + 1 + b] -= 2.0 * n[a] * n[b];
  return m;
}
// implicit3.rs:214-270
void cell_blocks3(const C5& wk, const C5& wm, const C5& wp, const Face3& fl, const Face3& fr, double vol, double dt, const orc::ImplicitParams& p,
                  M5& lo, M5& d, M5& up) {
  double s = 0.5 * dt / vol;
  double al = fl.area, ar = fr.area;
  M5 dl{}, dr{};
  if (p.roe) {
    dl = abs_jacobian3(wm, wk, fl.n, p.eps_fix);
    dr = abs_jacobian3(wk, wp, fr.n, p.eps_fix);
    double tl = orc::shock_weight(wm[4], wk[4]), tr = orc::shock_weight(wk[4], wp[4]);
    if (tl > 0.0 || tr > 0.0) {
      double lam_l = fmax_rs(spectral3(wk, fl.n), spectral3(wm, fl.n));
      double lam_r = fmax_rs(spectral3(wk, fr.n), spectral3(wp, fr.n));
      for (double& x : dl) x *= 1.0 - tl;
      for (double& x : dr) x *= 1.0 - tr;
      for (int q = 0; q < 5; ++q) dl[6 * q] += tl * lam_l, dr[6 * q] += tr * lam_r;
    }
  } else {
    double lam_l = fmax_rs(spectral3(wk, fl.n), spectral3(wm, fl.n));
    double lam_r = fmax_rs(spectral3(wk, fr.n), spectral3(wp, fr.n));
    for (int q = 0; q < 5; ++q) dl[6 * q] = lam_l, dr[6 * q] = lam_r;
  }
  d = eye5();
  axpy5(d, s * ar, flux_jacobian3(wk, fr.n));
  axpy5(d, -s * al, flux_jacobian3(wk, fl.n));
  axpy5(d, s * ar, dr);
  axpy5(d, s * al, dl);
  if (!p.lines) {
    lo = M5{}, up = M5{};
    return;
  }
  lo = flux_jacobian3(wm, fl.n);
  axpy5(lo, 1.0, dl);
  for (double& x : lo) x *= -s * al;
  up = flux_jacobian3(wp, fr.n);
  axpy5(up, -1.0, dr);
  for (double& x : up) x *= s * ar;
}
// implicit3.rs:133-156: lo_m x_{m-1} + d_m x_m + up_m x_{m+1} = rhs_m in place
void block_thomas5(size_t n, const M5* lo, const M5* d, const M5* up, C5* rhs) {
  std::vector<M5> y(n);
  for (size_t k = 0; k < n; ++k) {
    M5 m = d[k];
    C5 r = rhs[k];
    if (k > 0) {
      M5 t = mm5(lo[k], y[k - 1]);
      axpy5(m, -1.0, t);
      C5 lg = mv5(lo[k], rhs[k - 1]);
      for (int q = 0; q < 5; ++q) r[q] -= lg[q];
    }
    M5 minv = inv5(m);
    rhs[k] = mv5(minv, r);
    if (k + 1 < n) y[k] = mm5(minv, up[k]);
  }
  for (size_t k = n - 1; k-- > 0;) {
    C5 t = mv5(y[k], rhs[k + 1]);
    for (int q = 0; q < 5; ++q) rhs[k][q] -= t[q];
  }
}

// ---------------------------------------------------------------- solver3.rs
struct Solver3 {
  Grid3 grid;
  C5 fs;
  double cfl = 0.5;
  int limiter = orc::MINMOD;
  size_t first_order_iters = 0;
  bool low_mach = false;
  bool implicit = true;
  orc::ImplicitParams ip;
  std::vector<C5> u, w, res, fi, fj, fk, u0;
  std::vector<double> dt;
  size_t iter = 0, ramp_k = 0, n_active = 0;
  std::vector<size_t> axis_k;
  std::vector<std::array<double, 2>> rot_i, rot_j, rot_k;
  // solver3.rs:84-97: per cell, inside a solid box; n_active counts the fluid cells
  std::vector<uint8_t> solid;
  bool has_solid = false;

  size_t pidx(long i, long j, long k) const {
    return ((size_t)(k + NG) * (grid.nj + 2 * NG) + (size_t)(j + NG)) * (grid.ni + 2 * NG) + (size_t)(i + NG);
  }
  void init() {  // solver3.rs:84-140
    size_t ni = grid.ni, nj = grid.nj, nk = grid.nk, nc = ni * nj * nk;
    n_active = nc;
    auto theta = [&](size_t i, size_t k) {
      const auto& c = grid.xc[(k * nj) * ni + i];
      return std::atan2(c[1], c[2]);
    };
    size_t na = std::min(grid.axis_cells, ni);
    axis_k.assign(na * nk, 0);
    for (size_t i = 0; i < na; ++i)
      for (size_t k = 0; k < nk; ++k) {
        double target = M_PI - theta(i, k);
        double best = INFINITY;
        size_t bk = 0;
        for (size_t kk = 0; kk < nk; ++kk) {
          double d = std::fabs(theta(i, kk) - target);
          if (d < best) best = d, bk = kk;
        }
        axis_k[i * nk + k] = bk;
      }
    auto rot = [](const std::vector<Face3>& f, std::vector<std::array<double, 2>>& out) {
      out.resize(f.size());
      for (size_t q = 0; q < f.size(); ++q) out[q] = face_rot(f[q].c);
    };
    rot(grid.iface, rot_i), rot(grid.jface, rot_j), rot(grid.kface, rot_k);
    C5 q = prim_to_cons3(fs);
    u.assign(nc, q);
    w.assign((ni + 2 * NG) * (nj + 2 * NG) * (nk + 2 * NG), fs);
    res.assign(nc, C5{});
    dt.assign(nc, 0.0);
    fi.assign(grid.iface.size(), C5{}), fj.assign(grid.jface.size(), C5{}), fk.assign(grid.kface.size(), C5{});
    u0.assign(nc, C5{});
    iter = ramp_k = 0;
    solid.assign(nc, 0);
    has_solid = false;
  }
  // boxes: 6 per box, half-open ranges [i0, i1) [j0, j1) [k0, k1) (grid3.rs:17-24 SolidBox)
  void set_solid(size_t nbox, const uint64_t* boxes) {
    size_t ni = grid.ni, nj = grid.nj, nk = grid.nk;
    solid.assign(ni * nj * nk, 0);
    for (size_t b = 0; b < nbox; ++b) {
      const uint64_t* q = boxes + 6 * b;
      for (uint64_t k = q[4]; k < std::min<uint64_t>(q[5], nk); ++k)
        for (uint64_t j = q[2]; j < std::min<uint64_t>(q[3], nj); ++j)
          for (uint64_t i = q[0]; i < std::min<uint64_t>(q[1], ni); ++i) solid[(k * nj + j) * ni + i] = 1;
    }
    n_active = 0;
    for (uint8_t v : solid) n_active += v ? 0 : 1;
    has_solid = n_active != solid.size();
  }
  // solver3.rs:343-353: out-of-range (ghost) positions are not solid
  bool is_solid(long i, long j, long k) const {
    return has_solid && i >= 0 && j >= 0 && k >= 0 && (size_t)i < grid.ni && (size_t)j < grid.nj && (size_t)k < grid.nk &&
           solid[((size_t)k * grid.nj + (size_t)j) * grid.ni + (size_t)i];
  }
  double density_residual() const {  // solver3.rs:152-155
    double s = 0.0;
    for (const auto& r : res) s += r[0] * r[0];
    return std::sqrt(s / (double)n_active);
  }
  void fill_ghosts() {  // solver3.rs:171-219
    long ni = (long)grid.ni, nj = (long)grid.nj, nk = (long)grid.nk;
    auto ghost_char = [&](const C5& edge, const double* n, double outward) {
      double o[3] = {outward * n[0], outward * n[1], outward * n[2]};
      return characteristic_ghost3(fs, edge, o);
    };
    for (long k = 0; k < nk; ++k) {
      for (long j = 0; j < nj; ++j) {
        size_t base = ((size_t)k * grid.nj + (size_t)j) * (grid.ni + 1);
        const Face3& fl = grid.iface[base];
        const Face3& fr = grid.iface[base + grid.ni];
        C5 gl = ghost_char(w[pidx(0, j, k)], fl.n, -1.0);
        C5 gr = ghost_char(w[pidx(ni - 1, j, k)], fr.n, 1.0);
        for (long m = 1; m <= NG; ++m) w[pidx(-m, j, k)] = gl, w[pidx(ni + m - 1, j, k)] = gr;
      }
      for (long i = 0; i < ni; ++i) {
        if ((size_t)i < grid.axis_cells) {
          long kp = (long)axis_k[(size_t)i * grid.nk + (size_t)k];
          for (long m = 1; m <= NG; ++m) {
            C5 s = w[pidx(i, m - 1, kp)];
            s[2] = -s[2];
            w[pidx(i, -m, k)] = s;
          }
        } else {
          const Face3& f = grid.jface[((size_t)k * (grid.nj + 1)) * grid.ni + (size_t)i];
          for (long m = 1; m <= NG; ++m) w[pidx(i, -m, k)] = reflect3(w[pidx(i, m - 1, k)], f.n);
        }
        const Face3& f = grid.jface[((size_t)k * (grid.nj + 1) + grid.nj) * grid.ni + (size_t)i];
        C5 gh = ghost_char(w[pidx(i, nj - 1, k)], f.n, 1.0);
        for (long m = 1; m <= NG; ++m) w[pidx(i, nj + m - 1, k)] = gh;
      }
    }
    for (long j = 0; j < nj; ++j)
      for (long i = 0; i < ni; ++i) {
        const Face3& fl = grid.kface[(size_t)j * grid.ni + (size_t)i];
        const Face3& fh = grid.kface[((size_t)nk * grid.nj + (size_t)j) * grid.ni + (size_t)i];
        for (long m = 1; m <= NG; ++m) {
          w[pidx(i, j, -m)] = reflect3(w[pidx(i, j, m - 1)], fl.n);
          w[pidx(i, j, nk + m - 1)] = reflect3(w[pidx(i, j, nk - m)], fh.n);
        }
      }
  }
  void fluxes(int dir, const std::vector<Face3>& faces, const std::vector<std::array<double, 2>>& rots, std::vector<C5>& out, int lim) {
    size_t ni = grid.ni, nj = grid.nj, nk = grid.nk;
    size_t nfi = ni + (dir == 0), nfj = nj + (dir == 1), nfk = nk + (dir == 2);
    size_t plane = nfi * nfj;
    long e[3] = {dir == 0, dir == 1, dir == 2};
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)nfk; ++k)
      for (size_t j = 0; j < nfj; ++j)
        for (size_t i = 0; i < nfi; ++i) {
          size_t fidx = (size_t)k * plane + j * nfi + i;
          const Face3& f = faces[fidx];
          if (f.area == 0.0) {
            out[fidx] = C5{};
            continue;
          }
          long p0[3] = {(long)i, (long)j, k};
          auto at = [&](long s) { return w[pidx(p0[0] + s * e[0], p0[1] + s * e[1], p0[2] + s * e[2])]; };
          auto sol = [&](long s) { return is_solid(p0[0] + s * e[0], p0[1] + s * e[1], p0[2] + s * e[2]); };
          C5 wm2 = at(-2), wm1 = at(-1), wp0 = at(0), wp1 = at(1);
          if (has_solid) {  // solver3.rs:362-405: solid cells as slip walls of their fluid neighbours
            const size_t fstride = dir == 0 ? 1 : dir == 1 ? nfi : plane;
            bool sm1 = sol(-1), sp0 = sol(0);
            if (sm1 && sp0) {
              out[fidx] = C5{};
              continue;
            }
            if (sm1) {
              wm1 = reflect3(wp0, f.n);
              wm2 = sol(1) ? wm1 : reflect3(wp1, f.n);
            } else if (sp0) {
              wp0 = reflect3(wm1, f.n);
              wp1 = sol(-2) ? wp0 : reflect3(wm2, f.n);
            } else {
              if (sol(-2)) wm2 = reflect3(wm1, faces[fidx - fstride].n);
              if (sol(1)) wp1 = reflect3(wp0, faces[fidx + fstride].n);
            }
          }
          out[fidx] = face_flux_lm3(wm2, wm1, wp0, wp1, lim, f.n, rots[fidx], low_mach);
        }
  }
  void eval_residual() {  // solver3.rs:222-270
    size_t ni = grid.ni, nj = grid.nj, nk = grid.nk;
    int lim = iter < first_order_iters ? orc::FIRST_ORDER : limiter;
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)nk; ++k)
      for (size_t j = 0; j < nj; ++j)
        for (size_t i = 0; i < ni; ++i) w[pidx((long)i, (long)j, k)] = cons_to_prim3(u[((size_t)k * nj + j) * ni + i]);
    fill_ghosts();
    fluxes(0, grid.iface, rot_i, fi, lim);
    fluxes(1, grid.jface, rot_j, fj, lim);
    fluxes(2, grid.kface, rot_k, fk, lim);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)nk; ++k)
      for (size_t j = 0; j < nj; ++j)
        for (size_t i = 0; i < ni; ++i) {
          size_t c = ((size_t)k * nj + j) * ni + i;
          if (solid[c]) {
            res[c] = C5{};
            continue;
          }
          size_t il = ((size_t)k * nj + j) * (ni + 1) + i, jl = ((size_t)k * (nj + 1) + j) * ni + i;
          size_t ir = il + 1, jr = jl + ni, kr = c + ni * nj;
          double inv_v = 1.0 / grid.vol[c];
          C5 out;
          for (int q = 0; q < 5; ++q)
            out[q] = -((fi[ir][q] * grid.iface[ir].area - fi[il][q] * grid.iface[il].area) +
                       (fj[jr][q] * grid.jface[jr].area - fj[jl][q] * grid.jface[jl].area) +
                       (fk[kr][q] * grid.kface[kr].area - fk[c][q] * grid.kface[c].area)) *
                     inv_v;
          res[c] = out;
        }
  }
  void compute_dt(double cfl_, int mode) {  // solver3.rs:274-300
    size_t ni = grid.ni, nj = grid.nj, nk = grid.nk;
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)nk; ++k)
      for (size_t j = 0; j < nj; ++j)
        for (size_t i = 0; i < ni; ++i) {
          size_t c = ((size_t)k * nj + j) * ni + i;
          if (solid[c]) {
            dt[c] = 0.0;
            continue;
          }
          const C5& wc = w[pidx((long)i, (long)j, k)];
          double cs = sound_speed3(wc);
          auto lam = [&](const Face3& f) { return (std::fabs(wc[1] * f.n[0] + wc[2] * f.n[1] + wc[3] * f.n[2]) + cs) * f.area; };
          size_t il = ((size_t)k * nj + j) * (ni + 1) + i, jl = ((size_t)k * (nj + 1) + j) * ni + i;
          double li = 0.5 * (lam(grid.iface[il]) + lam(grid.iface[il + 1]));
          double lj = 0.5 * (lam(grid.jface[jl]) + lam(grid.jface[jl + ni]));
          double lk = 0.5 * (lam(grid.kface[c]) + lam(grid.kface[c + ni * nj]));
          dt[c] = mode == orc::DT_SUM ? cfl_ * grid.vol[c] / (li + lj + lk) : cfl_ * grid.vol[c] / (3.0 * fmin_rs(fmin_rs(li, lj), lk));
        }
  }
  void stage(double a, double b) {  // solver3.rs:317-327 (fluid cells)
    for (size_t c = 0; c < u.size(); ++c)
      if (!solid[c])
        for (int k = 0; k < 5; ++k) u[c][k] = a * (u[c][k] + dt[c] * res[c][k]) + b * u0[c][k];
  }
  double rk3_step() {  // solver3.rs:303-314
    eval_residual();
    double rn = density_residual();
    compute_dt(cfl, orc::DT_SUM);
    u0 = u;
    stage(1.0, 0.0);
    eval_residual();
    stage(0.25, 0.75);
    eval_residual();
    stage(2.0 / 3.0, 1.0 / 3.0);
    return rn;
  }
  // implicit3.rs:274-355: blocks of direction dir, ghost Jacobians folded at the line ends; a solid cell is the identity
  // row, a fluid cell next to one along the line folds B T (T the reflection about the face) into its diagonal
  void assemble3(int dir, std::vector<M5>& LO, std::vector<M5>& D, std::vector<M5>& UP) {
    size_t ni = grid.ni, nj = grid.nj, nk = grid.nk, n = ni * nj * nk, plane = ni * nj;
    LO.assign(n, M5{}), D.assign(n, M5{}), UP.assign(n, M5{});
    long e[3] = {dir == 0, dir == 1, dir == 2};
    auto ghost_t = [&](bool lower, const Face3& f, size_t i) -> M5 {
      if (!ip.implicit_bc) return M5{};
      if (dir == 0 || (dir == 1 && !lower)) return M5{};
      if (dir == 1 && lower) return i < grid.axis_cells ? M5{} : reflection3(f.n);
      return reflection3(f.n);
    };
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)nk; ++k)
      for (size_t j = 0; j < nj; ++j)
        for (size_t i = 0; i < ni; ++i) {
          size_t c = ((size_t)k * nj + j) * ni + i;
          if (solid[c]) {
            D[c] = eye5();
            continue;
          }
          size_t m = dir == 0 ? i : dir == 1 ? j : (size_t)k;
          size_t nl = dir == 0 ? ni : dir == 1 ? nj : nk;
          const size_t stride = dir == 0 ? 1 : dir == 1 ? ni : plane;
          const C5& wk = w[pidx((long)i, (long)j, k)];
          const Face3 *fl, *fr;
          if (dir == 0) {
            size_t il = ((size_t)k * nj + j) * (ni + 1) + i;
            fl = &grid.iface[il], fr = &grid.iface[il + 1];
          } else if (dir == 1) {
            size_t jl = ((size_t)k * (nj + 1) + j) * ni + i;
            fl = &grid.jface[jl], fr = &grid.jface[jl + ni];
          } else {
            fl = &grid.kface[c], fr = &grid.kface[c + plane];
          }
          const bool lower_solid = m > 0 && solid[c - stride], upper_solid = m + 1 < nl && solid[c + stride];
          const C5 wm = lower_solid ? reflect3(wk, fl->n) : w[pidx((long)i - e[0], (long)j - e[1], k - e[2])];
          const C5 wp = upper_solid ? reflect3(wk, fr->n) : w[pidx((long)i + e[0], (long)j + e[1], k + e[2])];
          M5 l, dd, uu;
          cell_blocks3(wk, wm, wp, *fl, *fr, grid.vol[c], dt[c], ip, l, dd, uu);
          if (m == 0) {
            axpy5(dd, 1.0, mm5(l, ghost_t(true, *fl, i)));
            l = M5{};
          } else if (lower_solid) {
            axpy5(dd, 1.0, mm5(l, reflection3(fl->n)));
            l = M5{};
          }
          if (m == nl - 1) {
            axpy5(dd, 1.0, mm5(uu, ghost_t(false, *fr, i)));
            uu = M5{};
          } else if (upper_solid) {
            axpy5(dd, 1.0, mm5(uu, reflection3(fr->n)));
            uu = M5{};
          }
          LO[c] = l, D[c] = dd, UP[c] = uu;
        }
  }
  void solve_lines3(int dir, const std::vector<M5>& LO, const std::vector<M5>& D, const std::vector<M5>& UP, std::vector<C5>& x) {
    size_t ni = grid.ni, nj = grid.nj, nk = grid.nk;
    size_t nl = dir == 0 ? ni : dir == 1 ? nj : nk;
    size_t stride = dir == 0 ? 1 : dir == 1 ? ni : ni * nj;
    size_t nlines = dir == 0 ? nj * nk : dir == 1 ? ni * nk : ni * nj;
    auto base_of = [&](size_t l) { return dir == 0 ? l * ni : dir == 1 ? (l / ni) * ni * nj + l % ni : l; };
#pragma omp parallel for schedule(static)
    for (long l = 0; l < (long)nlines; ++l) {
      size_t base = base_of((size_t)l);
      std::vector<M5> lo(nl), d(nl), up(nl);
      std::vector<C5> rhs(nl);
      for (size_t m = 0; m < nl; ++m) {
        size_t c = base + m * stride;
        lo[m] = LO[c], d[m] = D[c], up[m] = UP[c], rhs[m] = x[c];
      }
      block_thomas5(nl, lo.data(), d.data(), up.data(), rhs.data());
      for (size_t m = 0; m < nl; ++m) x[base + m * stride] = rhs[m];
    }
  }
  std::vector<C5> apply_factor3(int dir, const std::vector<M5>& LO, const std::vector<M5>& D, const std::vector<M5>& UP,
                                const std::vector<C5>& x) {  // implicit3.rs:384-410
    size_t ni = grid.ni, nj = grid.nj, nk = grid.nk;
    size_t stride = dir == 0 ? 1 : dir == 1 ? ni : ni * nj;
    std::vector<C5> out(ni * nj * nk);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)nk; ++k)
      for (size_t j = 0; j < nj; ++j)
        for (size_t i = 0; i < ni; ++i) {
          size_t c = ((size_t)k * nj + j) * ni + i;
          size_t m = dir == 0 ? i : dir == 1 ? j : (size_t)k;
          size_t nl = dir == 0 ? ni : dir == 1 ? nj : nk;
          C5 v = mv5(D[c], x[c]);
          if (m > 0) {
            C5 a = mv5(LO[c], x[c - stride]);
            for (int q = 0; q < 5; ++q) v[q] += a[q];
          }
          if (m + 1 < nl) {
            C5 a = mv5(UP[c], x[c + stride]);
            for (int q = 0; q < 5; ++q) v[q] += a[q];
          }
          out[c] = v;
        }
    return out;
  }
  double implicit_step() {  // implicit3.rs:416-469
    double cflv = fmin_rs(ip.cfl0 * std::pow(ip.growth, (int)std::min<size_t>(ramp_k, 10000)), ip.cfl_max);
    ramp_k += 1;
    eval_residual();
    double rn = density_residual();
    compute_dt(cflv, ip.dt_mode);
    size_t n = u.size();
    std::vector<M5> LO[3], D[3], UP[3];
    for (int dir = 0; dir < 3; ++dir) assemble3(dir, LO[dir], D[dir], UP[dir]);
    std::vector<C5> b(n);
    for (size_t c = 0; c < n; ++c)
      for (int q = 0; q < 5; ++q) b[c][q] = res[c][q] * dt[c];
    auto af = [&](const std::vector<C5>& rhs) {
      std::vector<C5> x = rhs;
      for (int dir = 0; dir < 3; ++dir) solve_lines3(dir, LO[dir], D[dir], UP[dir], x);
      return x;
    };
    std::vector<C5> du = af(b);
    for (size_t s = 1; s < std::max<size_t>(ip.sub_iters, 1); ++s) {
      std::vector<C5> a[3];
      for (int dir = 0; dir < 3; ++dir) a[dir] = apply_factor3(dir, LO[dir], D[dir], UP[dir], du);
      std::vector<C5> r(n);
      for (size_t c = 0; c < n; ++c)
        for (int q = 0; q < 5; ++q) r[c][q] = b[c][q] - (a[0][c][q] + a[1][c][q] + a[2][c][q] - 2.0 * du[c][q]);
      std::vector<C5> corr = af(r);
      for (size_t c = 0; c < n; ++c)
        for (int q = 0; q < 5; ++q) du[c][q] += corr[c][q];
    }
    for (size_t c = 0; c < n; ++c) {
      if (solid[c]) continue;
      const C5& dq = du[c];
      double alpha = 1.0;
      for (int t = 0; t < 8; ++t) {
        C5 q;
        for (int m = 0; m < 5; ++m) q[m] = u[c][m] + alpha * dq[m];
        C5 wq = cons_to_prim3(q);
        bool fin = true;
        for (double v : q) fin = fin && std::isfinite(v);
        if (wq[0] > 0.0 && wq[4] > 0.0 && fin) {
          u[c] = q;
          break;
        }
        alpha *= 0.5;
      }
    }
    return rn;
  }
  double step() {  // solver3.rs:158-165
    double rn = implicit ? implicit_step() : rk3_step();
    iter += 1;
    return rn;
  }
};

// ---------------------------------------------------------------- run3.rs (forces)
struct Forces3 {
  double cn = 0, ca = 0, x_cp = NAN;
};
// run3.rs:130-212 `accumulate` summed over its parts: the j = 0 faces with i >= axis_cells over fluid cells, and every face
// between a fluid and a solid cell (the fin sides, edges and tips); faces with centroid x <= x_max. The wall pressure is
// extrapolated from the first fluid cell a and the fluid cell b behind it, pw = p_a + (p_a - p_b) d_a / (d_b - d_a), or p_a
// where there is none; dF = (pw - p_inf) area n_into_body; coefficients of the half domain doubled, S_ref = pi/4.
Forces3 forces_on(const Solver3& s, double mach, double x_max) {
  const Grid3& g = s.grid;
  size_t ni = g.ni, nj = g.nj, nk = g.nk;
  double p_inf = s.fs[4];
  auto p = [&](size_t c) { return cons_to_prim3(s.u[c])[4]; };
  auto dist = [&](size_t c, const Face3& f) {
    const auto& x = g.xc[c];
    return std::sqrt(std::pow(x[0] - f.c[0], 2) + std::pow(x[1] - f.c[1], 2) + std::pow(x[2] - f.c[2], 2));
  };
  auto sol = [&](size_t i, size_t j, size_t k) { return s.solid[g.cell(i, j, k)] != 0; };
  double fx = 0, fz = 0, mz = 0;
  auto add = [&](size_t a, long b, const Face3& f, double sign) {
    if (f.c[0] > x_max) return;
    double p0 = p(a), pw = p0;
    if (b >= 0) {
      double d0 = dist(a, f), d1 = dist((size_t)b, f);
      pw = p0 + (p0 - p((size_t)b)) * d0 / (d1 - d0);
    }
    double d = (pw - p_inf) * f.area * sign;
    fx += d * f.n[0];
    fz += d * f.n[2];
    mz += d * f.n[2] * f.c[0];
  };
  for (size_t k = 0; k < nk; ++k)
    for (size_t i = g.axis_cells; i < ni; ++i)
      if (!sol(i, 0, k)) add(g.cell(i, 0, k), nj > 1 && !sol(i, 1, k) ? (long)g.cell(i, 1, k) : -1, g.jface[k * (nj + 1) * ni + i], -1.0);
  if (s.has_solid) {
    for (size_t k = 0; k < nk; ++k)
      for (size_t j = 0; j < nj; ++j)
        for (size_t i = 1; i < ni; ++i) {
          const Face3& f = g.iface[(k * nj + j) * (ni + 1) + i];
          bool a = sol(i - 1, j, k), b = sol(i, j, k);
          if (!a && b) add(g.cell(i - 1, j, k), i >= 2 && !sol(i - 2, j, k) ? (long)g.cell(i - 2, j, k) : -1, f, 1.0);
          if (a && !b) add(g.cell(i, j, k), i + 1 < ni && !sol(i + 1, j, k) ? (long)g.cell(i + 1, j, k) : -1, f, -1.0);
        }
    for (size_t k = 0; k < nk; ++k)
      for (size_t j = 1; j < nj; ++j)
        for (size_t i = 0; i < ni; ++i) {
          const Face3& f = g.jface[(k * (nj + 1) + j) * ni + i];
          bool a = sol(i, j - 1, k), b = sol(i, j, k);
          if (!a && b) add(g.cell(i, j - 1, k), j >= 2 && !sol(i, j - 2, k) ? (long)g.cell(i, j - 2, k) : -1, f, 1.0);
          if (a && !b) add(g.cell(i, j, k), j + 1 < nj && !sol(i, j + 1, k) ? (long)g.cell(i, j + 1, k) : -1, f, -1.0);
        }
    for (size_t k = 1; k < nk; ++k)
      for (size_t j = 0; j < nj; ++j)
        for (size_t i = 0; i < ni; ++i) {
          const Face3& f = g.kface[(k * nj + j) * ni + i];
          bool a = sol(i, j, k - 1), b = sol(i, j, k);
          if (!a && b) add(g.cell(i, j, k - 1), k >= 2 && !sol(i, j, k - 2) ? (long)g.cell(i, j, k - 2) : -1, f, 1.0);
          if (a && !b) add(g.cell(i, j, k), k + 1 < nk && !sol(i, j, k + 1) ? (long)g.cell(i, j, k + 1) : -1, f, -1.0);
        }
  }
  double q = 0.5 * mach * mach, s_ref = M_PI / 4.0;
  double norm = 2.0 / (q * s_ref);
  Forces3 r;
  r.cn = norm * fz;
  r.ca = norm * fx;
  r.x_cp = std::fabs(fz) < 1e-12 ? NAN : mz / fz;
  return r;
}

// run3.rs:85-127 `breakdown_on` (the parts of `accumulate`, run3.rs:130-212): nose (body wall with centroid x <= x_nose),
// afterbody, fin sides (k faces), fin edges (i faces), fin tips (j faces); (cn, ca, x_cp) per part
std::array<Forces3, 5> forces_parts(const Solver3& s, double mach, double x_max, double x_nose) {
  const Grid3& g = s.grid;
  size_t ni = g.ni, nj = g.nj, nk = g.nk;
  double p_inf = s.fs[4];
  auto p = [&](size_t c) { return cons_to_prim3(s.u[c])[4]; };
  auto dist = [&](size_t c, const Face3& f) {
    const auto& x = g.xc[c];
    return std::sqrt(std::pow(x[0] - f.c[0], 2) + std::pow(x[1] - f.c[1], 2) + std::pow(x[2] - f.c[2], 2));
  };
  auto sol = [&](size_t i, size_t j, size_t k) { return s.solid[g.cell(i, j, k)] != 0; };
  double acc[5][3] = {};
  auto add = [&](int part, size_t a, long b, const Face3& f, double sign) {
    if (f.c[0] > x_max) return;
    if (part == 0 && f.c[0] > x_nose) part = 1;
    double p0 = p(a), pw = p0;
    if (b >= 0) {
      double d0 = dist(a, f), d1 = dist((size_t)b, f);
      pw = p0 + (p0 - p((size_t)b)) * d0 / (d1 - d0);
    }
    double d = (pw - p_inf) * f.area * sign;
    acc[part][0] += d * f.n[0];
    acc[part][1] += d * f.n[2];
    acc[part][2] += d * f.n[2] * f.c[0];
  };
  for (size_t k = 0; k < nk; ++k)
    for (size_t i = g.axis_cells; i < ni; ++i)
      if (!sol(i, 0, k)) add(0, g.cell(i, 0, k), nj > 1 && !sol(i, 1, k) ? (long)g.cell(i, 1, k) : -1, g.jface[k * (nj + 1) * ni + i], -1.0);
  if (s.has_solid) {
    for (size_t k = 0; k < nk; ++k)
      for (size_t j = 0; j < nj; ++j)
        for (size_t i = 1; i < ni; ++i) {
          const Face3& f = g.iface[(k * nj + j) * (ni + 1) + i];
          bool a = sol(i - 1, j, k), b = sol(i, j, k);
          if (!a && b) add(3, g.cell(i - 1, j, k), i >= 2 && !sol(i - 2, j, k) ? (long)g.cell(i - 2, j, k) : -1, f, 1.0);
          if (a && !b) add(3, g.cell(i, j, k), i + 1 < ni && !sol(i + 1, j, k) ? (long)g.cell(i + 1, j, k) : -1, f, -1.0);
        }
    for (size_t k = 0; k < nk; ++k)
      for (size_t j = 1; j < nj; ++j)
        for (size_t i = 0; i < ni; ++i) {
          const Face3& f = g.jface[(k * (nj + 1) + j) * ni + i];
          bool a = sol(i, j - 1, k), b = sol(i, j, k);
          if (!a && b) add(4, g.cell(i, j - 1, k), j >= 2 && !sol(i, j - 2, k) ? (long)g.cell(i, j - 2, k) : -1, f, 1.0);
          if (a && !b) add(4, g.cell(i, j, k), j + 1 < nj && !sol(i, j + 1, k) ? (long)g.cell(i, j + 1, k) : -1, f, -1.0);
        }
    for (size_t k = 1; k < nk; ++k)
      for (size_t j = 0; j < nj; ++j)
        for (size_t i = 0; i < ni; ++i) {
          const Face3& f = g.kface[(k * nj + j) * ni + i];
          bool a = sol(i, j, k - 1), b = sol(i, j, k);
          if (!a && b) add(2, g.cell(i, j, k - 1), k >= 2 && !sol(i, j, k - 2) ? (long)g.cell(i, j, k - 2) : -1, f, 1.0);
          if (a && !b) add(2, g.cell(i, j, k), k + 1 < nk && !sol(i, j, k + 1) ? (long)g.cell(i, j, k + 1) : -1, f, -1.0);
        }
  }
  double q = 0.5 * mach * mach, s_ref = M_PI / 4.0;
  double norm = 2.0 / (q * s_ref);
  std::array<Forces3, 5> out;
  for (int k = 0; k < 5; ++k) {
    out[k].cn = norm * acc[k][1];
    out[k].ca = norm * acc[k][0];
    out[k].x_cp = std::fabs(acc[k][1]) < 1e-12 ? NAN : acc[k][2] / acc[k][1];
  }
  return out;
}

}  // namespace orc3

// ---------------------------------------------------------------- C API
using namespace orc3;
extern "C" {

struct Orc3Result {
  double cn, ca, x_cp;
  uint64_t iterations;
  int32_t stop_reason;  // 0 max iterations, 1 residual drop, 2 CN stationary, 5 non-finite
  double drop_orders;
};

// Solver on the 2D grid (x2, r2: (ni+1)(nj+1) nodes, r >= 0) revolved over theta (nk+1 angles in [0, pi]).
void* orc3_new(uint64_t ni, uint64_t nj, const double* x2, const double* r2, uint64_t nk, const double* theta, uint64_t axis_cells,
               double mach, double alpha, int limiter, uint64_t first_order_iters, int low_mach, int implicit, const orc::ImplicitParams* ip,
               double cfl, char* err, uint64_t err_len) {
  auto* s = new Solver3();
  std::string e;
  if (!revolve(ni, nj, x2, r2, nk, theta, s->grid, &e)) {
    if (err && err_len) std::snprintf(err, err_len, "%s", e.c_str());
    delete s;
    return nullptr;
  }
  s->grid.axis_cells = axis_cells;
  s->fs = freestream3(mach, alpha);
  s->limiter = limiter;
  s->first_order_iters = first_order_iters;
  s->low_mach = low_mach != 0;
  s->implicit = implicit != 0;
  if (ip) s->ip = *ip;
  s->cfl = cfl;
  s->init();
  return s;
}
void orc3_free(void* h) { delete static_cast<Solver3*>(h); }
// solid boxes (6 per box: i0, i1, j0, j1, k0, k1, half-open), before the first step
void orc3_set_solid(void* h, uint64_t nbox, const uint64_t* boxes) { static_cast<Solver3*>(h)->set_solid(nbox, boxes); }
// the i / j / k face fluxes of the last residual evaluation (5 per face, flux per unit area)
uint64_t orc3_face_fluxes(void* h, int dir, double* out) {
  auto* s = static_cast<Solver3*>(h);
  const std::vector<C5>& f = dir == 0 ? s->fi : dir == 1 ? s->fj : s->fk;
  if (out) std::memcpy(out, f.data(), f.size() * 40);
  return 5 * f.size();
}
void orc3_dims(void* h, uint64_t* ni, uint64_t* nj, uint64_t* nk) {
  auto* s = static_cast<Solver3*>(h);
  *ni = s->grid.ni, *nj = s->grid.nj, *nk = s->grid.nk;
}
// fields: 0 u (5/cell), 1 res (5/cell), 2 dt, 3 vol, 4 xc (3/cell), 5 i faces (n[3], area, c[3] = 7/face), 6 j faces, 7 k faces
uint64_t orc3_get(void* h, int field, double* out) {
  auto* s = static_cast<Solver3*>(h);
  const Grid3& g = s->grid;
  auto faces = [&](const std::vector<Face3>& f) {
    if (out)
      for (size_t q = 0; q < f.size(); ++q) {
        std::memcpy(out + 7 * q, f[q].n, 24);
        out[7 * q + 3] = f[q].area;
        std::memcpy(out + 7 * q + 4, f[q].c, 24);
      }
    return 7 * f.size();
  };
  switch (field) {
    case 0:
      if (out) std::memcpy(out, s->u.data(), s->u.size() * 40);
      return 5 * s->u.size();
    case 1:
      if (out) std::memcpy(out, s->res.data(), s->res.size() * 40);
      return 5 * s->res.size();
    case 2:
      if (out) std::memcpy(out, s->dt.data(), s->dt.size() * 8);
      return s->dt.size();
    case 3:
      if (out) std::memcpy(out, g.vol.data(), g.vol.size() * 8);
      return g.vol.size();
    case 4:
      if (out) std::memcpy(out, g.xc.data(), g.xc.size() * 24);
      return 3 * g.xc.size();
    case 5:
      return faces(g.iface);
    case 6:
      return faces(g.jface);
    case 7:
      return faces(g.kface);
  }
  return 0;
}
void orc3_set_state(void* h, const double* u) {
  auto* s = static_cast<Solver3*>(h);
  std::memcpy(s->u.data(), u, s->u.size() * 40);
}
void orc3_set_iter(void* h, uint64_t it, uint64_t ramp) {
  auto* s = static_cast<Solver3*>(h);
  s->iter = it, s->ramp_k = ramp;
}
// one residual evaluation (and the local time step at `cfl`, sum mode) of the current state; returns the density residual
double orc3_eval_residual(void* h, double cfl) {
  auto* s = static_cast<Solver3*>(h);
  s->eval_residual();
  s->compute_dt(cfl, orc::DT_SUM);
  return s->density_residual();
}
void orc3_steps(void* h, uint64_t n, double* residual) {
  auto* s = static_cast<Solver3*>(h);
  for (uint64_t k = 0; k < n; ++k) {
    double r = s->step();
    if (residual) residual[k] = r;
  }
}
void orc3_forces_parts(void* h, double mach, double x_max, double x_nose, double* out15) {
  std::array<Forces3, 5> f = forces_parts(*static_cast<Solver3*>(h), mach, x_max, x_nose);
  for (int k = 0; k < 5; ++k) out15[3 * k] = f[k].cn, out15[3 * k + 1] = f[k].ca, out15[3 * k + 2] = f[k].x_cp;
}
void orc3_forces(void* h, double mach, double x_max, double* out3) {
  Forces3 f = forces_on(*static_cast<Solver3*>(h), mach, x_max);
  out3[0] = f.cn, out3[1] = f.ca, out3[2] = f.x_cp;
}
// run3.rs:220-330: iterate to the stop rules (drop 6 orders below the peak after iteration 20; CN stationary within rel_tol over
// `window` iterations once it + 1 >= max(window, 1000); a frozen state without a residual drop counts as non-finite)
void orc3_run(void* h, double mach, double x_max, uint64_t max_iter, double rel_tol, uint64_t window, Orc3Result* out) {
  auto* s = static_cast<Solver3*>(h);
  s->ramp_k = 0;
  const size_t SAMPLE = 50, MIN_IT = 1000, skip = 20;
  size_t nwin = std::max<size_t>(window / SAMPLE, 1);
  double rmax = 0.0, rl = NAN;
  std::vector<double> hist;
  int reason = 0;
  size_t it = 0;
  while (it < max_iter) {
    double r = s->step();
    bool sample = (it + 1) % SAMPLE == 0;
    double cn = sample ? forces_on(*s, mach, x_max).cn : NAN;
    it += 1;
    size_t i0 = it - 1;
    rl = r;
    if (!std::isfinite(r)) {
      reason = 5;
      break;
    }
    if (i0 >= skip) rmax = fmax_rs(rmax, r);
    double drop = rmax > 0.0 ? std::log10(rmax / fmax_rs(r, 1e-300)) : 0.0;
    if (drop >= 6.0) {
      reason = 1;
      break;
    }
    if (sample) {
      if (!std::isfinite(cn) || std::fabs(cn) > orc::MONITOR_LIMIT) {
        reason = 5;
        break;
      }
      hist.push_back(cn);
      if (i0 + 1 >= std::max(window, MIN_IT) && hist.size() >= nwin) {
        const double* wv = hist.data() + hist.size() - nwin;
        bool frozen = true;
        for (size_t q = 0; q < nwin; ++q) frozen = frozen && std::memcmp(&wv[q], &wv[0], 8) == 0;
        if (drop < 1.0 && frozen) {
          reason = 5;
          break;
        }
        double lo = INFINITY, hi = -INFINITY, sum = 0.0;
        for (size_t q = 0; q < nwin; ++q) lo = fmin_rs(lo, wv[q]), hi = fmax_rs(hi, wv[q]), sum += wv[q];
        if (hi - lo < rel_tol * std::fabs(sum / (double)nwin)) {
          reason = 2;
          break;
        }
      }
    }
  }
  Forces3 f = forces_on(*s, mach, x_max);
  out->cn = f.cn, out->ca = f.ca, out->x_cp = f.x_cp;
  out->iterations = it;
  out->stop_reason = reason;
  out->drop_orders = rmax > 0.0 && rl > 0.0 ? std::log10(rmax / rl) : 0.0;
}
// kernels for the ported unit tests
void orc3_face_flux(const double* m2, const double* m1, const double* p0, const double* p1, int lim, const double* n, const double* rot,
                    int low_mach, double* out) {
  C5 a, b, c, d;
  std::memcpy(a.data(), m2, 40), std::memcpy(b.data(), m1, 40), std::memcpy(c.data(), p0, 40), std::memcpy(d.data(), p1, 40);
  std::array<double, 2> r = {rot[0], rot[1]};
  C5 f = face_flux_lm3(a, b, c, d, lim, n, r, low_mach != 0);
  std::memcpy(out, f.data(), 40);
}
void orc3_hllc(const double* wl, const double* wr, const double* n, double* out) {
  C5 a, b;
  std::memcpy(a.data(), wl, 40), std::memcpy(b.data(), wr, 40);
  C5 f = hllc3(a, b, n);
  std::memcpy(out, f.data(), 40);
}
void orc3_physical_flux(const double* w, const double* n, double* out) {
  C5 a;
  std::memcpy(a.data(), w, 40);
  C5 f = physical_flux3(a, n);
  std::memcpy(out, f.data(), 40);
}
void orc3_char_ghost(const double* fs, const double* in, const double* n, double* out) {
  C5 a, b;
  std::memcpy(a.data(), fs, 40), std::memcpy(b.data(), in, 40);
  C5 g = characteristic_ghost3(a, b, n);
  std::memcpy(out, g.data(), 40);
}
void orc3_flux_jacobian(const double* w, const double* n, double* out) {
  C5 a;
  std::memcpy(a.data(), w, 40);
  M5 m = flux_jacobian3(a, n);
  std::memcpy(out, m.data(), 200);
}
void orc3_abs_jacobian(const double* wl, const double* wr, const double* n, double eps_fix, double* out) {
  C5 a, b;
  std::memcpy(a.data(), wl, 40), std::memcpy(b.data(), wr, 40);
  M5 m = abs_jacobian3(a, b, n, eps_fix);
  std::memcpy(out, m.data(), 200);
}
void orc3_inv5(const double* m, double* out) {
  M5 a;
  std::memcpy(a.data(), m, 200);
  M5 r = inv5(a);
  std::memcpy(out, r.data(), 200);
}
void orc3_block_thomas5(uint64_t n, const double* lo, const double* d, const double* up, double* rhs) {
  block_thomas5(n, reinterpret_cast<const M5*>(lo), reinterpret_cast<const M5*>(d), reinterpret_cast<const M5*>(up), reinterpret_cast<C5*>(rhs));
}
void orc3_reflection(const double* n, double* out) {
  M5 m = reflection3(n);
  std::memcpy(out, m.data(), 200);
}
}
