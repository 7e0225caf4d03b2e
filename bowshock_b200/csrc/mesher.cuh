// Host mesher of the case layer: the reference's body-fitted H-grids about a nose + aft-segment body
// (crates/bowshock-core/src/engine/body_grid.rs:134-452, with grid.rs:199-228 and the ogive of
// crates/bowshock-reference/src/shock_expansion.rs:42-82), in FP64. It lets a sweep of many seeded bodies be meshed by
// this library instead of by the caller.
#pragma once
#include <cmath>
#include <string>
#include <vector>

namespace bk {
namespace mesh {

enum { NOSE_TANGENT_OGIVE = 0, NOSE_CONE = 1, NOSE_POWER = 2, NOSE_PARABOLIC = 3, NOSE_HAACK = 4 };

struct Body {
  int nose = NOSE_TANGENT_OGIVE;
  double fineness = 3, half_angle = 0, param = 0;
  std::vector<double> seg_len, seg_slope;
  double sting_radius = 0;

  double nose_length() const { return nose == NOSE_CONE ? 0.5 / std::tan(half_angle) : fineness; }  // body_grid.rs:62-67
  double nose_r(double x) const {                                                                     // body_grid.rs:69-88
    if (x <= 0.0) return 0.0;
    double ln = nose_length(), R = 0.5;
    if (x >= ln) return R;
    double eta = x / ln;
    switch (nose) {
      case NOSE_TANGENT_OGIVE: {
        double l = fineness, rho = (l * l + R * R) / (2.0 * R), xx = std::fmax(x, 0.0);
        return std::sqrt(std::fmax(rho * rho - (l - xx) * (l - xx), 0.0)) - (rho - R);
      }
      case NOSE_CONE:
        return x * std::tan(half_angle);
      case NOSE_POWER:
        return R * std::pow(eta, param);
      case NOSE_PARABOLIC:
        return R * (2.0 * eta - param * eta * eta) / (2.0 - param);
      default: {
        double t = 1.0 - 2.0 * eta;
        t = t < -1.0 ? -1.0 : (t > 1.0 ? 1.0 : t);
        double th = std::acos(t), s = std::sin(th);
        return R * std::sqrt(std::fmax((th - 0.5 * std::sin(2.0 * th) + param * s * s * s) / M_PI, 0.0));
      }
    }
  }
  std::pair<double, double> station(size_t k) const {  // body_grid.rs:269-276
    double x = nose_length(), r = 0.5;
    for (size_t t = 0; t < k; ++t) {
      x += seg_len[t];
      r += seg_len[t] * seg_slope[t];
    }
    return {x, r};
  }
  double aft_length() const {
    double a = 0;
    for (double l : seg_len) a = a + l;
    return a;
  }
  double x_base() const { return station(seg_len.size()).first; }
  double base_radius() const { return station(seg_len.size()).second; }
  double r(double x) const {  // body_grid.rs:303-311
    if (x <= nose_length()) return nose_r(x);
    double x0 = nose_length(), r0 = 0.5;
    for (size_t k = 0; k < seg_len.size(); ++k) {
      double x1 = x0 + seg_len[k];
      if (x < x1) return r0 + (x - x0) * seg_slope[k];
      x0 = x1;
      r0 += seg_len[k] * seg_slope[k];
    }
    return base_radius();
  }
};

inline std::vector<double> geometric_offsets(double first, double length, size_t n) {  // grid.rs:199-228
  auto sum = [&](double q) {
    double s = 0, d = first;
    for (size_t k = 0; k < n; ++k) s += d, d *= q;
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
  double s = 0, d = first;
  for (size_t k = 0; k < n; ++k) v.push_back(s), s += d, d *= q;
  v.push_back(length);
  return v;
}

inline std::vector<double> two_sided_nodes(double len, size_t n, double dx) {  // body_grid.rs:134-157
  auto node = [&](double delta, size_t k) {
    double t = (double)k / (double)n;
    if (delta < 1e-9) return len * t;
    return 0.5 * len * (1.0 + std::tanh(delta * (t - 0.5)) / std::tanh(0.5 * delta));
  };
  std::vector<double> out(n + 1);
  double delta = 0.0;
  if (!(dx >= len / (double)n)) {
    double lo = 0.0, hi = 40.0;
    for (int it = 0; it < 200; ++it) {
      double mid = 0.5 * (lo + hi);
      if (node(mid, 1) > dx)
        lo = mid;
      else
        hi = mid;
    }
    delta = 0.5 * (lo + hi);
  }
  for (size_t k = 0; k <= n; ++k) out[k] = node(delta, k);
  return out;
}

struct BaseGrid {  // body_grid.rs:330-355 (power-off)
  double x_up, x_down, r_far;
  size_t n_up, n_nose;
  std::vector<size_t> n_seg;
  size_t n_wake, n_sting, n_gap, nj_out;
  double dx_tip, dr_wall;
  bool gap_one_sided;
};
struct StingGrid {  // body_grid.rs:112-131
  double x_up, x_down, r_far;
  size_t n_up, n_nose;
  std::vector<size_t> n_seg;
  size_t n_ext, nj;
  double dx_tip, dr_wall;
};

// The argument checks of base_domain_grid (body_grid.rs:360-375), shared with the device mesher
inline bool base_grid_check(const Body& bb, const BaseGrid& p, std::string& err) {
  double ln = bb.nose_length();
  if (!(p.n_up >= 1 && p.n_nose >= 2 && p.n_wake >= 2 && p.n_gap >= 2 && p.nj_out >= 1)) return err = "cell counts", false;
  if (bb.seg_len.empty() || p.n_seg.size() != bb.seg_len.size()) return err = "n_seg needs one entry per body segment", false;
  for (size_t k = 0; k < bb.seg_len.size(); ++k)
    if (!(bb.seg_len[k] > 0.0) || p.n_seg[k] < 1) return err = "segments need a positive length and >= 1 cell", false;
  if (!(p.n_sting == 0 || p.n_sting >= 2)) return err = "n_sting must be 0 or >= 2", false;
  if (bb.sting_radius >= bb.base_radius()) return err = "sting thicker than the base", false;
  if (!(ln > 0.0 && p.x_up > 0.0 && p.x_down > 0.0 && p.dx_tip > 0.0 && p.dr_wall > 0.0 && p.r_far > bb.base_radius()))
    return err = "x_up, x_down, dx_tip, dr_wall must be positive, r_far must exceed the base radius", false;
  return true;
}

// body_grid.rs:360-452
inline bool base_domain_grid(const Body& bb, const BaseGrid& p, size_t& ni, size_t& nj, std::vector<double>& x, std::vector<double>& r,
                             size_t blk[3], std::string& err) {
  double ln = bb.nose_length();
  if (!base_grid_check(bb, p, err)) return false;
  std::vector<double> nose = two_sided_nodes(ln, p.n_nose, p.dx_tip);
  std::vector<double> xs, up = geometric_offsets(nose[1] - nose[0], p.x_up, p.n_up);
  for (size_t k = p.n_up; k >= 1; --k) xs.push_back(-up[k]);
  for (double v : nose) xs.push_back(v);
  for (size_t k = 0; k < bb.seg_len.size(); ++k) {
    std::vector<double> sn = two_sided_nodes(bb.seg_len[k], p.n_seg[k], p.dx_tip);
    double x0 = bb.station(k).first;
    for (size_t i = 1; i <= p.n_seg[k]; ++i) xs.push_back(x0 + sn[i]);
  }
  size_t i_end = xs.size() - 1;
  std::vector<double> wake = geometric_offsets(xs[i_end] - xs[i_end - 1], p.x_down, p.n_wake);
  double x_base = bb.x_base();
  for (size_t k = 1; k <= p.n_wake; ++k) xs.push_back(x_base + wake[k]);
  ni = xs.size() - 1;
  size_t j_sting = p.n_sting, j_end = p.n_sting + p.n_gap;
  nj = j_end + p.nj_out;
  double re = bb.base_radius(), rs = bb.sting_radius;
  std::vector<double> gap(p.n_gap + 1);
  if (p.gap_one_sided) {
    std::vector<double> off = geometric_offsets(p.dr_wall, re - rs, p.n_gap);
    for (size_t k = 0; k <= p.n_gap; ++k) gap[k] = (re - rs) - off[p.n_gap - k];
  } else {
    gap = two_sided_nodes(re - rs, p.n_gap, p.dr_wall);
  }
  std::vector<double> sj = geometric_offsets(p.dr_wall / (p.r_far - re), 1.0, p.nj_out);
  x.assign((ni + 1) * (nj + 1), 0.0);
  r.assign((ni + 1) * (nj + 1), 0.0);
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
  blk[0] = i_end;
  blk[1] = j_end;
  blk[2] = j_sting;
  return true;
}

// The argument checks of large_domain_grid (body_grid.rs:160-175), shared with the device mesher
inline bool large_grid_check(const Body& bb, const StingGrid& p, std::string& err) {
  size_t nseg = bb.seg_len.size();
  double ln = bb.nose_length();
  if (!(p.x_up > 0.0 && p.x_down > bb.aft_length() && nseg >= 1 && ln > 0.0 && p.dx_tip > 0.0))
    return err = "x_up and dx_tip must be positive and x_down must exceed the aft length", false;
  if (p.n_seg.size() != nseg) return err = "n_seg needs one entry per body segment", false;
  for (size_t k = 0; k < nseg; ++k)
    if (!(bb.seg_len[k] > 0.0) || p.n_seg[k] < 1) return err = "segments need a positive length and >= 1 cell", false;
  if (!(p.n_up >= 1 && p.n_nose >= 2 && p.n_ext >= 1 && p.nj >= 1 && p.dr_wall > 0.0 && p.r_far > 0.0)) return err = "cell counts", false;
  return true;
}

// body_grid.rs:160-231
inline bool large_domain_grid(const Body& bb, const StingGrid& p, size_t& ni, size_t& nj, std::vector<double>& x, std::vector<double>& r,
                              std::string& err) {
  size_t nseg = bb.seg_len.size();
  double ln = bb.nose_length();
  if (!large_grid_check(bb, p, err)) return false;
  std::vector<double> nose = two_sided_nodes(ln, p.n_nose, p.dx_tip);
  double d_tip = nose[1] - nose[0], d_sh = nose[p.n_nose] - nose[p.n_nose - 1];
  std::vector<double> xs, up = geometric_offsets(d_tip, p.x_up, p.n_up);
  for (size_t k = p.n_up; k >= 1; --k) xs.push_back(-up[k]);
  for (double v : nose) xs.push_back(v);
  double d_prev = d_sh;
  for (size_t k = 0; k < nseg; ++k) {
    size_t n = p.n_seg[k];
    double x0 = bb.station(k).first;
    bool geometric_fits = d_prev * (1.0 - std::pow(0.2, (int)n)) / 0.8 < bb.seg_len[k];
    std::vector<double> offs = (k == nseg - 1 && bb.seg_slope[k] == 0.0 && geometric_fits) ? geometric_offsets(d_prev, bb.seg_len[k], n)
                                                                                          : two_sided_nodes(bb.seg_len[k], n, p.dx_tip);
    for (size_t i = 1; i <= n; ++i) xs.push_back(x0 + offs[i]);
    d_prev = offs[n] - offs[n - 1];
  }
  std::vector<double> ext = geometric_offsets(d_prev, p.x_down - bb.aft_length(), p.n_ext);
  for (size_t k = 1; k <= p.n_ext; ++k) xs.push_back(bb.x_base() + ext[k]);
  ni = xs.size() - 1;
  nj = p.nj;
  std::vector<double> sj = geometric_offsets(p.dr_wall / p.r_far, 1.0, nj);
  x.assign((ni + 1) * (nj + 1), 0.0);
  r.assign((ni + 1) * (nj + 1), 0.0);
  for (size_t i = 0; i <= ni; ++i) {
    double r_in = bb.r(xs[i]);
    for (size_t j = 0; j <= nj; ++j) {
      x[j * (ni + 1) + i] = xs[i];
      r[j * (ni + 1) + i] = r_in + sj[j] * (p.r_far - r_in);
    }
  }
  return true;
}

}  // namespace mesh
}  // namespace bk
