// Device arithmetic of the finite-volume path, templated on the real type (float for the iteration, double for the
// boundary ghosts, the ghost Jacobians and the final-stage residual). Each function names the reference function it
// computes; the expression order follows the reference so the FP32 results track the FP64 oracle to rounding.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define BK_HD __host__ __device__ __forceinline__

namespace bk {

constexpr double GAMMA_D = 1.4;

template <typename T>
struct V4 {
  T v[4];
  BK_HD T& operator[](int k) { return v[k]; }
  BK_HD const T& operator[](int k) const { return v[k]; }
};
template <typename T>
struct M4 {
  T a[16];
  BK_HD T& operator[](int k) { return a[k]; }
  BK_HD const T& operator[](int k) const { return a[k]; }
};

template <typename T>
BK_HD V4<T> mk4(T a, T b, T c, T d) {
  V4<T> r;
  r.v[0] = a;
  r.v[1] = b;
  r.v[2] = c;
  r.v[3] = d;
  return r;
}
BK_HD V4<float> from_f4(float4 f) { return mk4(f.x, f.y, f.z, f.w); }
BK_HD float4 to_f4(const V4<float>& v) { return make_float4(v.v[0], v.v[1], v.v[2], v.v[3]); }
BK_HD V4<double> f4d(float4 f) { return mk4<double>(f.x, f.y, f.z, f.w); }
template <typename T>
BK_HD float4 to_f4c(const V4<T>& v) {
  return make_float4((float)v.v[0], (float)v.v[1], (float)v.v[2], (float)v.v[3]);
}
template <typename T>
BK_HD V4<T> cvt4(const V4<float>& v) {
  return mk4<T>((T)v.v[0], (T)v.v[1], (T)v.v[2], (T)v.v[3]);
}

template <typename T>
BK_HD T gam() {
  return (T)1.4;
}
template <typename T>
BK_HD T g1() {
  return (T)0.4;  // GAMMA - 1
}

// ------------------------------------------------------------------ gas.rs
template <typename T>
BK_HD V4<T> prim_to_cons(const V4<T>& w) {  // gas.rs:12-16
  T rho = w[0], u = w[1], v = w[2], p = w[3];
  return mk4<T>(rho, rho * u, rho * v, p / g1<T>() + (T)0.5 * rho * (u * u + v * v));
}
template <typename T>
BK_HD V4<T> cons_to_prim(const V4<T>& q) {  // gas.rs:18-24
  T rho = q[0];
  T u = q[1] / rho;
  T v = q[2] / rho;
  T p = g1<T>() * (q[3] - (T)0.5 * rho * (u * u + v * v));
  return mk4<T>(rho, u, v, p);
}
template <typename T>
BK_HD T sound_speed(const V4<T>& w) {  // gas.rs:27-29
  return sqrt(gam<T>() * w[3] / w[0]);
}
template <typename T>
BK_HD V4<T> physical_flux(const V4<T>& w, T nx, T nr) {  // gas.rs:33-38
  T rho = w[0], u = w[1], v = w[2], p = w[3];
  T un = u * nx + v * nr;
  T e = p / g1<T>() + (T)0.5 * rho * (u * u + v * v);
  return mk4<T>(rho * un, rho * u * un + p * nx, rho * v * un + p * nr, (e + p) * un);
}
template <typename T>
BK_HD V4<T> reflect(const V4<T>& w, T nx, T nr) {  // gas.rs:47-50
  T un = w[1] * nx + w[2] * nr;
  return mk4<T>(w[0], w[1] - (T)2 * un * nx, w[2] - (T)2 * un * nr, w[3]);
}
template <typename T>
BK_HD V4<T> wall_ghost(const V4<T>& w, T nx, T nr, bool noslip) {  // viscous.rs:67-73
  if (noslip) return mk4<T>(w[0], -w[1], -w[2], w[3]);
  return reflect(w, nx, nr);
}
template <typename T>
BK_HD T temperature(const V4<T>& w) {  // viscous.rs:61-63
  return gam<T>() * w[3] / w[0];
}

// ------------------------------------------------------------------ flux.rs
enum { LIM_FIRST = 0, LIM_MINMOD = 1, LIM_VAN_ALBADA = 2, LIM_VENKAT = 3 };
template <typename T>
BK_HD T limited_slope(T a, T b, int lim) {  // flux.rs:18-50
  if (lim == LIM_FIRST) return (T)0;
  if (a * b <= (T)0) return (T)0;
  if (lim == LIM_MINMOD) return fabs(a) < fabs(b) ? a : b;
  const T EPS = (T)1e-14;
  if (lim == LIM_VAN_ALBADA) return (a * (b * b + EPS) + b * (a * a + EPS)) / (a * a + b * b + (T)2 * EPS);
  return (T)2 * b * (a * a + a * b + EPS) / ((T)2 * a * a + a * b + b * b + (T)2 * EPS);
}
template <typename T>
BK_HD void reconstruct(const V4<T>& m2, const V4<T>& m1, const V4<T>& p0, const V4<T>& p1, int lim, V4<T>& l, V4<T>& r) {
  // flux.rs:56-72
  l = m1;
  r = p0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    T phi_l = limited_slope(m1[k] - m2[k], p0[k] - m1[k], lim);
    T phi_r = limited_slope(p0[k] - m1[k], p1[k] - p0[k], lim);
    l[k] = m1[k] + (T)0.5 * phi_l;
    r[k] = p0[k] - (T)0.5 * phi_r;
  }
  if (l[0] <= (T)0 || l[3] <= (T)0) l = m1;
  if (r[0] <= (T)0 || r[3] <= (T)0) r = p0;
}
template <typename T>
BK_HD V4<T> hllc(const V4<T>& wl, const V4<T>& wr, T nx, T nr) {  // flux.rs:79-126
  T rl = wl[0], ul = wl[1], vl = wl[2], pl = wl[3];
  T rr = wr[0], ur = wr[1], vr = wr[2], pr = wr[3];
  T unl = ul * nx + vl * nr;
  T unr = ur * nx + vr * nr;
  T cl = sqrt(gam<T>() * pl / rl);
  T cr = sqrt(gam<T>() * pr / rr);
  T el = pl / g1<T>() + (T)0.5 * rl * (ul * ul + vl * vl);
  T er = pr / g1<T>() + (T)0.5 * rr * (ur * ur + vr * vr);
  T sql = sqrt(rl), sqr = sqrt(rr);
  T inv = (T)1 / (sql + sqr);
  T uh = (sql * ul + sqr * ur) * inv;
  T vh = (sql * vl + sqr * vr) * inv;
  T hl = (el + pl) / rl;
  T hr = (er + pr) / rr;
  T hh = (sql * hl + sqr * hr) * inv;
  T ch2 = g1<T>() * (hh - (T)0.5 * (uh * uh + vh * vh));
  T floor_ = sizeof(T) == 8 ? (T)1e-300 : (T)1e-30;
  T ch = sqrt(fmax(ch2, floor_));
  T unh = uh * nx + vh * nr;
  T sl = fmin(unl - cl, unh - ch);
  T sr = fmax(unr + cr, unh + ch);
  if (sl >= (T)0) return physical_flux(wl, nx, nr);
  if (sr <= (T)0) return physical_flux(wr, nx, nr);
  T sm = (pr - pl + rl * unl * (sl - unl) - rr * unr * (sr - unr)) / (rl * (sl - unl) - rr * (sr - unr));
  if (sm >= (T)0) {
    V4<T> f = physical_flux(wl, nx, nr);
    T fac = rl * (sl - unl) / (sl - sm);
    V4<T> us = mk4<T>(fac, fac * (ul + (sm - unl) * nx), fac * (vl + (sm - unl) * nr), fac * (el / rl + (sm - unl) * (sm + pl / (rl * (sl - unl)))));
    V4<T> q = mk4<T>(rl, rl * ul, rl * vl, el);
    return mk4<T>(f[0] + sl * (us[0] - q[0]), f[1] + sl * (us[1] - q[1]), f[2] + sl * (us[2] - q[2]), f[3] + sl * (us[3] - q[3]));
  } else {
    V4<T> f = physical_flux(wr, nx, nr);
    T fac = rr * (sr - unr) / (sr - sm);
    V4<T> us = mk4<T>(fac, fac * (ur + (sm - unr) * nx), fac * (vr + (sm - unr) * nr), fac * (er / rr + (sm - unr) * (sm + pr / (rr * (sr - unr)))));
    V4<T> q = mk4<T>(rr, rr * ur, rr * vr, er);
    return mk4<T>(f[0] + sr * (us[0] - q[0]), f[1] + sr * (us[1] - q[1]), f[2] + sr * (us[2] - q[2]), f[3] + sr * (us[3] - q[3]));
  }
}
template <typename T>
BK_HD V4<T> rusanov(const V4<T>& wl, const V4<T>& wr, T nx, T nr) {  // flux.rs:132-147
  T rl = wl[0], ul = wl[1], vl = wl[2], pl = wl[3];
  T rr = wr[0], ur = wr[1], vr = wr[2], pr = wr[3];
  T unl = ul * nx + vl * nr;
  T unr = ur * nx + vr * nr;
  T smax = fmax(fabs(unl) + sqrt(gam<T>() * pl / rl), fabs(unr) + sqrt(gam<T>() * pr / rr));
  V4<T> fl = physical_flux(wl, nx, nr), fr = physical_flux(wr, nx, nr);
  V4<T> ql = mk4<T>(rl, rl * ul, rl * vl, pl / g1<T>() + (T)0.5 * rl * (ul * ul + vl * vl));
  V4<T> qr = mk4<T>(rr, rr * ur, rr * vr, pr / g1<T>() + (T)0.5 * rr * (ur * ur + vr * vr));
  V4<T> out;
#pragma unroll
  for (int k = 0; k < 4; ++k) out[k] = (T)0.5 * (fl[k] + fr[k]) - (T)0.5 * smax * (qr[k] - ql[k]);
  return out;
}
template <typename T>
BK_HD T shock_weight(T pl, T pr) {  // flux.rs:158-162 (thresholds 0.002 / 0.02)
  T s = fabs(pr - pl) / fmin(pl, pr);
  T t = (s - (T)0.002) / ((T)0.02 - (T)0.002);
  t = t < (T)0 ? (T)0 : (t > (T)1 ? (T)1 : t);
  return t * t * ((T)3 - (T)2 * t);
}
template <typename T>
BK_HD void low_mach_states(V4<T>& l, V4<T>& r, T nx, T nr) {  // flux.rs:206-219 (floor 0.05)
  T unl = l[1] * nx + l[2] * nr;
  T unr = r[1] * nx + r[2] * nr;
  T ml = sqrt(l[1] * l[1] + l[2] * l[2]) / sqrt(gam<T>() * l[3] / l[0]);
  T mr = sqrt(r[1] * r[1] + r[2] * r[2]) / sqrt(gam<T>() * r[3] / r[0]);
  T z = fmax(ml, mr);
  z = z < (T)0.05 ? (T)0.05 : (z > (T)1 ? (T)1 : z);
  if (z >= (T)1) return;
  T avg = (T)0.5 * (unl + unr);
  T dl = avg + z * (unl - avg) - unl;
  T dr = avg + z * (unr - avg) - unr;
  l[1] = l[1] + dl * nx;
  l[2] = l[2] + dl * nr;
  r[1] = r[1] + dr * nx;
  r[2] = r[2] + dr * nr;
}
template <typename T>
BK_HD V4<T> face_flux_lm(const V4<T>& m2, const V4<T>& m1, const V4<T>& p0, const V4<T>& p1, int lim, T nx, T nr, bool low_mach) {
  // flux.rs:173-186 and 224-241
  V4<T> l, r;
  reconstruct(m2, m1, p0, p1, lim, l, r);
  if (low_mach) low_mach_states(l, r, nx, nr);
  V4<T> c = hllc(l, r, nx, nr);
  T t = shock_weight(m1[3], p0[3]);
  if (t == (T)0) return c;
  V4<T> f = rusanov(l, r, nx, nr);
  V4<T> out;
#pragma unroll
  for (int k = 0; k < 4; ++k) out[k] = ((T)1 - t) * c[k] + t * f[k];
  return out;
}

// ------------------------------------------------------------------ bc.rs
enum { BC_FREESTREAM = 0, BC_EXTRAPOLATE = 1, BC_SLIPWALL = 2, BC_CHARACTERISTIC = 3, BC_PRESSURE_OUTFLOW = 4 };
template <typename T>
BK_HD V4<T> characteristic_ghost(const V4<T>& fs, const V4<T>& in, T nx, T nr) {  // bc.rs:69-93
  T m = (in[1] * nx + in[2] * nr) / sound_speed(in);
  if (m <= (T)-1) return fs;
  if (m >= (T)1) return in;
  T ci = sound_speed(in), ce = sound_speed(fs);
  T uni = in[1] * nx + in[2] * nr;
  T une = fs[1] * nx + fs[2] * nr;
  T r_out = uni + (T)2 * ci / g1<T>();
  T r_in = une - (T)2 * ce / g1<T>();
  T un_b = (T)0.5 * (r_out + r_in);
  T c_b = fmax((T)0.25 * g1<T>() * (r_out - r_in), (T)1e-8);
  bool out = un_b >= (T)0;
  const V4<T>& rf = out ? in : fs;
  T un_ref = out ? uni : une;
  T s = rf[3] / pow(rf[0], gam<T>());
  T rho = pow(c_b * c_b / (gam<T>() * s), (T)1 / g1<T>());
  T p = rho * c_b * c_b / gam<T>();
  T dn = un_b - un_ref;
  return mk4<T>(rho, rf[1] + dn * nx, rf[2] + dn * nr, p);
}
template <typename T>
BK_HD V4<T> pressure_outflow_ghost(T p_back, const V4<T>& in, T nx, T nr) {  // bc.rs:97-103
  if ((in[1] * nx + in[2] * nr) / sound_speed(in) >= (T)1) return in;
  return mk4<T>(in[0], in[1], in[2], p_back);
}
template <typename T>
BK_HD V4<T> ghost_state(int bc, const V4<T>& fs, const V4<T>& edge, const V4<T>& mirror, T nx, T nr, T outward) {  // solver.rs:413-421
  switch (bc) {
    case BC_FREESTREAM:
      return fs;
    case BC_EXTRAPOLATE:
      return edge;
    case BC_SLIPWALL:
      return reflect(mirror, nx, nr);
    case BC_CHARACTERISTIC:
      return characteristic_ghost(fs, edge, outward * nx, outward * nr);
    default:
      return pressure_outflow_ghost(fs[3], edge, outward * nx, outward * nr);
  }
}

// ------------------------------------------------------------------ 4x4 blocks (implicit.rs:45-175)
template <typename T>
BK_HD M4<T> zero4() {
  M4<T> m;
#pragma unroll
  for (int k = 0; k < 16; ++k) m[k] = (T)0;
  return m;
}
template <typename T>
BK_HD M4<T> eye4() {
  M4<T> m = zero4<T>();
  m[0] = m[5] = m[10] = m[15] = (T)1;
  return m;
}
template <typename T>
BK_HD M4<T> mm(const M4<T>& a, const M4<T>& b) {  // implicit.rs:111-122
  M4<T> c;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
      c[4 * i + j] = a[4 * i] * b[j] + a[4 * i + 1] * b[4 + j] + a[4 * i + 2] * b[8 + j] + a[4 * i + 3] * b[12 + j];
  return c;
}
template <typename T>
BK_HD V4<T> mv(const M4<T>& a, const V4<T>& x) {  // implicit.rs:125-131
  V4<T> y;
#pragma unroll
  for (int i = 0; i < 4; ++i) y[i] = a[4 * i] * x[0] + a[4 * i + 1] * x[1] + a[4 * i + 2] * x[2] + a[4 * i + 3] * x[3];
  return y;
}
template <typename T>
BK_HD void axpy(M4<T>& a, T s, const M4<T>& b) {
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] += s * b[k];
}
// Gauss-Jordan inverse with partial pivoting (implicit.rs:141-175), written with register-resident selects (no dynamic
// indexing) so the block stays in registers.
template <typename T>
BK_HD M4<T> inv4(const M4<T>& m) {
  T a[4][4], v[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      a[r][c] = m[4 * r + c];
      v[r][c] = r == c ? (T)1 : (T)0;
    }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    // pivot row: first row r >= c with the largest |a[r][c]| (strictly larger replaces, as in the reference)
    int piv = c;
    T best = fabs(a[c][c]);
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      T x = fabs(a[r][c]);
      if (x > best) {
        best = x;
        piv = r;
      }
    }
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      bool sw = piv == r;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        T t0 = a[c][k], t1 = a[r][k];
        a[c][k] = sw ? t1 : t0;
        a[r][k] = sw ? t0 : t1;
        T u0 = v[c][k], u1 = v[r][k];
        v[c][k] = sw ? u1 : u0;
        v[r][k] = sw ? u0 : u1;
      }
    }
    T d = (T)1 / a[c][c];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      a[c][k] *= d;
      v[c][k] *= d;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (r == c) continue;
      T f = a[r][c];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        a[r][k] -= f * a[c][k];
        v[r][k] -= f * v[c][k];
      }
    }
  }
  M4<T> out;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) out[4 * r + c] = v[r][c];
  return out;
}

template <typename T>
BK_HD M4<T> flux_jacobian(const V4<T>& w, T nx, T nr) {  // implicit.rs:95-108
  T rho = w[0], u = w[1], v = w[2], p = w[3];
  T G = gam<T>(), G1 = g1<T>();
  T q2 = u * u + v * v;
  T th = u * nx + v * nr;
  T phi = (T)0.5 * G1 * q2;
  T h = G * p / (G1 * rho) + (T)0.5 * q2;
  M4<T> a;
  a[0] = 0;
  a[1] = nx;
  a[2] = nr;
  a[3] = 0;
  a[4] = phi * nx - u * th;
  a[5] = th + ((T)2 - G) * u * nx;
  a[6] = u * nr - G1 * v * nx;
  a[7] = G1 * nx;
  a[8] = phi * nr - v * th;
  a[9] = v * nx - G1 * u * nr;
  a[10] = th + ((T)2 - G) * v * nr;
  a[11] = G1 * nr;
  a[12] = th * (phi - h);
  a[13] = h * nx - G1 * u * th;
  a[14] = h * nr - G1 * v * th;
  a[15] = G * th;
  return a;
}
template <typename T>
BK_HD M4<T> abs_jacobian(const V4<T>& wl, const V4<T>& wr, T nx, T nr, T eps_fix) {  // implicit.rs:209-241
  T G = gam<T>(), G1 = g1<T>();
  T sl = sqrt(wl[0]), sr = sqrt(wr[0]);
  T inv = (T)1 / (sl + sr);
  T u = (sl * wl[1] + sr * wr[1]) * inv, v = (sl * wl[2] + sr * wr[2]) * inv;
  T hl = G * wl[3] / (G1 * wl[0]) + (T)0.5 * (wl[1] * wl[1] + wl[2] * wl[2]);
  T hr = G * wr[3] / (G1 * wr[0]) + (T)0.5 * (wr[1] * wr[1] + wr[2] * wr[2]);
  T h = (sl * hl + sr * hr) * inv;
  T floor_ = sizeof(T) == 8 ? (T)1e-300 : (T)1e-30;
  T c = sqrt(fmax(G1 * (h - (T)0.5 * (u * u + v * v)), floor_));
  T a = u * nx + v * nr;
  T eps = eps_fix * c;
  auto fix = [&](T l) { return fabs(l) >= eps ? fabs(l) : (T)0.5 * (l * l / eps + eps); };
  T e1 = fix(a), e2 = fix(a + c), e3 = fix(a - c);
  T d1 = (e2 - e1) / c;
  T d2 = (e2 + e3 - (T)2 * e1) / ((T)2 * c * c);
  V4<T> wa = mk4<T>((T)1, u, v, G1 / G * (h - (T)0.5 * (u * u + v * v)));
  M4<T> am = flux_jacobian(wa, nx, nr);
  M4<T> b1 = am, b2 = am;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    b1[5 * q] -= a;
    b2[5 * q] -= a + c;
  }
  M4<T> prod = mm(b1, b2);
  M4<T> out;
#pragma unroll
  for (int k = 0; k < 16; ++k) out[k] = d1 * b1[k] + d2 * prod[k];
#pragma unroll
  for (int q = 0; q < 4; ++q) out[5 * q] += e1;
  return out;
}
template <typename T>
BK_HD T spectral(const V4<T>& w, T nx, T nr) {  // implicit.rs:244-246
  return fabs(w[1] * nx + w[2] * nr) + sound_speed(w);
}
template <typename T>
BK_HD M4<T> reflection(T nx, T nr) {  // implicit.rs:249-251
  M4<T> m = zero4<T>();
  m[0] = 1;
  m[5] = (T)1 - (T)2 * nx * nx;
  m[6] = (T)-2 * nx * nr;
  m[9] = (T)-2 * nx * nr;
  m[10] = (T)1 - (T)2 * nr * nr;
  m[15] = 1;
  return m;
}
template <typename T>
BK_HD M4<T> noslip4() {  // implicit.rs:254
  M4<T> m = zero4<T>();
  m[0] = 1;
  m[5] = -1;
  m[10] = -1;
  m[15] = 1;
  return m;
}
// T = dU_ghost / dU_interior of the first ghost layer (implicit.rs:257-279), evaluated in FP64 (finite differences with the
// reference's step 1e-7 (1 + |u|) need the double-precision ghost state).
BK_HD M4<double> ghost_jacobian(int bc, const V4<double>& fs, const V4<double>& edge, double nx, double nr, double outward) {
  if (bc == BC_FREESTREAM) return zero4<double>();
  if (bc == BC_EXTRAPOLATE) return eye4<double>();
  if (bc == BC_SLIPWALL) return reflection<double>(nx, nr);
  V4<double> u0 = prim_to_cons(edge);
  V4<double> g0 = prim_to_cons(ghost_state<double>(bc, fs, edge, edge, nx, nr, outward));
  M4<double> t = zero4<double>();
  for (int q = 0; q < 4; ++q) {
    double h = 1e-7 * (1.0 + fabs(u0[q]));
    V4<double> up = u0;
    up[q] += h;
    V4<double> e = cons_to_prim(up);
    V4<double> g = prim_to_cons(ghost_state<double>(bc, fs, e, e, nx, nr, outward));
    for (int r = 0; r < 4; ++r) t[4 * r + q] = (g[r] - g0[r]) / h;
  }
  return t;
}

// Blocks (lo, d, up) of I - dt J for one cell (implicit.rs:284-367).
template <typename T>
BK_HD void cell_blocks(const V4<T>& wk, const V4<T>& wm, const V4<T>& wp, T fl_nx, T fl_nr, T fl_w, T fr_nx, T fr_nr, T fr_w, T vol, T dt,
                       bool lines, T src, bool roe, T eps_fix, T visc_l, T visc_r, M4<T>& lo, M4<T>& d, M4<T>& up) {
  T s = (T)0.5 * dt / vol;
  M4<T> dis_l, dis_r;
  if (roe) {
    dis_l = abs_jacobian(wm, wk, fl_nx, fl_nr, eps_fix);
    dis_r = abs_jacobian(wk, wp, fr_nx, fr_nr, eps_fix);
    T tl = shock_weight(wm[3], wk[3]), tr = shock_weight(wk[3], wp[3]);
    if (tl > (T)0 || tr > (T)0) {
      T lam_l = fmax(spectral(wk, fl_nx, fl_nr), spectral(wm, fl_nx, fl_nr));
      T lam_r = fmax(spectral(wk, fr_nx, fr_nr), spectral(wp, fr_nx, fr_nr));
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        dis_l[k] *= (T)1 - tl;
        dis_r[k] *= (T)1 - tr;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        dis_l[5 * q] += tl * lam_l;
        dis_r[5 * q] += tr * lam_r;
      }
    }
  } else {
    T lam_l = fmax(spectral(wk, fl_nx, fl_nr), spectral(wm, fl_nx, fl_nr));
    T lam_r = fmax(spectral(wk, fr_nx, fr_nr), spectral(wp, fr_nx, fr_nr));
    dis_l = zero4<T>();
    dis_r = zero4<T>();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      dis_l[5 * q] = lam_l;
      dis_r[5 * q] = lam_r;
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    dis_l[5 * q] += (T)2 * visc_l;
    dis_r[5 * q] += (T)2 * visc_r;
  }
  d = eye4<T>();
  axpy(d, s * fr_w, flux_jacobian(wk, fr_nx, fr_nr));
  axpy(d, -s * fl_w, flux_jacobian(wk, fl_nx, fl_nr));
  axpy(d, s * fr_w, dis_r);
  axpy(d, s * fl_w, dis_l);
  if (src != (T)0) {
    T c = -dt * src * g1<T>();
    d[8] += c * (T)0.5 * (wk[1] * wk[1] + wk[2] * wk[2]);
    d[9] += -c * wk[1];
    d[10] += -c * wk[2];
    d[11] += c;
  }
  if (!lines) {
    lo = zero4<T>();
    up = zero4<T>();
    return;
  }
  lo = flux_jacobian(wm, fl_nx, fl_nr);
  axpy(lo, (T)1, dis_l);
  T sl_ = -s * fl_w;
#pragma unroll
  for (int k = 0; k < 16; ++k) lo[k] *= sl_;
  up = flux_jacobian(wp, fr_nx, fr_nr);
  axpy(up, (T)-1, dis_r);
  T sr_ = s * fr_w;
#pragma unroll
  for (int k = 0; k < 16; ++k) up[k] *= sr_;
}

// Aupoix (2015) "Colebrook" rough-wall state of a no-slip wall cell (turbulence.rs:292-320): kinematic viscosity nu, speed
// |u|, wall distance d, equivalent sand-grain roughness ks > 0 -> (k_w, omega_w, nu_t,w), omega_w bounded by the smooth
// wall value 60 nu / (beta_1 d^2) and nu_t,w by 1e5 nu; u_tau^2 = (nu + nu_t,w) |u| / d by 16 fixed-point steps from
// the laminar u_tau^2 = nu |u| / d. FP64: it runs once per wall cell and iteration.
__device__ inline void aupoix_state(double nu, double speed, double d, double ks, double u2, double out[3]) {
  const double u_tau = sqrt(u2);
  const double ks_plus = fmax(u_tau * ks / nu, 1e-30);
  const double t = tanh(ks_plus / 125.0);
  const double k_plus = fmax(tanh((log10(ks_plus / 30.0) + 1.0 - t) * t), 0.0) / sqrt(0.09);
  const double om_rough = 300.0 * nu / (ks * ks) / tanh(15.0 / (4.0 * ks_plus)) + 191.0 * u_tau / ks * (1.0 - exp(-ks_plus / 250.0));
  out[0] = k_plus * u2;
  out[1] = fmin(om_rough, 60.0 * nu / (0.075 * d * d));
  out[2] = fmin(out[0] / out[1], 1e5 * nu);
}
__device__ inline void aupoix_wall(double nu, double speed, double d, double ks, double out[3]) {
  double u2 = nu * speed / d;
  for (int k = 0; k < 16; ++k) {
    aupoix_state(nu, speed, d, ks, u2, out);
    u2 = (nu + out[2]) * speed / d;
  }
  aupoix_state(nu, speed, d, ks, u2, out);
}

}  // namespace bk
