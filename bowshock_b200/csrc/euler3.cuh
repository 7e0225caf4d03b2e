// 3D Euler path (crates/bowshock-cfd/src/{gas3,bc3,flux3,grid3,solver3,implicit3}.rs; forces and stop rules of
// crates/bowshock-core/src/engine/run3.rs) on the B200: a batch of cases (Mach number, incidence) that share one revolved
// grid, so the geometry is stored once and read through L2 by every case. Per case the state is SoA FP32 planes
// [case][var][cell]; the face fluxes and the cell residual are evaluated in FP64 from the FP32 primitives; the three-factor
// line-implicit operator (5x5 blocks, Roe |A| with the entropy fix, shock-sensor blend) is assembled once per iteration,
// thread per cell, into line records, factorised and solved one thread per line (block Thomas), i then j then k, and the
// defect-correction passes reuse the kept blocks and factors.
//   k3_prims      conserved -> primitive (padded, 2 ghost layers)                    (solver3.rs:222-236)
//   k3_ghosts     characteristic far field (FP64), axis (the cell across the axis), slip wall, symmetry planes (solver3.rs:171-219)
//   k3_flux       MUSCL in the face's cylindrical frame + HLLC / Rusanov blend + low-Mach correction, FP64 (flux3.rs, solver3.rs:365-418)
//   k3_residual   R = -(1/V) sum S F (FP64 accumulation), local time step, FP64 density norm (solver3.rs:251-300)
//   k3_assemble   blocks of I - dt J_i, J_j, J_k per cell into the line records           (implicit3.rs:214-355)
//   k3_lines      first pass: block Thomas along every line of direction dir on the kept blocks, factors kept
//   k3_lines_subst the defect-correction passes with the kept factors                  (implicit3.rs:274-382)
//   k3_defect     dt R - (A_i du + A_j du + A_k du - 2 du) with the kept blocks         (implicit3.rs:384-455)
//   k3_stage      SSP-RK3 stage                                                       (solver3.rs:303-327)
//   k3_forces     FP64 wall-pressure force integration: CN, CA, centre of pressure     (run3.rs:130-212)
// Solid boxes (fins, solver3.rs:13): cells of B.solid are never updated (zero residual and time step, identity rows of the
// line systems) and act as slip walls of their fluid neighbours (reflected states in the flux stencils and in the blocks).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device_math.cuh"

namespace bk3 {
using bk::LIM_FIRST;
using bk::LIM_MINMOD;
using bk::limited_slope;
using bk::shock_weight;

constexpr double GD = 1.4;

template <typename T>
struct V5 {
  T v[5];
  __host__ __device__ __forceinline__ T& operator[](int k) { return v[k]; }
  __host__ __device__ __forceinline__ const T& operator[](int k) const { return v[k]; }
};
template <typename T>
struct M5 {
  T a[25];
  __host__ __device__ __forceinline__ T& operator[](int k) { return a[k]; }
  __host__ __device__ __forceinline__ const T& operator[](int k) const { return a[k]; }
};
template <typename T>
__device__ __forceinline__ V5<T> cons_to_prim3(const V5<T>& q) {  // gas3.rs:20-25
  T rho = q[0];
  T u = q[1] / rho, v = q[2] / rho, w = q[3] / rho;
  T p = (T)(GD - 1.0) * (q[4] - (T)0.5 * rho * (u * u + v * v + w * w));
  return V5<T>{{rho, u, v, w, p}};
}
template <typename T>
__device__ __forceinline__ V5<T> prim_to_cons3(const V5<T>& w) {  // gas3.rs:14-17
  return V5<T>{{w[0], w[0] * w[1], w[0] * w[2], w[0] * w[3], w[4] / (T)(GD - 1.0) + (T)0.5 * w[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3])}};
}
template <typename T>
__device__ __forceinline__ V5<T> physical_flux3(const V5<T>& w, T nx, T ny, T nz) {  // gas3.rs:34-39
  T un = w[1] * nx + w[2] * ny + w[3] * nz;
  T e = w[4] / (T)(GD - 1.0) + (T)0.5 * w[0] * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
  return V5<T>{{w[0] * un, w[0] * w[1] * un + w[4] * nx, w[0] * w[2] * un + w[4] * ny, w[0] * w[3] * un + w[4] * nz, (e + w[4]) * un}};
}
template <typename T>
__device__ __forceinline__ V5<T> reflect3(const V5<T>& w, T nx, T ny, T nz) {  // gas3.rs:48-51
  T un = w[1] * nx + w[2] * ny + w[3] * nz;
  return V5<T>{{w[0], w[1] - (T)2 * un * nx, w[2] - (T)2 * un * ny, w[3] - (T)2 * un * nz, w[4]}};
}
__device__ __forceinline__ V5<double> char_ghost3(const V5<double>& fs, const V5<double>& in, double nx, double ny, double nz) {  // bc3.rs:30-56
  double ci = sqrt(GD * in[4] / in[0]);
  double uni = in[1] * nx + in[2] * ny + in[3] * nz;
  double m = uni / ci;
  if (m <= -1.0) return fs;
  if (m >= 1.0) return in;
  const double g1 = GD - 1.0;
  double ce = sqrt(GD * fs[4] / fs[0]);
  double une = fs[1] * nx + fs[2] * ny + fs[3] * nz;
  double r_out = uni + 2.0 * ci / g1, r_in = une - 2.0 * ce / g1;
  double un_b = 0.5 * (r_out + r_in);
  double c_b = fmax(0.25 * g1 * (r_out - r_in), 1e-8);
  const V5<double>& rf = un_b >= 0.0 ? in : fs;
  double un_ref = un_b >= 0.0 ? uni : une;
  double s = rf[4] / pow(rf[0], GD);
  double rho = pow(c_b * c_b / (GD * s), 1.0 / g1);
  double p = rho * c_b * c_b / GD;
  double dn = un_b - un_ref;
  return V5<double>{{rho, rf[1] + dn * nx, rf[2] + dn * ny, rf[3] + dn * nz, p}};
}
// flux3.rs:27-54: MUSCL with the lateral velocity limited in the face's cylindrical frame (s, co)
__device__ __forceinline__ void reconstruct3(const V5<double>& m2, const V5<double>& m1, const V5<double>& p0, const V5<double>& p1, int lim,
                                             double s, double co, V5<double>& lo, V5<double>& ro) {
  auto fwd = [&](const V5<double>& w) { return V5<double>{{w[0], w[1], w[2] * s + w[3] * co, w[2] * co - w[3] * s, w[4]}}; };
  V5<double> a = fwd(m2), b = fwd(m1), c = fwd(p0), d = fwd(p1);
  V5<double> l = b, r = c;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    l[k] = b[k] + 0.5 * limited_slope<double>(b[k] - a[k], c[k] - b[k], lim);
    r[k] = c[k] - 0.5 * limited_slope<double>(c[k] - b[k], d[k] - c[k], lim);
  }
  if (l[0] <= 0.0 || l[4] <= 0.0) l = b;
  if (r[0] <= 0.0 || r[4] <= 0.0) r = c;
  bool lb = true, rc = true;
#pragma unroll
  for (int k = 0; k < 5; ++k) lb = lb && l[k] == b[k], rc = rc && r[k] == c[k];
  lo = lb ? m1 : V5<double>{{l[0], l[1], l[2] * s + l[3] * co, l[2] * co - l[3] * s, l[4]}};
  ro = rc ? p0 : V5<double>{{r[0], r[1], r[2] * s + r[3] * co, r[2] * co - r[3] * s, r[4]}};
}
__device__ __forceinline__ V5<double> hllc3(const V5<double>& wl, const V5<double>& wr, double nx, double ny, double nz) {  // flux3.rs:59-117
  double rl = wl[0], ul = wl[1], vl = wl[2], zl = wl[3], pl = wl[4];
  double rr = wr[0], ur = wr[1], vr = wr[2], zr = wr[3], pr = wr[4];
  double unl = ul * nx + vl * ny + zl * nz, unr = ur * nx + vr * ny + zr * nz;
  double cl = sqrt(GD * pl / rl), cr = sqrt(GD * pr / rr);
  double el = pl / (GD - 1.0) + 0.5 * rl * (ul * ul + vl * vl + zl * zl);
  double er = pr / (GD - 1.0) + 0.5 * rr * (ur * ur + vr * vr + zr * zr);
  double sql = sqrt(rl), sqr = sqrt(rr), inv = 1.0 / (sql + sqr);
  double uh = (sql * ul + sqr * ur) * inv, vh = (sql * vl + sqr * vr) * inv, wh = (sql * zl + sqr * zr) * inv;
  double hh = (sql * ((el + pl) / rl) + sqr * ((er + pr) / rr)) * inv;
  double ch = sqrt(fmax((GD - 1.0) * (hh - 0.5 * (uh * uh + vh * vh + wh * wh)), 1e-300));
  double unh = uh * nx + vh * ny + wh * nz;
  double sl = fmin(unl - cl, unh - ch), sr = fmax(unr + cr, unh + ch);
  if (sl >= 0.0) return physical_flux3<double>(wl, nx, ny, nz);
  if (sr <= 0.0) return physical_flux3<double>(wr, nx, ny, nz);
  double sm = (pr - pl + rl * unl * (sl - unl) - rr * unr * (sr - unr)) / (rl * (sl - unl) - rr * (sr - unr));
  V5<double> out;
  if (sm >= 0.0) {
    V5<double> f = physical_flux3<double>(wl, nx, ny, nz);
    double fac = rl * (sl - unl) / (sl - sm), d = sm - unl;
    double st[5] = {fac, fac * (ul + d * nx), fac * (vl + d * ny), fac * (zl + d * nz), fac * (el / rl + d * (sm + pl / (rl * (sl - unl))))};
    double q[5] = {rl, rl * ul, rl * vl, rl * zl, el};
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = f[k] + sl * (st[k] - q[k]);
  } else {
    V5<double> f = physical_flux3<double>(wr, nx, ny, nz);
    double fac = rr * (sr - unr) / (sr - sm), d = sm - unr;
    double st[5] = {fac, fac * (ur + d * nx), fac * (vr + d * ny), fac * (zr + d * nz), fac * (er / rr + d * (sm + pr / (rr * (sr - unr))))};
    double q[5] = {rr, rr * ur, rr * vr, rr * zr, er};
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = f[k] + sr * (st[k] - q[k]);
  }
  return out;
}
__device__ __forceinline__ V5<double> rusanov3(const V5<double>& wl, const V5<double>& wr, double nx, double ny, double nz) {  // flux3.rs:121-135
  double unl = wl[1] * nx + wl[2] * ny + wl[3] * nz, unr = wr[1] * nx + wr[2] * ny + wr[3] * nz;
  double smax = fmax(fabs(unl) + sqrt(GD * wl[4] / wl[0]), fabs(unr) + sqrt(GD * wr[4] / wr[0]));
  V5<double> fl = physical_flux3<double>(wl, nx, ny, nz), fr = physical_flux3<double>(wr, nx, ny, nz);
  V5<double> ql = prim_to_cons3<double>(wl), qr = prim_to_cons3<double>(wr);
  V5<double> out;
#pragma unroll
  for (int k = 0; k < 5; ++k) out[k] = 0.5 * (fl[k] + fr[k]) - 0.5 * smax * (qr[k] - ql[k]);
  return out;
}
__device__ __forceinline__ V5<double> face_flux_lm3(const V5<double>& m2, const V5<double>& m1, const V5<double>& p0, const V5<double>& p1,
                                                    int lim, double nx, double ny, double nz, double s, double co, bool low_mach) {
  V5<double> l, r;
  reconstruct3(m2, m1, p0, p1, lim, s, co, l, r);
  if (low_mach) {  // flux3.rs:163-176
    double unl = l[1] * nx + l[2] * ny + l[3] * nz, unr = r[1] * nx + r[2] * ny + r[3] * nz;
    double ml = sqrt(l[1] * l[1] + l[2] * l[2] + l[3] * l[3]) / sqrt(GD * l[4] / l[0]);
    double mr = sqrt(r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) / sqrt(GD * r[4] / r[0]);
    double z = fmin(fmax(fmax(ml, mr), 0.05), 1.0);
    if (z < 1.0) {
      double avg = 0.5 * (unl + unr);
      double dl = avg + z * (unl - avg) - unl, dr = avg + z * (unr - avg) - unr;
      l[1] += dl * nx, l[2] += dl * ny, l[3] += dl * nz;
      r[1] += dr * nx, r[2] += dr * ny, r[3] += dr * nz;
    }
  }
  V5<double> c = hllc3(l, r, nx, ny, nz);  // flux3.rs:146-158
  double t = shock_weight<double>(m1[4], p0[4]);
  if (t == 0.0) return c;
  V5<double> f = rusanov3(l, r, nx, ny, nz);
#pragma unroll
  for (int k = 0; k < 5; ++k) c[k] = (1.0 - t) * c[k] + t * f[k];
  return c;
}

// ---------------------------------------------------------------- 5x5 blocks (implicit3.rs)
__device__ __forceinline__ M5<float> zero5() {
  M5<float> m;
#pragma unroll
  for (int k = 0; k < 25; ++k) m[k] = 0.f;
  return m;
}
__device__ __forceinline__ M5<float> eye5() {
  M5<float> m = zero5();
#pragma unroll
  for (int q = 0; q < 5; ++q) m[6 * q] = 1.f;
  return m;
}
__device__ __forceinline__ M5<float> flux_jacobian3(const V5<float>& w, float nx, float ny, float nz) {  // implicit3.rs:44-60
  const float G = 1.4f, g1 = 0.4f;
  float rho = w[0], u = w[1], v = w[2], ww = w[3], p = w[4];
  float q2 = u * u + v * v + ww * ww, th = u * nx + v * ny + ww * nz, phi = 0.5f * g1 * q2, h = G * p / (g1 * rho) + 0.5f * q2;
  return M5<float>{{0.f, nx, ny, nz, 0.f,                                                                                   //
                    phi * nx - u * th, th + (2.f - G) * u * nx, u * ny - g1 * v * nx, u * nz - g1 * ww * nx, g1 * nx,        //
                    phi * ny - v * th, v * nx - g1 * u * ny, th + (2.f - G) * v * ny, v * nz - g1 * ww * ny, g1 * ny,        //
                    phi * nz - ww * th, ww * nx - g1 * u * nz, ww * ny - g1 * v * nz, th + (2.f - G) * ww * nz, g1 * nz,     //
                    th * (phi - h), h * nx - g1 * u * th, h * ny - g1 * v * th, h * nz - g1 * ww * th, G * th}};
}
__device__ __forceinline__ M5<float> mm5(const M5<float>& a, const M5<float>& b) {
  M5<float> c;
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      float s = 0.f;
#pragma unroll
      for (int k = 0; k < 5; ++k) s += a[5 * i + k] * b[5 * k + j];
      c[5 * i + j] = s;
    }
  return c;
}
__device__ __forceinline__ V5<float> mv5(const M5<float>& a, const V5<float>& x) {
  V5<float> y;
#pragma unroll
  for (int i = 0; i < 5; ++i) y[i] = a[5 * i] * x[0] + a[5 * i + 1] * x[1] + a[5 * i + 2] * x[2] + a[5 * i + 3] * x[3] + a[5 * i + 4] * x[4];
  return y;
}
__device__ __forceinline__ void axpy5(M5<float>& a, float s, const M5<float>& b) {
#pragma unroll
  for (int k = 0; k < 25; ++k) a[k] += s * b[k];
}
// Gauss-Jordan with partial pivoting (implicit3.rs:94-125), register-resident: row swaps by selects
__device__ __forceinline__ M5<float> inv5(const M5<float>& m) {
  float a[5][5], v[5][5];
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) a[r][c] = m[5 * r + c], v[r][c] = r == c ? 1.f : 0.f;
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    int piv = c;
    float best = fabsf(a[c][c]);
#pragma unroll
    for (int r = c + 1; r < 5; ++r) {
      float x = fabsf(a[r][c]);
      if (x > best) best = x, piv = r;
    }
#pragma unroll
    for (int r = c + 1; r < 5; ++r) {
      bool sw = piv == r;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        float t0 = a[c][k], t1 = a[r][k], u0 = v[c][k], u1 = v[r][k];
        a[c][k] = sw ? t1 : t0, a[r][k] = sw ? t0 : t1;
        v[c][k] = sw ? u1 : u0, v[r][k] = sw ? u0 : u1;
      }
    }
    float d = 1.f / a[c][c];
#pragma unroll
    for (int k = 0; k < 5; ++k) a[c][k] *= d, v[c][k] *= d;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      if (r == c) continue;
      float f = a[r][c];
#pragma unroll
      for (int k = 0; k < 5; ++k) a[r][k] -= f * a[c][k], v[r][k] -= f * v[c][k];
    }
  }
  M5<float> out;
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) out[5 * r + c] = v[r][c];
  return out;
}
__device__ __forceinline__ M5<float> abs_jacobian3(const V5<float>& wl, const V5<float>& wr, float nx, float ny, float nz, float eps_fix) {
  const float G = 1.4f, g1 = 0.4f;  // implicit3.rs:160-193
  float sl = sqrtf(wl[0]), sr = sqrtf(wr[0]), inv = 1.f / (sl + sr);
  float u = (sl * wl[1] + sr * wr[1]) * inv, v = (sl * wl[2] + sr * wr[2]) * inv, ww = (sl * wl[3] + sr * wr[3]) * inv;
  float hl = G * wl[4] / (g1 * wl[0]) + 0.5f * (wl[1] * wl[1] + wl[2] * wl[2] + wl[3] * wl[3]);
  float hr = G * wr[4] / (g1 * wr[0]) + 0.5f * (wr[1] * wr[1] + wr[2] * wr[2] + wr[3] * wr[3]);
  float h = (sl * hl + sr * hr) * inv, q2h = 0.5f * (u * u + v * v + ww * ww);
  float c = sqrtf(fmaxf(g1 * (h - q2h), 1e-30f));
  float a = u * nx + v * ny + ww * nz, eps = eps_fix * c;
  auto fix = [&](float l) { return fabsf(l) >= eps ? fabsf(l) : 0.5f * (l * l / eps + eps); };
  float e1 = fix(a), e2 = fix(a + c), e3 = fix(a - c);
  float d1 = (e2 - e1) / c, d2 = (e2 + e3 - 2.f * e1) / (2.f * c * c);
  V5<float> wa{{1.f, u, v, ww, g1 / G * (h - q2h)}};
  M5<float> b1 = flux_jacobian3(wa, nx, ny, nz), b2 = b1;
#pragma unroll
  for (int q = 0; q < 5; ++q) b1[6 * q] -= a, b2[6 * q] -= a + c;
  M5<float> prod = mm5(b1, b2);
#pragma unroll
  for (int k = 0; k < 25; ++k) prod[k] = d1 * b1[k] + d2 * prod[k];
#pragma unroll
  for (int q = 0; q < 5; ++q) prod[6 * q] += e1;
  return prod;
}
__device__ __forceinline__ float spectral3(const V5<float>& w, float nx, float ny, float nz) {
  return fabsf(w[1] * nx + w[2] * ny + w[3] * nz) + sqrtf(1.4f * w[4] / w[0]);
}
__device__ __forceinline__ M5<float> reflection3(float nx, float ny, float nz) {  // implicit3.rs:202-210
  M5<float> m = eye5();
  float n[3] = {nx, ny, nz};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) m[5 * (1 + a) + 1 + b] -= 2.f * n[a] * n[b];
  return m;
}

// ---------------------------------------------------------------- batch layout
struct Case3Dev {
  double fs[5];
  float cfl, cfl0, cfl_max, growth, eps_fix;
  int limiter, low_mach, first_order_iters, implicit, dt_mode, sub_iters, roe, implicit_bc, lines;
};

struct B3 {
  int ni, nj, nk, nb, axis_cells;
  int b0;  // the first case of a launch: blockIdx.y + b0 is the case (a group of the batch's cases)
  long long nc, npad, nfi, nfj, nfk;
  const float4 *fi, *fj, *fk;  // (nx, ny, nz, area)
  const float2 *ri, *rj, *rk;  // face_rot (s, co)
  const float* vol;
  const unsigned char* solid;  // per cell, inside a solid box (null: no solid cells)
  const int* axis_k;  // [i * nk + k], i < axis_cells
  const Case3Dev* cs;
  int *iter, *ramp, *active;
  float *U, *U0, *W, *R, *X, *DU, *RR, *dt, *scr;  // [case][var][cell]; W [case][var][padded]; scr: line records (rec3)
  double *FI, *FJ, *FK;                             // face flux x area, [case][var][face]
  double* rsum;                                     // [slot][case]
};

__device__ __forceinline__ long long pidx3(const B3& B, int i, int j, int k) {
  return ((long long)(k + 2) * (B.nj + 4) + (j + 2)) * (B.ni + 4) + (i + 2);
}
__device__ __forceinline__ long long cell3(const B3& B, int i, int j, int k) { return ((long long)k * B.nj + j) * B.ni + i; }
// solver3.rs:343-353: positions outside the grid (ghosts) are not solid
__device__ __forceinline__ bool sol3(const B3& B, int i, int j, int k) {
  return B.solid && i >= 0 && j >= 0 && k >= 0 && i < B.ni && j < B.nj && k < B.nk && B.solid[cell3(B, i, j, k)];
}
__device__ __forceinline__ V5<float> ldU(const B3& B, const float* a, int b, long long c) {
  const float* p = a + (long long)b * 5 * B.nc + c;
  return V5<float>{{p[0], p[B.nc], p[2 * B.nc], p[3 * B.nc], p[4 * B.nc]}};
}
__device__ __forceinline__ void stU(const B3& B, float* a, int b, long long c, const V5<float>& v) {
  float* p = a + (long long)b * 5 * B.nc + c;
#pragma unroll
  for (int q = 0; q < 5; ++q) p[q * B.nc] = v[q];
}
__device__ __forceinline__ V5<float> ldW(const B3& B, int b, long long pi) {
  const float* p = B.W + (long long)b * 5 * B.npad + pi;
  return V5<float>{{p[0], p[B.npad], p[2 * B.npad], p[3 * B.npad], p[4 * B.npad]}};
}
__device__ __forceinline__ void stW(const B3& B, int b, long long pi, const V5<double>& v) {
  float* p = B.W + (long long)b * 5 * B.npad + pi;
#pragma unroll
  for (int q = 0; q < 5; ++q) p[q * B.npad] = (float)v[q];
}
__device__ __forceinline__ V5<double> f2d5(const V5<float>& v) { return V5<double>{{v[0], v[1], v[2], v[3], v[4]}}; }
__device__ __forceinline__ V5<double> fs3(const Case3Dev& c) { return V5<double>{{c.fs[0], c.fs[1], c.fs[2], c.fs[3], c.fs[4]}}; }

// ---------------------------------------------------------------- kernels
__global__ void k3_prims(B3 B) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  if (t >= B.nc || !B.active[b]) return;
  int i = (int)(t % B.ni), j = (int)((t / B.ni) % B.nj), k = (int)(t / ((long long)B.ni * B.nj));
  V5<float> w = cons_to_prim3<float>(ldU(B, B.U, b, t));
  stW(B, b, pidx3(B, i, j, k), f2d5(w));
}

// ghosts of every boundary face column: i ends, j = 0 (axis or slip wall), j = nj, k ends (symmetry planes)
__global__ void k3_ghosts(B3 B) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  if (!B.active[b]) return;
  const Case3Dev& c = B.cs[b];
  const long long njk = (long long)B.nj * B.nk, nik = (long long)B.ni * B.nk, nij = (long long)B.ni * B.nj;
  if (t < 2 * njk) {  // i ends: characteristic far field (FP64)
    bool hi = t >= njk;
    long long q = hi ? t - njk : t;
    int j = (int)(q % B.nj), k = (int)(q / B.nj);
    long long f = ((long long)k * B.nj + j) * (B.ni + 1) + (hi ? B.ni : 0);
    float4 n = B.fi[f];
    double o = hi ? 1.0 : -1.0;
    V5<double> g = char_ghost3(fs3(c), f2d5(ldW(B, b, pidx3(B, hi ? B.ni - 1 : 0, j, k))), o * n.x, o * n.y, o * n.z);
    for (int m = 1; m <= 2; ++m) stW(B, b, pidx3(B, hi ? B.ni + m - 1 : -m, j, k), g);
    return;
  }
  t -= 2 * njk;
  if (t < nik) {  // j = 0: the axis (the cell across it, lateral velocity mirrored) or the slip wall
    int i = (int)(t % B.ni), k = (int)(t / B.ni);
    if (i < B.axis_cells) {
      int kp = B.axis_k[i * B.nk + k];
      for (int m = 1; m <= 2; ++m) {
        V5<float> s = ldW(B, b, pidx3(B, i, m - 1, kp));
        s[2] = -s[2];
        stW(B, b, pidx3(B, i, -m, k), f2d5(s));
      }
    } else {
      float4 n = B.fj[((long long)k * (B.nj + 1)) * B.ni + i];
      for (int m = 1; m <= 2; ++m)
        stW(B, b, pidx3(B, i, -m, k), reflect3<double>(f2d5(ldW(B, b, pidx3(B, i, m - 1, k))), n.x, n.y, n.z));
    }
    return;
  }
  t -= nik;
  if (t < nik) {  // j = nj: characteristic far field
    int i = (int)(t % B.ni), k = (int)(t / B.ni);
    float4 n = B.fj[((long long)k * (B.nj + 1) + B.nj) * B.ni + i];
    V5<double> g = char_ghost3(fs3(c), f2d5(ldW(B, b, pidx3(B, i, B.nj - 1, k))), n.x, n.y, n.z);
    for (int m = 1; m <= 2; ++m) stW(B, b, pidx3(B, i, B.nj + m - 1, k), g);
    return;
  }
  t -= nik;
  if (t < 2 * nij) {  // k ends: symmetry planes
    bool hi = t >= nij;
    long long q = hi ? t - nij : t;
    int i = (int)(q % B.ni), j = (int)(q / B.ni);
    float4 n = B.fk[(hi ? (long long)B.nk * nij : 0) + (long long)j * B.ni + i];
    for (int m = 1; m <= 2; ++m) {
      int src = hi ? B.nk - m : m - 1, dst = hi ? B.nk + m - 1 : -m;
      stW(B, b, pidx3(B, i, j, dst), reflect3<double>(f2d5(ldW(B, b, pidx3(B, i, j, src))), n.x, n.y, n.z));
    }
  }
}

// face fluxes of direction dir (0 i, 1 j, 2 k), FP64, times the face area
__global__ void k3_flux(B3 B, int dir) {
  long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  const long long nf = dir == 0 ? B.nfi : dir == 1 ? B.nfj : B.nfk;
  if (f >= nf || !B.active[b]) return;
  const Case3Dev& c = B.cs[b];
  const int nfi = B.ni + (dir == 0), nfj = B.nj + (dir == 1);
  int i = (int)(f % nfi), j = (int)((f / nfi) % nfj), k = (int)(f / ((long long)nfi * nfj));
  float4 n = dir == 0 ? B.fi[f] : dir == 1 ? B.fj[f] : B.fk[f];
  double* out = (dir == 0 ? B.FI : dir == 1 ? B.FJ : B.FK) + (long long)b * 5 * nf + f;
  if (n.w == 0.f) {
#pragma unroll
    for (int q = 0; q < 5; ++q) out[q * nf] = 0.0;
    return;
  }
  float2 rot = dir == 0 ? B.ri[f] : dir == 1 ? B.rj[f] : B.rk[f];
  int ei = dir == 0, ej = dir == 1, ek = dir == 2;
  auto at = [&](int s) { return f2d5(ldW(B, b, pidx3(B, i + s * ei, j + s * ej, k + s * ek))); };
  int lim = B.iter[b] < c.first_order_iters ? LIM_FIRST : c.limiter;
  V5<double> wm2 = at(-2), wm1 = at(-1), wp0 = at(0), wp1 = at(1);
  if (B.solid) {  // solver3.rs:362-405: a solid cell is a slip wall of its fluid neighbour
    auto sol = [&](int s) { return sol3(B, i + s * ei, j + s * ej, k + s * ek); };
    const bool sm1 = sol(-1), sp0 = sol(0);
    if (sm1 && sp0) {
#pragma unroll
      for (int q = 0; q < 5; ++q) out[q * nf] = 0.0;
      return;
    }
    if (sm1) {
      wm1 = reflect3<double>(wp0, n.x, n.y, n.z);
      wm2 = sol(1) ? wm1 : reflect3<double>(wp1, n.x, n.y, n.z);
    } else if (sp0) {
      wp0 = reflect3<double>(wm1, n.x, n.y, n.z);
      wp1 = sol(-2) ? wp0 : reflect3<double>(wm2, n.x, n.y, n.z);
    } else {
      const float4* fam = dir == 0 ? B.fi : dir == 1 ? B.fj : B.fk;
      const long long fs = dir == 0 ? 1 : dir == 1 ? nfi : (long long)nfi * nfj;
      if (sol(-2)) {
        const float4 m = fam[f - fs];
        wm2 = reflect3<double>(wm1, m.x, m.y, m.z);
      }
      if (sol(1)) {
        const float4 m = fam[f + fs];
        wp1 = reflect3<double>(wp0, m.x, m.y, m.z);
      }
    }
  }
  V5<double> fl = face_flux_lm3(wm2, wm1, wp0, wp1, lim, n.x, n.y, n.z, rot.x, rot.y, c.low_mach != 0);
  double area = n.w;
#pragma unroll
  for (int q = 0; q < 5; ++q) out[q * nf] = fl[q] * area;
}

// cell residual (FP64 sums, stored FP32), the local time step (dt_kind 1 explicit CFL, 2 implicit ramp), the density norm
__global__ void k3_residual(B3 B, int dt_kind, int slot) {
  __shared__ double sred[8];
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  if (!B.active[b]) return;
  const Case3Dev& cs = B.cs[b];
  double rr = 0.0;
  if (c < B.nc && B.solid && B.solid[c]) {  // solver3.rs:251-254, 281-284: zero residual and time step
    stU(B, B.R, b, c, V5<float>{{0.f, 0.f, 0.f, 0.f, 0.f}});
    if (dt_kind) B.dt[(long long)b * B.nc + c] = 0.f;
  } else if (c < B.nc) {
    int i = (int)(c % B.ni), j = (int)((c / B.ni) % B.nj), k = (int)(c / ((long long)B.ni * B.nj));
    long long il = ((long long)k * B.nj + j) * (B.ni + 1) + i, jl = ((long long)k * (B.nj + 1) + j) * B.ni + i, kl = c;
    long long ir = il + 1, jr = jl + B.ni, kr = c + (long long)B.ni * B.nj;
    const double *FI = B.FI + (long long)b * 5 * B.nfi, *FJ = B.FJ + (long long)b * 5 * B.nfj, *FK = B.FK + (long long)b * 5 * B.nfk;
    double inv_v = 1.0 / (double)B.vol[c];
    V5<float> r;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      double s = -((FI[q * B.nfi + ir] - FI[q * B.nfi + il]) + (FJ[q * B.nfj + jr] - FJ[q * B.nfj + jl]) + (FK[q * B.nfk + kr] - FK[q * B.nfk + kl])) * inv_v;
      r[q] = (float)s;
      if (q == 0) rr = s * s;
    }
    stU(B, B.R, b, c, r);
    if (dt_kind) {
      V5<float> w = ldW(B, b, pidx3(B, i, j, k));
      float csnd = sqrtf(1.4f * w[4] / w[0]);
      auto lam = [&](float4 f) { return (fabsf(w[1] * f.x + w[2] * f.y + w[3] * f.z) + csnd) * f.w; };
      float li = 0.5f * (lam(B.fi[il]) + lam(B.fi[ir])), lj = 0.5f * (lam(B.fj[jl]) + lam(B.fj[jr])), lk = 0.5f * (lam(B.fk[kl]) + lam(B.fk[kr]));
      float cfl = cs.cfl;
      int mode = 0;
      if (dt_kind == 2) {
        int rk = B.ramp[b];
        cfl = (float)fmin((double)cs.cfl0 * pow((double)cs.growth, (double)(rk < 10000 ? rk : 10000)), (double)cs.cfl_max);
        mode = cs.dt_mode;
      }
      float v = B.vol[c];
      B.dt[(long long)b * B.nc + c] = mode == 0 ? cfl * v / (li + lj + lk) : cfl * v / (3.f * fminf(fminf(li, lj), lk));
    }
  }
  if (slot >= 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rr += __shfl_down_sync(0xffffffffu, rr, o);
    if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = rr;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += sred[q];
      atomicAdd(&B.rsum[(long long)slot * B.nb + b], s);
    }
  }
}

__global__ void k3_stage(B3 B, float a, float bb, int copy, int last) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  if (c >= B.nc || !B.active[b]) return;
  if (last && c == 0) B.iter[b] += 1;
  if (B.solid && B.solid[c]) return;  // solver3.rs:317-327: fluid cells only
  V5<float> u = ldU(B, B.U, b, c);
  if (copy) stU(B, B.U0, b, c, u);
  V5<float> u0 = copy ? u : ldU(B, B.U0, b, c);
  V5<float> r = ldU(B, B.R, b, c);
  float d = B.dt[(long long)b * B.nc + c];
#pragma unroll
  for (int q = 0; q < 5; ++q) u[q] = a * (u[q] + d * r[q]) + bb * u0[q];
  stU(B, B.U, b, c, u);
}

// blocks (lo, d, up) of I - dt J_dir of cell (i, j, k) with the line-end ghost Jacobians folded in (implicit3.rs:214-355)
__device__ void blocks3(const B3& B, int b, int dir, int i, int j, int k, M5<float>& lo, M5<float>& d, M5<float>& up) {
  const Case3Dev& cs = B.cs[b];
  const int ei = dir == 0, ej = dir == 1, ek = dir == 2;
  const int m = dir == 0 ? i : dir == 1 ? j : k, nl = dir == 0 ? B.ni : dir == 1 ? B.nj : B.nk;
  const long long c = cell3(B, i, j, k);
  float4 fl, fr;
  if (dir == 0) {
    long long il = ((long long)k * B.nj + j) * (B.ni + 1) + i;
    fl = B.fi[il], fr = B.fi[il + 1];
  } else if (dir == 1) {
    long long jl = ((long long)k * (B.nj + 1) + j) * B.ni + i;
    fl = B.fj[jl], fr = B.fj[jl + B.ni];
  } else {
    fl = B.fk[c], fr = B.fk[c + (long long)B.ni * B.nj];
  }
  // implicit3.rs:329-332: a solid neighbour along the line enters as the reflection of this cell about the face
  const bool lower_solid = m > 0 && sol3(B, i - ei, j - ej, k - ek), upper_solid = m + 1 < nl && sol3(B, i + ei, j + ej, k + ek);
  V5<float> wk = ldW(B, b, pidx3(B, i, j, k));
  V5<float> wm = lower_solid ? reflect3<float>(wk, fl.x, fl.y, fl.z) : ldW(B, b, pidx3(B, i - ei, j - ej, k - ek));
  V5<float> wp = upper_solid ? reflect3<float>(wk, fr.x, fr.y, fr.z) : ldW(B, b, pidx3(B, i + ei, j + ej, k + ek));
  const float s = 0.5f * B.dt[(long long)b * B.nc + c] / B.vol[c], al = fl.w, ar = fr.w;
  M5<float> dl, dr;
  if (cs.roe) {
    dl = abs_jacobian3(wm, wk, fl.x, fl.y, fl.z, cs.eps_fix);
    dr = abs_jacobian3(wk, wp, fr.x, fr.y, fr.z, cs.eps_fix);
    float tl = shock_weight<float>(wm[4], wk[4]), tr = shock_weight<float>(wk[4], wp[4]);
    if (tl > 0.f || tr > 0.f) {
      float lam_l = fmaxf(spectral3(wk, fl.x, fl.y, fl.z), spectral3(wm, fl.x, fl.y, fl.z));
      float lam_r = fmaxf(spectral3(wk, fr.x, fr.y, fr.z), spectral3(wp, fr.x, fr.y, fr.z));
#pragma unroll
      for (int q = 0; q < 25; ++q) dl[q] *= 1.f - tl, dr[q] *= 1.f - tr;
#pragma unroll
      for (int q = 0; q < 5; ++q) dl[6 * q] += tl * lam_l, dr[6 * q] += tr * lam_r;
    }
  } else {
    float lam_l = fmaxf(spectral3(wk, fl.x, fl.y, fl.z), spectral3(wm, fl.x, fl.y, fl.z));
    float lam_r = fmaxf(spectral3(wk, fr.x, fr.y, fr.z), spectral3(wp, fr.x, fr.y, fr.z));
    dl = zero5(), dr = zero5();
#pragma unroll
    for (int q = 0; q < 5; ++q) dl[6 * q] = lam_l, dr[6 * q] = lam_r;
  }
  d = eye5();
  axpy5(d, s * ar, flux_jacobian3(wk, fr.x, fr.y, fr.z));
  axpy5(d, -s * al, flux_jacobian3(wk, fl.x, fl.y, fl.z));
  axpy5(d, s * ar, dr);
  axpy5(d, s * al, dl);
  if (!cs.lines) {
    lo = zero5(), up = zero5();
    return;
  }
  lo = flux_jacobian3(wm, fl.x, fl.y, fl.z);
  axpy5(lo, 1.f, dl);
#pragma unroll
  for (int q = 0; q < 25; ++q) lo[q] *= -s * al;
  up = flux_jacobian3(wp, fr.x, fr.y, fr.z);
  axpy5(up, -1.f, dr);
#pragma unroll
  for (int q = 0; q < 25; ++q) up[q] *= s * ar;
  // ghost Jacobians: far field (i ends, j = nj) frozen, T = 0; the axis frozen; slip wall and symmetry planes reflect
  if (m == 0) {
    bool refl = cs.implicit_bc && ((dir == 1 && i >= B.axis_cells) || dir == 2);
    if (refl) axpy5(d, 1.f, mm5(lo, reflection3(fl.x, fl.y, fl.z)));
    lo = zero5();
  } else if (lower_solid) {  // implicit3.rs:338-345: B T folded into the diagonal, the line cut
    axpy5(d, 1.f, mm5(lo, reflection3(fl.x, fl.y, fl.z)));
    lo = zero5();
  }
  if (m == nl - 1) {
    if (cs.implicit_bc && dir == 2) axpy5(d, 1.f, mm5(up, reflection3(fr.x, fr.y, fr.z)));
    up = zero5();
  } else if (upper_solid) {
    axpy5(d, 1.f, mm5(up, reflection3(fr.x, fr.y, fr.z)));
    up = zero5();
  }
}

__device__ __forceinline__ void damped_update3(const B3& B, int b, long long c, const V5<float>& dq) {  // implicit3.rs:456-469
  V5<float> u = ldU(B, B.U, b, c);
  float alpha = 1.f;
  for (int t = 0; t < 8; ++t) {
    V5<float> q;
#pragma unroll
    for (int m = 0; m < 5; ++m) q[m] = u[m] + alpha * dq[m];
    V5<float> w = cons_to_prim3<float>(q);
    bool fin = true;
#pragma unroll
    for (int m = 0; m < 5; ++m) fin = fin && isfinite(q[m]);
    if (w[0] > 0.f && w[4] > 0.f && fin) {
      stU(B, B.U, b, c, q);
      return;
    }
    alpha *= 0.5f;
  }
}

// Line records of case b, direction dir, in a region of 130 planes of ncell floats: the blocks lo (25), d (25), up (25)
// assembled by k3_assemble and the factors M^-1 (25), Y = M^-1 up (25) of the factorising pass as 125 planes of ncell
// FP16 values at the start of the region (half its first 125 float planes), and g (5 FP32 planes from plane R_G), the
// forward sweep of the current right-hand side. FP16 halves the bytes the assembly writes and the line passes and the
// defect read; the blocks and factors only precondition the defect correction (the fixed point is the residual's), and
// their entries (the blocks of I - dt J at CFL <= 10, the inverse and the Y of a diagonally dominant block) lie far
// inside FP16's range.
constexpr int REC3 = 130, R_LO = 0, R_D = 25, R_UP = 50, R_MINV = 75, R_Y = 100, R_G = 125;
__device__ __forceinline__ float* rec3(const B3& B, int b, int dir) { return B.scr + ((long long)b * 3 + dir) * REC3 * B.nc; }
__device__ __forceinline__ __half* rec3h(const B3& B, int b, int dir) { return reinterpret_cast<__half*>(rec3(B, b, dir)); }
// Index of cell (i, j, k) in the records of direction dir: the i-direction records are transposed (j fastest) so that the
// threads of neighbouring i lines, which walk the lines side by side, read neighbouring addresses.
__device__ __forceinline__ long long rcell(const B3& B, int dir, int i, int j, int k) {
  return dir == 0 ? ((long long)k * B.ni + i) * B.nj + j : cell3(B, i, j, k);
}
__device__ __forceinline__ M5<float> ld5(const float* p, long long stride) {
  M5<float> m;
#pragma unroll
  for (int q = 0; q < 25; ++q) m[q] = p[q * stride];
  return m;
}
__device__ __forceinline__ void st5(float* p, long long stride, const M5<float>& m) {
#pragma unroll
  for (int q = 0; q < 25; ++q) p[q * stride] = m[q];
}
__device__ __forceinline__ M5<float> ld5(const __half* p, long long stride) {
  M5<float> m;
#pragma unroll
  for (int q = 0; q < 25; ++q) m[q] = __half2float(p[q * stride]);
  return m;
}
__device__ __forceinline__ void st5(__half* p, long long stride, const M5<float>& m) {
#pragma unroll
  for (int q = 0; q < 25; ++q) p[q * stride] = __float2half_rn(m[q]);
}

// Blocks of every cell into the line records (thread per cell). part 0: the i direction, threads ordered j fastest so that
// the transposed i records are written side by side; part 1: the j and k directions, threads ordered i fastest.
__global__ void __launch_bounds__(128, 4) k3_assemble(B3 B, int part) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  if (t >= B.nc || !B.active[b]) return;
  int i, j, k;
  if (part == 0) {
    j = (int)(t % B.nj), i = (int)((t / B.nj) % B.ni), k = (int)(t / ((long long)B.ni * B.nj));
  } else {
    i = (int)(t % B.ni), j = (int)((t / B.ni) % B.nj), k = (int)(t / ((long long)B.ni * B.nj));
  }
  const bool solid = B.solid && B.solid[cell3(B, i, j, k)];
#pragma unroll 1
  for (int dir = part == 0 ? 0 : 1; dir < (part == 0 ? 1 : 3); ++dir) {
    M5<float> lo, d, up;
    if (solid)  // implicit3.rs:311-314: the identity row
      lo = zero5(), d = eye5(), up = zero5();
    else
      blocks3(B, b, dir, i, j, k, lo, d, up);
    __half* r = rec3h(B, b, dir) + rcell(B, dir, i, j, k);
    st5(r + R_LO * B.nc, B.nc, lo);
    st5(r + R_D * B.nc, B.nc, d);
    st5(r + R_UP * B.nc, B.nc, up);
  }
}

// line of direction dir through line index L: first cell, cell stride, length
__device__ __forceinline__ void line3(const B3& B, int dir, long long L, long long& c0, long long& stride, int& n, long long& r0,
                                      long long& rstride) {
  int i0, j0, k0;
  if (dir == 0) i0 = 0, j0 = (int)(L % B.nj), k0 = (int)(L / B.nj);
  else if (dir == 1) i0 = (int)(L % B.ni), j0 = 0, k0 = (int)(L / B.ni);
  else i0 = (int)(L % B.ni), j0 = (int)(L / B.ni), k0 = 0;
  n = dir == 0 ? B.ni : dir == 1 ? B.nj : B.nk;
  stride = dir == 0 ? 1 : dir == 1 ? B.ni : (long long)B.ni * B.nj;
  c0 = cell3(B, i0, j0, k0);
  r0 = rcell(B, dir, i0, j0, k0);
  rstride = dir == 0 ? B.nj : stride;
}
__device__ __forceinline__ long long nlines3(const B3& B, int dir) {
  return dir == 0 ? (long long)B.nj * B.nk : dir == 1 ? (long long)B.ni * B.nk : (long long)B.ni * B.nj;
}

// x of cell c: epilogue 0: x -> out; 1: du = x; 2: du += x; `update` applies the damped update
__device__ __forceinline__ void emit3(const B3& B, int b, int epilogue, bool update, float* out, long long c, const V5<float>& x) {
  if (epilogue == 0) {
    stU(B, out, b, c, x);
    return;
  }
  V5<float> du = x;
  if (epilogue == 2) {
    V5<float> o = ldU(B, B.DU, b, c);
#pragma unroll
    for (int q = 0; q < 5; ++q) du[q] += o[q];
  }
  stU(B, B.DU, b, c, du);
  if (update && !(B.solid && B.solid[c])) damped_update3(B, b, c, du);
}

// First pass of an iteration, one thread per line: block Thomas on the kept blocks (implicit3.rs:133-156), keeping M^-1,
// Y and g for the defect-correction passes. in: the right-hand side (from_res: dt R).
__global__ void __launch_bounds__(64) k3_lines(B3 B, int dir, const float* in, int from_res, float* out, int epilogue) {
  long long L = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  if (L >= nlines3(B, dir) || !B.active[b]) return;
  const Case3Dev& cs = B.cs[b];
  const bool update = epilogue != 0 && (cs.sub_iters > 1 ? cs.sub_iters : 1) == 1;
  long long c0, stride, r0, rs;
  int n;
  line3(B, dir, L, c0, stride, n, r0, rs);
  float* R = rec3(B, b, dir) + r0;        // g (FP32 planes)
  __half* H = rec3h(B, b, dir) + r0;      // blocks and factors (FP16 planes)
  const long long nc = B.nc;
  M5<float> Y = zero5();
  V5<float> g{{0, 0, 0, 0, 0}};
  for (int m = 0; m < n; ++m) {
    long long c = c0 + m * stride, rr = m * rs;
    M5<float> d = ld5(H + R_D * nc + rr, nc);
    V5<float> r = ldU(B, in, b, c);
    if (from_res) {
      float dtc = B.dt[(long long)b * nc + c];
#pragma unroll
      for (int q = 0; q < 5; ++q) r[q] *= dtc;
    }
    if (m > 0) {
      M5<float> lo = ld5(H + R_LO * nc + rr, nc);
      axpy5(d, -1.f, mm5(lo, Y));
      V5<float> t = mv5(lo, g);
#pragma unroll
      for (int q = 0; q < 5; ++q) r[q] -= t[q];
    }
    M5<float> Minv = inv5(d);
    g = mv5(Minv, r);
    Y = mm5(Minv, ld5(H + R_UP * nc + rr, nc));
    st5(H + R_MINV * nc + rr, nc, Minv);
    st5(H + R_Y * nc + rr, nc, Y);
#pragma unroll
    for (int q = 0; q < 5; ++q) R[(R_G + q) * nc + rr] = g[q];
  }
  V5<float> xn = g;
  emit3(B, b, epilogue, update, out, c0 + (long long)(n - 1) * stride, xn);
  for (int m = n - 2; m >= 0; --m) {
    long long c = c0 + m * stride, rr = m * rs;
    M5<float> Ym = ld5(H + R_Y * nc + rr, nc);
    V5<float> gm;
#pragma unroll
    for (int q = 0; q < 5; ++q) gm[q] = R[(R_G + q) * nc + rr];
    V5<float> t = mv5(Ym, xn);
#pragma unroll
    for (int q = 0; q < 5; ++q) gm[q] -= t[q];
    emit3(B, b, epilogue, update, out, c, gm);
    xn = gm;
  }
  if (update && L == 0) B.iter[b] += 1, B.ramp[b] += 1;
}

// cp.async helpers of the staged line walk (16-byte chunks, bypassing L1)
__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpa_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// The first pass with the walk staged through shared memory: one warp per block walks 32 adjacent lines, whose records
// are adjacent in every plane, and the blocks lo, d, up of step m + 2 (75 FP16 planes, 64 bytes per plane and step) are
// copied by cp.async while step m is computed; the right-hand side and time step of step m + 1 are loaded into registers
// before the arithmetic of step m (for the i lines they are strided by ni across the lanes). The loads of the unstaged
// walk cannot move above the previous step's stores of M^-1 and Y, so every step of it waits a memory latency; the
// arithmetic here is the same, in the same order, so the results are the unstaged kernel's bit for bit. One warp per
// block and 14.4 KB of stages let 14 blocks share an SM, all the i lines of the 15-case sweep batch in one wave. The host
// runs it where the lines of a warp are adjacent, which also aligns every copy to 16 bytes (Batch3::staged_ok).
constexpr int ST3N = 3;  // stages: the copies run two steps ahead
struct Stage3 {
  __half blk[75][32];  // planes R_LO .. R_UP + 24 of the warp's 32 lines
};
__global__ void __launch_bounds__(32) k3_lines_st(B3 B, int dir, const float* in, int from_res, float* out, int epilogue) {
  __shared__ __align__(16) Stage3 S[ST3N];
  const long long L = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = B.b0 + (int)blockIdx.y, lane = threadIdx.x & 31;
  if (L >= nlines3(B, dir) || !B.active[b]) return;  // whole warps: the host launches it for line counts in multiples of 32
  const Case3Dev& cs = B.cs[b];
  const bool update = epilogue != 0 && (cs.sub_iters > 1 ? cs.sub_iters : 1) == 1;
  long long c0, stride, r0, rs;
  int n;
  line3(B, dir, L, c0, stride, n, r0, rs);
  float* R = rec3(B, b, dir) + r0;
  __half* H = rec3h(B, b, dir) + r0;
  const long long nc = B.nc;
  const __half* Hw = rec3h(B, b, dir) + (r0 - lane);  // lane 0's records: the lanes' records are adjacent
  auto issue = [&](int m) {
    if (m < n) {
      Stage3& st = S[m % ST3N];
      const long long rr = (long long)m * rs;
      for (int t = lane; t < 75 * 4; t += 32) {
        const int q = t >> 2, ch = t & 3;
        cpa16(&st.blk[q][8 * ch], Hw + (long long)(R_LO + q) * nc + rr + 8 * ch);
      }
    }
    cpa_commit();
  };
  auto rhs = [&](int m, V5<float>& r, float& dtc) {
    const long long c = c0 + (long long)m * stride;
    r = ldU(B, in, b, c);
    dtc = from_res ? B.dt[(long long)b * nc + c] : 1.f;
  };
  issue(0);
  issue(1);
  V5<float> r_n;
  float dt_n;
  rhs(0, r_n, dt_n);
  M5<float> Y = zero5();
  V5<float> g{{0, 0, 0, 0, 0}};
  for (int m = 0; m < n; ++m) {
    cpa_wait1();  // the copies of step m are done (those of step m + 1 may still run)
    __syncwarp();
    issue(m + 2);  // into the stage step m - 1 used, which every lane has finished with
    const Stage3& st = S[m % ST3N];
    const long long rr = (long long)m * rs;
    V5<float> r = r_n;
    const float dtc = dt_n;
    if (m + 1 < n) rhs(m + 1, r_n, dt_n);
    M5<float> d;
#pragma unroll
    for (int q = 0; q < 25; ++q) d[q] = __half2float(st.blk[R_D + q][lane]);
    if (from_res) {
#pragma unroll
      for (int q = 0; q < 5; ++q) r[q] *= dtc;
    }
    if (m > 0) {
      M5<float> lo;
#pragma unroll
      for (int q = 0; q < 25; ++q) lo[q] = __half2float(st.blk[R_LO + q][lane]);
      axpy5(d, -1.f, mm5(lo, Y));
      V5<float> t = mv5(lo, g);
#pragma unroll
      for (int q = 0; q < 5; ++q) r[q] -= t[q];
    }
    M5<float> Minv = inv5(d);
    g = mv5(Minv, r);
    M5<float> up;
#pragma unroll
    for (int q = 0; q < 25; ++q) up[q] = __half2float(st.blk[R_UP + q][lane]);
    Y = mm5(Minv, up);
    st5(H + R_MINV * nc + rr, nc, Minv);
    st5(H + R_Y * nc + rr, nc, Y);
#pragma unroll
    for (int q = 0; q < 5; ++q) R[(R_G + q) * nc + rr] = g[q];
  }
  V5<float> xn = g;
  emit3(B, b, epilogue, update, out, c0 + (long long)(n - 1) * stride, xn);
  for (int m = n - 2; m >= 0; --m) {
    long long c = c0 + m * stride, rr = m * rs;
    M5<float> Ym = ld5(H + R_Y * nc + rr, nc);
    V5<float> gm;
#pragma unroll
    for (int q = 0; q < 5; ++q) gm[q] = R[(R_G + q) * nc + rr];
    V5<float> t = mv5(Ym, xn);
#pragma unroll
    for (int q = 0; q < 5; ++q) gm[q] -= t[q];
    emit3(B, b, epilogue, update, out, c, gm);
    xn = gm;
  }
  if (update && L == 0) B.iter[b] += 1, B.ramp[b] += 1;
}

// The defect-correction pass staged as k3_lines_st: the forward walk copies lo and M^-1 of step m + 2 (50 FP16 planes),
// the backward walk Y of step m - 2 (25 planes), by cp.async into shared memory while it computes step m; the
// right-hand side and g are loaded into registers one step ahead. Same arithmetic, same order: the results are
// k3_lines_subst's bit for bit.
struct StageS3 {
  __half blk[50][32];  // forward: lo (0..24), M^-1 (25..49); backward: Y (0..24)
};
__global__ void __launch_bounds__(32) k3_lines_subst_st(B3 B, int dir, const float* in, float* out, int epilogue, int pass) {
  __shared__ __align__(16) StageS3 S[ST3N];
  const long long L = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = B.b0 + (int)blockIdx.y, lane = threadIdx.x & 31;
  if (L >= nlines3(B, dir) || !B.active[b]) return;  // whole warps
  const Case3Dev& cs = B.cs[b];
  const int s = cs.sub_iters > 1 ? cs.sub_iters : 1;
  if (pass >= s) return;
  const bool update = epilogue != 0 && pass == s - 1;
  long long c0, stride, r0, rs;
  int n;
  line3(B, dir, L, c0, stride, n, r0, rs);
  float* R = rec3(B, b, dir) + r0;
  const long long nc = B.nc;
  const __half* Hw = rec3h(B, b, dir) + (r0 - lane);
  auto issue_f = [&](int m) {  // lo and M^-1 of step m
    if (m < n) {
      StageS3& st = S[m % ST3N];
      const long long rr = (long long)m * rs;
      for (int t = lane; t < 50 * 4; t += 32) {
        const int q = t >> 2, ch = t & 3;
        const int plane = q < 25 ? R_LO + q : R_MINV + (q - 25);
        cpa16(&st.blk[q][8 * ch], Hw + (long long)plane * nc + rr + 8 * ch);
      }
    }
    cpa_commit();
  };
  auto issue_b = [&](int m, int k) {  // Y of step m into stage k
    if (m >= 0) {
      StageS3& st = S[k % ST3N];
      const long long rr = (long long)m * rs;
      for (int t = lane; t < 25 * 4; t += 32) {
        const int q = t >> 2, ch = t & 3;
        cpa16(&st.blk[q][8 * ch], Hw + (long long)(R_Y + q) * nc + rr + 8 * ch);
      }
    }
    cpa_commit();
  };
  issue_f(0);
  issue_f(1);
  V5<float> g{{0, 0, 0, 0, 0}};
  V5<float> r_n = ldU(B, in, b, c0);
  for (int m = 0; m < n; ++m) {
    cpa_wait1();
    __syncwarp();
    issue_f(m + 2);
    const StageS3& st = S[m % ST3N];
    const long long rr = (long long)m * rs;
    V5<float> r = r_n;
    if (m + 1 < n) r_n = ldU(B, in, b, c0 + (m + 1) * stride);
    if (m > 0) {
      M5<float> lo;
#pragma unroll
      for (int q = 0; q < 25; ++q) lo[q] = __half2float(st.blk[q][lane]);
      V5<float> t = mv5(lo, g);
#pragma unroll
      for (int q = 0; q < 5; ++q) r[q] -= t[q];
    }
    M5<float> mi;
#pragma unroll
    for (int q = 0; q < 25; ++q) mi[q] = __half2float(st.blk[25 + q][lane]);
    g = mv5(mi, r);
#pragma unroll
    for (int q = 0; q < 5; ++q) R[(R_G + q) * nc + rr] = g[q];
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");  // the forward walk's trailing (empty) groups
  __syncwarp();  // every lane's g stores and reads of the stages are done before the backward walk reuses them
  V5<float> xn = g;
  emit3(B, b, epilogue, update, out, c0 + (long long)(n - 1) * stride, xn);
  if (n >= 2) {
    // backward step k = 0, 1, ... handles cell m = n - 2 - k; its Y goes through stage k
    issue_b(n - 2, 0);
    issue_b(n - 3, 1);
    V5<float> g_n;
#pragma unroll
    for (int q = 0; q < 5; ++q) g_n[q] = R[(R_G + q) * nc + (n - 2) * rs];
    for (int k = 0, m = n - 2; m >= 0; ++k, --m) {
      cpa_wait1();
      __syncwarp();
      issue_b(m - 2, k + 2);
      const StageS3& st = S[k % ST3N];
      const long long c = c0 + m * stride;
      M5<float> ym;
#pragma unroll
      for (int q = 0; q < 25; ++q) ym[q] = __half2float(st.blk[q][lane]);
      V5<float> gm = g_n;
      if (m > 0) {
#pragma unroll
        for (int q = 0; q < 5; ++q) g_n[q] = R[(R_G + q) * nc + (m - 1) * rs];
      }
      V5<float> t = mv5(ym, xn);
#pragma unroll
      for (int q = 0; q < 5; ++q) gm[q] -= t[q];
      emit3(B, b, epilogue, update, out, c, gm);
      xn = gm;
    }
  }
  if (update && L == 0) B.iter[b] += 1, B.ramp[b] += 1;
}

// Defect-correction pass `pass` >= 1: the same line solve with the kept factors (forward g = M^-1 (r - lo g_prev),
// backward x = g - Y x_next).
__global__ void __launch_bounds__(128) k3_lines_subst(B3 B, int dir, const float* in, float* out, int epilogue, int pass) {
  long long L = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  if (L >= nlines3(B, dir) || !B.active[b]) return;
  const Case3Dev& cs = B.cs[b];
  const int s = cs.sub_iters > 1 ? cs.sub_iters : 1;
  if (pass >= s) return;
  const bool update = epilogue != 0 && pass == s - 1;
  long long c0, stride, r0, rs;
  int n;
  line3(B, dir, L, c0, stride, n, r0, rs);
  float* R = rec3(B, b, dir) + r0;        // g (FP32 planes)
  __half* H = rec3h(B, b, dir) + r0;      // blocks and factors (FP16 planes)
  const long long nc = B.nc;
  // both walks load the next cell's factors before the arithmetic of the current one (software pipelining)
  V5<float> g{{0, 0, 0, 0, 0}};
  M5<float> lo_n = ld5(H + R_LO * nc, nc), mi_n = ld5(H + R_MINV * nc, nc);
  V5<float> r_n = ldU(B, in, b, c0);
  for (int m = 0; m < n; ++m) {
    const long long rr = m * rs;
    const M5<float> lo = lo_n, mi = mi_n;
    V5<float> r = r_n;
    if (m + 1 < n) {
      const long long rn = (m + 1) * rs;
      lo_n = ld5(H + R_LO * nc + rn, nc), mi_n = ld5(H + R_MINV * nc + rn, nc);
      r_n = ldU(B, in, b, c0 + (m + 1) * stride);
    }
    if (m > 0) {
      V5<float> t = mv5(lo, g);
#pragma unroll
      for (int q = 0; q < 5; ++q) r[q] -= t[q];
    }
    g = mv5(mi, r);
#pragma unroll
    for (int q = 0; q < 5; ++q) R[(R_G + q) * nc + rr] = g[q];
  }
  V5<float> xn = g;
  emit3(B, b, epilogue, update, out, c0 + (long long)(n - 1) * stride, xn);
  if (n >= 2) {
    M5<float> y_n = ld5(H + R_Y * nc + (n - 2) * rs, nc);
    V5<float> g_n;
#pragma unroll
    for (int q = 0; q < 5; ++q) g_n[q] = R[(R_G + q) * nc + (n - 2) * rs];
    for (int m = n - 2; m >= 0; --m) {
      const long long c = c0 + m * stride;
      const M5<float> ym = y_n;
      V5<float> gm = g_n;
      if (m > 0) {
        const long long rn = (m - 1) * rs;
        y_n = ld5(H + R_Y * nc + rn, nc);
#pragma unroll
        for (int q = 0; q < 5; ++q) g_n[q] = R[(R_G + q) * nc + rn];
      }
      V5<float> t = mv5(ym, xn);
#pragma unroll
      for (int q = 0; q < 5; ++q) gm[q] -= t[q];
      emit3(B, b, epilogue, update, out, c, gm);
      xn = gm;
    }
  }
  if (update && L == 0) B.iter[b] += 1, B.ramp[b] += 1;
}

// A_dir du of cell (i, j, k) with the kept blocks of direction dir (implicit3.rs:384-410)
__device__ __forceinline__ V5<float> apply3(const B3& B, int b, int dir, int i, int j, int k, long long c, const V5<float>& du) {
  const long long nc = B.nc;
  const __half* H = rec3h(B, b, dir) + rcell(B, dir, i, j, k);
  const int m = dir == 0 ? i : dir == 1 ? j : k, nl = dir == 0 ? B.ni : dir == 1 ? B.nj : B.nk;
  const long long stride = dir == 0 ? 1 : dir == 1 ? B.ni : (long long)B.ni * B.nj;
  V5<float> v = mv5(ld5(H + R_D * nc, nc), du);
  if (m > 0) {
    V5<float> t = mv5(ld5(H + R_LO * nc, nc), ldU(B, B.DU, b, c - stride));
#pragma unroll
    for (int q = 0; q < 5; ++q) v[q] += t[q];
  }
  if (m + 1 < nl) {
    V5<float> t = mv5(ld5(H + R_UP * nc, nc), ldU(B, B.DU, b, c + stride));
#pragma unroll
    for (int q = 0; q < 5; ++q) v[q] += t[q];
  }
  return v;
}

// the i-direction product A_i du into X (free between passes), threads ordered j fastest like the transposed i records
__global__ void __launch_bounds__(128) k3_defect_i(B3 B, int pass) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  if (t >= B.nc || !B.active[b] || pass >= B.cs[b].sub_iters) return;
  int j = (int)(t % B.nj), i = (int)((t / B.nj) % B.ni), k = (int)(t / ((long long)B.ni * B.nj));
  long long c = cell3(B, i, j, k);
  stU(B, B.X, b, c, apply3(B, b, 0, i, j, k, c, ldU(B, B.DU, b, c)));
}

// defect of the unfactored operator (implicit3.rs:440-446): rr = dt R - (A_i du + A_j du + A_k du - 2 du), A_i du from X
__global__ void __launch_bounds__(128) k3_defect(B3 B, int pass) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int b = B.b0 + (int)blockIdx.y;
  if (c >= B.nc || !B.active[b]) return;
  const Case3Dev& cs = B.cs[b];
  if (pass >= cs.sub_iters) return;
  int i = (int)(c % B.ni), j = (int)((c / B.ni) % B.nj), k = (int)(c / ((long long)B.ni * B.nj));
  V5<float> du = ldU(B, B.DU, b, c);
  V5<float> acc = ldU(B, B.X, b, c);
#pragma unroll 1
  for (int dir = 1; dir < 3; ++dir) {
    V5<float> v = apply3(B, b, dir, i, j, k, c, du);
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[q] += v[q];
  }
  V5<float> r = ldU(B, B.R, b, c);
  float d = B.dt[(long long)b * B.nc + c];
  V5<float> o;
#pragma unroll
  for (int q = 0; q < 5; ++q) o[q] = r[q] * d - (acc[q] - 2.f * du[q]);
  stU(B, B.RR, b, c, o);
}

// the conserved states of case b at the listed cells, 5 per cell in Cons3 order (GpuSolver3::read_boundary_into)
__global__ void k3_gather(B3 B, int b, const long long* cells, int n, double* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const V5<float> u = ldU(B, B.U, b, cells[q]);
#pragma unroll
  for (int v = 0; v < 5; ++v) out[5 * (long long)q + v] = u[v];
}

// FP64 wall forces of every case (run3.rs:130-212): one block per case. wall: WALL3 doubles per wall face, the j = 0 body
// faces (i >= axis_cells, fluid cells) and every face between a fluid and a solid cell: n[3], area, c[3], the centroid of
// the first fluid cell a and of the fluid cell b behind it, a, b (-1: none), the sign that turns n into the body, and the
// part of the surface (0 body wall, 2 fin sides (k faces), 3 fin edges (i faces), 4 fin tips (j faces)).
constexpr int WALL3 = 17;
// the wall pressure of face record w of case b (run3.rs:150-160): extrapolated from the first two fluid cells
__device__ __forceinline__ double wall_pressure3(const B3& B, int b, const double* w) {
  auto pres = [&](long long cc) {
    const float* p = B.U + (long long)b * 5 * B.nc + cc;
    double rho = p[0], u = p[B.nc] / rho, v = p[2 * B.nc] / rho, ww = p[3 * B.nc] / rho;
    return (GD - 1.0) * ((double)p[4 * B.nc] - 0.5 * rho * (u * u + v * v + ww * ww));
  };
  const long long ca = (long long)w[13], cb = (long long)w[14];
  double p0 = pres(ca), pw = p0;
  if (cb >= 0) {
    double d0 = sqrt((w[7] - w[4]) * (w[7] - w[4]) + (w[8] - w[5]) * (w[8] - w[5]) + (w[9] - w[6]) * (w[9] - w[6]));
    double d1 = sqrt((w[10] - w[4]) * (w[10] - w[4]) + (w[11] - w[5]) * (w[11] - w[5]) + (w[12] - w[6]) * (w[12] - w[6]));
    pw = p0 + (p0 - pres(cb)) * d0 / (d1 - d0);
  }
  return pw;
}
// run3.rs:85-127 `breakdown_on`: the forces of every case split into nose (body wall with centroid x <= x_nose),
// afterbody, fin sides, fin edges and fin tips; out: (cn, ca, x_cp) x 5 parts x cases
__global__ void k3_forces_parts(B3 B, const double* wall, int nwall, double x_max, double x_nose, double* out) {
  __shared__ double acc[15][128];
  int b = blockIdx.x;
  double p_inf = B.cs[b].fs[4];
  double a[15];
#pragma unroll
  for (int q = 0; q < 15; ++q) a[q] = 0.0;
  for (int q = threadIdx.x; q < nwall; q += blockDim.x) {
    const double* w = wall + WALL3 * (long long)q;
    if (w[4] > x_max) continue;
    int part = (int)w[16];
    if (part == 0 && w[4] > x_nose) part = 1;
    const double dd = (wall_pressure3(B, b, w) - p_inf) * w[3] * w[15];
#pragma unroll
    for (int k = 0; k < 5; ++k)
      if (k == part) a[3 * k] += dd * w[0], a[3 * k + 1] += dd * w[2], a[3 * k + 2] += dd * w[2] * w[4];
  }
#pragma unroll
  for (int q = 0; q < 15; ++q) acc[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int q = 0; q < 15; ++q) acc[q][threadIdx.x] += acc[q][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 5) {
    const int k = threadIdx.x;
    double mach = sqrt(B.cs[b].fs[1] * B.cs[b].fs[1] + B.cs[b].fs[3] * B.cs[b].fs[3]);
    double norm = 2.0 / (0.5 * mach * mach * (M_PI / 4.0));
    const double fx = acc[3 * k][0], fz = acc[3 * k + 1][0], mz = acc[3 * k + 2][0];
    out[15 * b + 3 * k] = norm * fz;
    out[15 * b + 3 * k + 1] = norm * fx;
    out[15 * b + 3 * k + 2] = fabs(fz) < 1e-12 ? NAN : mz / fz;
  }
}
__global__ void k3_forces(B3 B, const double* wall, int nwall, double x_max, double* out) {
  __shared__ double acc[3][256];
  int b = blockIdx.x;
  double p_inf = B.cs[b].fs[4];
  double fx = 0, fz = 0, mz = 0;
  for (int q = threadIdx.x; q < nwall; q += blockDim.x) {
    const double* w = wall + WALL3 * (long long)q;
    if (w[4] > x_max) continue;
    auto pres = [&](long long cc) {
      const float* p = B.U + (long long)b * 5 * B.nc + cc;
      double rho = p[0], u = p[B.nc] / rho, v = p[2 * B.nc] / rho, ww = p[3 * B.nc] / rho;
      return (GD - 1.0) * ((double)p[4 * B.nc] - 0.5 * rho * (u * u + v * v + ww * ww));
    };
    const long long ca = (long long)w[13], cb = (long long)w[14];
    double p0 = pres(ca), pw = p0;
    if (cb >= 0) {
      double d0 = sqrt((w[7] - w[4]) * (w[7] - w[4]) + (w[8] - w[5]) * (w[8] - w[5]) + (w[9] - w[6]) * (w[9] - w[6]));
      double d1 = sqrt((w[10] - w[4]) * (w[10] - w[4]) + (w[11] - w[5]) * (w[11] - w[5]) + (w[12] - w[6]) * (w[12] - w[6]));
      pw = p0 + (p0 - pres(cb)) * d0 / (d1 - d0);
    }
    double dd = (pw - p_inf) * w[3] * w[15];
    fx += dd * w[0];
    fz += dd * w[2];
    mz += dd * w[2] * w[4];
  }
  acc[0][threadIdx.x] = fx, acc[1][threadIdx.x] = fz, acc[2][threadIdx.x] = mz;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int q = 0; q < 3; ++q) acc[q][threadIdx.x] += acc[q][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double mach = sqrt(B.cs[b].fs[1] * B.cs[b].fs[1] + B.cs[b].fs[3] * B.cs[b].fs[3]);
    double norm = 2.0 / (0.5 * mach * mach * (M_PI / 4.0));
    out[3 * b] = norm * acc[1][0];
    out[3 * b + 1] = norm * acc[0][0];
    out[3 * b + 2] = fabs(acc[1][0]) < 1e-12 ? NAN : acc[2][0] / acc[1][0];
  }
}

}  // namespace bk3
