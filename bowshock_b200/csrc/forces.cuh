// FP64 surface-force integration on the device (crates/bowshock-core/src/engine/run.rs:188-313): wall pressure extrapolated
// linearly from the two first cells, CD = sum Cp d(r^2 / R^2) over the nose and each aft segment, base drag and area-mean
// base Cp from the two first cells behind the base, skin friction tau = mu(T) u_t / d_n and the largest first-cell y+.
// One block per case; node and centroid coordinates are kept in FP64 on the device for this pass.
#pragma once
#include "arena.cuh"
#include "device_math.cuh"

namespace bk {

constexpr int MAX_SEG = 8;
struct BodyDev {
  double nose_length, rb2, x_base;
  double stations[MAX_SEG + 1];
  int nseg;
  int has_body;
};

// output layout per case (NF doubles)
enum {
  F_CD_NOSE = 0,
  F_CD_NOSE_CELL,
  F_CD_BASE,
  F_CP_BASE,
  F_CP_BASE_CELL,
  F_CD_FRICTION,
  F_YPLUS,
  F_CD_AFT0,
  F_NF = F_CD_AFT0 + MAX_SEG
};

__device__ __forceinline__ double dpress(const Arena& A, const CaseDev& c, int i, int j) {
  V4<double> q = state_of(A, cidx(c, i, j));
  double rho = q[0], u = q[1] / rho, v = q[2] / rho;
  return 0.4 * (q[3] - 0.5 * rho * (u * u + v * v));
}

__global__ void k_forces(Arena A, const BodyDev* bodies, const double* nx, const double* nr, const long long* node_off, const double* dxc,
                         const double* drc, double* out) {
  __shared__ double acc[F_NF + 1];  // + the base area sum
  __shared__ unsigned long long yplus_bits;
  const int ci = blockIdx.x;
  const CaseDev& c = A.cases[ci];
  const BodyDev& b = bodies[ci];
  for (int k = threadIdx.x; k <= F_NF; k += blockDim.x) acc[k] = 0.0;
  if (threadIdx.x == 0) yplus_bits = 0ull;
  __syncthreads();
  const int ni = c.ni;
  const long long no = node_off[ci];
  auto X = [&](int i, int j) { return nx[no + (long long)j * (ni + 1) + i]; };
  auto R = [&](int i, int j) { return nr[no + (long long)j * (ni + 1) + i]; };
  const double p_inf = c.fs[3], q_inf = 0.5 * c.fs[0] * c.fs[1] * c.fs[1];
  auto cp = [&](double p) { return (p - p_inf) / q_inf; };
  const double rb2 = b.rb2;
  // wall distribution and segment drag (run.rs:188-199, 252-282)
  const int i_wall_end = c.has_block ? c.i_end : ni;
  for (int i = threadIdx.x; i < i_wall_end; i += blockDim.x) {
    int j0 = col_start(c, i);
    double x0 = X(i, j0), r0 = R(i, j0), x1 = X(i + 1, j0), r1 = R(i + 1, j0);
    double xm = 0.5 * (x0 + x1), rm = 0.5 * (r0 + r1);
    if (xm <= 0.0) continue;
    double p0 = dpress(A, c, i, j0), p1 = dpress(A, c, i, j0 + 1);
    long long c0 = c.cell_off + (long long)j0 * ni + i, c1 = c0 + ni;
    double d0 = hypot(dxc[c0] - xm, drc[c0] - rm), d1 = hypot(dxc[c1] - xm, drc[c1] - rm);
    double pw = p0 + (p0 - p1) * d0 / (d1 - d0);
    double s0 = r0 * r0 / rb2, s1 = r1 * r1 / rb2;
    if (x1 <= b.nose_length + 1e-12) {
      atomicAdd(&acc[F_CD_NOSE], cp(pw) * (s1 - s0));
      atomicAdd(&acc[F_CD_NOSE_CELL], cp(p0) * (s1 - s0));
    }
    for (int k = 0; k < b.nseg; ++k)
      if (xm >= b.stations[k] && xm < b.stations[k + 1]) {
        atomicAdd(&acc[F_CD_AFT0 + k], cp(pw) * (s1 - s0));
        break;
      }
  }
  // base (run.rs:286-313)
  if (c.has_block) {
    int ie = c.i_end;
    int jb = c.has_nozzle ? c.nz_j_end : c.j_sting;
    for (int j = jb + threadIdx.x; j < c.j_end; j += blockDim.x) {
      double x0 = X(ie, j), r0 = R(ie, j), r1 = R(ie, j + 1);
      double xm = x0, rm = 0.5 * (r0 + r1);
      double p0 = dpress(A, c, ie, j), p1 = dpress(A, c, ie + 1, j);
      long long c0 = c.cell_off + (long long)j * ni + ie, c1 = c0 + 1;
      double d0 = hypot(dxc[c0] - xm, drc[c0] - rm), d1 = hypot(dxc[c1] - xm, drc[c1] - rm);
      double pw = p0 + (p0 - p1) * d0 / (d1 - d0);
      double ds = (r1 * r1 - r0 * r0) / rb2;
      atomicAdd(&acc[F_CD_BASE], -cp(pw) * ds);
      atomicAdd(&acc[F_CP_BASE], cp(pw) * ds);
      atomicAdd(&acc[F_CP_BASE_CELL], cp(p0) * ds);
      atomicAdd(&acc[F_NF], ds);
    }
  }
  // skin friction and y+ (run.rs:207-248); a rough wall adds its mu_t,w (Aupoix state at the full roughness)
  if (c.viscous) {
    int rows[2] = {c.has_block ? c.j_end : 0, c.has_block ? c.j_sting : -1};
    for (int rr = 0; rr < 2; ++rr) {
      int j = rows[rr];
      if (j < 0) continue;
      for (int i = threadIdx.x; i < ni; i += blockDim.x) {
        if (!noslip_jface(c, i, j)) continue;
        double x0 = X(i, j), r0 = R(i, j), x1 = X(i + 1, j), r1 = R(i + 1, j);
        double xm = 0.5 * (x0 + x1);
        if (xm >= b.x_base) continue;
        double dx = x1 - x0, dr = r1 - r0, len = hypot(dx, dr);
        double fnx = -dr / len, fnr = dx / len, frm = 0.5 * (r0 + r1);
        long long cc = c.cell_off + (long long)j * ni + i;
        V4<double> q = state_of(A, cc);
        double rho = q[0], u = q[1] / rho, v = q[2] / rho;
        double p = 0.4 * (q[3] - 0.5 * rho * (u * u + v * v));
        double tx = fnr, tr = -fnx;
        double u_t = u * tx + v * tr;
        double d_n = fabs((dxc[cc] - xm) * fnx + (drc[cc] - frm) * fnr);
        double T = 1.4 * p / rho;
        double mu = pow(T, 1.5) * (1.0 + c.sutherland) / (T + c.sutherland) / c.re_c;
        double mu_tw = 0.0;
        if (is_rough(c)) {
          double a[3];
          aupoix_wall(mu / rho, hypot(u, v), d_n, c.roughness, a);
          mu_tw = rho * a[2];
        }
        double tau = (mu + mu_tw) * u_t / d_n;
        atomicAdd(&acc[F_CD_FRICTION], 2.0 * tau * tx * frm * len / (q_inf * rb2));
        double yp = d_n * sqrt(rho * fabs(tau)) / mu;
        atomicMax(&yplus_bits, (unsigned long long)__double_as_longlong(yp));  // yp >= 0: the bit patterns order like the values
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double* o = out + (long long)ci * F_NF;
    for (int k = 0; k < F_NF; ++k) o[k] = acc[k];
    if (c.has_block) {
      double s_sum = acc[F_NF];  // area-mean base Cp: sum Cp ds / sum ds
      o[F_CP_BASE] = acc[F_CP_BASE] / s_sum;
      o[F_CP_BASE_CELL] = acc[F_CP_BASE_CELL] / s_sum;
    } else {
      o[F_CP_BASE] = o[F_CP_BASE_CELL] = nan("");
    }
    o[F_YPLUS] = c.viscous ? __longlong_as_double((long long)yplus_bits) : nan("");
  }
}

}  // namespace bk
