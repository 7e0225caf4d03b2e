// FAS multigrid on the arena (crates/bowshock-cfd/src/multigrid.rs:72-218). Every level of a case is a case of the arena
// (the coarse grids drop every second node line, grid.rs:129-144), so the smoother is the same SSP-RK3 kernels; a level
// mask selects which level a launch works on. Transfers:
//   k_restrict_state    U_c = sum V U / sum V over the fluid children, U_c^0 = U_c, forcing zeroed   (multigrid.rs:115-146)
//   k_restrict_forcing  P_c = sum V R / sum V - R_c(U_c)                                            (multigrid.rs:147-171)
//   k_prolong           U += I (U_c - U_c^0): cell-centred bilinear weights 9/3/3/1 over the non-solid parents, the
//                       correction halved up to 6 times until density and pressure stay positive    (multigrid.rs:177-218)
#pragma once
#include "arena.cuh"
#include "device_math.cuh"

namespace bk {

// active[k] = enabled[k] && level(k) == level
__global__ void k_level_mask(Arena A, int level) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= A.ncases) return;
  A.active[k] = (A.enabled[k] && A.cases[k].level == level) ? 1 : 0;
}

// over the tiles of the coarse cases of `level` (their fine level is level - 1)
__global__ void k_restrict_state(Arena A, int level) {
  int t = blockIdx.x;
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (c.level != level || c.fine_case < 0 || !A.enabled[ci]) return;
  const CaseDev& f = A.cases[c.fine_case];
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (i >= c.ni || j >= c.nj) return;
  double s[4] = {0, 0, 0, 0}, v = 0;
  for (int d = 0; d < 4; ++d) {
    int fi = 2 * i + (d & 1), fj = 2 * j + (d >> 1);
    if (is_solid(f, fi, fj)) continue;
    long long fc = cidx(f, fi, fj);
    double vol = A.cellg[fc].x;
    float4 u = A.U[fc];
    s[0] += vol * u.x, s[1] += vol * u.y, s[2] += vol * u.z, s[3] += vol * u.w;
    v += vol;
  }
  long long cc = cidx(c, i, j);
  if (v > 0.0) A.U[cc] = make_float4((float)(s[0] / v), (float)(s[1] / v), (float)(s[2] / v), (float)(s[3] / v));
  A.MG0[cc] = A.U[cc];
  A.FORCE[cc] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void k_restrict_forcing(Arena A, int level) {
  int t = blockIdx.x;
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (c.level != level || c.fine_case < 0 || !A.enabled[ci]) return;
  const CaseDev& f = A.cases[c.fine_case];
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (i >= c.ni || j >= c.nj) return;
  double s[4] = {0, 0, 0, 0}, v = 0;
  for (int d = 0; d < 4; ++d) {
    int fi = 2 * i + (d & 1), fj = 2 * j + (d >> 1);
    if (is_solid(f, fi, fj)) continue;
    long long fc = cidx(f, fi, fj);
    double vol = A.cellg[fc].x;
    float4 r = A.R[fc];
    s[0] += vol * r.x, s[1] += vol * r.y, s[2] += vol * r.z, s[3] += vol * r.w;
    v += vol;
  }
  if (v > 0.0) {
    long long cc = cidx(c, i, j);
    float4 rc = A.R[cc];
    A.FORCE[cc] = make_float4((float)(s[0] / v - rc.x), (float)(s[1] / v - rc.y), (float)(s[2] / v - rc.z), (float)(s[3] / v - rc.w));
  }
}

// over the tiles of the fine cases of `level` (their coarse level is level + 1)
__global__ void k_prolong(Arena A, int level) {
  int t = blockIdx.x;
  int fi_case = A.tile_case[t];
  const CaseDev& f = A.cases[fi_case];
  if (f.level != level || f.coarse_case < 0 || !A.enabled[fi_case]) return;
  const CaseDev& c = A.cases[f.coarse_case];
  int lt = t - f.tile_off;
  int i = (lt % f.ntx) * TI + threadIdx.x % TI, j = (lt / f.ntx) * TJ + threadIdx.x / TI;
  if (i >= f.ni || j >= f.nj || is_solid(f, i, j)) return;
  int ci = i / 2, cj = j / 2;
  int ci2 = (i % 2 == 0) ? (ci > 0 ? ci - 1 : 0) : min(ci + 1, c.ni - 1);
  int cj2 = (j % 2 == 0) ? (cj > 0 ? cj - 1 : 0) : min(cj + 1, c.nj - 1);
  const int ca[4] = {ci, ci2, ci, ci2}, cb[4] = {cj, cj, cj2, cj2};
  const float wt[4] = {9.f, 3.f, 3.f, 1.f};
  float d[4] = {0, 0, 0, 0}, wsum = 0.f;
  for (int q = 0; q < 4; ++q) {
    if (is_solid(c, ca[q], cb[q])) continue;
    long long cc = cidx(c, ca[q], cb[q]);
    float4 u = A.U[cc], u0 = A.MG0[cc];
    d[0] += wt[q] * (u.x - u0.x), d[1] += wt[q] * (u.y - u0.y), d[2] += wt[q] * (u.z - u0.z), d[3] += wt[q] * (u.w - u0.w);
    wsum += wt[q];
  }
  for (int q = 0; q < 4; ++q) d[q] /= wsum;
  long long fc = cidx(f, i, j);
  float4 u = A.U[fc];
  float alpha = 1.f;
  for (int it = 0; it < 6; ++it) {
    V4<float> q = mk4<float>(u.x + alpha * d[0], u.y + alpha * d[1], u.z + alpha * d[2], u.w + alpha * d[3]);
    V4<float> w = cons_to_prim(q);
    if (w[0] > 0.f && w[3] > 0.f) {
      A.U[fc] = to_f4(q);
      return;
    }
    alpha *= 0.5f;
  }
}

}  // namespace bk
