// FAS multigrid on the arena (crates/bowshock-cfd/src/multigrid.rs:72-218). Every level of a case is a case of the arena
// (the coarse grids drop every second node line, grid.rs:129-144), so the smoother is the same SSP-RK3 kernels; a level
// mask selects which level a launch works on. Transfers:
//   k_restrict_state    U_c = sum V U / sum V over the fluid children, U_c^0 = U_c, forcing zeroed   (multigrid.rs:115-146)
//   k_restrict_forcing  P_c = sum V R / sum V - R_c(U_c)                                            (multigrid.rs:147-171)
// By default the restriction is folded into the coarse level's own kernels: k_prims_restrict restricts the state while
// it converts it to primitives, and the coarse residual evaluation (k_residual<..., true>) writes the forcing; the two stand-alone kernels remain for the unfused order (Arena::mg_fused). The prolongation stays a
// kernel of its own: the fine primitives' ghost cells read states that other threads of that launch would correct.
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

// The volume-weighted mean state of the fluid children of coarse cell (i, j) in its fine case f (multigrid.rs:115-146);
// `has` false where every child is solid (the coarse state is then left as it is)
__device__ __forceinline__ V4<double> restrict_mean(const Arena& A, const CaseDev& f, int i, int j, bool& has) {
  double s[4] = {0, 0, 0, 0}, v = 0;
  for (int d = 0; d < 4; ++d) {
    int fi = 2 * i + (d & 1), fj = 2 * j + (d >> 1);
    if (is_solid(f, fi, fj)) continue;
    long long fc = cidx(f, fi, fj);
    double vol = A.cellg[fc].x;
    V4<double> u = state_of(A, fc);
    s[0] += vol * u[0], s[1] += vol * u[1], s[2] += vol * u[2], s[3] += vol * u[3];
    v += vol;
  }
  has = v > 0.0;
  return mk4<double>(s[0] / v, s[1] / v, s[2] / v, s[3] / v);
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
  bool has;
  const V4<double> q = restrict_mean(A, f, i, j, has);
  long long cc = cidx(c, i, j);
  if (has) pair_st(A.U, A.Ulo, cc, q);
  A.MG0[cc] = A.U[cc];
  A.MG0lo[cc] = A.Ulo[cc];
  A.FORCE[cc] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// k_prims on the coarse cases of the current level with k_restrict_state folded in: every padded position computes its
// primitives from the restricted states of the cells it reads (rounded to the state pair, as k_restrict_state stores
// them), and the owner of each interior cell stores that state, its copy U^0 and a zero forcing. The primitives and
// states are those of k_restrict_state followed by k_prims, in one launch; no thread reads a state another one writes
// (the fine states are only read, and a coarse state is read as it is only where no restriction replaces it).
__global__ void k_prims_restrict(Arena A) {
  int b = pblk_at(A);
  int ci = A.pblk_case[b];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || c.fine_case < 0) return;
  int p = (b - c.pblk_off) * blockDim.x + threadIdx.x;
  int pw = c.ni + 4;
  if (p >= pw * (c.nj + 4)) return;
  int i = p % pw - 2, j = p / pw - 2;
  const CaseDev& f = A.cases[c.fine_case];
  auto st = [&](int a, int bb) {
    bool has;
    const V4<double> q = restrict_mean(A, f, a, bb, has);
    return has ? pair_round(q) : state_of(A, cidx(c, a, bb));
  };
  pair_st(A.W, A.Wlo, pidx(c, i, j), prims_at(A, c, i, j, st));
  if (i >= 0 && i < c.ni && j >= 0 && j < c.nj) {
    const long long cc = cidx(c, i, j);
    bool has;
    const V4<double> q = restrict_mean(A, f, i, j, has);
    if (has) pair_st(A.U, A.Ulo, cc, q);
    A.MG0[cc] = A.U[cc];
    A.MG0lo[cc] = A.Ulo[cc];
    A.FORCE[cc] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

__global__ void k_restrict_forcing(Arena A, int level) {
  int t = blockIdx.x;
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (c.level != level || c.fine_case < 0 || !A.enabled[ci]) return;
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (i >= c.ni || j >= c.nj) return;
  restrict_forcing_cell(A, c, i, j);
}

// over the tiles of the fine cases of `level` (their coarse level is level + 1)
// relax: the fraction of the interpolated correction applied (1: the reference's full correction)
__global__ void k_prolong(Arena A, int level, double relax) {
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
  const double wt[4] = {9.0, 3.0, 3.0, 1.0};
  double d[4] = {0, 0, 0, 0}, wsum = 0.0;
  for (int q = 0; q < 4; ++q) {
    if (is_solid(c, ca[q], cb[q])) continue;
    long long cc = cidx(c, ca[q], cb[q]);
    V4<double> u = state_of(A, cc), u0 = pair_ld(A.MG0[cc], A.MG0lo[cc]);
    for (int k = 0; k < 4; ++k) d[k] += wt[q] * (u[k] - u0[k]);
    wsum += wt[q];
  }
  for (int q = 0; q < 4; ++q) d[q] = relax * (d[q] / wsum);
  long long fc = cidx(f, i, j);
  V4<double> u = state_of(A, fc);
  double alpha = 1.0;
  for (int it = 0; it < 6; ++it) {
    V4<double> q = mk4<double>(u[0] + alpha * d[0], u[1] + alpha * d[1], u[2] + alpha * d[2], u[3] + alpha * d[3]);
    V4<double> w = cons_to_prim(q);
    if (w[0] > 0.0 && w[3] > 0.0) {
      pair_st(A.U, A.Ulo, fc, q);
      return;
    }
    alpha *= 0.5;
  }
}

}  // namespace bk
