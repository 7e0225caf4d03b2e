// Device layout of a case arena: every case of a sweep (one or many, uneven grid sizes) packed into the same
// structure-of-arrays buffers, so one launch of each kernel serves all cases. A single-case solver is an arena of one.
//
// Per case (ni x nj cells, row-major with i fastest, as the reference's grid.rs:1-4):
//   cells     U, R, X, DU, RR, U0, FORCE (float4 = 4 conserved vars), dt, geometry cellg = {V, A, xc, rc}
//   padded    W = primitives with 2 ghost layers, (ni+4) x (nj+4)            (solver.rs:200-203)
//   i-faces   iface = {nx, nr, len, w = len*r_mid}, (ni+1) x nj                (grid.rs:22-47)
//   j-faces   jface, ni x (nj+1)
// Case descriptors, iteration counters and convergence masks live in device memory so that an iteration launched
// from a CUDA graph reads everything it needs on the device.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_math.cuh"

namespace bk {

enum { SCHEME_EXPLICIT = 0, SCHEME_SMOOTHED = 1, SCHEME_MULTIGRID = 2, SCHEME_IMPLICIT = 3 };
enum { DT_SUM = 0, DT_MIN_DIRECTION = 1 };

struct CaseDev {
  int ni, nj;
  long long cell_off, pad_off, if_off, jf_off;
  int tile_off, ntx, nty;           // residual tiles (TI x TJ cells)
  int iline_off, jline_off;         // first global i-line / j-line of this case
  int pblk_off;                     // first block of the padded-cell kernels
  int has_block, i_end, j_end, j_sting;
  int has_nozzle, nz_j_end;
  float nz_state[4], nz_turb[2];
  int bc[4];
  double fs[4];
  float cfl;
  int limiter, first_order_iters, low_mach;
  int scheme;
  float cfl0, cfl_max, growth, eps_fix;
  int dt_mode, lines, implicit_bc, sub_iters, roe;
  float cfl_star;  // implicit residual smoothing of the SSP-RK3 stages (solver.rs:104-120): > 0 on, per-direction CFL limit
  int viscous, sst, wall_i_start;
  double re_c, sutherland, roughness;
  int n_active;
  // FAS multigrid: level of this case (0 = fine) and the arena indices of its finer / coarser level (-1: none)
  int level, fine_case, coarse_case;
};

struct Arena {
  int ncases;
  const CaseDev* cases;
  int* iter;    // per case: iterations since the last reset (first-order phase, solver.rs:477)
  int* ramp_k;  // per case: CFL-ramp counter (implicit.rs:602-603)
  int* active;  // per case: 1 = iterate, 0 = frozen (converged or stopped)
  float4 *U, *W, *R, *X, *DU, *RR, *U0, *FORCE;
  // Low words of the state and of the primitives: the state is the unevaluated pair U + Ulo (about 48 significant bits),
  // so that the FP64 residual, not FP32 rounding of the state, decides the converged state. Everything that only
  // preconditions (Jacobians, line solves, turbulence, viscous gradients) reads the high words alone.
  float4 *Ulo, *Wlo, *U0lo;
  // per case two tensor maps (W, then Wlo) over its padded primitives, 16-byte elements as 4 floats, boxes of the
  // residual tile and its 2-cell halo: the residual kernel stages its tile with TMA
  const CUtensorMap* wmaps;
  float* dt;
  float2* irs_eps;  // implicit residual smoothing: (eps_i, eps_j) of every cell, set with the explicit time step
  float* irs_c;     // its Thomas multipliers
  const float4 *iface, *jface, *cellg;
  const float2 *ifc, *jfc;  // face centres (mean of the end nodes)
  float* scratch;  // line-solve records (fv_kernels.cu: line_rec, pcr_rec)
  float4* lend;    // ghost Jacobian T of every line end, 4 float4 each (fv_kernels.cu: lend_slot)
  long long ncell;
  double* rsum;    // sum of R_rho^2, [slot * ncases + case]
  const int* tile_case;
  int ntiles;
  const int* iline_case;
  int nilines;
  const int* jline_case;
  int njlines;
  const int* pblk_case;
  int npblk;
  // viscous / SST fields (null for an inviscid arena)
  float4* grad4;   // (u_x, u_r, v_x, v_r)
  float2* gradT;   // (T_x, T_r)
  float* mu;
  float* mu_t;
  float4* rough;   // rough-wall runs: (k_w, omega_w, mu_t,w, 0) of the cells next to a no-slip face (null: no rough case)
  float4* fvi;     // viscous i-face fluxes
  float4* fvj;     // viscous j-face fluxes
  float2* turb;    // (k, omega)
  float2* turb_new;
  float* dwall;
  float* mflux_i;  // inviscid mass flux F[0] of the i-faces (turbulence convection)
  float* mflux_j;
  double* tsum;    // sum of (rho dk/dt)^2, [slot * ncases + case]
  float4* tcoef;   // SST line coefficients, 3 per cell
  float2* trhs;    // SST right-hand side / solution per cell
  float4* grad_kw; // (k_x, k_r, omega_x, omega_r)
  float2* blend;   // (F1, X)
  // coupled SST lines: per cell the derivatives of V R_k, V R_omega with respect to the mass fluxes of the cell's four
  // faces and to its density, 3 per cell (null: loosely coupled, the reference's scheme)
  float4* tcpl;
  // FP64-derived stencil of every face: (|d|, e_x, e_r, 0) between the two side positions (viscous.rs:233-250)
  const float4 *ifs, *jfs;
  // FAS multigrid: the restricted state at the start of a coarse cycle, and the user's mask the level masks derive from
  float4 *MG0, *MG0lo;
  int* enabled;
  // Compaction: when some cases are masked out, the launches run over the active cases' tiles, padded-array blocks and
  // lines only; the kernels map their block / line index through these lists (null: every entry).
  const int *tile_list, *pblk_list, *iline_list, *jline_list;
  int n_tl, n_pb, n_il, n_jl;
  // Smallest segment (cells per lane) of the block line solves, i and j lines (>= 2; the same for a first pass and the
  // substitution passes that reuse its factors)
  int mmin_i = 2, mmin_j = 2;
};

constexpr int TI = 32, TJ = 8;  // residual tile

__device__ __forceinline__ bool is_solid(const CaseDev& c, int i, int j) {
  if (!c.has_block) return false;
  return i < c.i_end ? j < c.j_end : j < c.j_sting;
}
__device__ __forceinline__ int col_start(const CaseDev& c, int i) { return c.has_block ? (i < c.i_end ? c.j_end : c.j_sting) : 0; }
// first fluid cell of row j; ni when the whole row is solid (implicit.rs:471-477)
__device__ __forceinline__ int row_start(const CaseDev& c, int j) {
  if (!c.has_block) return 0;
  if (j < c.j_sting) return c.ni;
  return j < c.j_end ? c.i_end : 0;
}
// viscous.rs:97-127
__device__ __forceinline__ bool noslip_jface(const CaseDev& c, int i, int j) {
  if (!c.viscous) return false;
  if (!c.has_block) return j == 0 && c.bc[2] == 2 && i >= c.wall_i_start;
  return (j == c.j_end && i >= c.wall_i_start && i < c.i_end) || (j == c.j_sting && c.j_sting > 0 && i >= c.i_end);
}
__device__ __forceinline__ bool noslip_iface(const CaseDev& c, int i, int j) {
  return c.viscous && c.has_block && i == c.i_end && j >= c.j_sting && j < c.j_end && !(c.has_nozzle && j < c.nz_j_end);
}
// SST with a sand-grain roughness (viscous.rs:52-56)
__device__ __forceinline__ bool is_rough(const CaseDev& c) { return c.sst && c.roughness > 0.0; }
// viscous.rs:111-121: the body surface is the rough wall; the base wall and the sting keep the smooth state
__device__ __forceinline__ bool rough_jface(const CaseDev& c, int i, int j) {
  if (!is_rough(c)) return false;
  if (!c.has_block) return j == 0 && c.bc[2] == 2 && i >= c.wall_i_start;
  return j == c.j_end && i >= c.wall_i_start && i < c.i_end;
}
// turbulence.rs:280-290: the roughness is phased in over the first 8 wall cells
__device__ __forceinline__ double rough_ramp(const CaseDev& c, int i) {
  int a = i + 1 - c.wall_i_start;
  return fmin((double)(a > 0 ? a : 0) / 8.0, 1.0);
}
__device__ __forceinline__ bool jet_iface(const CaseDev& c, int i, int j) { return c.has_block && i == c.i_end && c.has_nozzle && j < c.nz_j_end; }

// a pair (hi, lo) as one double, and a double split into the nearest float and its remainder
__device__ __forceinline__ V4<double> pair_ld(float4 h, float4 l) {
  return mk4<double>((double)h.x + (double)l.x, (double)h.y + (double)l.y, (double)h.z + (double)l.z, (double)h.w + (double)l.w);
}
__device__ __forceinline__ void pair_st(float4* hi, float4* lo, long long k, const V4<double>& q) {
  float4 h = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
  hi[k] = h;
  lo[k] = make_float4((float)(q[0] - (double)h.x), (float)(q[1] - (double)h.y), (float)(q[2] - (double)h.z), (float)(q[3] - (double)h.w));
}
__device__ __forceinline__ V4<double> state_of(const Arena& A, long long k) { return pair_ld(A.U[k], A.Ulo[k]); }
// q as pair_st stores it and state_of reads it back
__device__ __forceinline__ V4<double> pair_round(const V4<double>& q) {
  float4 h = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
  float4 l = make_float4((float)(q[0] - (double)h.x), (float)(q[1] - (double)h.y), (float)(q[2] - (double)h.z), (float)(q[3] - (double)h.w));
  return pair_ld(h, l);
}

__device__ __forceinline__ int tile_at(const Arena& A) { return A.tile_list ? A.tile_list[blockIdx.x] : (int)blockIdx.x; }
__device__ __forceinline__ int pblk_at(const Arena& A) { return A.pblk_list ? A.pblk_list[blockIdx.x] : (int)blockIdx.x; }
__device__ __forceinline__ int lines_of(const Arena& A, bool dir_i) {
  return dir_i ? (A.iline_list ? A.n_il : A.nilines) : (A.jline_list ? A.n_jl : A.njlines);
}
// the idx-th line of direction dir of this launch, -1 past the end
__device__ __forceinline__ int line_at(const Arena& A, bool dir_i, int idx) {
  if (idx >= lines_of(A, dir_i)) return -1;
  const int* l = dir_i ? A.iline_list : A.jline_list;
  return l ? l[idx] : idx;
}

__device__ __forceinline__ long long cidx(const CaseDev& c, int i, int j) { return c.cell_off + (long long)j * c.ni + i; }
__device__ __forceinline__ long long pidx(const CaseDev& c, int i, int j) { return c.pad_off + (long long)(j + 2) * (c.ni + 4) + (i + 2); }
__device__ __forceinline__ long long ifidx(const CaseDev& c, int i, int j) { return c.if_off + (long long)j * (c.ni + 1) + i; }
__device__ __forceinline__ long long jfidx(const CaseDev& c, int i, int j) { return c.jf_off + (long long)j * c.ni + i; }

}  // namespace bk
