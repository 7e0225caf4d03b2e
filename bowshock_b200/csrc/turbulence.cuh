// Menter SST k-omega update (crates/bowshock-cfd/src/turbulence.rs:542-611) on the arena, loosely coupled after each
// mean-flow iteration as in the reference:
//   k_turb_grad   Green-Gauss gradients of k and omega with the boundary states of the two scalars (turbulence.rs:337-372),
//                 then F1 and the cross-diffusion X of the cell (turbulence.rs:375-397)
//   k_turb_cell   face convection / diffusion data of the tile's faces, each once in shared memory (turbulence.rs:413-435),
//                 and the cell terms: residual, diag0 and the coefficients of the i- and j-line systems
//                 (turbulence.rs:477-519, 559-579)
//   k_turb_lines  the two scalar tridiagonal line systems, i then j, one thread per (line, scalar) (turbulence.rs:580-581);
//                 k_turb_lines_w the same with one warp per line (partitioned Thomas), used for lines up to 512 cells
//   k_turb_update clipped update and the new eddy viscosity (turbulence.rs:584-603)
// Host helpers: the turbulence initialisation (free stream, wall distance in FP64, mu_t; turbulence.rs:128-138).
#pragma once
#include "arena.cuh"
#include "device_math.cuh"
#include "viscous.cuh"

namespace bk {

constexpr float K_INF = 9e-9f;
constexpr float A1 = 0.31f, BETA_STAR = 0.09f, SIGMA_K1 = 0.85f, SIGMA_K2 = 1.0f, SIGMA_W1 = 0.5f, SIGMA_W2 = 0.856f, BETA1 = 0.075f,
                BETA2 = 0.0828f, GAMMA1 = 5.0f / 9.0f, GAMMA2 = 0.44f;

enum { KIND_CELL = 0, KIND_INF = 1, KIND_FIXED = 2, KIND_WALL = 3 };
__device__ __forceinline__ int bc_kind(int bc) { return (bc == BC_FREESTREAM || bc == BC_CHARACTERISTIC || bc == BC_PRESSURE_OUTFLOW) ? KIND_INF : KIND_CELL; }
__device__ __forceinline__ float omega_inf(const CaseDev& c) { return (float)(1e-6 * c.re_c); }

// Ctx::iface / jface (turbulence.rs:188-221): the origin of the ghost state of the two scalars
__device__ __forceinline__ int ikind(const CaseDev& c, int i, const SidesD& s) {
  if (i == 0) return bc_kind(c.bc[0]);
  if (i == c.ni) return bc_kind(c.bc[1]);
  if (s.l.ghost && s.l.fixed && c.has_nozzle) return KIND_FIXED;
  if (s.l.ghost && s.noslip) return KIND_WALL;
  return KIND_CELL;
}
__device__ __forceinline__ int jkind(const CaseDev& c, int j, const SidesD& s) {
  if (s.l.ghost) {
    if (s.noslip) return KIND_WALL;
    if (j == 0) return bc_kind(c.bc[2]);
    return KIND_CELL;
  }
  if (s.r.ghost) return bc_kind(c.bc[3]);
  return KIND_CELL;
}
// Ctx::kw (turbulence.rs:224-245): a wall ghost mirrors (0, omega_w) of a smooth wall, or the rough-wall state of the
// wall cell stored by the last viscous pass
__device__ __forceinline__ float2 kw_side(const Arena& A, const CaseDev& c, const SideD& s, int kind) {
  float2 t = A.turb[s.cell];
  if (!s.ghost || kind == KIND_CELL) return t;
  if (kind == KIND_INF) return make_float2(K_INF, omega_inf(c));
  if (kind == KIND_FIXED) return make_float2(c.nz_turb[0], c.nz_turb[1]);
  long long cc = s.cell;
  if (is_rough(c)) {
    float4 r = A.rough[cc];
    return make_float2(2.f * r.x - t.x, 2.f * r.y - t.y);
  }
  int i = (int)((cc - c.cell_off) % c.ni), j = (int)((cc - c.cell_off) / c.ni);
  float rho = A.W[pidx(c, i, j)].x;
  float nu = A.mu[cc] / rho;
  float d = A.dwall[cc];
  return make_float2(-t.x, 2.f * (60.f * nu / (BETA1 * d * d)) - t.y);
}

// F1 and the cross-diffusion X of a fluid cell from its own gradient (turbulence.rs:375-397)
__device__ __forceinline__ float2 blend_of(const Arena& A, const CaseDev& c, int i, int j, long long cc, float4 g) {
  float rho = A.W[pidx(c, i, j)].x;
  float nu = A.mu[cc] / rho;
  float2 kw = A.turb[cc];
  float d = A.dwall[cc];
  float x = 2.f * rho * SIGMA_W2 * (g.x * g.z + g.y * g.w) / kw.y;
  float cd = fmaxf(x, 1e-20f);
  float t1 = sqrtf(kw.x) / (BETA_STAR * kw.y * d), t2 = 500.f * nu / (d * d * kw.y);
  float t3 = 4.f * rho * SIGMA_W2 * kw.x / (cd * d * d);
  float a = fminf(fmaxf(t1, t2), t3);
  float a2 = a * a;
  return make_float2(tanhf(a2 * a2), x);
}

// Green-Gauss gradients of k and omega (turbulence.rs:337-372) and, from the cell's own gradient, its blend (F1, X)
__global__ void k_turb_grad(Arena A) {
  int t = tile_at(A);
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || !c.sst) return;
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (i >= c.ni || j >= c.nj) return;
  long long cc = cidx(c, i, j);
  if (is_solid(c, i, j)) {
    A.grad_kw[cc] = make_float4(0.f, 0.f, 0.f, 0.f);
    A.blend[cc] = make_float2(0.f, 0.f);
    return;
  }
  float2 pc = A.turb[cc];
  SidesD sl, sr, sb, st;
  iface_sides_d(A, c, i, j, sl);
  iface_sides_d(A, c, i + 1, j, sr);
  jface_sides_d(A, c, i, j, sb);
  jface_sides_d(A, c, i, j + 1, st);
  float2 nb[4] = {kw_side(A, c, sr.r, ikind(c, i + 1, sr)), kw_side(A, c, sl.l, ikind(c, i, sl)), kw_side(A, c, st.r, jkind(c, j + 1, st)),
                  kw_side(A, c, sb.l, jkind(c, j, sb))};
  float4 fs4[4] = {A.iface[ifidx(c, i + 1, j)], A.iface[ifidx(c, i, j)], A.jface[jfidx(c, i, j + 1)], A.jface[jfidx(c, i, j)]};
  const float sg[4] = {1.f, -1.f, 1.f, -1.f};
  float g[4] = {0, 0, 0, 0};
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    float pk = 0.5f * (pc.x + nb[f].x), pw = 0.5f * (pc.y + nb[f].y);
    g[0] += sg[f] * pk * fs4[f].x * fs4[f].z;
    g[1] += sg[f] * pk * fs4[f].y * fs4[f].z;
    g[2] += sg[f] * pw * fs4[f].x * fs4[f].z;
    g[3] += sg[f] * pw * fs4[f].y * fs4[f].z;
  }
  float inv_a = 1.f / A.cellg[cc].y;
  const float4 gk = make_float4(g[0] * inv_a, g[1] * inv_a, g[2] * inv_a, g[3] * inv_a);
  A.grad_kw[cc] = gk;
  A.blend[cc] = blend_of(A, c, i, j, cc, gk);
}

struct TFaceD {
  float m, g0, g1, f0, f1;
  float2 l, r;
};

// turbulence.rs:413-435
__device__ TFaceD tface_d(const Arena& A, const CaseDev& c, const SidesD& s, int kind, float4 f, float4 st, float m) {
  TFaceD o;
  o.m = m;
  o.l = kw_side(A, c, s.l, kind);
  o.r = kw_side(A, c, s.r, kind);
  o.g0 = o.g1 = o.f0 = o.f1 = 0.f;
  if (f.w == 0.f) return o;
  float dd = st.x, ex = st.y, er = st.z;
  float4 gl = A.grad_kw[s.l.cell], gr = A.grad_kw[s.r.cell];
  float mu_f, mut_f;
  face_mu_d(A, c, s, mu_f, mut_f);
  float f1l = A.blend[s.l.cell].x, f1r = A.blend[s.r.cell].x;
  {
    float sigma = 0.5f * (f1l * SIGMA_K1 + (1.f - f1l) * SIGMA_K2 + f1r * SIGMA_K1 + (1.f - f1r) * SIGMA_K2);
    float coef = mu_f + sigma * mut_f;
    float gbx = 0.5f * (gl.x + gr.x), gbr = 0.5f * (gl.y + gr.y);
    float corr = (o.r.x - o.l.x) / dd - (gbx * ex + gbr * er);
    float gn = (gbx + corr * ex) * f.x + (gbr + corr * er) * f.y;
    o.f0 = coef * gn * f.w;
    o.g0 = coef * f.w / dd;
  }
  {
    float sigma = 0.5f * (f1l * SIGMA_W1 + (1.f - f1l) * SIGMA_W2 + f1r * SIGMA_W1 + (1.f - f1r) * SIGMA_W2);
    float coef = mu_f + sigma * mut_f;
    float gbx = 0.5f * (gl.z + gr.z), gbr = 0.5f * (gl.w + gr.w);
    float corr = (o.r.y - o.l.y) / dd - (gbx * ex + gbr * er);
    float gn = (gbx + corr * ex) * f.x + (gbr + corr * er) * f.y;
    o.f1 = coef * gn * f.w;
    o.g1 = coef * f.w / dd;
  }
  return o;
}

__device__ __forceinline__ float strain2(float4 g, float v, float r) {  // turbulence.rs:250-255
  float vr = v / r;
  float div = g.x + g.w + vr;
  float shear = g.y + g.z;
  return 2.f * (g.x * g.x + g.w * g.w + vr * vr) + shear * shear - 2.f / 3.f * div * div;
}

// Cell terms and line coefficients (turbulence.rs:477-519, 559-579). Coefficients per cell:
//   tcoef[3c+0] = (lo_i k, lo_i w, up_i k, up_i w), [3c+1] = (d_i k, d_i w, lo_j k / d0k, lo_j w / d0w),
//   [3c+2] = (up_j k / d0k, up_j w / d0w, d_j k, d_j w); trhs[c] = V R (the i-line right-hand side).
// CPL: also store the coupling derivatives of the coupled SST lines (A.tcpl); the loosely coupled instance compiles
// without them.
template <bool CPL>
__global__ void k_turb_cell(Arena A, int slot) {
  __shared__ double sred[TI * TJ / 32];
  __shared__ TFaceD sFI[TJ][TI + 1];  // the tile's face data, each face once (turbulence.rs:413-435)
  __shared__ TFaceD sFJ[TJ + 1][TI];
  int t = tile_at(A);
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || !c.sst) return;
  int lt = t - c.tile_off;
  const int i0 = (lt % c.ntx) * TI, j0 = (lt / c.ntx) * TJ;
  for (int idx = threadIdx.x; idx < TJ * (TI + 1) + (TJ + 1) * TI; idx += blockDim.x) {
    SidesD s;
    if (idx < TJ * (TI + 1)) {
      const int r = idx / (TI + 1), q = idx % (TI + 1), fi = i0 + q, fj = j0 + r;
      if (fi > c.ni || fj >= c.nj) continue;
      if (!((fi < c.ni && !is_solid(c, fi, fj)) || (fi > 0 && !is_solid(c, fi - 1, fj)))) continue;  // no fluid side
      iface_sides_d(A, c, fi, fj, s);
      sFI[r][q] = tface_d(A, c, s, ikind(c, fi, s), A.iface[ifidx(c, fi, fj)], A.ifs[ifidx(c, fi, fj)],
                          A.mflux_i[ifidx(c, fi, fj)] * A.iface[ifidx(c, fi, fj)].w);
    } else {
      const int k = idx - TJ * (TI + 1), r = k / TI, q = k % TI, fi = i0 + q, fj = j0 + r;
      if (fi >= c.ni || fj > c.nj) continue;
      if (!((fj < c.nj && !is_solid(c, fi, fj)) || (fj > 0 && !is_solid(c, fi, fj - 1)))) continue;
      jface_sides_d(A, c, fi, fj, s);
      sFJ[r][q] = tface_d(A, c, s, jkind(c, fj, s), A.jface[jfidx(c, fi, fj)], A.jfs[jfidx(c, fi, fj)],
                          A.mflux_j[jfidx(c, fi, fj)] * A.jface[jfidx(c, fi, fj)].w);
    }
  }
  __syncthreads();
  const int q = threadIdx.x % TI, r = threadIdx.x / TI;
  int i = i0 + q, j = j0 + r;
  double rr = 0.0;
  if (i < c.ni && j < c.nj) {
    long long cc = cidx(c, i, j);
    if (is_solid(c, i, j)) {
      A.tcoef[3 * cc] = make_float4(0.f, 0.f, 0.f, 0.f);
      A.tcoef[3 * cc + 1] = make_float4(1.f, 1.f, 0.f, 0.f);
      A.tcoef[3 * cc + 2] = make_float4(0.f, 0.f, 1.f, 1.f);
      A.trhs[cc] = make_float2(0.f, 0.f);
      if constexpr (CPL)
        for (int q3 = 0; q3 < 3; ++q3) A.tcpl[3 * cc + q3] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
      float4 g = A.cellg[cc];
      float vol = g.x;
      float4 wc = A.W[pidx(c, i, j)];
      float rho = wc.x;
      float2 kw = A.turb[cc];
      float2 bl = A.blend[cc];
      float f1 = bl.x;
      float s2 = strain2(A.grad4[cc], wc.z, g.w);
      float mut_c = A.mu_t[cc];
      float prod = fminf(mut_c * s2, 10.f * BETA_STAR * rho * kw.x * kw.y);
      float beta = f1 * BETA1 + (1.f - f1) * BETA2;
      float gamma = f1 * GAMMA1 + (1.f - f1) * GAMMA2;
      float src0 = prod - BETA_STAR * rho * kw.y * kw.x;
      float src1 = gamma * rho * prod / fmaxf(mut_c, 1e-30f) - beta * rho * kw.y * kw.y + (1.f - f1) * bl.y;
      float dest0 = BETA_STAR * kw.y, dest1 = 2.f * beta * kw.y;
      // the four faces
      const TFaceD fa[4] = {sFI[r][q], sFI[r][q + 1], sFJ[r][q], sFJ[r + 1][q]};
      bool ends_lo[2] = {i == row_start(c, j), j == col_start(c, i)};
      bool ends_up[2] = {i == c.ni - 1, j == c.nj - 1};
      float rate0 = 0.f, rate1 = 0.f;
      float lo[2][2], dd[2][2], up[2][2];
      float4 cpl[2] = {};
#pragma unroll
      for (int dir = 0; dir < 2; ++dir) {
        const TFaceD& lf = fa[2 * dir];
        const TFaceD& uf = fa[2 * dir + 1];
        float a_lo = fmaxf(lf.m, 0.f), a_up = fmaxf(-uf.m, 0.f);
        rate0 += a_lo * (lf.l.x - kw.x) + a_up * (uf.r.x - kw.x) + uf.f0 - lf.f0;
        rate1 += a_lo * (lf.l.y - kw.y) + a_up * (uf.r.y - kw.y) + uf.f1 - lf.f1;
        lo[dir][0] = ends_lo[dir] ? 0.f : -(a_lo + lf.g0);
        lo[dir][1] = ends_lo[dir] ? 0.f : -(a_lo + lf.g1);
        up[dir][0] = ends_up[dir] ? 0.f : -(a_up + uf.g0);
        up[dir][1] = ends_up[dir] ? 0.f : -(a_up + uf.g1);
        dd[dir][0] = a_lo + a_up + lf.g0 + uf.g0;
        dd[dir][1] = a_lo + a_up + lf.g1 + uf.g1;
        if constexpr (CPL) {
          // d(rate)/d(m) of the two faces: inflow through the lower face (m > 0), through the upper face (m < 0)
          const bool cl = !ends_lo[dir] && lf.m > 0.f, cu = !ends_up[dir] && uf.m < 0.f;
          cpl[dir] = make_float4(cl ? lf.l.x - kw.x : 0.f, cl ? lf.l.y - kw.y : 0.f, cu ? kw.x - uf.r.x : 0.f, cu ? kw.y - uf.r.y : 0.f);
        }
      }
      float r0 = rate0 / vol + src0, r1 = rate1 / vol + src1;
      float dtc = A.dt[cc];
      float d00 = rho * vol / dtc + rho * vol * dest0, d01 = rho * vol / dtc + rho * vol * dest1;
      A.tcoef[3 * cc] = make_float4(lo[0][0], lo[0][1], up[0][0], up[0][1]);
      A.tcoef[3 * cc + 1] = make_float4(d00 + dd[0][0], d01 + dd[0][1], lo[1][0] / d00, lo[1][1] / d01);
      A.tcoef[3 * cc + 2] = make_float4(up[1][0] / d00, up[1][1] / d01, 1.f + dd[1][0] / d00, 1.f + dd[1][1] / d01);
      A.trhs[cc] = make_float2(vol * r0, vol * r1);
      if constexpr (CPL) {
        // d(V source)/d(rho) with mu_t, F1 and the strain frozen: the production limiter's branch, the destruction
        // terms, and the cross-diffusion term (linear in rho)
        const bool lim = mut_c * s2 > 10.f * BETA_STAR * rho * kw.x * kw.y;
        const float dprod = lim ? 10.f * BETA_STAR * kw.x * kw.y : 0.f;
        const float ds0 = dprod - BETA_STAR * kw.y * kw.x;
        const float ds1 = gamma * (prod + rho * dprod) / fmaxf(mut_c, 1e-30f) - beta * kw.y * kw.y + (1.f - f1) * bl.y / rho;
        A.tcpl[3 * cc] = cpl[0];
        A.tcpl[3 * cc + 1] = cpl[1];
        A.tcpl[3 * cc + 2] = make_float4(vol * ds0, vol * ds1, 0.f, 0.f);
      }
      rr = (double)r0 * (double)r0;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) rr += __shfl_down_sync(0xffffffffu, rr, o);
  if ((threadIdx.x & 31) == 0) sred[threadIdx.x >> 5] = rr;
  __syncthreads();
  if (threadIdx.x == 0 && slot >= 0) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sred[k];
    atomicAdd(&A.tsum[(long long)slot * A.ncases + ci], s);
  }
}

// Scalar tridiagonal solve along every i (dir 1) or j (dir 0) line, one thread per (line, scalar): x <- A^-1 x in place
// in trhs (turbulence.rs:580-581 with the block solver's diagonal blocks, implicit.rs:179-204).
__global__ void k_turb_lines(Arena A, int dir_i) {
  int gt = blockIdx.x * blockDim.x + threadIdx.x;
  int line = line_at(A, dir_i != 0, gt >> 1), e = gt & 1;
  if (line < 0) return;
  int ci = dir_i ? A.iline_case[line] : A.jline_case[line];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || !c.sst) return;
  int L = line - (dir_i ? c.iline_off : c.jline_off);
  int n = dir_i ? c.ni : c.nj;
  int k0 = dir_i ? row_start(c, L) : col_start(c, L);
  if (n - k0 <= 0) return;
  float* cp = A.scratch;  // the mean-flow line records are spent by now: floats 36 c + 0 / 1 hold the Thomas c' of the scalars
  float xprev = 0.f, cprev = 0.f;
  for (int k = k0; k < n; ++k) {
    long long cc = dir_i ? cidx(c, k, L) : cidx(c, L, k);
    float4 t0 = A.tcoef[3 * cc], t1 = A.tcoef[3 * cc + 1], t2 = A.tcoef[3 * cc + 2];
    float lo, d, up;
    if (dir_i) {
      lo = e ? t0.y : t0.x;
      up = e ? t0.w : t0.z;
      d = e ? t1.y : t1.x;
    } else {
      lo = e ? t1.w : t1.z;
      up = e ? t2.y : t2.x;
      d = e ? t2.w : t2.z;
    }
    float2 r2 = A.trhs[cc];
    float r = e ? r2.y : r2.x;
    float m = d, rhs = r;
    if (k > k0) {
      m -= lo * cprev;
      rhs -= lo * xprev;
    }
    float minv = 1.f / m;
    float x = minv * rhs;
    float cpk = minv * up;
    cp[36 * cc + e] = cpk;
    if (e)
      A.trhs[cc].y = x;
    else
      A.trhs[cc].x = x;
    xprev = x;
    cprev = cpk;
  }
  for (int k = n - 2; k >= k0; --k) {
    long long cc = dir_i ? cidx(c, k, L) : cidx(c, L, k);
    long long cn = dir_i ? cidx(c, k + 1, L) : cidx(c, L, k + 1);
    float xn = e ? A.trhs[cn].y : A.trhs[cn].x;
    float v = (e ? A.trhs[cc].y : A.trhs[cc].x) - cp[36 * cc + e] * xn;
    if (e)
      A.trhs[cc].y = v;
    else
      A.trhs[cc].x = v;
  }
}

// The same two scalar line systems, one warp per line and both scalars per lane (partitioned Thomas): lane s eliminates
// its segment of m = max(2, ceil(len/32)) cells (m <= TL_MAXM, so the spikes stay in registers), expressing every interior
// unknown through the separators on either side (the last cell of each segment but the last); the separator rows form a
// tridiagonal system solved by parallel cyclic reduction with warp shuffles; each lane then back-substitutes its segment.
// Coefficient reads per cell are the same as the thread-per-line kernel's, but 32 lanes share a line, so the grid has
// 32x the threads and every read is used once.
constexpr int TL_WARPS = 4, TL_MAXM = 16;  // lines of up to 32 * TL_MAXM = 512 cells
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 f2neg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 f2rcp(float2 a) { return make_float2(1.f / a.x, 1.f / a.y); }
__device__ __forceinline__ float2 shfl_up2(float2 v, int h) {
  return make_float2(__shfl_up_sync(0xffffffffu, v.x, h), __shfl_up_sync(0xffffffffu, v.y, h));
}
__device__ __forceinline__ float2 shfl_down2(float2 v, int h) {
  return make_float2(__shfl_down_sync(0xffffffffu, v.x, h), __shfl_down_sync(0xffffffffu, v.y, h));
}

template <int W>  // lines (warps) per block, chosen by the arena's autotuner
__global__ void __launch_bounds__(32 * W) k_turb_lines_w(Arena A, int dir_i) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int line = line_at(A, dir_i != 0, blockIdx.x * W + warp);
  if (line < 0) return;  // uniform per warp
  const int ci = dir_i ? A.iline_case[line] : A.jline_case[line];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || !c.sst) return;
  const int L = line - (dir_i ? c.iline_off : c.jline_off);
  const int n = dir_i ? c.ni : c.nj;
  const int k0 = dir_i ? row_start(c, L) : col_start(c, L);
  const int len = n - k0;
  if (len <= 0) return;
  int m = (len + 31) / 32;
  if (m < 2) m = 2;
  const int P = (len + m - 1) / m, N = P - 1;
  const int s = lane;
  const bool act = s < P;
  const int a = k0 + s * m;
  const int e = act ? min(a + m, n) : a;
  const bool has_sep = act && s < N;
  const int cnt = act ? (has_sep ? e - 1 - a : e - a) : 0;  // interior cells of the segment
  auto cell = [&](int k) { return dir_i ? cidx(c, k, L) : cidx(c, L, k); };
  auto coef = [&](long long cc, float2& lo, float2& d, float2& up) {
    if (dir_i) {
      float4 t0 = A.tcoef[3 * cc], t1 = A.tcoef[3 * cc + 1];
      lo = make_float2(t0.x, t0.y), up = make_float2(t0.z, t0.w), d = make_float2(t1.x, t1.y);
    } else {
      float4 t1 = A.tcoef[3 * cc + 1], t2 = A.tcoef[3 * cc + 2];
      lo = make_float2(t1.z, t1.w), up = make_float2(t2.x, t2.y), d = make_float2(t2.z, t2.w);
    }
  };
  float2 Y[TL_MAXM], G[TL_MAXM], GE[TL_MAXM];
  const float2 z2 = make_float2(0.f, 0.f);
  float2 yl = z2, gl = z2, gel = z2;
#pragma unroll
  for (int t = 0; t < TL_MAXM; ++t) {
    if (t < cnt) {
      long long cc = cell(a + t);
      float2 lo, d, up;
      coef(cc, lo, d, up);
      float2 r = A.trhs[cc];
      float2 M = d, GEr = f2neg(lo);
      if (t > 0) {
        M = f2sub(M, f2mul(lo, yl));
        r = f2sub(r, f2mul(lo, gl));
        GEr = f2neg(f2mul(lo, gel));
      }
      float2 inv = f2rcp(M);
      gl = f2mul(inv, r);
      gel = f2mul(inv, GEr);
      yl = f2mul(inv, up);
      Y[t] = yl, G[t] = gl, GE[t] = gel;
    }
  }
  // x at the last interior cell = v_l + E_l l_{s-1} + F_l l_s; at the first, by the backward recurrence, v_f + E_f .. + F_f ..
  const float2 v_l = gl, E_l = gel, F_l = f2neg(yl);
  float2 v_f = v_l, E_f = E_l, F_f = F_l;
#pragma unroll
  for (int t = TL_MAXM - 2; t >= 0; --t) {
    if (t < cnt - 1) {
      v_f = f2sub(G[t], f2mul(Y[t], v_f));
      E_f = f2sub(GE[t], f2mul(Y[t], E_f));
      F_f = f2neg(f2mul(Y[t], F_f));
    }
  }
  const float2 v_n = shfl_down2(v_f, 1), E_n = shfl_down2(E_f, 1), F_n = shfl_down2(F_f, 1);
  // separator row: lo x_{last interior} + d x_sep + up x_{first of the next segment}
  float2 ra = z2, rb = make_float2(1.f, 1.f), rc = z2, rd = z2;
  if (has_sep) {
    long long cs = cell(e - 1);
    float2 lo, d, up;
    coef(cs, lo, d, up);
    float2 r = A.trhs[cs];
    ra = f2mul(lo, E_l);
    rb = f2add(f2add(d, f2mul(lo, F_l)), f2mul(up, E_n));
    rc = f2mul(up, F_n);
    rd = f2sub(f2sub(r, f2mul(lo, v_l)), f2mul(up, v_n));
  }
  // parallel cyclic reduction of the N separator rows
  for (int h = 1; h < N; h <<= 1) {
    float2 am = shfl_up2(ra, h), bm = shfl_up2(rb, h), cm = shfl_up2(rc, h), dm = shfl_up2(rd, h);
    float2 ap = shfl_down2(ra, h), bp = shfl_down2(rb, h), cp = shfl_down2(rc, h), dp = shfl_down2(rd, h);
    if (s < N) {
      float2 na = z2, nc = z2, nb = rb, nd = rd;
      if (s - h >= 0) {
        float2 al = f2neg(f2mul(ra, f2rcp(bm)));
        na = f2mul(al, am);
        nb = f2add(nb, f2mul(al, cm));
        nd = f2add(nd, f2mul(al, dm));
      }
      if (s + h < N) {
        float2 ga = f2neg(f2mul(rc, f2rcp(bp)));
        nc = f2mul(ga, cp);
        nb = f2add(nb, f2mul(ga, ap));
        nd = f2add(nd, f2mul(ga, dp));
      }
      ra = na, rb = nb, rc = nc, rd = nd;
    }
  }
  const float2 lsep = s < N ? f2mul(rd, f2rcp(rb)) : z2;
  float2 lprev = shfl_up2(lsep, 1);
  if (s == 0) lprev = z2;
  if (!act) return;
  if (has_sep) A.trhs[cell(e - 1)] = lsep;
  float2 xn = has_sep ? lsep : z2;
#pragma unroll
  for (int t = TL_MAXM - 1; t >= 0; --t) {
    if (t < cnt) {
      float2 x = f2sub(f2add(G[t], f2mul(GE[t], lprev)), f2mul(Y[t], xn));
      A.trhs[cell(a + t)] = x;
      xn = x;
    }
  }
}

// Coupled SST lines (an option beside the reference's loose coupling). Unknowns per cell: the mean-flow increment dU (4)
// and (dk, domega), so the line blocks are 6x6. The mean-flow rows do not depend on k and omega, because the mean-flow
// operator freezes mu_t (implicit.rs: the viscous Jacobian takes mu + mu_t as given), so every 6x6 block is lower
// block-triangular and the line system is solved exactly by block substitution: the 4x4 mean-flow lines first, then the
// turbulence rows with their coupling to dU moved to the right-hand side,
//   M_tt x = V R_t + (d(V R_t)/dU) dU,
// M_tt being the reference's two scalar line systems (same approximate factorisation, i then j). The coupling block
// holds what V R_t depends on through the mean-flow state on the line stencil: the mass flux m of each interior face
// of the cell's convection terms (d rate / d m from k_turb_cell, m linearised as the first row of the Rusanov-split
// flux Jacobian, dm = w/2 [n.(d(rho u)_L + d(rho u)_R) + lambda (d rho_L - d rho_R)], lambda = |u_n| + c of the face
// average), and the cell's density in its sources. The strain's dependence on the velocity gradients (a wider stencil)
// is left out, as the mean-flow operator leaves out its viscous cross terms. The residuals are the reference's, so the
// fixed point is the loosely coupled scheme's; only the path to it changes.
__device__ __forceinline__ float dmass(const Arena& A, float4 f, long long cl, long long pl, long long cr, long long pr) {
  const float4 wl = A.W[pl], wr = A.W[pr];
  const float4 dl = A.DU[cl], dr = A.DU[cr];
  const float rho = 0.5f * (wl.x + wr.x), p = 0.5f * (wl.w + wr.w);
  const float un = 0.5f * ((wl.y + wr.y) * f.x + (wl.z + wr.z) * f.y);
  const float lam = fabsf(un) + sqrtf(1.4f * p / rho);
  return 0.5f * f.w * (f.x * (dl.y + dr.y) + f.y * (dl.z + dr.z) + lam * (dl.x - dr.x));
}

// Adds (d(V R_t)/dU) dU to the turbulence right-hand side of every fluid cell of an SST case, after the mean-flow line
// solves have left the full increment dU in DU and before the turbulence line solves.
__global__ void k_turb_couple(Arena A) {
  int t = tile_at(A);
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || !c.sst) return;
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (i >= c.ni || j >= c.nj || is_solid(c, i, j)) return;
  const long long cc = cidx(c, i, j), pc = pidx(c, i, j);
  const float4 a = A.tcpl[3 * cc], b = A.tcpl[3 * cc + 1], s = A.tcpl[3 * cc + 2];
  float add0 = s.x * A.DU[cc].x, add1 = s.y * A.DU[cc].x;
  if (i > row_start(c, j)) {
    const float dm = dmass(A, A.iface[ifidx(c, i, j)], cidx(c, i - 1, j), pidx(c, i - 1, j), cc, pc);
    add0 += a.x * dm, add1 += a.y * dm;
  }
  if (i < c.ni - 1) {
    const float dm = dmass(A, A.iface[ifidx(c, i + 1, j)], cc, pc, cidx(c, i + 1, j), pidx(c, i + 1, j));
    add0 += a.z * dm, add1 += a.w * dm;
  }
  if (j > col_start(c, i)) {
    const float dm = dmass(A, A.jface[jfidx(c, i, j)], cidx(c, i, j - 1), pidx(c, i, j - 1), cc, pc);
    add0 += b.x * dm, add1 += b.y * dm;
  }
  if (j < c.nj - 1) {
    const float dm = dmass(A, A.jface[jfidx(c, i, j + 1)], cc, pc, cidx(c, i, j + 1), pidx(c, i, j + 1));
    add0 += b.z * dm, add1 += b.w * dm;
  }
  const float2 x = A.trhs[cc];
  A.trhs[cc] = make_float2(x.x + add0, x.y + add1);
}

__global__ void k_turb_update(Arena A) {  // turbulence.rs:584-603
  int t = tile_at(A);
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || !c.sst) return;
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (i >= c.ni || j >= c.nj) return;
  long long cc = cidx(c, i, j);
  if (is_solid(c, i, j)) {
    A.turb[cc] = make_float2(0.f, 0.f);
    A.mu_t[cc] = 0.f;
    return;
  }
  float2 kw0 = A.turb[cc];
  float2 x = A.trhs[cc];
  float winf = omega_inf(c);
  float k = fmaxf(fmaxf(kw0.x + x.x, 0.1f * kw0.x), 1e-3f * K_INF);
  float om = fmaxf(fmaxf(kw0.y + x.y, 0.1f * kw0.y), 1e-3f * winf);
  float4 wc = A.W[pidx(c, i, j)];
  float rho = wc.x;
  float nu = A.mu[cc] / rho;
  float strain = sqrtf(fmaxf(strain2(A.grad4[cc], wc.z, A.cellg[cc].w), 0.f));
  float d = A.dwall[cc];
  float t1 = sqrtf(k) / (BETA_STAR * om * d), t2 = 500.f * nu / (d * d * om);
  float b = fmaxf(2.f * t1, t2);
  float f2 = tanhf(b * b);
  float mut = fminf(rho * A1 * k / fmaxf(A1 * om, strain * f2), (float)(1e5 / c.re_c));
  A.turb[cc] = make_float2(k, om);
  A.mu_t[cc] = mut;
}

}  // namespace bk
