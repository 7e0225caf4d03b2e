// Mean-flow kernels of one iteration over a case arena (sm_100a):
//   k_prims     conserved -> primitive with both ghost layers and the block ghosts     (solver.rs:423-498)
//   k_residual  32x8 cell tiles staged in shared memory: every i/j face flux of the tile computed once (MUSCL + limiter,
//               HLLC blended to Rusanov, low-Mach correction), the cell residual with the axisymmetric source, the local
//               time step, and the FP64 density-residual norm (block reduce + one atomic per block)   (solver.rs:474-654)
//   k_stage     SSP-RK3 stage update                                                   (solver.rs:694-720)
//   k_assemble  blocks (lo, d, up) of I - dt J_i and I - dt J_j of every cell into its two line records
//               (implicit.rs:284-438); k_line_ends_T / _fold fold the line-end ghost Jacobians in (implicit.rs:440-467)
//   k_lines     line-implicit solve of (I - dt J_dir) x = b along every i or j line: one warp per line, a partitioned
//               block-tridiagonal (4x4) solver — each lane eliminates its own segment, the separator unknowns form a
//               reduced block-tridiagonal system solved by parallel cyclic reduction across the warp through shared
//               memory, then each lane back-substitutes its segment; factors kept in the records (implicit.rs:528-563)
//   k_lines_subst  the defect-correction passes with the kept factors                  (implicit.rs:622-639)
//   k_defect    defect r = dt R - (A_i du + A_j du - du) with the kept blocks           (implicit.rs:622-630)
#include "tma.cuh"
#include "arena.cuh"
#include "device_math.cuh"
#include "viscous.cuh"

namespace bk {

__device__ __forceinline__ V4<float> Wat(const Arena& A, const CaseDev& c, int i, int j) { return from_f4(A.W[pidx(c, i, j)]); }
__device__ __forceinline__ V4<double> fs_of(const CaseDev& c) { return mk4<double>(c.fs[0], c.fs[1], c.fs[2], c.fs[3]); }

// ==================================================================================== primitives + ghosts
// FP64 from the state pair, stored as the pair (W, Wlo); the ghosts in FP64 as well. prims_at: the primitives of padded
// position (i, j) of case c with both ghost layers and the block ghosts, from the conserved states `st(i, j)` of the
// interior cells (k_prims: the stored states; the multigrid transfers of multigrid.cuh: the states after a restriction
// or a prolongation, computed where they are read).
template <class ST>
__device__ __forceinline__ V4<double> prims_at(const Arena& A, const CaseDev& c, int i, int j, ST&& st) {
  auto prim = [&](int a, int b) { return cons_to_prim(st(a, b)); };
  int ni = c.ni, nj = c.nj;
  V4<double> out;
  bool in_i = i >= 0 && i < ni, in_j = j >= 0 && j < nj;
  if (in_i && in_j) {
    int j0 = col_start(c, i);
    if (c.has_block && j0 > 0 && j < j0 && j >= j0 - 2) {
      // block ghost below a body / sting surface (solver.rs:457-471)
      int src = j0 + (j0 - 1 - j);
      float4 f = A.jface[jfidx(c, i, j0)];
      out = wall_ghost<double>(prim(i, src), f.x, f.y, noslip_jface(c, i, j0));
    } else {
      out = prim(i, j);
    }
  } else if (in_j && !in_i) {
    // i ghosts (solver.rs:429-439)
    V4<double> fs = fs_of(c);
    if (i < 0) {
      int k = -i;
      float4 f = A.iface[ifidx(c, 0, j)];
      out = ghost_state<double>(c.bc[0], fs, prim(0, j), prim(k - 1, j), f.x, f.y, -1.0);
    } else {
      int k = i - ni + 1;
      float4 f = A.iface[ifidx(c, ni, j)];
      out = ghost_state<double>(c.bc[1], fs, prim(ni - 1, j), prim(ni - k, j), f.x, f.y, 1.0);
    }
  } else if (in_i && !in_j) {
    // j ghosts (solver.rs:440-451)
    V4<double> fs = fs_of(c);
    if (j < 0) {
      int k = -j;
      float4 f = A.jface[jfidx(c, i, 0)];
      V4<double> mir = prim(i, k - 1);
      if (noslip_jface(c, i, 0))
        out = wall_ghost<double>(mir, f.x, f.y, true);
      else
        out = ghost_state<double>(c.bc[2], fs, prim(i, 0), mir, f.x, f.y, -1.0);
    } else {
      int k = j - nj + 1;
      float4 f = A.jface[jfidx(c, i, nj)];
      out = ghost_state<double>(c.bc[3], fs, prim(i, nj - 1), prim(i, nj - k), f.x, f.y, 1.0);
    }
  } else {
    out = fs_of(c);  // corners: never read
  }
  return out;
}
__global__ void k_prims(Arena A) {
  int b = pblk_at(A);
  int ci = A.pblk_case[b];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci]) return;
  int p = (b - c.pblk_off) * blockDim.x + threadIdx.x;
  int pw = c.ni + 4;
  if (p >= pw * (c.nj + 4)) return;
  int i = p % pw - 2, j = p / pw - 2;
  V4<double> out = prims_at(A, c, i, j, [&](int a, int bb) { return state_of(A, cidx(c, a, bb)); });
  pair_st(A.W, A.Wlo, pidx(c, i, j), out);
}

// ==================================================================================== residual
// Inviscid flux of i-face (i, j) from the shared-memory stencil (solver.rs:505-542), with the base-wall stencils of a
// block. Evaluated in FP64 from the FP32 primitives: the flux balance of a cell and its axisymmetric pressure source cancel
// to round-off in a converged (and in a free-stream) state, and next to the axis that cancellation error grows like
// eps p / r_c; in FP32 it is large enough for the implicit operator to amplify it into a divergence, in FP64 it is not.
__device__ __forceinline__ V4<double> iface_flux(const Arena& A, const CaseDev& c, int i, int j, const V4<double>& m2_, const V4<double>& m1_,
                                                 const V4<double>& p0, const V4<double>& p1, int lim, float4 f) {
  V4<double> m2 = m2_, m1 = m1_;
  if (c.has_block && j < c.j_end) {
    if (j < c.j_sting || i < c.i_end) return mk4<double>(0, 0, 0, 0);
    if (i <= c.i_end + 1) {
      float4 fb = A.iface[ifidx(c, c.i_end, j)];
      if (jet_iface(c, c.i_end, j)) {
        V4<double> jw = mk4<double>(c.nz_state[0], c.nz_state[1], c.nz_state[2], c.nz_state[3]);
        m2 = jw;
        if (i == c.i_end) m1 = jw;
      } else if (i == c.i_end) {
        bool ns = noslip_iface(c, i, j);
        m2 = wall_ghost<double>(p1, fb.x, fb.y, ns);
        m1 = wall_ghost<double>(p0, fb.x, fb.y, ns);
      } else {
        m2 = wall_ghost<double>(m1, fb.x, fb.y, noslip_iface(c, c.i_end, j));
      }
    }
  }
  return face_flux_lm<double>(m2, m1, p0, p1, lim, f.x, f.y, c.low_mach != 0);
}

__device__ __forceinline__ float diffusion_rate(float mu_c, float mu_t_c, float rho_c, float len, float area) {  // viscous.rs:421-424
  float lv = 1.4f * (mu_c / 0.72f + mu_t_c / 0.9f) / rho_c;
  return 2.0f * lv * len * len / area;
}
__device__ __forceinline__ double hoop_stress(double mue, float4 g4, double v_c, double r_c) {  // viscous.rs:413-416
  double div = (double)g4.x + (double)g4.w + v_c / r_c;
  return mue * (2.0 * v_c / r_c - 2.0 / 3.0 * div);
}
__device__ __forceinline__ V4<double> d4(const double4& v) { return mk4<double>(v.x, v.y, v.z, v.w); }
__device__ __forceinline__ double4 to_d4(const V4<double>& v) { return make_double4(v[0], v[1], v[2], v[3]); }
__device__ __forceinline__ V4<double> f2d(const float4& v) { return mk4<double>(v.x, v.y, v.z, v.w); }

// dt_kind: 0 = keep dt, 1 = explicit local time step (solver.rs:614-643), 2 = implicit pseudo-time step (implicit.rs:666-695)
// NT threads per block (>= TI * TJ; the first TI * TJ also own a cell each): the tile's TJ (TI + 1) + (TJ + 1) TI = 552 face
// fluxes are spread over all NT, so with NT = 288 no thread computes more than two of them (three with 256); MINB blocks
// per SM bound the registers. The arena's autotuner picks NT for the implicit iteration, with MINB = 3: the two compile to
// the same arithmetic (checked bit for bit), whereas MINB = 2 rounds differently.
// FAS forcing of coarse cell (i, j) of case c (multigrid.rs:147-171): the volume-weighted mean residual of its fluid
// children in the fine case, less its own residual as stored; nothing where every child is solid
__device__ __forceinline__ void restrict_forcing_cell(const Arena& A, const CaseDev& c, int i, int j) {
  const CaseDev& f = A.cases[c.fine_case];
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

// FORCING: the coarse level of a multigrid transfer; each cell also writes its FAS forcing from the residual it has just
// stored (k_restrict_forcing folded into the coarse residual evaluation)
template <int NT, int MINB, bool FORCING = false>
__global__ void __launch_bounds__(NT, MINB) k_residual(Arena A, int dt_kind, int slot) {
  __shared__ __align__(128) float4 sW[TJ + 4][TI + 4];
  __shared__ __align__(128) float4 sWl[TJ + 4][TI + 4];
  __shared__ double4 sFI[TJ][TI + 1];
  __shared__ double4 sFJ[TJ + 1][TI];
  __shared__ double sred[NT / 32];
  __shared__ float s_cfl;
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ int s_ok;
  const int t = tile_at(A);
  const int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci]) return;
  const int lt = t - c.tile_off;
  const int i0 = (lt % c.ntx) * TI, j0 = (lt / c.ntx) * TJ;
  const int ni = c.ni, nj = c.nj;
  const int tid = threadIdx.x;
  const int iter = A.iter[ci];
  const int lim = iter < c.first_order_iters ? LIM_FIRST : c.limiter;
  if (tid == 0) {
    if (dt_kind == 2) {
      int k = A.ramp_k[ci];
      double cfl = (double)c.cfl0 * pow((double)c.growth, (double)(k < 10000 ? k : 10000));
      s_cfl = (float)fmin(cfl, (double)c.cfl_max);
    } else {
      s_cfl = c.cfl;
    }
    bktma::mbar_init(&s_bar, 1);
    bktma::mbar_init_fence();
  }
  __syncthreads();
  // stage the padded primitives of the tile and its 2-cell halo, (TJ + 4) x (TI + 4) cells of both words of the pair,
  // with two TMA box loads: the tile's padded origin (i0, j0) is cell (i0 - 2, j0 - 2), its x offset 4 i0 floats is
  // 16-byte aligned; cells beyond the padded array read zeros and are never used (faces past i = ni, j = nj are skipped)
  if (tid == 0) {
    const CUtensorMap* m = A.wmaps + 2 * ci;
    bktma::tensormap_acquire(m);
    bktma::tensormap_acquire(m + 1);
    bktma::mbar_expect_tx(&s_bar, (uint32_t)(2 * sizeof(sW)));
    bktma::tma_load_2d(&sW[0][0], m, &s_bar, 4 * i0, j0);
    bktma::tma_load_2d(&sWl[0][0], m + 1, &s_bar, 4 * i0, j0);
  }
  const bool staged = bktma::mbar_wait(&s_bar, 0);
  if (tid == 0) s_ok = 1;
  __syncthreads();
  if (!staged) s_ok = 0;
  __syncthreads();
  if (!s_ok) {  // the staging never completed (bounded wait): the tile's residual becomes NaN, which the host reports
    const int q = tid % TI, r = tid / TI;
    if (tid < TI * TJ && i0 + q < ni && j0 + r < nj) A.R[cidx(c, i0 + q, j0 + r)] = make_float4(NAN, NAN, NAN, NAN);
    if (tid == 0 && slot >= 0) atomicAdd(&A.rsum[(long long)slot * A.ncases + ci], (double)NAN);
    return;
  }
  auto wd = [&](int r, int q) { return pair_ld(sW[r][q], sWl[r][q]); };
  // i faces (TI+1 per row) and j faces (TJ+1 per column), FP64
  for (int idx = tid; idx < TJ * (TI + 1) + (TJ + 1) * TI; idx += blockDim.x) {
    if (idx < TJ * (TI + 1)) {
      int r = idx / (TI + 1), q = idx % (TI + 1);
      int i = i0 + q, j = j0 + r;
      if (i <= ni && j < nj) {
        V4<double> fl = iface_flux(A, c, i, j, wd(r + 2, q), wd(r + 2, q + 1), wd(r + 2, q + 2), wd(r + 2, q + 3), lim,
                                   A.iface[ifidx(c, i, j)]);
        sFI[r][q] = to_d4(fl);
      }
    } else {
      int k = idx - TJ * (TI + 1);
      int r = k / TI, q = k % TI;
      int i = i0 + q, j = j0 + r;
      if (i < ni && j <= nj) {
        V4<double> fl;
        if (c.has_block && j < col_start(c, i)) {
          fl = mk4<double>(0, 0, 0, 0);
        } else {
          float4 f = A.jface[jfidx(c, i, j)];
          fl = face_flux_lm<double>(wd(r, q + 2), wd(r + 1, q + 2), wd(r + 2, q + 2), wd(r + 3, q + 2), lim, f.x, f.y,
                                    c.low_mach != 0);
        }
        sFJ[r][q] = to_d4(fl);
        // inviscid mass flux of the face for the turbulence convection (turbulence.rs:445-456)
        if (A.mflux_j && c.sst) A.mflux_j[jfidx(c, i, j)] = (float)fl[0];
      }
    }
  }
  __syncthreads();
  if (A.mflux_i && c.sst) {
    for (int idx = tid; idx < TJ * (TI + 1); idx += blockDim.x) {
      int r = idx / (TI + 1), q = idx % (TI + 1);
      int i = i0 + q, j = j0 + r;
      if (i <= ni && j < nj && (q < TI || i == ni)) A.mflux_i[ifidx(c, i, j)] = (float)sFI[r][q].x;
    }
  }
  const int q = tid % TI, r = tid / TI;
  const int i = i0 + q, j = j0 + r;
  double rr = 0.0;
  if (tid < TI * TJ && i < ni && j < nj) {
    long long cc = cidx(c, i, j);
    if (is_solid(c, i, j)) {
      A.R[cc] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (dt_kind) A.dt[cc] = 0.f;
      if (dt_kind == 1 && c.cfl_star > 0.f) A.irs_eps[cc] = make_float2(0.f, 0.f);
    } else {
      float4 fl = A.iface[ifidx(c, i, j)], fr = A.iface[ifidx(c, i + 1, j)];
      float4 fb = A.jface[jfidx(c, i, j)], ft = A.jface[jfidx(c, i, j + 1)];
      float4 g = A.cellg[cc];  // (V, A, xc, rc)
      V4<double> gl = d4(sFI[r][q]), gr = d4(sFI[r][q + 1]), gb = d4(sFJ[r][q]), gt = d4(sFJ[r + 1][q]);
      V4<float> wc = from_f4(sW[r + 2][q + 2]);
      const V4<double> wcd = wd(r + 2, q + 2);
      const double wl = fl.w, wr = fr.w, wb = fb.w, wt = ft.w, inv_v = 1.0 / (double)g.x;
      V4<double> out;
      float mu_c = 0.f, mut_c = 0.f;
      if (c.viscous) {
        V4<double> hl = f2d(A.fvi[ifidx(c, i, j)]), hr = f2d(A.fvi[ifidx(c, i + 1, j)]);
        V4<double> hb = f2d(A.fvj[jfidx(c, i, j)]), ht = f2d(A.fvj[jfidx(c, i, j + 1)]);
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k] = -((gr[k] - hr[k]) * wr - (gl[k] - hl[k]) * wl + (gt[k] - ht[k]) * wt - (gb[k] - hb[k]) * wb) * inv_v;
        mu_c = A.mu[cc];
        mut_c = A.mu_t[cc];
        double t_tt = hoop_stress((double)mu_c + (double)mut_c, A.grad4[cc], wcd[2], g.w);
        out[2] += (wcd[3] - t_tt) * (double)g.y * inv_v;
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k] = -(gr[k] * wr - gl[k] * wl + gt[k] * wt - gb[k] * wb) * inv_v;
        out[2] += wcd[3] * (double)g.y * inv_v;
      }
      if (A.FORCE) {
        float4 fo = A.FORCE[cc];
        out[0] += fo.x;
        out[1] += fo.y;
        out[2] += fo.z;
        out[3] += fo.w;
      }
      A.R[cc] = make_float4((float)out[0], (float)out[1], (float)out[2], (float)out[3]);
      rr = out[0] * out[0];
      if (dt_kind) {
        float cs = sqrtf(1.4f * wc[3] / wc[0]);
        auto lam = [&](float4 f) { return (fabsf(wc[1] * f.x + wc[2] * f.y) + cs) * f.z; };
        float xi = 0.f, xj = 0.f;
        if (c.viscous) {
          xi = diffusion_rate(mu_c, mut_c, wc[0], 0.5f * (fl.z + fr.z), g.y);
          xj = diffusion_rate(mu_c, mut_c, wc[0], 0.5f * (fb.z + ft.z), g.y);
        }
        float cfl = s_cfl, d;
        if (dt_kind == 1 && c.cfl_star > 0.f) {
          // with implicit residual smoothing: dt = CFL A / (L_i + L_j), and each direction whose CFL number
          // c_d = dt L_d / A exceeds cfl_star smoothed with eps_d = ((c_d / cfl_star)^2 - 1) / 4 (solver.rs:631-641)
          float li = 0.5f * (lam(fl) + lam(fr)), lj = 0.5f * (lam(fb) + lam(ft));
          if (c.viscous) li += xi, lj += xj;
          d = cfl * g.y / (li + lj);
          auto coef = [&](float l) {
            const float rr = d * l / g.y / c.cfl_star;
            return fmaxf(0.25f * (rr * rr - 1.f), 0.f);
          };
          A.irs_eps[cc] = make_float2(coef(li), coef(lj));
        } else if (dt_kind == 1) {
          float sum = lam(fl) + lam(fr) + lam(fb) + lam(ft);
          d = c.viscous ? cfl * g.y / (0.5f * sum + xi + xj) : cfl * g.y / (0.5f * sum);
        } else {
          float li = 0.5f * (lam(fl) + lam(fr)) + xi, lj = 0.5f * (lam(fb) + lam(ft)) + xj;
          d = c.dt_mode == DT_SUM ? cfl * g.y / (li + lj) : cfl * g.y / (2.0f * fminf(li, lj));
        }
        A.dt[cc] = d;
      }
    }
    if constexpr (FORCING) restrict_forcing_cell(A, c, i, j);
  }
  if (slot >= 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rr += __shfl_down_sync(0xffffffffu, rr, o);
    if ((tid & 31) == 0) sred[tid >> 5] = rr;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sred[k];
      atomicAdd(&A.rsum[(long long)slot * A.ncases + ci], s);
    }
  }
}

// ==================================================================================== explicit stage
// u = a (u + dt R) + b u0 on the fluid cells; `copy` first saves u0 = u; `last` advances the iteration counter.
__global__ void k_stage(Arena A, float a, float b, int copy, int last) {
  int t = tile_at(A);
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci]) return;
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (last && lt == 0 && threadIdx.x == 0) A.iter[ci] += 1;
  if (i >= c.ni || j >= c.nj || is_solid(c, i, j)) return;
  long long cc = cidx(c, i, j);
  float4 uh = A.U[cc], ul = A.Ulo[cc];
  if (copy) A.U0[cc] = uh, A.U0lo[cc] = ul;
  V4<double> u = pair_ld(uh, ul), u0 = copy ? u : pair_ld(A.U0[cc], A.U0lo[cc]);
  float4 r = A.R[cc];
  double d = A.dt[cc];
  V4<double> rd = f2d(r);
#pragma unroll
  for (int k = 0; k < 4; ++k) u[k] = (double)a * (u[k] + d * rd[k]) + (double)b * u0[k];
  pair_st(A.U, A.Ulo, cc, u);
}

// ==================================================================================== implicit residual smoothing
// One factor of (1 - eps_i d_ii)(1 - eps_j d_jj) R_bar = R along every i line (dir_i) or j line: the conservative scalar
// tridiagonal system -e_- x_{k-1} + (1 + e_- + e_+) x_k - e_+ x_{k+1} = r_k with face coefficients e = (eps_k +
// eps_{k+1}) / 2, zero next to solid cells, solved by the Thomas algorithm, one thread per line, the four conserved
// components together (solver.rs:722-803). in -> out (the i factor R -> X, then the j factor X -> R).
__global__ void k_irs(Arena A, int dir_i, const float4* __restrict__ in, float4* __restrict__ out) {
  const int gw = blockIdx.x * blockDim.x + threadIdx.x;
  if (gw >= (dir_i ? A.nilines : A.njlines)) return;
  const int ci = dir_i ? A.iline_case[gw] : A.jline_case[gw];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || !(c.cfl_star > 0.f)) return;
  const int L = gw - (dir_i ? c.iline_off : c.jline_off);
  const int n = dir_i ? c.ni : c.nj;
  auto cell = [&](int k) { return dir_i ? cidx(c, k, L) : cidx(c, L, k); };
  auto solid = [&](int k) { return dir_i ? is_solid(c, k, L) : is_solid(c, L, k); };
  auto eps = [&](int k) {
    const float2 v = A.irs_eps[cell(k)];
    return dir_i ? v.x : v.y;
  };
  auto face = [&](int k) { return (solid(k) || solid(k + 1)) ? 0.f : 0.5f * (eps(k) + eps(k + 1)); };  // between k and k + 1
  float4 prev = make_float4(0.f, 0.f, 0.f, 0.f);
  float cprev = 0.f, fprev = 0.f;
  for (int k = 0; k < n; ++k) {
    const float a = k > 0 ? fprev : 0.f;
    const float up = k + 1 < n ? face(k) : 0.f;
    const float m = (1.f + a + up) + a * (k > 0 ? cprev : 0.f);
    const float cp = -up / m;
    const long long cc = cell(k);
    const float4 r = in[cc];
    const float4 x = make_float4((r.x + a * prev.x) / m, (r.y + a * prev.y) / m, (r.z + a * prev.z) / m, (r.w + a * prev.w) / m);
    out[cc] = x;
    A.irs_c[cc] = cp;
    prev = x, cprev = cp, fprev = up;
  }
  float4 nx = prev;
  for (int k = n - 2; k >= 0; --k) {
    const long long cc = cell(k);
    const float cp = A.irs_c[cc];
    float4 x = out[cc];
    x.x -= cp * nx.x, x.y -= cp * nx.y, x.z -= cp * nx.z, x.w -= cp * nx.w;
    out[cc] = x;
    nx = x;
  }
}

// ==================================================================================== implicit operator

// Blocks (lo, d, up) of I - dt J_dir for fluid cell (i, j) of a line (implicit.rs:379-467).
__device__ void assemble(const Arena& A, const CaseDev& c, bool dir_i, int i, int j, M4<float>& lo, M4<float>& d, M4<float>& up) {
  const int k = dir_i ? i : j;
  const int k0 = dir_i ? row_start(c, j) : col_start(c, i);
  const long long cc = cidx(c, i, j);
  V4<float> wk = Wat(A, c, i, j);
  float4 fl = dir_i ? A.iface[ifidx(c, i, j)] : A.jface[jfidx(c, i, j)];
  float4 fr = dir_i ? A.iface[ifidx(c, i + 1, j)] : A.jface[jfidx(c, i, j + 1)];
  float4 g = A.cellg[cc];
  float src = dir_i ? 0.f : g.y / g.x;
  bool wall_lower = k == k0 && k0 > 0;
  bool jet = wall_lower && dir_i && jet_iface(c, k0, j);
  V4<float> wm;
  if (jet) {
    wm = mk4<float>(c.nz_state[0], c.nz_state[1], c.nz_state[2], c.nz_state[3]);
  } else if (wall_lower && dir_i) {
    float4 fb = A.iface[ifidx(c, k0, j)];
    wm = wall_ghost(wk, fb.x, fb.y, noslip_iface(c, k0, j));
  } else {
    wm = dir_i ? Wat(A, c, i - 1, j) : Wat(A, c, i, j - 1);
  }
  V4<float> wp = dir_i ? Wat(A, c, i + 1, j) : Wat(A, c, i, j + 1);
  float lam_l = 0.f, lam_r = 0.f;
  if (c.viscous) {
    lam_l = dir_i ? face_lambda_dev(A, c, true, i, j) : face_lambda_dev(A, c, false, i, j);
    lam_r = dir_i ? face_lambda_dev(A, c, true, i + 1, j) : face_lambda_dev(A, c, false, i, j + 1);
  }
  cell_blocks<float>(wk, wm, wp, fl.x, fl.y, fl.w, fr.x, fr.y, fr.w, g.x, A.dt[cc], c.lines != 0, src, c.roe != 0, c.eps_fix, lam_l, lam_r,
                     lo, d, up);
}

// right-hand side of a line solve for cell cc: dt R (first pass) or the stored vector
__device__ __forceinline__ V4<float> rhs_of(const Arena& A, const float4* in, bool from_res, long long cc) {
  V4<float> r = from_f4(in[cc]);
  if (from_res) {
    float d = A.dt[cc];
#pragma unroll
    for (int k = 0; k < 4; ++k) r[k] *= d;
  }
  return r;
}

// Line-solve records in A.scratch: per direction (i lines first, then j lines) a plane per field over the arena's cells,
//   F_LO, F_D, F_UP  the assembled blocks lo, d, up of I - dt J_dir (line ends folded in),
//   F_MINV, F_Y, F_GE, F_T  the factors M^-1, Y = M^-1 up, the left spike GE and the weight T of the cell's forward value
//                    in its segment's first interior cell   (a 4x4 block = 4 float4 per cell each),
//   F_G              g, the right-hand side's forward sweep (1 float4 per cell);
// then for every line and lane of the reduced separator system 44 float4 = 5 PCR levels x (alpha, gamma) + b^-1.
// A plane keeps one field of consecutive cells contiguous: the per-cell kernels (assembly, defect) store and load whole
// sectors across a warp, and a lane walking its segment of an i line reads consecutive 64-byte blocks.
// The first pass of an iteration assembles and factorises (k_assemble, k_line_ends_fold, k_lines); later passes
// (k_lines_subst) and the defect (k_defect) only read them.
enum { F_LO = 0, F_D, F_UP, F_MINV, F_Y, F_GE, F_T, F_G };
constexpr int REC = 29, PREC = 44, PCR_LEVELS = 5;  // REC: float4 per cell and direction
// float4 per direction, rounded up to whole 64-byte blocks so that the j planes start on sector boundaries
__host__ __device__ __forceinline__ long long rec_dir_stride(long long ncell) { return (ncell * REC + 3) & ~3LL; }
struct Rec {  // the record of one cell in one direction
  float4* base;
  long long n, cc;
  __device__ __forceinline__ float4* blk(int f) const { return base + (n * f + cc) * 4; }
  __device__ __forceinline__ float4* g() const { return base + n * 28 + cc; }
};
__device__ __forceinline__ Rec line_rec(const Arena& A, bool dir_i, long long cc) {
  return Rec{reinterpret_cast<float4*>(A.scratch) + (dir_i ? 0 : rec_dir_stride(A.ncell)), A.ncell, cc};
}
__device__ __forceinline__ float4* pcr_rec(const Arena& A, bool dir_i, int gw, int lane) {
  float4* base = reinterpret_cast<float4*>(A.scratch) + 2 * rec_dir_stride(A.ncell);
  if (!dir_i) base += (long long)A.nilines * 32 * PREC;
  return base + ((long long)gw * 32 + lane) * PREC;
}
__device__ __forceinline__ void st_m4(float4* p, const M4<float>& m) {
#pragma unroll
  for (int q = 0; q < 4; ++q) p[q] = make_float4(m[4 * q], m[4 * q + 1], m[4 * q + 2], m[4 * q + 3]);
}
__device__ __forceinline__ M4<float> ld_m4(const float4* p) {
  M4<float> m;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float4 v = p[q];
    m[4 * q] = v.x, m[4 * q + 1] = v.y, m[4 * q + 2] = v.z, m[4 * q + 3] = v.w;
  }
  return m;
}

// Positivity-damped update u += alpha du, alpha halved up to 8 times (implicit.rs:641-660), on the state pair in FP64.
// u: the cell's state before the update (state_of(A, cc), or the same pair fetched ahead of time)
__device__ __forceinline__ void damped_update_from(const Arena& A, long long cc, const V4<float>& dq, const V4<double>& u) {
  double alpha = 1.0;
  for (int t = 0; t < 8; ++t) {
    V4<double> q = mk4<double>(u[0] + alpha * dq[0], u[1] + alpha * dq[1], u[2] + alpha * dq[2], u[3] + alpha * dq[3]);
    V4<double> w = cons_to_prim(q);
    if (w[0] > 0.0 && w[3] > 0.0 && isfinite(q[0]) && isfinite(q[1]) && isfinite(q[2]) && isfinite(q[3])) {
      pair_st(A.U, A.Ulo, cc, q);
      return;
    }
    alpha *= 0.5;
  }
}
__device__ __forceinline__ void damped_update(const Arena& A, long long cc, const V4<float>& dq) {
  damped_update_from(A, cc, dq, state_of(A, cc));
}

constexpr int LINE_WARPS = 4;  // default lines per block of the line kernels
struct PcrSlot {  // one reduced row: a, b^-1 (or b), c, d
  float a[16], b[16], c[16], d[4];
};

// Line geometry shared by the factorisation and substitution kernels: warp `gw` solves line L of case c; lane s owns the
// segment [a, e) of m = max(m_min, ceil(len/32)) cells, the last cell of every segment but the last is a separator.
// m_min >= 2 (Arena::mmin_i / mmin_j: 2 unless pinned by bowshock_arena_set_tuning): short lines with a larger m_min
// have fewer separators, so fewer reduction multipliers to store and read (22.5 KB per line at 31 separators), and longer
// segments per lane; the rounding of the solve changes with it.
struct LineSeg {
  int gw, ci, L, n, k0, len, m, P, N, a, e, ke;
  bool act, has_sep;
};
// idx: the line's position in this launch (mapped through the compaction list)
__device__ __forceinline__ bool line_seg(const Arena& A, int dir_i, int idx, int lane, LineSeg& g) {
  const int gw = line_at(A, dir_i != 0, idx);
  if (gw < 0) return false;
  g.gw = gw;
  g.ci = dir_i ? A.iline_case[gw] : A.jline_case[gw];
  const CaseDev& c = A.cases[g.ci];
  g.L = gw - (dir_i ? c.iline_off : c.jline_off);
  g.n = dir_i ? c.ni : c.nj;
  g.k0 = dir_i ? row_start(c, g.L) : col_start(c, g.L);
  g.len = g.n - g.k0;
  if (g.len <= 0) return false;
  g.m = (g.len + 31) / 32;
  const int mmin = dir_i ? A.mmin_i : A.mmin_j;
  if (g.m < mmin) g.m = mmin;
  g.P = (g.len + g.m - 1) / g.m;
  g.N = g.P - 1;
  g.act = lane < g.P;
  g.a = g.k0 + lane * g.m;
  g.e = g.act ? min(g.a + g.m, g.n) : g.a;
  g.has_sep = g.act && lane < g.P - 1;
  g.ke = g.has_sep ? g.e - 2 : g.e - 1;  // last interior cell
  return true;
}

// Result x of cell cc of a line solve: i-sweeps write x to `out`; j-sweeps write du (pass 0) or add the correction to
// du, and the last pass of a case applies the positivity-damped update.
__device__ __forceinline__ void line_emit(const Arena& A, int epilogue, bool update, float4* out, long long cc, const V4<float>& x) {
  if (epilogue == 0) {
    out[cc] = to_f4(x);
    return;
  }
  V4<float> du = x;
  if (epilogue == 2) {
    V4<float> o = from_f4(A.DU[cc]);
#pragma unroll
    for (int q = 0; q < 4; ++q) du[q] += o[q];
  }
  A.DU[cc] = to_f4(du);
  if (update) damped_update(A, cc, du);
}

// Blocks (lo, d, up) of I - dt J_i and I - dt J_j of every fluid cell into its two line records (implicit.rs:379-467),
// one thread per cell and direction (two blocks per tile): the assembly is the arithmetic-heavy part of the operator and
// has no dependence along the lines. The direction loop and the register budget (3 blocks per SM) are kept: in this
// form the compiled arithmetic, and so every result, is bit for bit that of one thread doing both directions; a
// straight-line form and a budget of 2 blocks per SM were measured to round differently (ptxas contracts multiply-adds
// by register budget).
__global__ void __launch_bounds__(TI* TJ, 3) k_assemble(Arena A) {
  int t = tile_at(A);
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci]) return;
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (i >= c.ni || j >= c.nj || is_solid(c, i, j)) return;
  const long long cc = cidx(c, i, j);
#pragma unroll 1
  for (int dir = 0; dir < 2; ++dir) {
    if (dir != (int)blockIdx.y) continue;  // blockIdx.y: the direction of this block (0 = i lines, 1 = j lines)
    M4<float> lo, d, up;
    assemble(A, c, dir == 0, i, j, lo, d, up);
    Rec rec = line_rec(A, dir == 0, cc);
    st_m4(rec.blk(F_LO), lo);
    st_m4(rec.blk(F_D), d);
    st_m4(rec.blk(F_UP), up);
  }
}

// Ghost Jacobians of the two ends of line `L` folded into the diagonal blocks (implicit.rs:440-467): at the first cell
// d += lo T and lo = 0, with T the wall reflection / no-slip, the jet's zero, or the far-field ghost Jacobian (FP64 finite
// differences); at the last cell d += up T and up = 0. In two launches: k_line_ends_T computes every end's T from the
// primitives alone (so it can run beside the residual and the assembly), k_line_ends_fold folds them in after k_assemble.

// T of end `end` (0 first, 1 last) of line L; zero where the line has no fluid cell
__device__ __forceinline__ M4<float> line_end_T(const Arena& A, const CaseDev& c, bool dir_i, int L, int end) {
  const int n = dir_i ? c.ni : c.nj;
  const int k0 = dir_i ? row_start(c, L) : col_start(c, L);
  M4<float> T = zero4<float>();
  if (k0 >= n) return T;
  if (end == 0) {
    const int i = dir_i ? k0 : L, j = dir_i ? L : k0;
    float4 fl = dir_i ? A.iface[ifidx(c, i, j)] : A.jface[jfidx(c, i, j)];
    bool wall_lower = k0 > 0;
    bool jet = wall_lower && dir_i && jet_iface(c, k0, j);
    if (jet) {
      T = zero4<float>();
    } else if (wall_lower) {
      bool ns = dir_i ? noslip_iface(c, k0, j) : noslip_jface(c, i, k0);
      T = ns ? noslip4<float>() : reflection<float>(fl.x, fl.y);
    } else if (!c.implicit_bc) {
      T = zero4<float>();
    } else {
      int bc = dir_i ? c.bc[0] : c.bc[2];
      if (!dir_i && noslip_jface(c, i, 0) && bc == BC_SLIPWALL) {
        T = noslip4<float>();
      } else {
        M4<double> Td = ghost_jacobian(bc, fs_of(c), cvt4<double>(Wat(A, c, i, j)), fl.x, fl.y, -1.0);
#pragma unroll
        for (int q = 0; q < 16; ++q) T[q] = (float)Td[q];
      }
    }
  } else {
    const int i = dir_i ? n - 1 : L, j = dir_i ? L : n - 1;
    float4 fr = dir_i ? A.iface[ifidx(c, i + 1, j)] : A.jface[jfidx(c, i, j + 1)];
    if (!c.implicit_bc) {
      T = zero4<float>();
    } else {
      M4<double> Td = ghost_jacobian(dir_i ? c.bc[1] : c.bc[3], fs_of(c), cvt4<double>(Wat(A, c, i, j)), fr.x, fr.y, 1.0);
#pragma unroll
      for (int q = 0; q < 16; ++q) T[q] = (float)Td[q];
    }
  }
  return T;
}
// d += lo T, lo = 0 (first end) or d += up T, up = 0 (last end) in the end cell's line record
__device__ __forceinline__ void fold_line_end(const Arena& A, const CaseDev& c, bool dir_i, int L, int end, const M4<float>& T) {
  const int n = dir_i ? c.ni : c.nj;
  const int k0 = dir_i ? row_start(c, L) : col_start(c, L);
  if (k0 >= n) return;
  const int k = end == 0 ? k0 : n - 1;
  const long long cc = dir_i ? cidx(c, k, L) : cidx(c, L, k);
  const int f = end == 0 ? F_LO : F_UP;
  Rec rec = line_rec(A, dir_i, cc);
  M4<float> d = ld_m4(rec.blk(F_D));
  axpy(d, 1.f, mm(ld_m4(rec.blk(f)), T));
  st_m4(rec.blk(f), zero4<float>());
  st_m4(rec.blk(F_D), d);
}
// the slot of end `end` of global line gw in A.lend (4 float4 per end; i lines first)
__device__ __forceinline__ float4* lend_slot(const Arena& A, bool dir_i, int gw, int end) {
  return A.lend + ((long long)(dir_i ? gw : A.nilines + gw) * 2 + end) * 4;
}
// thread t: line t / 2 of the launch (every i line, then every j line, of the active cases), end t % 2
__device__ __forceinline__ bool line_end_of(const Arena& A, int t, bool& dir_i, int& gw, int& e) {
  e = t & 1;
  const int l = t >> 1, nli = lines_of(A, true);
  dir_i = l < nli;
  gw = line_at(A, dir_i, dir_i ? l : l - nli);
  return gw >= 0;
}
__global__ void k_line_ends_T(Arena A) {
  bool dir_i;
  int gw, e;
  if (!line_end_of(A, blockIdx.x * blockDim.x + threadIdx.x, dir_i, gw, e)) return;
  const int ci = dir_i ? A.iline_case[gw] : A.jline_case[gw];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci]) return;
  const int L = gw - (dir_i ? c.iline_off : c.jline_off);
  st_m4(lend_slot(A, dir_i, gw, e), line_end_T(A, c, dir_i, L, e));
}
__global__ void k_line_ends_fold(Arena A) {
  bool dir_i;
  int gw, e;
  if (!line_end_of(A, blockIdx.x * blockDim.x + threadIdx.x, dir_i, gw, e)) return;
  const int ci = dir_i ? A.iline_case[gw] : A.jline_case[gw];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci]) return;
  const int L = gw - (dir_i ? c.iline_off : c.jline_off);
  const int n = dir_i ? c.ni : c.nj;
  const int k0 = dir_i ? row_start(c, L) : col_start(c, L);
  if (n - k0 == 1) {  // one cell: both ends in the first thread (the two folds update the same diagonal block)
    if (e == 0) {
      fold_line_end(A, c, dir_i, L, 0, ld_m4(lend_slot(A, dir_i, gw, 0)));
      fold_line_end(A, c, dir_i, L, 1, ld_m4(lend_slot(A, dir_i, gw, 1)));
    }
    return;
  }
  fold_line_end(A, c, dir_i, L, e, ld_m4(lend_slot(A, dir_i, gw, e)));
}

// cp.async copies of 16 (or 4) bytes from global into shared memory, one commit group per call of cp_commit; cp_wait<N>
// waits until at most N of this thread's groups are in flight (the staged walks below keep one group per cell, SUB_SD
// cells ahead of the arithmetic).
constexpr int SUB_SD = 3;
__device__ __forceinline__ void cp16(float4* smem, const float4* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp4(float* smem, const float* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// a 4x4 block whose rows lie 32 float4 apart (one lane's slots of a staging array)
__device__ __forceinline__ M4<float> ld_m4s(const float4* p) {
  M4<float> m;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float4 v = p[32 * q];
    m[4 * q] = v.x, m[4 * q + 1] = v.y, m[4 * q + 2] = v.z, m[4 * q + 3] = v.w;
  }
  return m;
}
__device__ __forceinline__ void cp_m4(float4* smem, const float4* gmem) {
#pragma unroll
  for (int q = 0; q < 4; ++q) cp16(smem + 32 * q, gmem + q);
}

// First pass of an iteration (implicit.rs:619-621): with the blocks k_assemble and k_line_ends_fold left in the line records, factorise
// with the partitioned solver (each lane eliminates its segment, the separator unknowns form a
// reduced 4x4-block tridiagonal system solved by parallel cyclic reduction through shared memory, each lane
// back-substitutes), solve for the first right-hand side, and keep blocks, factors and reduction multipliers in the line
// records for the later passes and the defect.
// W: lines (warps) per block; PF 1: the walks load the next cell's record before the arithmetic of the current one
// (software pipelining: more memory parallelism per lane, ~80 more registers, so fewer warps per SM); PF 2: each lane's
// records staged through shared memory SUB_SD cells ahead (cp.async, one line per block), for directions with few lines
// left, whose walks otherwise wait for one memory round trip per cell. The arena's autotuner picks W and PF 0 / 1 per
// direction; the results do not depend on them.
template <int W, int PF>
__global__ void __launch_bounds__(32 * W) k_lines(Arena A, int dir_i, const float4* in, int from_res, float4* out) {
  static_assert(PF != 2 || W == 1, "the staged walks run one line per block");
  __shared__ PcrSlot sp[W][32];
  __shared__ float4 sl[W][32];
  // PF == 2: per lane SUB_SD cells of records in flight (forward: lo 0-3, d 4-7, up 8-11, r 12; backward: Y 0-3, GE 4-7,
  // g 8), their time steps, and the separator row (lo, d, up, r and its time step)
  __shared__ float4 stg[PF == 2 ? SUB_SD : 1][PF == 2 ? 13 : 1][32];
  __shared__ float stg_dt[PF == 2 ? SUB_SD : 1][32];
  __shared__ float4 ssep[PF == 2 ? 13 : 1][32];
  __shared__ float ssep_dt[32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * W + warp;
  LineSeg G;
  if (!line_seg(A, dir_i, gw, lane, G)) return;
  const int ci = G.ci;
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci]) return;
  const int epilogue = dir_i ? 0 : 1;
  const bool update = !dir_i && c.sub_iters <= 1;
  const int L = G.L, n = G.n, P = G.P, N = G.N, a = G.a, e = G.e, ke = G.ke;
  const int s = lane;
  const bool act = G.act, has_sep = G.has_sep;
  auto cell = [&](int k) { return dir_i ? cidx(c, k, L) : cidx(c, L, k); };
  (void)n;
  (void)P;
  // ---- forward elimination of the segment interior. The segment's first interior cell in terms of the separators,
  // x_a = v_f + E_f l_left + F_f l_right, follows from the back substitution x_k = g_k + GE_k l_left - Y_k x_k+1 unrolled:
  // v_f = sum_k T_k g_k, E_f = sum_k T_k GE_k, F_f = T_ke+1 with T_a = I, T_k+1 = -T_k Y_k; the sums are accumulated
  // on the way down (no backward walk), and T_k is kept for the substitution passes' v_f.
  M4<float> Y = zero4<float>(), GE = zero4<float>(), T = eye4<float>(), E_f = zero4<float>();
  V4<float> g = mk4<float>(0, 0, 0, 0), v_f = mk4<float>(0, 0, 0, 0);
  if constexpr (PF == 2) {
    // the walk of k_lines<W, 0> with each lane's records staged SUB_SD cells ahead (the same arithmetic)
    const bool di = dir_i != 0;
    if (has_sep) {
      const long long cs = cell(e - 1);
      const Rec r = line_rec(A, di, cs);
      cp_m4(&ssep[0][lane], r.blk(F_LO));
      cp_m4(&ssep[4][lane], r.blk(F_D));
      cp_m4(&ssep[8][lane], r.blk(F_UP));
      cp16(&ssep[12][lane], in + cs);
      if (from_res) cp4(&ssep_dt[lane], A.dt + cs);
    }
    cp_commit();
    const int nk = act ? ke - a + 1 : 0, mk = G.m;
    auto issue_f = [&](int k, int slot) {
      const long long cc = cell(a + k);
      const Rec r = line_rec(A, di, cc);
      cp_m4(&stg[slot][0][lane], r.blk(F_LO));
      cp_m4(&stg[slot][4][lane], r.blk(F_D));
      cp_m4(&stg[slot][8][lane], r.blk(F_UP));
      cp16(&stg[slot][12][lane], in + cc);
      if (from_res) cp4(&stg_dt[slot][lane], A.dt + cc);
    };
#pragma unroll
    for (int q = 0; q < SUB_SD; ++q) {
      if (q < nk) issue_f(q, q);
      cp_commit();
    }
    for (int kk = 0; kk < mk; ++kk) {
      cp_wait<SUB_SD - 1>();
      const int slot = kk % SUB_SD;
      if (kk < nk) {
        const int k = a + kk;
        const Rec rec_k = line_rec(A, di, cell(k));
        const M4<float> Ak = ld_m4s(&stg[slot][0][lane]), Bk = ld_m4s(&stg[slot][4][lane]), Ck = ld_m4s(&stg[slot][8][lane]);
        V4<float> r = from_f4(stg[slot][12][lane]);
        if (from_res) {
          float d = stg_dt[slot][lane];
#pragma unroll
          for (int q = 0; q < 4; ++q) r[q] *= d;
        }
        M4<float> M = Bk;
        M4<float> GEr;
        if (k > a) {
          axpy(M, -1.f, mm(Ak, Y));
          V4<float> t = mv(Ak, g);
#pragma unroll
          for (int q = 0; q < 4; ++q) r[q] -= t[q];
          GEr = mm(Ak, GE);
        } else {
          GEr = Ak;
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) GEr[q] = -GEr[q];
        M4<float> Minv = inv4(M);
        g = mv(Minv, r);
        GE = mm(Minv, GEr);
        Y = mm(Minv, Ck);
        st_m4(rec_k.blk(F_MINV), Minv);
        st_m4(rec_k.blk(F_Y), Y);
        st_m4(rec_k.blk(F_GE), GE);
        st_m4(rec_k.blk(F_T), T);
        *rec_k.g() = to_f4(g);
        const V4<float> tg = mv(T, g);
#pragma unroll
        for (int q = 0; q < 4; ++q) v_f[q] += tg[q];
        axpy(E_f, 1.f, mm(T, GE));
        T = mm(T, Y);
#pragma unroll
        for (int q = 0; q < 16; ++q) T[q] = -T[q];
      }
      __syncwarp();
      if (kk + SUB_SD < nk) issue_f(kk + SUB_SD, slot);
      cp_commit();
    }
  } else if (act) {
    Rec rec = line_rec(A, dir_i != 0, cell(a));
    M4<float> An, Bn, Cn;
    V4<float> rn;
    if (PF == 1) {
      An = ld_m4(rec.blk(F_LO)), Bn = ld_m4(rec.blk(F_D)), Cn = ld_m4(rec.blk(F_UP));
      rn = rhs_of(A, in, from_res != 0, cell(a));
    }
    for (int k = a; k <= ke; ++k) {
      if (PF == 0) {
        rec = line_rec(A, dir_i != 0, cell(k));
        An = ld_m4(rec.blk(F_LO)), Bn = ld_m4(rec.blk(F_D)), Cn = ld_m4(rec.blk(F_UP));
        rn = rhs_of(A, in, from_res != 0, cell(k));
      }
      const M4<float> Ak = An, Bk = Bn, Ck = Cn;
      V4<float> r = rn;
      const Rec rec_k = rec;
      if (PF == 1 && k < ke) {
        const long long cn = cell(k + 1);
        rec = line_rec(A, dir_i != 0, cn);
        An = ld_m4(rec.blk(F_LO)), Bn = ld_m4(rec.blk(F_D)), Cn = ld_m4(rec.blk(F_UP));
        rn = rhs_of(A, in, from_res != 0, cn);
      }
      M4<float> M = Bk;
      M4<float> GEr;
      if (k > a) {
        axpy(M, -1.f, mm(Ak, Y));
        V4<float> t = mv(Ak, g);
#pragma unroll
        for (int q = 0; q < 4; ++q) r[q] -= t[q];
        GEr = mm(Ak, GE);
      } else {
        GEr = Ak;
      }
#pragma unroll
      for (int q = 0; q < 16; ++q) GEr[q] = -GEr[q];
      M4<float> Minv = inv4(M);
      g = mv(Minv, r);
      GE = mm(Minv, GEr);
      Y = mm(Minv, Ck);
      st_m4(rec_k.blk(F_MINV), Minv);
      st_m4(rec_k.blk(F_Y), Y);
      st_m4(rec_k.blk(F_GE), GE);
      st_m4(rec_k.blk(F_T), T);
      *rec_k.g() = to_f4(g);
      const V4<float> tg = mv(T, g);
#pragma unroll
      for (int q = 0; q < 4; ++q) v_f[q] += tg[q];
      axpy(E_f, 1.f, mm(T, GE));
      T = mm(T, Y);
#pragma unroll
      for (int q = 0; q < 16; ++q) T[q] = -T[q];
    }
  }
  // ---- (v, E, F) at the last interior cell (the forward sweep's last values) and at the first (the sums)
  const V4<float> v_l = g;
  const M4<float> E_l = GE;
  M4<float> F_l;
#pragma unroll
  for (int q = 0; q < 16; ++q) F_l[q] = -Y[q];
  const M4<float> F_f = T;
  // publish (v, E, F) of the first interior cell for the lane on the left
  PcrSlot* my = &sp[warp][s];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    my->a[q] = E_f[q];
    my->c[q] = F_f[q];
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) my->d[q] = v_f[q];
  __syncwarp();
  // ---- reduced row of the separator (the last cell of the segment)
  M4<float> ra = zero4<float>(), rb = eye4<float>(), rc = zero4<float>();
  V4<float> rd = mk4<float>(0, 0, 0, 0);
  if (has_sep) {
    M4<float> As, Bs, Cs;
    V4<float> r;
    if constexpr (PF == 2) {
      As = ld_m4s(&ssep[0][lane]), Bs = ld_m4s(&ssep[4][lane]), Cs = ld_m4s(&ssep[8][lane]);
      r = from_f4(ssep[12][lane]);
      if (from_res) {
        float d = ssep_dt[lane];
#pragma unroll
        for (int k = 0; k < 4; ++k) r[k] *= d;
      }
    } else {
      Rec rec = line_rec(A, dir_i != 0, cell(e - 1));
      As = ld_m4(rec.blk(F_LO)), Bs = ld_m4(rec.blk(F_D)), Cs = ld_m4(rec.blk(F_UP));
      r = rhs_of(A, in, from_res != 0, cell(e - 1));
    }
    const PcrSlot* nx = &sp[warp][s + 1];
    M4<float> En, Fn;
    V4<float> vn;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      En[q] = nx->a[q];
      Fn[q] = nx->c[q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) vn[q] = nx->d[q];
    ra = mm(As, E_l);
    rb = Bs;
    axpy(rb, 1.f, mm(As, F_l));
    axpy(rb, 1.f, mm(Cs, En));
    rc = mm(Cs, Fn);
    V4<float> t1 = mv(As, v_l), t2 = mv(Cs, vn);
#pragma unroll
    for (int q = 0; q < 4; ++q) rd[q] = r[q] - t1[q] - t2[q];
  }
  __syncwarp();
  // ---- parallel cyclic reduction of the N separator rows across the warp; multipliers kept per level
  float4* prec = pcr_rec(A, dir_i != 0, G.gw, s);
  int lvl = 0;
  for (int h = 1; h < N; h <<= 1, ++lvl) {
    M4<float> binv = inv4(rb);
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      my->a[q] = ra[q];
      my->b[q] = binv[q];
      my->c[q] = rc[q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) my->d[q] = rd[q];
    __syncwarp();
    if (s < N) {
      M4<float> na = zero4<float>(), nc = zero4<float>(), nb = rb;
      M4<float> al = zero4<float>(), ga = zero4<float>();
      V4<float> nd = rd;
      if (s - h >= 0) {
        const PcrSlot* o = &sp[warp][s - h];
        M4<float> oa, ob, oc;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          oa[q] = o->a[q];
          ob[q] = o->b[q];
          oc[q] = o->c[q];
        }
        al = mm(ra, ob);  // alpha = -a_i b_{i-h}^-1
#pragma unroll
        for (int q = 0; q < 16; ++q) al[q] = -al[q];
        na = mm(al, oa);
        axpy(nb, 1.f, mm(al, oc));
        V4<float> od = mk4<float>(o->d[0], o->d[1], o->d[2], o->d[3]);
        V4<float> t = mv(al, od);
#pragma unroll
        for (int q = 0; q < 4; ++q) nd[q] += t[q];
      }
      if (s + h < N) {
        const PcrSlot* o = &sp[warp][s + h];
        M4<float> oa, ob, oc;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          oa[q] = o->a[q];
          ob[q] = o->b[q];
          oc[q] = o->c[q];
        }
        ga = mm(rc, ob);  // gamma = -c_i b_{i+h}^-1
#pragma unroll
        for (int q = 0; q < 16; ++q) ga[q] = -ga[q];
        nc = mm(ga, oc);
        axpy(nb, 1.f, mm(ga, oa));
        V4<float> od = mk4<float>(o->d[0], o->d[1], o->d[2], o->d[3]);
        V4<float> t = mv(ga, od);
#pragma unroll
        for (int q = 0; q < 4; ++q) nd[q] += t[q];
      }
      // only the multipliers the substitution passes read (they skip the same out-of-range neighbours)
      if (s - h >= 0) st_m4(prec + 8 * lvl, al);
      if (s + h < N) st_m4(prec + 8 * lvl + 4, ga);
      ra = na;
      rb = nb;
      rc = nc;
      rd = nd;
    }
    __syncwarp();
  }
  V4<float> lsep = mk4<float>(0, 0, 0, 0);
  if (s < N) {
    M4<float> binv = inv4(rb);
    st_m4(prec + 8 * PCR_LEVELS, binv);
    lsep = mv(binv, rd);
  }
  sl[warp][s] = to_f4(lsep);
  __syncwarp();
  if constexpr (PF == 2) {
    // the back substitution with Y, GE and g (this lane's own forward results) staged SUB_SD cells ahead
    const bool di = dir_i != 0;
    V4<float> lprev = s > 0 ? from_f4(sl[warp][s - 1]) : mk4<float>(0, 0, 0, 0);
    V4<float> xn = has_sep ? lsep : mk4<float>(0, 0, 0, 0);
    if (has_sep) line_emit(A, epilogue, update, out, cell(e - 1), lsep);
    const int nk = act ? ke - a + 1 : 0, mk = G.m;
    auto issue_b = [&](int k, int slot) {
      const Rec r = line_rec(A, di, cell(ke - k));
      cp_m4(&stg[slot][0][lane], r.blk(F_Y));
      cp_m4(&stg[slot][4][lane], r.blk(F_GE));
      cp16(&stg[slot][8][lane], r.g());
    };
    __threadfence_block();  // the forward walk's stores before the copies that read them back
    __syncwarp();
#pragma unroll
    for (int q = 0; q < SUB_SD; ++q) {
      if (q < nk) issue_b(q, q);
      cp_commit();
    }
    for (int kk = 0; kk < mk; ++kk) {
      cp_wait<SUB_SD - 1>();
      const int slot = kk % SUB_SD;
      if (kk < nk) {
        const long long cc = cell(ke - kk);
        const M4<float> Yk = ld_m4s(&stg[slot][0][lane]), GEk = ld_m4s(&stg[slot][4][lane]);
        const V4<float> gk = from_f4(stg[slot][8][lane]);
        V4<float> t1 = mv(GEk, lprev), t2 = mv(Yk, xn);
        V4<float> x;
#pragma unroll
        for (int q = 0; q < 4; ++q) x[q] = gk[q] + t1[q] - t2[q];
        line_emit(A, epilogue, update, out, cc, x);
        xn = x;
      }
      __syncwarp();
      if (kk + SUB_SD < nk) issue_b(kk + SUB_SD, slot);
      cp_commit();
    }
    cp_wait<0>();
    if (update && L == 0 && lane == 0) {
      A.iter[ci] += 1;
      A.ramp_k[ci] += 1;
    }
    return;
  }
  if (!act) return;
  // ---- back substitution of the segment
  V4<float> lprev = s > 0 ? from_f4(sl[warp][s - 1]) : mk4<float>(0, 0, 0, 0);
  V4<float> xn = has_sep ? lsep : mk4<float>(0, 0, 0, 0);
  if (has_sep) line_emit(A, epilogue, update, out, cell(e - 1), lsep);
  long long cn = cell(ke);
  Rec recb = line_rec(A, dir_i != 0, cn);
  M4<float> Yn, GEn;
  float4 gn;
  if (PF == 1) Yn = ld_m4(recb.blk(F_Y)), GEn = ld_m4(recb.blk(F_GE)), gn = *recb.g();
  for (int k = ke; k >= a; --k) {
    if (PF == 0) {
      cn = cell(k);
      recb = line_rec(A, dir_i != 0, cn);
      Yn = ld_m4(recb.blk(F_Y)), GEn = ld_m4(recb.blk(F_GE)), gn = *recb.g();
    }
    const long long cc = cn;
    const M4<float> Yk = Yn, GEk = GEn;
    const V4<float> gk = from_f4(gn);
    if (PF == 1 && k > a) {
      cn = cell(k - 1);
      recb = line_rec(A, dir_i != 0, cn);
      Yn = ld_m4(recb.blk(F_Y)), GEn = ld_m4(recb.blk(F_GE));
      gn = *recb.g();
    }
    V4<float> t1 = mv(GEk, lprev), t2 = mv(Yk, xn);
    V4<float> x;
#pragma unroll
    for (int q = 0; q < 4; ++q) x[q] = gk[q] + t1[q] - t2[q];
    line_emit(A, epilogue, update, out, cc, x);
    xn = x;
  }
  // the line through cell 0 of the case advances its iteration counters after the update
  if (update && L == 0 && lane == 0) {
    A.iter[ci] += 1;
    A.ramp_k[ci] += 1;
  }
}

__device__ __forceinline__ V4<float> shfl_up4(const V4<float>& v, int h) {
  V4<float> r;
#pragma unroll
  for (int q = 0; q < 4; ++q) r[q] = __shfl_up_sync(0xffffffffu, v[q], h);
  return r;
}
__device__ __forceinline__ V4<float> shfl_down4(const V4<float>& v, int h) {
  V4<float> r;
#pragma unroll
  for (int q = 0; q < 4; ++q) r[q] = __shfl_down_sync(0xffffffffu, v[q], h);
  return r;
}

// Defect-correction pass `pass` >= 1 (implicit.rs:622-639) of every case with more than `pass` passes: the same solve
// with the factors of the first pass. Per cell: g = M^-1 (r - lo g_prev) forward, the separators' right-hand sides, the
// reduction of the right-hand side alone with the kept multipliers (warp shuffles), x = g + GE l_left - Y x_next backward.
// W: lines (warps) per block; PF: the walks load the next cell's record before the arithmetic of the current one (more
// loads in flight per warp, ~60 more registers, so fewer warps per SM). The arena's autotuner picks both per direction;
// the arithmetic is the same.
template <int W, bool PF>
__global__ void __launch_bounds__(32 * W) k_lines_subst(Arena A, int dir_i, const float4* in, float4* out, int pass) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * W + warp;
  LineSeg G;
  if (!line_seg(A, dir_i, gw, lane, G)) return;
  const int ci = G.ci;
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || pass >= c.sub_iters) return;
  const int epilogue = dir_i ? 0 : 2;
  const bool update = !dir_i && pass == c.sub_iters - 1;
  const int L = G.L, N = G.N, a = G.a, e = G.e, ke = G.ke;
  const int s = lane;
  auto cell = [&](int k) { return dir_i ? cidx(c, k, L) : cidx(c, L, k); };
  // the forward sweep also sums the first interior cell's value v_f = sum_k T_k g_k with the kept weights
  V4<float> g = mk4<float>(0, 0, 0, 0), v_f = mk4<float>(0, 0, 0, 0);
  if (G.act) {
    long long cc = cell(a);
    Rec rec = line_rec(A, dir_i != 0, cc);
    M4<float> Lo, Mi, Tk;
    float4 rin;
    if (PF) Lo = ld_m4(rec.blk(F_LO)), Mi = ld_m4(rec.blk(F_MINV)), Tk = ld_m4(rec.blk(F_T)), rin = in[cc];
    for (int k = a; k <= ke; ++k) {
      if (!PF) {
        cc = cell(k);
        rec = line_rec(A, dir_i != 0, cc);
        Lo = ld_m4(rec.blk(F_LO)), Mi = ld_m4(rec.blk(F_MINV)), Tk = ld_m4(rec.blk(F_T)), rin = in[cc];
      }
      M4<float> Lo_n = Lo, Mi_n = Mi, T_n = Tk;
      float4 rin_n = rin;
      Rec rec_n = rec;
      if (PF && k < ke) {
        long long cn = cell(k + 1);
        rec_n = line_rec(A, dir_i != 0, cn);
        Lo_n = ld_m4(rec_n.blk(F_LO)), Mi_n = ld_m4(rec_n.blk(F_MINV)), T_n = ld_m4(rec_n.blk(F_T));
        rin_n = in[cn];
      }
      V4<float> r = from_f4(rin);
      if (k > a) {
        V4<float> t = mv(Lo, g);
#pragma unroll
        for (int q = 0; q < 4; ++q) r[q] -= t[q];
      }
      g = mv(Mi, r);
      *rec.g() = to_f4(g);
      const V4<float> tg = mv(Tk, g);
#pragma unroll
      for (int q = 0; q < 4; ++q) v_f[q] += tg[q];
      rec = rec_n, Lo = Lo_n, Mi = Mi_n, Tk = T_n, rin = rin_n;
    }
  }
  const V4<float> v_l = g;
  const V4<float> vn = shfl_down4(v_f, 1);
  V4<float> rd = mk4<float>(0, 0, 0, 0);
  if (G.has_sep) {
    long long cs = cell(e - 1);
    Rec rec = line_rec(A, dir_i != 0, cs);
    V4<float> r = from_f4(in[cs]);
    V4<float> t1 = mv(ld_m4(rec.blk(F_LO)), v_l), t2 = mv(ld_m4(rec.blk(F_UP)), vn);
#pragma unroll
    for (int q = 0; q < 4; ++q) rd[q] = r[q] - t1[q] - t2[q];
  }
  const float4* prec = pcr_rec(A, dir_i != 0, G.gw, s);
  int lvl = 0;
  for (int h = 1; h < N; h <<= 1, ++lvl) {
    V4<float> dm = shfl_up4(rd, h), dp = shfl_down4(rd, h);
    if (s < N) {
      V4<float> nd = rd;
      if (s - h >= 0) {
        V4<float> t = mv(ld_m4(prec + 8 * lvl), dm);
#pragma unroll
        for (int q = 0; q < 4; ++q) nd[q] += t[q];
      }
      if (s + h < N) {
        V4<float> t = mv(ld_m4(prec + 8 * lvl + 4), dp);
#pragma unroll
        for (int q = 0; q < 4; ++q) nd[q] += t[q];
      }
      rd = nd;
    }
  }
  V4<float> lsep = mk4<float>(0, 0, 0, 0);
  if (s < N) lsep = mv(ld_m4(prec + 8 * PCR_LEVELS), rd);
  V4<float> lprev = shfl_up4(lsep, 1);
  if (s == 0) lprev = mk4<float>(0, 0, 0, 0);
  if (!G.act) return;
  V4<float> xn = G.has_sep ? lsep : mk4<float>(0, 0, 0, 0);
  if (G.has_sep) line_emit(A, epilogue, update, out, cell(e - 1), lsep);
  {
    long long cc = cell(ke);
    Rec rec = line_rec(A, dir_i != 0, cc);
    M4<float> GEk, Yk;
    float4 gk4;
    if (PF) GEk = ld_m4(rec.blk(F_GE)), Yk = ld_m4(rec.blk(F_Y)), gk4 = *rec.g();
    for (int k = ke; k >= a; --k) {
      if (!PF) {
        cc = cell(k);
        rec = line_rec(A, dir_i != 0, cc);
        GEk = ld_m4(rec.blk(F_GE)), Yk = ld_m4(rec.blk(F_Y)), gk4 = *rec.g();
      }
      M4<float> GE_n = GEk, Y_n = Yk;
      float4 g_n = gk4;
      long long cn = cc;
      if (PF && k > a) {
        cn = cell(k - 1);
        Rec rn = line_rec(A, dir_i != 0, cn);
        GE_n = ld_m4(rn.blk(F_GE)), Y_n = ld_m4(rn.blk(F_Y)), g_n = *rn.g();
      }
      V4<float> t1 = mv(GEk, lprev), t2 = mv(Yk, xn);
      V4<float> gk = from_f4(gk4);
      V4<float> x;
#pragma unroll
      for (int q = 0; q < 4; ++q) x[q] = gk[q] + t1[q] - t2[q];
      line_emit(A, epilogue, update, out, cc, x);
      xn = x;
      cc = cn, GEk = GE_n, Yk = Y_n, gk4 = g_n;
    }
  }
  if (update && L == 0 && lane == 0) {
    A.iter[ci] += 1;
    A.ramp_k[ci] += 1;
  }
}

// ---- substitution passes with the walks' records staged through shared memory
// Each lane copies the records of the next SUB_SD cells of its segment into shared memory ahead of the arithmetic
// (cp.async, one commit group per cell), and the separator row and the reduction multipliers it will read are fetched at
// the start: a walk waits for one memory round trip per SUB_SD cells instead of one per cell, which is what bounds the
// passes when few lines are left (a lane's segment of a handful of cells is a chain of dependent loads otherwise). One
// line per block, 47 KB of shared memory. Every lane copies and reads only its own slots, so the copies need no barrier
// across the warp; the __syncwarp before each refill orders a slot's reads before the copy that overwrites it.
struct SubstStage {
  float4 w[SUB_SD][13][32];  // forward: lo 0-3, M^-1 4-7, T 8-11, r 12; backward: GE 0-3, Y 4-7, g 8, du 9, U 10, Ulo 11
  float4 p[PREC][32];        // the lane's reduction multipliers
  float4 sp[9][32];          // the separator row: lo 0-3, up 4-7, r 8
};
static_assert(sizeof(SubstStage) <= 48 * 1024, "static shared memory");
// The defect-correction pass of k_lines_subst (same arithmetic, same results) with the staged records.
__global__ void __launch_bounds__(32) k_lines_subst_st(Arena A, int dir_i, const float4* in, float4* out, int pass) {
  __shared__ SubstStage S;
  const int lane = threadIdx.x;
  LineSeg G;
  if (!line_seg(A, dir_i, blockIdx.x, lane, G)) return;
  const int ci = G.ci;
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || pass >= c.sub_iters) return;
  const bool di = dir_i != 0;
  const int epilogue = dir_i ? 0 : 2;
  const bool update = !dir_i && pass == c.sub_iters - 1;
  const int L = G.L, N = G.N, a = G.a, e = G.e, ke = G.ke;
  const int s = lane;
  auto cell = [&](int k) { return dir_i ? cidx(c, k, L) : cidx(c, L, k); };
  // the separator row and the multipliers this lane reads (the predicates of the reduction below)
  if (G.has_sep) {
    const long long cs = cell(e - 1);
    const Rec r = line_rec(A, di, cs);
    cp_m4(&S.sp[0][lane], r.blk(F_LO));
    cp_m4(&S.sp[4][lane], r.blk(F_UP));
    cp16(&S.sp[8][lane], in + cs);
  }
  const float4* prec = pcr_rec(A, di, G.gw, s);
  if (s < N) {
    int lvl = 0;
    for (int h = 1; h < N; h <<= 1, ++lvl) {
      if (s - h >= 0) cp_m4(&S.p[8 * lvl][lane], prec + 8 * lvl);
      if (s + h < N) cp_m4(&S.p[8 * lvl + 4][lane], prec + 8 * lvl + 4);
    }
    cp_m4(&S.p[8 * PCR_LEVELS][lane], prec + 8 * PCR_LEVELS);
  }
  cp_commit();
  const int nk = G.act ? ke - a + 1 : 0, mk = G.m;  // cells of this lane's walks; mk >= nk for every lane
  // forward: g = M^-1 (r - lo g_prev), v_f = sum_k T_k g_k
  auto issue_f = [&](int k, int slot) {
    const long long cc = cell(a + k);
    const Rec r = line_rec(A, di, cc);
    cp_m4(&S.w[slot][0][lane], r.blk(F_LO));
    cp_m4(&S.w[slot][4][lane], r.blk(F_MINV));
    cp_m4(&S.w[slot][8][lane], r.blk(F_T));
    cp16(&S.w[slot][12][lane], in + cc);
  };
#pragma unroll
  for (int q = 0; q < SUB_SD; ++q) {
    if (q < nk) issue_f(q, q);
    cp_commit();
  }
  V4<float> g = mk4<float>(0, 0, 0, 0), v_f = mk4<float>(0, 0, 0, 0);
  for (int k = 0; k < mk; ++k) {
    cp_wait<SUB_SD - 1>();
    const int slot = k % SUB_SD;
    if (k < nk) {
      const long long cc = cell(a + k);
      const M4<float> Lo = ld_m4s(&S.w[slot][0][lane]), Mi = ld_m4s(&S.w[slot][4][lane]), Tk = ld_m4s(&S.w[slot][8][lane]);
      V4<float> r = from_f4(S.w[slot][12][lane]);
      if (k > 0) {
        V4<float> t = mv(Lo, g);
#pragma unroll
        for (int q = 0; q < 4; ++q) r[q] -= t[q];
      }
      g = mv(Mi, r);
      *line_rec(A, di, cc).g() = to_f4(g);
      const V4<float> tg = mv(Tk, g);
#pragma unroll
      for (int q = 0; q < 4; ++q) v_f[q] += tg[q];
    }
    __syncwarp();
    if (k + SUB_SD < nk) issue_f(k + SUB_SD, slot);
    cp_commit();
  }
  const V4<float> v_l = g;
  const V4<float> vn = shfl_down4(v_f, 1);
  V4<float> rd = mk4<float>(0, 0, 0, 0);
  if (G.has_sep) {
    V4<float> r = from_f4(S.sp[8][lane]);
    V4<float> t1 = mv(ld_m4s(&S.sp[0][lane]), v_l), t2 = mv(ld_m4s(&S.sp[4][lane]), vn);
#pragma unroll
    for (int q = 0; q < 4; ++q) rd[q] = r[q] - t1[q] - t2[q];
  }
  int lvl = 0;
  for (int h = 1; h < N; h <<= 1, ++lvl) {
    V4<float> dm = shfl_up4(rd, h), dp = shfl_down4(rd, h);
    if (s < N) {
      V4<float> nd = rd;
      if (s - h >= 0) {
        V4<float> t = mv(ld_m4s(&S.p[8 * lvl][lane]), dm);
#pragma unroll
        for (int q = 0; q < 4; ++q) nd[q] += t[q];
      }
      if (s + h < N) {
        V4<float> t = mv(ld_m4s(&S.p[8 * lvl + 4][lane]), dp);
#pragma unroll
        for (int q = 0; q < 4; ++q) nd[q] += t[q];
      }
      rd = nd;
    }
  }
  V4<float> lsep = mk4<float>(0, 0, 0, 0);
  if (s < N) lsep = mv(ld_m4s(&S.p[8 * PCR_LEVELS][lane]), rd);
  V4<float> lprev = shfl_up4(lsep, 1);
  if (s == 0) lprev = mk4<float>(0, 0, 0, 0);
  V4<float> xn = G.has_sep ? lsep : mk4<float>(0, 0, 0, 0);
  if (G.has_sep) line_emit(A, epilogue, update, out, cell(e - 1), lsep);
  // backward: x = g + GE l_left - Y x_next, from the last interior cell down; the j passes also fetch du (and the
  // state, for the last pass's update) ahead of time
  auto issue_b = [&](int k, int slot) {
    const long long cc = cell(ke - k);
    const Rec r = line_rec(A, di, cc);
    cp_m4(&S.w[slot][0][lane], r.blk(F_GE));
    cp_m4(&S.w[slot][4][lane], r.blk(F_Y));
    cp16(&S.w[slot][8][lane], r.g());
    if (epilogue == 2) cp16(&S.w[slot][9][lane], A.DU + cc);
    if (update) {
      cp16(&S.w[slot][10][lane], A.U + cc);
      cp16(&S.w[slot][11][lane], A.Ulo + cc);
    }
  };
  __threadfence_block();  // the forward walk's g stores before the copies that read them back
  __syncwarp();
#pragma unroll
  for (int q = 0; q < SUB_SD; ++q) {
    if (q < nk) issue_b(q, q);
    cp_commit();
  }
  for (int k = 0; k < mk; ++k) {
    cp_wait<SUB_SD - 1>();
    const int slot = k % SUB_SD;
    if (k < nk) {
      const long long cc = cell(ke - k);
      const M4<float> GEk = ld_m4s(&S.w[slot][0][lane]), Yk = ld_m4s(&S.w[slot][4][lane]);
      V4<float> t1 = mv(GEk, lprev), t2 = mv(Yk, xn);
      V4<float> gk = from_f4(S.w[slot][8][lane]);
      V4<float> x;
#pragma unroll
      for (int q = 0; q < 4; ++q) x[q] = gk[q] + t1[q] - t2[q];
      if (epilogue == 0) {
        out[cc] = to_f4(x);
      } else {
        V4<float> du = x;
        V4<float> o = from_f4(S.w[slot][9][lane]);
#pragma unroll
        for (int q = 0; q < 4; ++q) du[q] += o[q];
        A.DU[cc] = to_f4(du);
        if (update) damped_update_from(A, cc, du, pair_ld(S.w[slot][10][lane], S.w[slot][11][lane]));
      }
      xn = x;
    }
    __syncwarp();
    if (k + SUB_SD < nk) issue_b(k + SUB_SD, slot);
    cp_commit();
  }
  cp_wait<0>();
  if (update && L == 0 && lane == 0) {
    A.iter[ci] += 1;
    A.ramp_k[ci] += 1;
  }
}

// Defect of the unfactored operator (implicit.rs:622-630): rr = dt R - (A_i du + A_j du - du), per fluid cell, with the
// blocks the first pass kept in the line records.
__global__ void k_defect(Arena A, int pass) {
  int t = tile_at(A);
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || pass >= c.sub_iters) return;
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (i >= c.ni || j >= c.nj) return;
  long long cc = cidx(c, i, j);
  if (is_solid(c, i, j)) {
    A.RR[cc] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  V4<float> du = from_f4(A.DU[cc]);
  V4<float> acc = mk4<float>(0, 0, 0, 0);
  for (int dir = 0; dir < 2; ++dir) {
    bool di = dir == 0;
    Rec rec = line_rec(A, di, cc);
    V4<float> v = mv(ld_m4(rec.blk(F_D)), du);
    int k = di ? i : j, kn = di ? c.ni : c.nj;
    int k0 = di ? row_start(c, j) : col_start(c, i);
    if (k > k0) {
      V4<float> t2 = mv(ld_m4(rec.blk(F_LO)), from_f4(A.DU[di ? cidx(c, i - 1, j) : cidx(c, i, j - 1)]));
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] += t2[q];
    }
    if (k + 1 < kn) {
      V4<float> t2 = mv(ld_m4(rec.blk(F_UP)), from_f4(A.DU[di ? cidx(c, i + 1, j) : cidx(c, i, j + 1)]));
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] += t2[q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] += v[q];
  }
  float4 r = A.R[cc];
  float d = A.dt[cc];
  float4 o;
  o.x = r.x * d - (acc[0] - du[0]);
  o.y = r.y * d - (acc[1] - du[1]);
  o.z = r.z * d - (acc[2] - du[2]);
  o.w = r.w * d - (acc[3] - du[3]);
  A.RR[cc] = o;
}

}  // namespace bk
