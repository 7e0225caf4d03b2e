// Viscous terms of the axisymmetric RANS residual (crates/bowshock-cfd/src/viscous.rs), FP32 on the arena:
//   face sides with the ghost / wall / jet rules (viscous.rs:150-215), the face stencils (|d|, e) between the side
//   positions (viscous.rs:233-250; derived in FP64 on the host, stored per face), the face viscosities (viscous.rs:256-270), the Green-Gauss cell gradients (cell pass,
//   viscous.rs:280-316), the viscous face fluxes (face pass, viscous.rs:319-381) and the diffusive spectral radius of the
//   implicit operator (viscous.rs:429-454). Smooth walls only: the rough-wall (Aupoix) state is not on the GPU path.
#pragma once
#include "arena.cuh"
#include "device_math.cuh"

namespace bk {

constexpr float PR = 0.72f, PR_T = 0.9f;

struct SideD {
  V4<float> w;
  long long cell;  // fluid cell the side belongs to (a ghost: the adjacent fluid cell)
  bool ghost;
  bool fixed;      // jet ghost: fixed mu, mu_t
  float fmu, fmut;
};
struct SidesD {
  SideD l, r;
  bool noslip;
};

__device__ __forceinline__ float mu_of(const CaseDev& c, float t) {  // viscous.rs:48-50 (Sutherland)
  float s = (float)c.sutherland;
  return powf(t, 1.5f) * (1.0f + s) / (t + s) / (float)c.re_c;
}

// viscous.rs:150-188; false inside the solid block
__device__ bool iface_sides_d(const Arena& A, const CaseDev& c, int i, int j, SidesD& o) {
  o.noslip = false;
  o.l.fixed = o.r.fixed = false;
  if (c.has_block && j < c.j_end) {
    if (j < c.j_sting || i < c.i_end) return false;
    if (i == c.i_end) {
      long long cc = cidx(c, i, j);
      V4<float> wr = from_f4(A.W[pidx(c, i, j)]);
      if (c.has_nozzle && j < c.nz_j_end) {
        V4<float> js = mk4<float>(c.nz_state[0], c.nz_state[1], c.nz_state[2], c.nz_state[3]);
        o.l = SideD{js, cc, true, true, mu_of(c, temperature(js)), c.sst ? js[0] * c.nz_turb[0] / c.nz_turb[1] : 0.f};
        o.r = SideD{wr, cc, false, false, 0.f, 0.f};
        return true;
      }
      bool ns = noslip_iface(c, i, j);
      float4 f = A.iface[ifidx(c, i, j)];
      o.l = SideD{wall_ghost(wr, f.x, f.y, ns), cc, true, false, 0.f, 0.f};
      o.r = SideD{wr, cc, false, false, 0.f, 0.f};
      o.noslip = ns;
      return true;
    }
  }
  if (i == 0) {
    long long cc = cidx(c, 0, j);
    o.l = SideD{from_f4(A.W[pidx(c, -1, j)]), cc, true, false, 0.f, 0.f};
    o.r = SideD{from_f4(A.W[pidx(c, 0, j)]), cc, false, false, 0.f, 0.f};
  } else if (i == c.ni) {
    long long cc = cidx(c, c.ni - 1, j);
    o.l = SideD{from_f4(A.W[pidx(c, i - 1, j)]), cc, false, false, 0.f, 0.f};
    o.r = SideD{from_f4(A.W[pidx(c, i, j)]), cc, true, false, 0.f, 0.f};
  } else {
    o.l = SideD{from_f4(A.W[pidx(c, i - 1, j)]), cidx(c, i - 1, j), false, false, 0.f, 0.f};
    o.r = SideD{from_f4(A.W[pidx(c, i, j)]), cidx(c, i, j), false, false, 0.f, 0.f};
  }
  return true;
}

// viscous.rs:191-215
__device__ bool jface_sides_d(const Arena& A, const CaseDev& c, int i, int j, SidesD& o) {
  o.noslip = false;
  o.l.fixed = o.r.fixed = false;
  if (c.has_block) {
    int j0 = col_start(c, i);
    if (j < j0) return false;
    if (j == j0 && j0 > 0) {
      long long cc = cidx(c, i, j);
      o.l = SideD{from_f4(A.W[pidx(c, i, j - 1)]), cc, true, false, 0.f, 0.f};
      o.r = SideD{from_f4(A.W[pidx(c, i, j)]), cc, false, false, 0.f, 0.f};
      o.noslip = noslip_jface(c, i, j);
      return true;
    }
  }
  if (j == 0) {
    long long cc = cidx(c, i, 0);
    o.l = SideD{from_f4(A.W[pidx(c, i, -1)]), cc, true, false, 0.f, 0.f};
    o.r = SideD{from_f4(A.W[pidx(c, i, 0)]), cc, false, false, 0.f, 0.f};
    o.noslip = noslip_jface(c, i, 0);
  } else if (j == c.nj) {
    long long cc = cidx(c, i, c.nj - 1);
    o.l = SideD{from_f4(A.W[pidx(c, i, j - 1)]), cc, false, false, 0.f, 0.f};
    o.r = SideD{from_f4(A.W[pidx(c, i, j)]), cc, true, false, 0.f, 0.f};
  } else {
    o.l = SideD{from_f4(A.W[pidx(c, i, j - 1)]), cidx(c, i, j - 1), false, false, 0.f, 0.f};
    o.r = SideD{from_f4(A.W[pidx(c, i, j)]), cidx(c, i, j), false, false, 0.f, 0.f};
  }
  return true;
}

// viscous.rs:256-270: the ghost across a no-slip face carries -mu_t (smooth walls: the face value is 0), or
// 2 mu_t,w - mu_t with the rough-wall state of the wall cell (the face value is the wall's mu_t,w)
__device__ __forceinline__ void face_mu_d(const Arena& A, const CaseDev& c, const SidesD& s, float& mu_f, float& mut_f) {
  auto mus = [&](const SideD& d) { return d.fixed ? d.fmu : A.mu[d.cell]; };
  auto muts = [&](const SideD& d) {
    if (d.fixed) return d.fmut;
    if (d.ghost && s.noslip) return is_rough(c) ? 2.f * A.rough[d.cell].z - A.mu_t[d.cell] : -A.mu_t[d.cell];
    return A.mu_t[d.cell];
  };
  mu_f = 0.5f * (mus(s.l) + mus(s.r));
  mut_f = 0.5f * (muts(s.l) + muts(s.r));
}

__device__ __forceinline__ V4<float> phi3(const V4<float>& w) { return mk4<float>(w[1], w[2], temperature(w), 0.f); }  // viscous.rs:274-276

// Cell pass (viscous.rs:280-316): Sutherland viscosity and Green-Gauss gradient (u_x, u_r, v_x, v_r, T_x, T_r).
__global__ void k_visc_cell(Arena A) {
  int t = tile_at(A);
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || !c.viscous) return;
  int lt = t - c.tile_off;
  int i = (lt % c.ntx) * TI + threadIdx.x % TI, j = (lt / c.ntx) * TJ + threadIdx.x / TI;
  if (i >= c.ni || j >= c.nj) return;
  long long cc = cidx(c, i, j);
  if (is_solid(c, i, j)) {
    A.grad4[cc] = make_float4(0.f, 0.f, 0.f, 0.f);
    A.gradT[cc] = make_float2(0.f, 0.f);
    A.mu[cc] = 0.f;
    return;
  }
  V4<float> wc = from_f4(A.W[pidx(c, i, j)]);
  const float mu_c = mu_of(c, temperature(wc));
  A.mu[cc] = mu_c;
  if (is_rough(c)) {  // viscous.rs:387-409: the wall state of the cells next to a no-slip face, from this pass's mu
    float4 rw = make_float4(0.f, 0.f, 0.f, 0.f);
    const bool rough = rough_jface(c, i, j);
    if (rough || noslip_jface(c, i, j) || noslip_iface(c, i, j)) {
      const double rho = wc[0], nu = (double)mu_c / rho, d = A.dwall[cc];
      if (rough) {
        double a[3];
        aupoix_wall(nu, hypot((double)wc[1], (double)wc[2]), d, c.roughness * rough_ramp(c, i), a);
        rw = make_float4((float)a[0], (float)a[1], (float)(rho * a[2]), 0.f);
      } else {
        rw = make_float4(0.f, (float)(60.0 * nu / (0.075 * d * d)), 0.f, 0.f);
      }
    }
    A.rough[cc] = rw;
  }
  V4<float> pc = phi3(wc);
  SidesD s;
  iface_sides_d(A, c, i, j, s);
  V4<float> nb_l = s.l.w;
  iface_sides_d(A, c, i + 1, j, s);
  V4<float> nb_r = s.r.w;
  jface_sides_d(A, c, i, j, s);
  V4<float> nb_b = s.l.w;
  jface_sides_d(A, c, i, j + 1, s);
  V4<float> nb_t = s.r.w;
  float4 fs4[4] = {A.iface[ifidx(c, i + 1, j)], A.iface[ifidx(c, i, j)], A.jface[jfidx(c, i, j + 1)], A.jface[jfidx(c, i, j)]};
  const float sg[4] = {1.f, -1.f, 1.f, -1.f};
  V4<float> nbs[4] = {nb_r, nb_l, nb_t, nb_b};
  float g[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    V4<float> pn = phi3(nbs[f]);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      float pf = 0.5f * (pc[m] + pn[m]);
      g[2 * m] += sg[f] * pf * fs4[f].x * fs4[f].z;
      g[2 * m + 1] += sg[f] * pf * fs4[f].y * fs4[f].z;
    }
  }
  float inv_a = 1.f / A.cellg[cc].y;
  A.grad4[cc] = make_float4(g[0] * inv_a, g[1] * inv_a, g[2] * inv_a, g[3] * inv_a);
  A.gradT[cc] = make_float2(g[4] * inv_a, g[5] * inv_a);
}

__device__ __forceinline__ void grad6(const Arena& A, long long cc, float* g) {
  float4 a = A.grad4[cc];
  float2 b = A.gradT[cc];
  g[0] = a.x, g[1] = a.y, g[2] = a.z, g[3] = a.w, g[4] = b.x, g[5] = b.y;
}

// Viscous flux of one face (viscous.rs:319-343).
__device__ V4<float> viscous_flux_d(const Arena& A, const CaseDev& c, const SidesD& s, float4 f, float4 st) {
  if (f.w == 0.f) return mk4<float>(0, 0, 0, 0);  // r_mid = 0 (axis): weight len * r_mid is 0 exactly
  float dd = st.x, ex = st.y, er = st.z;
  float gl[6], gr[6];
  grad6(A, s.l.cell, gl);
  grad6(A, s.r.cell, gr);
  V4<float> pl = phi3(s.l.w), pr = phi3(s.r.w);
  float gf[6];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    float gbx = 0.5f * (gl[2 * m] + gr[2 * m]), gbr = 0.5f * (gl[2 * m + 1] + gr[2 * m + 1]);
    float corr = (pr[m] - pl[m]) / dd - (gbx * ex + gbr * er);
    gf[2 * m] = gbx + corr * ex;
    gf[2 * m + 1] = gbr + corr * er;
  }
  float mu_f, mut_f;
  face_mu_d(A, c, s, mu_f, mut_f);
  float uf = 0.5f * (s.l.w[1] + s.r.w[1]), vf = 0.5f * (s.l.w[2] + s.r.w[2]);
  float rm = f.w / f.z;
  float div = gf[0] + gf[3] + vf / rm;
  float mue = mu_f + mut_f;
  float txx = mue * (2.f * gf[0] - 2.f / 3.f * div);
  float trr = mue * (2.f * gf[3] - 2.f / 3.f * div);
  float txr = mue * (gf[1] + gf[2]);
  float kappa = (mu_f / PR + mut_f / PR_T) / 0.4f;
  return mk4<float>(0.f, txx * f.x + txr * f.y, txr * f.x + trr * f.y,
                    (uf * txx + vf * txr + kappa * gf[4]) * f.x + (uf * txr + vf * trr + kappa * gf[5]) * f.y);
}

// Face pass (viscous.rs:347-381): one thread per face of a residual tile's rows / columns.
__global__ void k_visc_face(Arena A) {
  int t = tile_at(A);
  int ci = A.tile_case[t];
  const CaseDev& c = A.cases[ci];
  if (!A.active[ci] || !c.viscous) return;
  int lt = t - c.tile_off;
  int i0 = (lt % c.ntx) * TI, j0 = (lt / c.ntx) * TJ;
  // The tile owns its TJ x TI left i faces and TJ x TI lower j faces (two per thread); a tile at the case's right or top
  // edge also owns the case's last i faces (q = TI) or last j faces (r = TJ), taken last.
  const int n_own = 2 * TI * TJ;
  for (int e = threadIdx.x; e < n_own + TJ + TI; e += blockDim.x) {
    int idx;
    if (e < TI * TJ) {
      idx = (e / TI) * (TI + 1) + e % TI;  // i face (r, q < TI)
    } else if (e < n_own) {
      idx = TJ * (TI + 1) + (e - TI * TJ);  // j face (r < TJ, q)
    } else if (e < n_own + TJ) {
      idx = (e - n_own) * (TI + 1) + TI;  // i face (r, q = TI)
    } else {
      idx = TJ * (TI + 1) + TJ * TI + (e - n_own - TJ);  // j face (r = TJ, q)
    }
    if (idx < TJ * (TI + 1)) {
      int r = idx / (TI + 1), q = idx % (TI + 1);
      int i = i0 + q, j = j0 + r;
      if (i > c.ni || j >= c.nj) continue;
      if (q == TI && i != c.ni) continue;  // owned by the next tile
      SidesD s;
      V4<float> fv = mk4<float>(0, 0, 0, 0);
      if (iface_sides_d(A, c, i, j, s)) fv = viscous_flux_d(A, c, s, A.iface[ifidx(c, i, j)], A.ifs[ifidx(c, i, j)]);
      A.fvi[ifidx(c, i, j)] = to_f4(fv);
    } else {
      int k = idx - TJ * (TI + 1);
      int r = k / TI, q = k % TI;
      int i = i0 + q, j = j0 + r;
      if (i >= c.ni || j > c.nj) continue;
      if (r == TJ && j != c.nj) continue;
      SidesD s;
      V4<float> fv = mk4<float>(0, 0, 0, 0);
      if (jface_sides_d(A, c, i, j, s)) fv = viscous_flux_d(A, c, s, A.jface[jfidx(c, i, j)], A.jfs[jfidx(c, i, j)]);
      A.fvj[jfidx(c, i, j)] = to_f4(fv);
    }
  }
}

// Diffusive spectral radius gamma (mu_f / Pr + mu_t,f / Pr_t) / (rho_f |d|) of one face (viscous.rs:429-454); 0 in the block.
__device__ float face_lambda_dev(const Arena& A, const CaseDev& c, bool dir_i, int fi, int fj) {
  SidesD s;
  float dd;
  if (dir_i) {
    if (!iface_sides_d(A, c, fi, fj, s)) return 0.f;
    dd = A.ifs[ifidx(c, fi, fj)].x;
  } else {
    if (!jface_sides_d(A, c, fi, fj, s)) return 0.f;
    dd = A.jfs[jfidx(c, fi, fj)].x;
  }
  float mu_f, mut_f;
  face_mu_d(A, c, s, mu_f, mut_f);
  float rho_f = 0.5f * (s.l.w[0] + s.r.w[0]);
  return 1.4f * (mu_f / PR + mut_f / PR_T) / (rho_f * dd);
}

}  // namespace bk
