// Host side of a case arena: FP64 grid metrics (grid.rs:65-119), device buffers, launch tables, the launch sequence of
// one iteration (solver.rs:658-676 with implicit.rs:601-663 or solver.rs:694-720), chunked residual read-back, and the
// state / turbulence transfers. One arena serves one case (the GpuSolver C ABI) or many (the batched sweep).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <vector>

#include "arena.cuh"
#include "tma.cuh"
#include "stream_copy.cuh"

namespace bk {

struct HostCase {
  int ni = 0, nj = 0;
  std::vector<double> x, r;                       // nodes
  std::vector<double> if_nx, if_nr, if_len, if_rm;  // (ni+1)*nj
  std::vector<double> jf_nx, jf_nr, jf_len, jf_rm;  // ni*(nj+1)
  std::vector<double> area, vol, xc, rc;
  std::vector<double> dwall;  // wall distance of the cells (turbulence.rs:91-125), computed once; empty until then
  // configuration (doubles as given by the caller)
  double cfl = 0.5;
  int limiter = 1;
  double fs[4] = {1, 0, 0, 1.0 / 1.4};
  int bc[4] = {3, 3, 2, 3};
  long long first_order_iters = 0;
  int low_mach = 0;
  int scheme = SCHEME_EXPLICIT;
  double cfl0 = 1, cfl_max = 30, growth = 1.02, eps_fix = 0.1;
  int dt_mode = 0, lines = 1, implicit_bc = 1, sub_iters = 2, roe = 1;
  double cfl_star = 0.0;  // implicit residual smoothing of the SSP-RK3 stages (Scheme::Smoothed, or the multigrid smoother)
  bool has_block = false;
  long long i_end = 0, j_end = 0, j_sting = 0;
  bool has_nozzle = false;
  long long nz_j_end = 0;
  double nz_state[4] = {0, 0, 0, 0}, nz_turb[2] = {0, 0};
  bool viscous = false;
  int turbulence = 0;
  long long wall_i_start = 0;
  double re_c = 1e6, sutherland = 0.368, roughness = 0;
  int level = 0, fine_case = -1, coarse_case = -1;  // FAS multigrid hierarchy inside the arena
  long long n_active() const {
    long long n = (long long)ni * nj;
    if (has_block) n -= i_end * j_end + ((long long)ni - i_end) * j_sting;
    return n;
  }
  bool solid(int i, int j) const { return has_block && (i < i_end ? j < j_end : j < j_sting); }
  int col_start(int i) const { return has_block ? (int)(i < i_end ? j_end : j_sting) : 0; }
  int row_start(int j) const { return !has_block ? 0 : j < j_sting ? ni : j < j_end ? (int)i_end : 0; }
  // viscous.rs:97-109 (host side: wall distance)
  bool noslip_jface(int i, int j) const {
    if (!viscous) return false;
    if (!has_block) return j == 0 && bc[2] == 2 && i >= wall_i_start;
    return (j == j_end && i >= wall_i_start && i < i_end) || (j == j_sting && j_sting > 0 && i >= i_end);
  }
  bool noslip_iface(int i, int j) const {
    return viscous && has_block && i == i_end && j >= j_sting && j < j_end && !(has_nozzle && j < nz_j_end);
  }
};

// Stencil (|d|, e_x, e_r) of every face between the positions of its two sides (a cell centroid, or for a ghost its
// mirror image in the face centre), viscous.rs:150-250, in FP64. Faces inside the block get |d| = 1 (never read).
inline void face_stencils(const HostCase& h, std::vector<float4>& fis, std::vector<float4>& fjs) {
  const int ni = h.ni, nj = h.nj;
  auto node = [&](int i, int j) { return std::make_pair(h.x[(size_t)j * (ni + 1) + i], h.r[(size_t)j * (ni + 1) + i]); };
  auto st = [&](int cl, bool gl, int cr, bool gr, double xf, double rf) {
    double xl = h.xc[cl], rl = h.rc[cl], xr = h.xc[cr], rr = h.rc[cr];
    if (gl) xl = 2.0 * xf - xl, rl = 2.0 * rf - rl;
    if (gr) xr = 2.0 * xf - xr, rr = 2.0 * rf - rr;
    double dx = xr - xl, dr = rr - rl, dd = std::hypot(dx, dr);
    return make_float4((float)dd, (float)(dx / dd), (float)(dr / dd), 0.f);
  };
  fis.assign((size_t)(ni + 1) * nj, make_float4(1.f, 1.f, 0.f, 0.f));
  fjs.assign((size_t)ni * (nj + 1), make_float4(1.f, 0.f, 1.f, 0.f));
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i <= ni; ++i) {
      auto a = node(i, j), b = node(i, j + 1);
      double xf = 0.5 * (a.first + b.first), rf = 0.5 * (a.second + b.second);
      float4& o = fis[(size_t)j * (ni + 1) + i];
      if (h.has_block && j < h.j_end) {
        if (j < h.j_sting || i < h.i_end) continue;
        if (i == h.i_end) {
          int c = j * ni + i;
          o = st(c, true, c, false, xf, rf);
          continue;
        }
      }
      if (i == 0)
        o = st(j * ni, true, j * ni, false, xf, rf);
      else if (i == ni)
        o = st(j * ni + ni - 1, false, j * ni + ni - 1, true, xf, rf);
      else
        o = st(j * ni + i - 1, false, j * ni + i, false, xf, rf);
    }
  for (int j = 0; j <= nj; ++j)
    for (int i = 0; i < ni; ++i) {
      auto a = node(i, j), b = node(i + 1, j);
      double xf = 0.5 * (a.first + b.first), rf = 0.5 * (a.second + b.second);
      float4& o = fjs[(size_t)j * ni + i];
      int j0 = h.col_start(i);
      if (h.has_block) {
        if (j < j0) continue;
        if (j == j0 && j0 > 0) {
          int c = j * ni + i;
          o = st(c, true, c, false, xf, rf);
          continue;
        }
      }
      if (j == 0)
        o = st(i, true, i, false, xf, rf);
      else if (j == nj)
        o = st((nj - 1) * ni + i, false, (nj - 1) * ni + i, true, xf, rf);
      else
        o = st((j - 1) * ni + i, false, j * ni + i, false, xf, rf);
    }
}

// Run f(k, err) for k in [0, n) over the host threads; false (with err of a failing k) if any call fails.
template <typename F>
inline bool parallel_cases(size_t n, F f, std::string& err) {
  const size_t nt = std::min<size_t>(n, std::max(1u, std::min(32u, std::thread::hardware_concurrency())));
  std::vector<std::string> errs(n);
  std::vector<char> ok(n, 1);
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (size_t k = next++; k < n; k = next++) ok[k] = f(k, errs[k]) ? 1 : 0;
  };
  std::vector<std::thread> th;
  for (size_t t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (auto& x : th) x.join();
  for (size_t k = 0; k < n; ++k)
    if (!ok[k]) {
      err = errs[k];
      return false;
    }
  return true;
}

// No-slip wall face segments of a case (turbulence.rs:91-125): endpoints and bounding box.
struct WallSegs {
  std::vector<double> s;  // x0, r0, x1, r1, xmin, xmax, rmin, rmax per segment
  explicit WallSegs(const HostCase& h) {
    const int ni = h.ni, nj = h.nj;
    auto node = [&](int i, int j) { return std::make_pair(h.x[(size_t)j * (ni + 1) + i], h.r[(size_t)j * (ni + 1) + i]); };
    auto add = [&](std::pair<double, double> a, std::pair<double, double> b) {
      s.insert(s.end(), {a.first, a.second, b.first, b.second, std::fmin(a.first, b.first), std::fmax(a.first, b.first),
                         std::fmin(a.second, b.second), std::fmax(a.second, b.second)});
    };
    for (int j = 0; j <= nj; ++j)
      for (int i = 0; i < ni; ++i)
        if (h.noslip_jface(i, j)) add(node(i, j), node(i + 1, j));
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i <= ni; ++i)
        if (h.noslip_iface(i, j)) add(node(i, j), node(i, j + 1));
    group();
  }
  static constexpr size_t GROUP = 8;  // consecutive segments (neighbours along the wall) under one bounding box
  std::vector<double> gb;              // xmin, xmax, rmin, rmax per group
  void group() {
    for (size_t q0 = 0; q0 < n(); q0 += GROUP) {
      double b[4] = {INFINITY, -INFINITY, INFINITY, -INFINITY};
      for (size_t q = q0; q < std::min(n(), q0 + GROUP); ++q) {
        const double* g = &s[8 * q];
        b[0] = std::fmin(b[0], g[4]), b[1] = std::fmax(b[1], g[5]), b[2] = std::fmin(b[2], g[6]), b[3] = std::fmax(b[3], g[7]);
      }
      gb.insert(gb.end(), b, b + 4);
    }
  }
  size_t n() const { return s.size() / 8; }
  static double box(const double* b, double px, double pr) {
    double dx = std::fmax(std::fmax(b[0] - px, px - b[1]), 0.0), dr = std::fmax(std::fmax(b[2] - pr, pr - b[3]), 0.0);
    return std::sqrt(dx * dx + dr * dr);
  }
  // distance of (px, pr) to segment q: the clamped projection, FP64
  double dist(size_t q, double px, double pr) const {
    const double* g = &s[8 * q];
    double ex = g[2] - g[0], er = g[3] - g[1];
    double t = ((px - g[0]) * ex + (pr - g[1]) * er) / (ex * ex + er * er);
    t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    return std::hypot(px - (g[0] + t * ex), pr - (g[1] + t * er));
  }
  // lower bounds of that distance: the distance to the segment's bounding box, and to its group's
  double bound(size_t q, double px, double pr) const { return box(&s[8 * q + 4], px, pr); }
  double group_bound(size_t g, double px, double pr) const { return box(&gb[4 * g], px, pr); }
};

// Distance of the centroids of rows [j0, j1) to the nearest wall segment, the minimum over every segment as the
// reference takes it. The minimum is the same: a segment is skipped only when its bounding box lies farther than the
// current minimum by a margin (1e-9 relative plus 1e-9 absolute, in nose diameters) far above the rounding of either
// distance (the bounds are tested per group of neighbouring segments, then per segment), and the segment nearest to the
// previous cell of the row is evaluated first.
inline void wall_distance_rows(const HostCase& h, const WallSegs& w, std::vector<double>& d, int j0, int j1) {
  const int ni = h.ni;
  const size_t ns = w.n();
  for (int j = j0; j < j1; ++j) {
    size_t hint = 0;
    for (int i = 0; i < ni; ++i) {
      if (h.solid(i, j)) continue;
      size_t c = (size_t)j * ni + i;
      double px = h.xc[c], pr = h.rc[c], best = d[c];
      if (ns == 0) continue;
      best = std::fmin(best, w.dist(hint, px, pr));
      size_t arg = hint;
      for (size_t g0 = 0; g0 < ns; g0 += WallSegs::GROUP) {
        if (w.group_bound(g0 / WallSegs::GROUP, px, pr) > best * (1.0 + 1e-9) + 1e-9) continue;
        for (size_t q = g0; q < std::min(ns, g0 + WallSegs::GROUP); ++q) {
          if (q == hint || w.bound(q, px, pr) > best * (1.0 + 1e-9) + 1e-9) continue;
          double dq = w.dist(q, px, pr);
          if (dq < best) arg = q;
          best = std::fmin(best, dq);
        }
      }
      d[c] = best;
      hint = arg;
    }
  }
}

// The wall distance of every cell of one case (infinity where no wall exists), rows split over the host threads.
inline std::vector<double> wall_distance(const HostCase& h) {
  const WallSegs w(h);
  std::vector<double> d((size_t)h.ni * h.nj, std::numeric_limits<double>::infinity());
  const int nj = h.nj;
  int nt = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] { wall_distance_rows(h, w, d, (int)((long long)nj * t / nt), (int)((long long)nj * (t + 1) / nt)); });
  for (auto& x : th) x.join();
  return d;
}

// grid.rs:65-119 in FP64; false (and a message) on a non-positive cell area
inline bool compute_metrics(HostCase& h, std::string& err) {
  const int ni = h.ni, nj = h.nj;
  auto nn = [&](int i, int j) { return (size_t)j * (ni + 1) + i; };
  const std::vector<double>&x = h.x, &r = h.r;
  h.if_nx.assign((size_t)(ni + 1) * nj, 0);
  h.if_nr = h.if_len = h.if_rm = h.if_nx;
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i <= ni; ++i) {
      size_t a = nn(i, j), b = nn(i, j + 1), f = (size_t)j * (ni + 1) + i;
      double dx = x[b] - x[a], dr = r[b] - r[a], len = std::hypot(dx, dr);
      h.if_nx[f] = dr / len;
      h.if_nr[f] = -dx / len;
      h.if_len[f] = len;
      h.if_rm[f] = 0.5 * (r[a] + r[b]);
    }
  h.jf_nx.assign((size_t)ni * (nj + 1), 0);
  h.jf_nr = h.jf_len = h.jf_rm = h.jf_nx;
  for (int j = 0; j <= nj; ++j)
    for (int i = 0; i < ni; ++i) {
      size_t a = nn(i, j), b = nn(i + 1, j), f = (size_t)j * ni + i;
      double dx = x[b] - x[a], dr = r[b] - r[a], len = std::hypot(dx, dr);
      h.jf_nx[f] = -dr / len;
      h.jf_nr[f] = dx / len;
      h.jf_len[f] = len;
      h.jf_rm[f] = 0.5 * (r[a] + r[b]);
    }
  size_t n = (size_t)ni * nj;
  h.area.assign(n, 0);
  h.vol = h.xc = h.rc = h.area;
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < ni; ++i) {
      size_t p[4] = {nn(i, j), nn(i + 1, j), nn(i + 1, j + 1), nn(i, j + 1)};
      double a = 0, v = 0, sx = 0, sr = 0;
      const int tri[2][3] = {{0, 1, 2}, {0, 2, 3}};
      for (auto& t : tri) {
        size_t k0 = p[t[0]], k1 = p[t[1]], k2 = p[t[2]];
        double at = 0.5 * ((x[k1] - x[k0]) * (r[k2] - r[k0]) - (x[k2] - x[k0]) * (r[k1] - r[k0]));
        double cx = (x[k0] + x[k1] + x[k2]) / 3.0, cr = (r[k0] + r[k1] + r[k2]) / 3.0;
        a += at;
        v += at * cr;
        sx += at * cx;
        sr += at * cr;
      }
      if (!(a > 0.0)) {
        err = "non-positive cell area at (" + std::to_string(i) + "," + std::to_string(j) + ")";
        return false;
      }
      size_t c = (size_t)j * ni + i;
      h.area[c] = a;
      h.vol[c] = v;
      h.xc[c] = sx / a;
      h.rc[c] = sr / a;
    }
  return true;
}

#define BK_CUDA(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);                          \
      return 3;                                                                          \
    }                                                                                    \
  } while (0)

template <class T>
inline int dalloc(T** p, size_t n, std::string& err) {
  *p = nullptr;
  if (n == 0) return 0;
  BK_CUDA(cudaMalloc((void**)p, n * sizeof(T)));
  return 0;
}

struct ArenaHost {
  std::vector<HostCase> cases;
  int device = 0;
  cudaStream_t stream = nullptr;
  // The captured iteration runs the SST chain up to its final step on a second branch of the graph, beside the
  // mean-flow line solves (both read this iteration's primitives, fluxes and time step; neither writes what the other
  // reads until k_turb_update, which joins them), and the line ends' ghost Jacobians beside the residual.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_ends = nullptr;
  bool capturing = false;
  std::string err;
  bool ready = false;
  int slots = 256;  // residual history slots per chunk
  // host copies of the tables
  std::vector<CaseDev> desc;
  long long ncell = 0, npad = 0, nif = 0, njf = 0;
  int ntiles = 0, nil = 0, njl = 0, npblk = 0;
  int max_line = 0;  // longest i or j line of any case
  int *d_tlist = nullptr, *d_pblist = nullptr, *d_illist = nullptr, *d_jllist = nullptr;  // compaction lists
  // launch sizes: the active entries when compacted, every entry otherwise
  int LT() const { return A.tile_list ? A.n_tl : ntiles; }
  int LP() const { return A.pblk_list ? A.n_pb : npblk; }
  int LI(int dir_i) const { return dir_i ? (A.iline_list ? A.n_il : nil) : (A.jline_list ? A.n_jl : njl); }
  // floats of the line-solve records: 29 float4 per cell and direction (rounded up to 64-byte blocks per direction),
  // 44 float4 per lane of every line
  size_t scratch_floats() const { return 4 * ((size_t)2 * rec_dir_stride(ncell) + (size_t)(nil + njl) * 32 * PREC); }
  bool any_viscous = false, any_sst = false, any_rough = false;
  // coupled SST lines (k_turb_couple) instead of the reference's loose coupling; A.tcpl is allocated on the first switch
  bool sst_coupled = false;
  // device buffers
  Arena A{};
  CaseDev* d_cases = nullptr;
  int *d_iter = nullptr, *d_ramp = nullptr, *d_active = nullptr;
  int *d_tile_case = nullptr, *d_iline = nullptr, *d_jline = nullptr, *d_pblk = nullptr;
  std::vector<double> h_rsum;
  cudaGraphExec_t graph = nullptr;
  int graph_len = 0;
  bool graph_dirty = false;  // `graph` is stale but has the topology of the next capture
  std::vector<int> h_active;
  // Case groups of the captured chunk: with groups_req > 1 the active cases are split into up to groups_req groups of
  // about equal cells, and each group's iterations are captured on a stream of its own, so the chunk's graph holds one
  // independent chain of iterations per group and the groups' kernels run side by side. Every kernel of an iteration
  // touches only its own cases' data (per-case counters, residual slots, records), so the states are the ones of the
  // ungrouped graph bit for bit; what changes is how many warps are in flight when few cases are left.
  struct Group {
    cudaStream_t st = nullptr, side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_ends = nullptr, ev_done = nullptr;
    int *d_act = nullptr, *d_tl = nullptr, *d_pb = nullptr, *d_il = nullptr, *d_jl = nullptr;
    int n_tl = 0, n_pb = 0, n_il = 0, n_jl = 0;
  };
  static constexpr int MAX_GROUPS = 4;
  std::vector<Group> grp;
  int groups_req = 1, ngroups = 1;
  cudaEvent_t ev_split = nullptr;

  ~ArenaHost() { release(); }

  void release() {
    if (graph) cudaGraphExecDestroy(graph), graph = nullptr;
    if (ev0) cudaEventDestroy(ev0), ev0 = nullptr;
    if (ev1) cudaEventDestroy(ev1), ev1 = nullptr;
    if (pe0) cudaEventDestroy(pe0), pe0 = nullptr;
    if (pe1) cudaEventDestroy(pe1), pe1 = nullptr;
    void* ptrs[] = {d_cases, d_iter, d_ramp, d_active, d_tile_case, d_iline, d_jline, d_pblk, A.U, A.W, A.R, A.X, A.DU, A.RR, A.U0, A.Ulo, A.Wlo, A.U0lo, A.MG0lo,
                    A.FORCE, A.dt, (void*)A.iface, (void*)A.jface, (void*)A.cellg, (void*)A.ifc, (void*)A.jfc, A.scratch, A.rsum,
                    A.grad4, A.gradT, A.mu, A.mu_t, A.rough, A.fvi, A.fvj, A.turb, A.turb_new, A.dwall, A.mflux_i, A.mflux_j, A.tsum, A.tcoef,
                    A.trhs, A.grad_kw, A.blend, (void*)A.ifs, (void*)A.jfs, A.MG0, d_enabled, d_tlist, d_pblist, d_illist, d_jllist,
                    A.lend, A.irs_eps, A.irs_c, (void*)A.wmaps, A.tcpl};
    d_enabled = nullptr;
    d_tlist = d_pblist = d_illist = d_jllist = nullptr;
    for (void* p : ptrs)
      if (p) cudaFree(p);
    d_cases = nullptr;
    d_iter = d_ramp = d_active = d_tile_case = d_iline = d_jline = d_pblk = nullptr;
    A = Arena{};
    if (stream) cudaStreamDestroy(stream), stream = nullptr;
    if (side) cudaStreamDestroy(side), side = nullptr;
    if (ev_fork) cudaEventDestroy(ev_fork), ev_fork = nullptr;
    if (ev_join) cudaEventDestroy(ev_join), ev_join = nullptr;
    if (ev_ends) cudaEventDestroy(ev_ends), ev_ends = nullptr;
    for (Group& q : grp) {
      for (cudaStream_t t : {q.st, q.side})
        if (t) cudaStreamDestroy(t);
      for (cudaEvent_t e : {q.ev_fork, q.ev_join, q.ev_ends, q.ev_done})
        if (e) cudaEventDestroy(e);
      for (int* p : {q.d_act, q.d_tl, q.d_pb, q.d_il, q.d_jl})
        if (p) cudaFree(p);
    }
    grp.clear();
    ngroups = 1;
    if (ev_split) cudaEventDestroy(ev_split), ev_split = nullptr;
    ready = false;
  }

  CaseDev make_desc(const HostCase& h) const {
    CaseDev c{};
    c.ni = h.ni;
    c.nj = h.nj;
    c.has_block = h.has_block;
    c.i_end = (int)h.i_end;
    c.j_end = (int)h.j_end;
    c.j_sting = (int)h.j_sting;
    c.has_nozzle = h.has_nozzle;
    c.nz_j_end = (int)h.nz_j_end;
    for (int k = 0; k < 4; ++k) c.nz_state[k] = (float)h.nz_state[k];
    c.nz_turb[0] = (float)h.nz_turb[0];
    c.nz_turb[1] = (float)h.nz_turb[1];
    for (int k = 0; k < 4; ++k) {
      c.bc[k] = h.bc[k];
      c.fs[k] = h.fs[k];
    }
    c.cfl = (float)h.cfl;
    c.limiter = h.limiter;
    c.first_order_iters = (int)std::min<long long>(h.first_order_iters, 1 << 30);
    c.low_mach = h.low_mach;
    c.scheme = h.scheme;
    c.cfl0 = (float)h.cfl0;
    c.cfl_max = (float)h.cfl_max;
    c.growth = (float)h.growth;
    c.eps_fix = (float)h.eps_fix;
    c.dt_mode = h.dt_mode;
    c.lines = h.lines;
    c.implicit_bc = h.implicit_bc;
    c.sub_iters = h.sub_iters;
    c.roe = h.roe;
    c.cfl_star = (h.scheme == SCHEME_SMOOTHED || h.scheme == SCHEME_MULTIGRID) && h.cfl_star > 0.0 ? (float)h.cfl_star : 0.f;
    c.viscous = h.viscous;
    c.sst = h.viscous && h.turbulence == 1;
    c.wall_i_start = (int)h.wall_i_start;
    c.re_c = h.re_c;
    c.sutherland = h.sutherland;
    c.roughness = h.roughness;
    c.n_active = (int)h.n_active();
    c.level = h.level;
    c.fine_case = h.fine_case;
    c.coarse_case = h.coarse_case;
    return c;
  }

  // The residual kernel's tensor maps: per case W then Wlo of its padded primitives as a 2D array of floats,
  // 4 (ni + 4) wide (each cell's float4 = 4 floats) and nj + 4 high, boxes of 4 (TI + 4) x (TJ + 4) floats.
  int build_wmaps() {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = bktma::encoder(err);
    if (!enc) return 3;
    const int nc = (int)cases.size();
    std::vector<CUtensorMap> maps(2 * (size_t)nc);
    for (int k = 0; k < nc; ++k)
      for (int w = 0; w < 2; ++w) {
        const CaseDev& c = desc[k];
        float4* base = (w ? A.Wlo : A.W) + c.pad_off;
        cuuint64_t dims[2] = {(cuuint64_t)4 * (c.ni + 4), (cuuint64_t)(c.nj + 4)};
        cuuint64_t strides[1] = {(cuuint64_t)(c.ni + 4) * sizeof(float4)};
        cuuint32_t box[2] = {(cuuint32_t)4 * (TI + 4), (cuuint32_t)(TJ + 4)};
        cuuint32_t es[2] = {1, 1};
        CUresult r = enc(&maps[2 * k + w], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
          err = "cuTensorMapEncodeTiled of the primitives of case " + std::to_string(k) + " failed (" + std::to_string((int)r) + ")";
          return 3;
        }
      }
    CUtensorMap* d = nullptr;
    BK_CUDA(cudaMalloc(&d, maps.size() * sizeof(CUtensorMap)));
    A.wmaps = d;
    BK_CUDA(copy_sync(stream, d, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    return 0;
  }

  // Lay out the arena, allocate and upload geometry (once; the case dimensions are fixed afterwards).
  int setup() {
    release();
    BK_CUDA(cudaSetDevice(device));
    BK_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    BK_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    BK_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    BK_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    BK_CUDA(cudaEventCreateWithFlags(&ev_ends, cudaEventDisableTiming));
    const int nc = (int)cases.size();
    desc.resize(nc);
    ncell = npad = nif = njf = 0;
    ntiles = nil = njl = npblk = 0;
    max_line = 0;
    std::vector<int> tile_case, iline, jline, pblk;
    for (int k = 0; k < nc; ++k) {
      HostCase& h = cases[k];
      CaseDev c = make_desc(h);
      c.cell_off = ncell;
      c.pad_off = npad;
      c.if_off = nif;
      c.jf_off = njf;
      c.ntx = (h.ni + TI - 1) / TI;
      c.nty = (h.nj + TJ - 1) / TJ;
      c.tile_off = ntiles;
      c.iline_off = nil;
      c.jline_off = njl;
      c.pblk_off = npblk;
      int nt = c.ntx * c.nty, nb = (int)(((long long)(h.ni + 4) * (h.nj + 4) + 255) / 256);
      tile_case.insert(tile_case.end(), nt, k);
      iline.insert(iline.end(), h.nj, k);
      jline.insert(jline.end(), h.ni, k);
      pblk.insert(pblk.end(), nb, k);
      ntiles += nt;
      nil += h.nj;
      njl += h.ni;
      max_line = std::max(max_line, std::max(h.ni, h.nj));
      npblk += nb;
      ncell += (long long)h.ni * h.nj;
      npad += (long long)(h.ni + 4) * (h.nj + 4);
      nif += (long long)(h.ni + 1) * h.nj;
      njf += (long long)h.ni * (h.nj + 1);
      desc[k] = c;
    }
    int rc = 0;
#define ALLOC(p, n) \
  if ((rc = dalloc(&(p), (size_t)(n), err))) return rc
    ALLOC(d_cases, nc);
    ALLOC(d_iter, nc);
    ALLOC(d_ramp, nc);
    ALLOC(d_active, nc);
    ALLOC(d_tile_case, ntiles);
    ALLOC(d_iline, nil);
    ALLOC(d_jline, njl);
    ALLOC(d_pblk, npblk);
    ALLOC(d_tlist, ntiles);
    ALLOC(d_pblist, npblk);
    ALLOC(d_illist, nil);
    ALLOC(d_jllist, njl);
    ALLOC(A.U, ncell);
    ALLOC(A.W, npad);
    ALLOC(A.R, ncell);
    ALLOC(A.X, ncell);
    ALLOC(A.DU, ncell);
    ALLOC(A.RR, ncell);
    ALLOC(A.U0, ncell);
    ALLOC(A.Ulo, ncell);
    ALLOC(A.Wlo, npad);
    ALLOC(A.U0lo, ncell);
    BK_CUDA(cudaMemsetAsync(A.Ulo, 0, ncell * sizeof(float4), stream));
    if ((rc = build_wmaps())) return rc;
    ALLOC(A.dt, ncell);
    ALLOC(A.irs_eps, ncell);
    ALLOC(A.irs_c, ncell);
    float4 *fi, *fj, *cg;
    float2 *ic, *jc;
    ALLOC(fi, nif);
    ALLOC(fj, njf);
    ALLOC(cg, ncell);
    ALLOC(ic, nif);
    ALLOC(jc, njf);
    A.iface = fi;
    A.jface = fj;
    A.cellg = cg;
    A.ifc = ic;
    A.jfc = jc;
    ALLOC(A.scratch, scratch_floats());
    ALLOC(A.lend, (size_t)8 * (nil + njl));
    ALLOC(A.rsum, (size_t)slots * nc);
    ALLOC(A.tsum, (size_t)slots * nc);
    ALLOC(d_enabled, nc);
    A.enabled = d_enabled;
    if (mg_levels > 1) {
      ALLOC(A.MG0, ncell);
      ALLOC(A.MG0lo, ncell);
      ALLOC(A.FORCE, ncell);
      BK_CUDA(cudaMemsetAsync(A.FORCE, 0, ncell * sizeof(float4), stream));
    }
    float4 *fis, *fjs;
    ALLOC(fis, nif);
    ALLOC(fjs, njf);
    A.ifs = fis;
    A.jfs = fjs;
    BK_CUDA(copy_sync(stream, d_tile_case, tile_case.data(), tile_case.size() * sizeof(int), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, d_iline, iline.data(), iline.size() * sizeof(int), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, d_jline, jline.data(), jline.size() * sizeof(int), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, d_pblk, pblk.data(), pblk.size() * sizeof(int), cudaMemcpyHostToDevice));
    // geometry
    std::vector<float4> hfi(nif), hfj(njf), hcg(ncell);
    std::vector<float2> hic(nif), hjc(njf);
    for (int k = 0; k < nc; ++k) {
      const HostCase& h = cases[k];
      const CaseDev& c = desc[k];
      for (int j = 0; j < h.nj; ++j)
        for (int i = 0; i <= h.ni; ++i) {
          size_t f = (size_t)j * (h.ni + 1) + i;
          hfi[c.if_off + f] = make_float4((float)h.if_nx[f], (float)h.if_nr[f], (float)h.if_len[f], (float)(h.if_len[f] * h.if_rm[f]));
          size_t a = (size_t)j * (h.ni + 1) + i, b = (size_t)(j + 1) * (h.ni + 1) + i;
          hic[c.if_off + f] = make_float2((float)(0.5 * (h.x[a] + h.x[b])), (float)(0.5 * (h.r[a] + h.r[b])));
        }
      for (int j = 0; j <= h.nj; ++j)
        for (int i = 0; i < h.ni; ++i) {
          size_t f = (size_t)j * h.ni + i;
          hfj[c.jf_off + f] = make_float4((float)h.jf_nx[f], (float)h.jf_nr[f], (float)h.jf_len[f], (float)(h.jf_len[f] * h.jf_rm[f]));
          size_t a = (size_t)j * (h.ni + 1) + i, b = a + 1;
          hjc[c.jf_off + f] = make_float2((float)(0.5 * (h.x[a] + h.x[b])), (float)(0.5 * (h.r[a] + h.r[b])));
        }
      for (int j = 0; j < h.nj; ++j)
        for (int i = 0; i < h.ni; ++i) {
          size_t cc = (size_t)j * h.ni + i;
          hcg[c.cell_off + cc] = make_float4((float)h.vol[cc], (float)h.area[cc], (float)h.xc[cc], (float)h.rc[cc]);
        }
    }
    BK_CUDA(copy_sync(stream, fi, hfi.data(), nif * sizeof(float4), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, fj, hfj.data(), njf * sizeof(float4), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, cg, hcg.data(), ncell * sizeof(float4), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, ic, hic.data(), nif * sizeof(float2), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, jc, hjc.data(), njf * sizeof(float2), cudaMemcpyHostToDevice));
    A.ncases = nc;
    A.cases = d_cases;
    A.iter = d_iter;
    A.ramp_k = d_ramp;
    A.active = d_active;
    A.tile_case = d_tile_case;
    A.ntiles = ntiles;
    A.iline_case = d_iline;
    A.nilines = nil;
    A.ncell = ncell;
    A.jline_case = d_jline;
    A.njlines = njl;
    A.pblk_case = d_pblk;
    A.npblk = npblk;
    std::vector<int> zero(nc, 0);
    h_active.assign(nc, 1);
    BK_CUDA(copy_sync(stream, d_iter, zero.data(), nc * sizeof(int), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, d_ramp, zero.data(), nc * sizeof(int), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, d_active, h_active.data(), nc * sizeof(int), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, d_enabled, h_active.data(), nc * sizeof(int), cudaMemcpyHostToDevice));
    ready = true;
    if ((rc = upload_desc())) return rc;
    for (int k = 0; k < nc; ++k)
      if ((rc = reset_case(k))) return rc;
    int nb = 0, sms = 0;
    BK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_lines_subst_st, 32, 0));
    BK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    staged_lines = 2 * nb * sms;
    return compact_lists();
  }

  // Re-derive the descriptors from the host configuration (config, scheme, block, viscous changes).
  int upload_desc() {
    any_viscous = any_sst = any_rough = false;
    for (size_t k = 0; k < cases.size(); ++k) {
      CaseDev c = make_desc(cases[k]);
      CaseDev& d = desc[k];
      c.cell_off = d.cell_off;
      c.pad_off = d.pad_off;
      c.if_off = d.if_off;
      c.jf_off = d.jf_off;
      c.tile_off = d.tile_off;
      c.ntx = d.ntx;
      c.nty = d.nty;
      c.iline_off = d.iline_off;
      c.jline_off = d.jline_off;
      c.pblk_off = d.pblk_off;
      d = c;
      any_viscous |= c.viscous != 0;
      any_sst |= c.sst != 0;
      any_rough |= c.sst != 0 && c.roughness > 0.0;
    }
    int rc = 0;
    if (any_viscous && !A.mu) {
      ALLOC(A.grad4, ncell);
      ALLOC(A.gradT, ncell);
      ALLOC(A.mu, ncell);
      ALLOC(A.mu_t, ncell);
      ALLOC(A.fvi, nif);
      ALLOC(A.fvj, njf);
      BK_CUDA(cudaMemsetAsync(A.mu_t, 0, ncell * sizeof(float), stream));
      BK_CUDA(cudaMemsetAsync(A.fvi, 0, nif * sizeof(float4), stream));
      BK_CUDA(cudaMemsetAsync(A.fvj, 0, njf * sizeof(float4), stream));
    }
    if (any_rough && !A.rough) {
      ALLOC(A.rough, ncell);
      BK_CUDA(cudaMemsetAsync(A.rough, 0, ncell * sizeof(float4), stream));
    }
    if (any_sst && !A.turb) {
      ALLOC(A.turb, ncell);
      ALLOC(A.dwall, ncell);
      ALLOC(A.mflux_i, nif);
      ALLOC(A.mflux_j, njf);
      ALLOC(A.tcoef, 3 * ncell);
      ALLOC(A.trhs, ncell);
      ALLOC(A.grad_kw, ncell);
      ALLOC(A.blend, ncell);
      BK_CUDA(cudaMemsetAsync(A.mflux_i, 0, nif * sizeof(float), stream));
      BK_CUDA(cudaMemsetAsync(A.mflux_j, 0, njf * sizeof(float), stream));
    }
    if (any_sst && sst_coupled && !A.tcpl) ALLOC(A.tcpl, 3 * ncell);
    if ((rc = upload_stencils())) return rc;
    BK_CUDA(copy_sync(stream, d_cases, desc.data(), desc.size() * sizeof(CaseDev), cudaMemcpyHostToDevice));
    if (graph) cudaGraphExecDestroy(graph), graph = nullptr;
    return 0;
  }
#undef ALLOC

  int upload_stencils() {
    std::vector<float4> fis, fjs;
    for (size_t k = 0; k < cases.size(); ++k) {
      face_stencils(cases[k], fis, fjs);
      BK_CUDA(copy_sync(stream, (void*)(A.ifs + desc[k].if_off), fis.data(), fis.size() * sizeof(float4), cudaMemcpyHostToDevice));
      BK_CUDA(copy_sync(stream, (void*)(A.jfs + desc[k].jf_off), fjs.data(), fjs.size() * sizeof(float4), cudaMemcpyHostToDevice));
    }
    return 0;
  }

  // The wall distances of every SST case not computed yet, the cases spread over the host threads (each case's rows
  // serially) and kept for the turbulence (re)initialisations of later runs.
  void wall_distances() {
    std::vector<size_t> todo;
    for (size_t k = 0; k < cases.size(); ++k)
      if (cases[k].viscous && cases[k].turbulence == 1 && cases[k].dwall.empty()) todo.push_back(k);
    std::string unused;
    parallel_cases(todo.size(), [&](size_t q, std::string&) {
      HostCase& h = cases[todo[q]];
      std::vector<double> d((size_t)h.ni * h.nj, std::numeric_limits<double>::infinity());
      wall_distance_rows(h, WallSegs(h), d, 0, h.nj);
      h.dwall = std::move(d);
      return true;
    }, unused);
  }
  // turbulence.rs:128-138: free-stream (k, omega) everywhere, the wall distance, mu_t = rho k / omega on fluid cells
  std::vector<double> last_turb_residual;
  int turb_init(int k) {
    const HostCase& h = cases[k];
    const CaseDev& c = desc[k];
    size_t n = (size_t)h.ni * h.nj;
    double winf = 1e-6 * h.re_c, kinf = 9e-9;
    if (cases[k].dwall.empty()) cases[k].dwall = wall_distance(h);
    const std::vector<double>& d = cases[k].dwall;
    std::vector<float> df(n), mt(n);
    std::vector<float2> t(n, make_float2((float)kinf, (float)winf));
    std::vector<double> u(4 * n);
    int rc = get_state(k, u.data());
    if (rc) return rc;
    for (size_t cc = 0; cc < n; ++cc) {
      df[cc] = std::isfinite(d[cc]) ? (float)d[cc] : 3.0e38f;
      mt[cc] = h.solid((int)(cc % h.ni), (int)(cc / h.ni)) ? 0.f : (float)(u[4 * cc] * kinf / winf);
    }
    BK_CUDA(copy_sync(stream, A.dwall + c.cell_off, df.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, A.turb + c.cell_off, t.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, A.mu_t + c.cell_off, mt.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    return 0;
  }
  int turb_upload(int k, const double* turb, const double* mu_t) {
    const CaseDev& c = desc[k];
    size_t n = (size_t)c.ni * c.nj;
    if (turb) {
      std::vector<float2> t(n);
      for (size_t i = 0; i < n; ++i) t[i] = make_float2((float)turb[2 * i], (float)turb[2 * i + 1]);
      BK_CUDA(copy_sync(stream, A.turb + c.cell_off, t.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    }
    if (mu_t) {
      std::vector<float> m(n);
      for (size_t i = 0; i < n; ++i) m[i] = (float)mu_t[i];
      BK_CUDA(copy_sync(stream, A.mu_t + c.cell_off, m.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    }
    return 0;
  }

  int reset_case(int k) {
    const HostCase& h = cases[k];
    double w[4] = {h.fs[0], h.fs[1], h.fs[2], h.fs[3]};
    double q[4] = {w[0], w[0] * w[1], w[0] * w[2], w[3] / 0.4 + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2])};
    std::vector<double> u((size_t)h.ni * h.nj * 4);
    for (size_t c = 0; c < (size_t)h.ni * h.nj; ++c)
      for (int m = 0; m < 4; ++m) u[4 * c + m] = q[m];
    return set_state(k, u.data());
  }

  int set_state(int k, const double* u) {
    const CaseDev& c = desc[k];
    size_t n = (size_t)c.ni * c.nj;
    std::vector<float4> h(n), l(n);
    for (size_t i = 0; i < n; ++i) {
      const double* q = u + 4 * i;
      h[i] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)q[3]);
      l[i] = make_float4((float)(q[0] - (double)h[i].x), (float)(q[1] - (double)h[i].y), (float)(q[2] - (double)h[i].z),
                         (float)(q[3] - (double)h[i].w));
    }
    BK_CUDA(copy_sync(stream, A.U + c.cell_off, h.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, A.Ulo + c.cell_off, l.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
    int z = 0;
    BK_CUDA(copy_sync(stream, d_iter + k, &z, sizeof(int), cudaMemcpyHostToDevice));
    BK_CUDA(copy_sync(stream, d_ramp + k, &z, sizeof(int), cudaMemcpyHostToDevice));
    return 0;
  }

  int get_state(int k, double* u) {
    const CaseDev& c = desc[k];
    size_t n = (size_t)c.ni * c.nj;
    std::vector<float4> h(n), l(n);
    BK_CUDA(cudaStreamSynchronize(stream));
    BK_CUDA(copy_sync(stream, h.data(), A.U + c.cell_off, n * sizeof(float4), cudaMemcpyDeviceToHost));
    BK_CUDA(copy_sync(stream, l.data(), A.Ulo + c.cell_off, n * sizeof(float4), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) {
      u[4 * i] = (double)h[i].x + (double)l[i].x;
      u[4 * i + 1] = (double)h[i].y + (double)l[i].y;
      u[4 * i + 2] = (double)h[i].z + (double)l[i].z;
      u[4 * i + 3] = (double)h[i].w + (double)l[i].w;
    }
    return 0;
  }

  int set_counter(int* d, int k, int v) {
    BK_CUDA(copy_sync(stream, d + k, &v, sizeof(int), cudaMemcpyHostToDevice));
    return 0;
  }
  int get_counter(const int* d, int k, int& v) {
    BK_CUDA(cudaStreamSynchronize(stream));
    BK_CUDA(copy_sync(stream, &v, d + k, sizeof(int), cudaMemcpyDeviceToHost));
    return 0;
  }
  int set_active(const int* act) {
    for (size_t k = 0; k < cases.size(); ++k) h_active[k] = act[k] ? 1 : 0;
    BK_CUDA(cudaMemcpyAsync(d_enabled, h_active.data(), cases.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    if (mg_levels > 1)
      k_level_mask<<<((int)cases.size() + 127) / 128, 128, 0, stream>>>(A, 0);
    else
      BK_CUDA(cudaMemcpyAsync(d_active, h_active.data(), cases.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    BK_CUDA(cudaStreamSynchronize(stream));
    return compact_lists();
  }
  // Launch only over the active cases' tiles, padded blocks and lines once some cases are masked out (not with a
  // multigrid hierarchy, whose level masks change inside an iteration). The line lists also order the lines longest
  // first, so the blocks with the longest per-lane chains start in the first wave of a line launch instead of trailing
  // it (a line's arithmetic does not depend on its position in the launch). A changed list invalidates the captured graph.
  int compact_lists() {
    const int nc = (int)cases.size();
    int n_act = 0;
    for (int k = 0; k < nc; ++k) n_act += h_active[k];
    const bool lists = mg_levels <= 1 && n_act > 0, want = lists && n_act < nc;
    std::vector<int> tl, pb, il, jl;
    if (lists) {
      std::vector<std::pair<int, int>> li, lj;  // (-fluid cells of the line, global line)
      for (int k = 0; k < nc; ++k) {
        if (!h_active[k]) continue;
        const CaseDev& c = desc[k];
        const HostCase& h = cases[k];
        int nt = c.ntx * c.nty, nb = (int)(((long long)(h.ni + 4) * (h.nj + 4) + 255) / 256);
        for (int q = 0; want && q < nt; ++q) tl.push_back(c.tile_off + q);
        for (int q = 0; want && q < nb; ++q) pb.push_back(c.pblk_off + q);
        for (int q = 0; q < h.nj; ++q) li.push_back({-(h.ni - h.row_start(q)), c.iline_off + q});
        for (int q = 0; q < h.ni; ++q) lj.push_back({-(h.nj - h.col_start(q)), c.jline_off + q});
      }
      std::stable_sort(li.begin(), li.end());
      std::stable_sort(lj.begin(), lj.end());
      for (auto& p : li) il.push_back(p.second);
      for (auto& p : lj) jl.push_back(p.second);
      if (want) {
        BK_CUDA(copy_sync(stream, d_tlist, tl.data(), tl.size() * sizeof(int), cudaMemcpyHostToDevice));
        BK_CUDA(copy_sync(stream, d_pblist, pb.data(), pb.size() * sizeof(int), cudaMemcpyHostToDevice));
      }
      BK_CUDA(copy_sync(stream, d_illist, il.data(), il.size() * sizeof(int), cudaMemcpyHostToDevice));
      BK_CUDA(copy_sync(stream, d_jllist, jl.data(), jl.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    A.tile_list = want ? d_tlist : nullptr;
    A.pblk_list = want ? d_pblist : nullptr;
    A.iline_list = lists ? d_illist : nullptr;
    A.jline_list = lists ? d_jllist : nullptr;
    A.n_tl = (int)tl.size(), A.n_pb = (int)pb.size(), A.n_il = (int)il.size(), A.n_jl = (int)jl.size();
    graph_dirty = true;  // same kernels, new grids and lists: the next capture updates the instantiated graph
    ngroups = 1;
    if (lists && groups_req > 1 && n_act >= 2) return group_lists(std::min(groups_req, n_act));
    return 0;
  }
  // The lists and masks of G case groups (Group): the active cases, largest first, each to the group with the fewest
  // cells so far; per group the tile, padded-block and line lists (lines longest first) and the per-case mask.
  int group_lists(int G) {
    const int nc = (int)cases.size();
    if (!ev_split) BK_CUDA(cudaEventCreateWithFlags(&ev_split, cudaEventDisableTiming));
    while ((int)grp.size() < G) {
      grp.emplace_back();
      Group& q = grp.back();
      BK_CUDA(cudaStreamCreateWithFlags(&q.st, cudaStreamNonBlocking));
      BK_CUDA(cudaStreamCreateWithFlags(&q.side, cudaStreamNonBlocking));
      for (cudaEvent_t* e : {&q.ev_fork, &q.ev_join, &q.ev_ends, &q.ev_done}) BK_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
      int rc;
      if ((rc = dalloc(&q.d_act, nc, err)) || (rc = dalloc(&q.d_tl, ntiles, err)) || (rc = dalloc(&q.d_pb, npblk, err)) ||
          (rc = dalloc(&q.d_il, nil, err)) || (rc = dalloc(&q.d_jl, njl, err)))
        return rc;
    }
    std::vector<int> order;
    for (int k = 0; k < nc; ++k)
      if (h_active[k]) order.push_back(k);
    auto cells = [&](int k) { return (long long)cases[k].ni * cases[k].nj; };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells(a) > cells(b); });
    std::vector<std::vector<int>> members(G);
    std::vector<long long> load(G, 0);
    for (int k : order) {
      const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      members[g].push_back(k);
      load[g] += cells(k);
    }
    for (int g = 0; g < G; ++g) {
      Group& q = grp[g];
      std::vector<int> act(nc, 0), tl, pb, il, jl;
      std::vector<std::pair<int, int>> li, lj;
      for (int k : members[g]) {
        act[k] = 1;
        const CaseDev& c = desc[k];
        const HostCase& h = cases[k];
        const int nt = c.ntx * c.nty, nb = (int)(((long long)(h.ni + 4) * (h.nj + 4) + 255) / 256);
        for (int t = 0; t < nt; ++t) tl.push_back(c.tile_off + t);
        for (int t = 0; t < nb; ++t) pb.push_back(c.pblk_off + t);
        for (int t = 0; t < h.nj; ++t) li.push_back({-(h.ni - h.row_start(t)), c.iline_off + t});
        for (int t = 0; t < h.ni; ++t) lj.push_back({-(h.nj - h.col_start(t)), c.jline_off + t});
      }
      std::sort(tl.begin(), tl.end());
      std::sort(pb.begin(), pb.end());
      std::stable_sort(li.begin(), li.end());
      std::stable_sort(lj.begin(), lj.end());
      for (auto& p : li) il.push_back(p.second);
      for (auto& p : lj) jl.push_back(p.second);
      BK_CUDA(copy_sync(stream, q.d_act, act.data(), nc * sizeof(int), cudaMemcpyHostToDevice));
      BK_CUDA(copy_sync(stream, q.d_tl, tl.data(), tl.size() * sizeof(int), cudaMemcpyHostToDevice));
      BK_CUDA(copy_sync(stream, q.d_pb, pb.data(), pb.size() * sizeof(int), cudaMemcpyHostToDevice));
      BK_CUDA(copy_sync(stream, q.d_il, il.data(), il.size() * sizeof(int), cudaMemcpyHostToDevice));
      BK_CUDA(copy_sync(stream, q.d_jl, jl.data(), jl.size() * sizeof(int), cudaMemcpyHostToDevice));
      q.n_tl = (int)tl.size(), q.n_pb = (int)pb.size(), q.n_il = (int)il.size(), q.n_jl = (int)jl.size();
    }
    ngroups = G;
    return 0;
  }
  // Point the launch state (A with the group's lists and mask, the streams and fork/join events) at group g, or back
  // (the same call again restores it).
  void swap_group(Group& q, Arena& saved) {
    std::swap(stream, q.st);
    std::swap(side, q.side);
    std::swap(ev_fork, q.ev_fork);
    std::swap(ev_join, q.ev_join);
    std::swap(ev_ends, q.ev_ends);
    std::swap(A, saved);
  }

  // ---------------------------------------------------------------- FAS multigrid (multigrid.rs:72-112)
  int mg_levels = 1, mg_pre = 1, mg_post = 1, mg_gamma = 1, mg_coarsest = 4;
  int* d_enabled = nullptr;
  void set_level(int l) { k_level_mask<<<((int)cases.size() + 127) / 128, 128, 0, stream>>>(A, l); }
  // one SSP-RK3 step of the active level (solver.rs:694-710); `slot` records the first stage's density residual
  void rk3(int slot, int last) {
    launch_mean_flow_prep();
    L(G_RESIDUAL, [&] { k_residual<TI * TJ, 3><<<ntiles, TI * TJ, 0, stream>>>(A, 1, slot); });
    launch_irs();
    L(G_STAGE, [&] { k_stage<<<ntiles, TI * TJ, 0, stream>>>(A, 1.f, 0.f, 1, 0); });
    launch_mean_flow_prep();
    L(G_RESIDUAL, [&] { k_residual<TI * TJ, 3><<<ntiles, TI * TJ, 0, stream>>>(A, 0, -1); });
    launch_irs();
    L(G_STAGE, [&] { k_stage<<<ntiles, TI * TJ, 0, stream>>>(A, 0.25f, 0.75f, 0, 0); });
    launch_mean_flow_prep();
    L(G_RESIDUAL, [&] { k_residual<TI * TJ, 3><<<ntiles, TI * TJ, 0, stream>>>(A, 0, -1); });
    launch_irs();
    L(G_STAGE, [&] { k_stage<<<ntiles, TI * TJ, 0, stream>>>(A, 2.f / 3.f, 1.f / 3.f, 0, last); });
  }
  // The smoother of a level: SSP-RK3 (the reference's, multigrid.rs:87-112), or with mg_implicit one line-implicit
  // iteration (the implicit scheme's residual, assembly, line solves, defect corrections and damped update) of the active
  // level, its time step from that level's own CFL ramp; the implicit iteration advances the level's iteration and ramp
  // counters itself (so the fine level's counters advance once per smoothing step).
  bool mg_implicit = false;
  double mg_relax = 1.0;  // fraction of the prolongated correction applied (1: the reference's FAS)
  void smooth(int slot, int last) {
    if (mg_implicit)
      implicit_step(slot);
    else
      rk3(slot, last);
  }
  // the multigrid restriction folded into the coarse level's primitives and residual evaluation (default), or the
  // reference's order of separate transfer kernels (the same states bit for bit)
  bool mg_fused = true;
  void mg_level(int l, int slot) {  // multigrid.rs:87-112
    const bool coarsest = l == mg_levels - 1;
    const int n_pre = coarsest ? mg_coarsest : mg_pre;
    set_level(l);
    for (int k = 0; k < n_pre; ++k) smooth(l == 0 && k == 0 ? slot : -1, 0);
    if (coarsest) return;
    launch_mean_flow_prep();
    L(G_RESIDUAL, [&] { k_residual<TI * TJ, 3><<<ntiles, TI * TJ, 0, stream>>>(A, 0, (l == 0 && n_pre == 0) ? slot : -1); });
    if (mg_fused) {  // the restriction folded into the coarse level's primitives and residual (the same states)
      set_level(l + 1);
      L(G_TRANSFER, [&] { k_prims_restrict<<<LP(), 256, 0, stream>>>(A); });
      if (any_viscous) {
        L(G_VISC, [&] { k_visc_cell<<<LT(), TI * TJ, 0, stream>>>(A); });
        L(G_VISC, [&] { k_visc_face<<<LT(), TI * TJ, 0, stream>>>(A); });
      }
      L(G_RESIDUAL, [&] { k_residual<TI * TJ, 3, true><<<ntiles, TI * TJ, 0, stream>>>(A, 0, -1); });
    } else {
      L(G_TRANSFER, [&] { k_restrict_state<<<ntiles, TI * TJ, 0, stream>>>(A, l + 1); });
      set_level(l + 1);
      launch_mean_flow_prep();
      L(G_RESIDUAL, [&] { k_residual<TI * TJ, 3><<<ntiles, TI * TJ, 0, stream>>>(A, 0, -1); });
      L(G_TRANSFER, [&] { k_restrict_forcing<<<ntiles, TI * TJ, 0, stream>>>(A, l + 1); });
    }
    for (int g = 0; g < std::max(mg_gamma, 1); ++g) mg_level(l + 1, -1);
    L(G_TRANSFER, [&] { k_prolong<<<ntiles, TI * TJ, 0, stream>>>(A, l, mg_relax); });
    set_level(l);
    for (int k = 0; k < mg_post; ++k) smooth(-1, l == 0 && k == mg_post - 1 ? 1 : 0);
    if (l == 0 && mg_post == 0 && !mg_implicit) {  // the cycle still counts one iteration
      launch_mean_flow_prep();
      L(G_STAGE, [&] { k_stage<<<ntiles, TI * TJ, 0, stream>>>(A, 1.f, 0.f, 0, 1); });
    }
  }

  // ---------------------------------------------------------------- one iteration (stream-ordered launches)
  // Kernel groups of the per-kernel profile (CUDA events around every launch when `profiling` is set).
  enum { G_PRIMS = 0, G_VISC, G_RESIDUAL, G_LINES_I, G_LINES_J, G_DEFECT, G_TURB, G_STAGE, G_SUBST_I, G_SUBST_J, G_ASSEMBLE, G_TURB_LINES, G_TRANSFER,
         G_N };
  bool profiling = false;
  double prof_ms[G_N] = {0};
  long long prof_launches[G_N] = {0};
  cudaEvent_t pe0 = nullptr, pe1 = nullptr;
  template <class F>
  void L(int g, F&& launch) {
    if (!profiling) {
      launch();
      return;
    }
    if (!pe0) cudaEventCreate(&pe0), cudaEventCreate(&pe1);
    cudaEventRecord(pe0, stream);
    launch();
    cudaEventRecord(pe1, stream);
    cudaEventSynchronize(pe1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, pe0, pe1);
    prof_ms[g] += ms;
    prof_launches[g] += 1;
  }
  // residual kernel of the implicit iteration: 0 = 256 threads, 1 = 288 threads (3 blocks per SM both; at most two
  // face fluxes per thread with 288). The two round differently, so the variant is fixed (288) and only a pinned
  // tuning changes it.
  int res_variant = 1;
  void launch_residual(int dt_kind, int slot) {
    if (res_variant == 1)
      k_residual<288, 3><<<LT(), 288, 0, stream>>>(A, dt_kind, slot);
    else
      k_residual<TI * TJ, 3><<<LT(), TI * TJ, 0, stream>>>(A, dt_kind, slot);
  }
  // Launch shapes of the line kernels, picked by autotune() per direction ([0] = j lines, [1] = i lines): lines per
  // block (1, 2, 4, or 8 except for the first pass, whose shared memory holds 4 lines at most) and, for the first pass,
  // whether the walks prefetch the next cell's record.
  int lw_lines[2] = {LINE_WARPS, LINE_WARPS}, pf_lines[2] = {0, 0}, lw_subst[2] = {LINE_WARPS, LINE_WARPS}, lw_turb = TL_WARPS;
  // how the substitution walks fetch their records: 0 one cell at a time, 1 the next cell's ahead (registers), 2 staged
  // through shared memory SUB_SD cells ahead (one line per block, lw_subst not used)
  int pf_subst[2] = {0, 0};
  // A direction with at most this many lines in the launch runs its line solves staged (pf_lines / pf_subst 2) whatever
  // pf_lines / pf_subst say: with few lines the walks wait on memory latency, not bandwidth, and the staged walks wait
  // once per SUB_SD cells. Set at setup to two waves of the staged substitution kernel (its blocks per SM x SMs x 2); 0
  // never.
  int staged_lines = 0;
  template <int PF>
  void launch_lines_pf(int dir_i, int w, const float4* in, int from_res, float4* out) {
    const int nl = LI(dir_i);
    const int nb = (nl + w - 1) / w;
    switch (w) {
      case 1: k_lines<1, PF><<<nb, 32, 0, stream>>>(A, dir_i, in, from_res, out); break;
      case 2: k_lines<2, PF><<<nb, 64, 0, stream>>>(A, dir_i, in, from_res, out); break;
      default: k_lines<4, PF><<<nb, 128, 0, stream>>>(A, dir_i, in, from_res, out); break;
    }
  }
  void launch_lines(int dir_i, const float4* in, int from_res, float4* out) {
    const int d = dir_i ? 1 : 0, w = lw_lines[d] > 4 ? 4 : lw_lines[d];
    if (pf_lines[d] == 2 || LI(dir_i) <= staged_lines)
      k_lines<1, 2><<<LI(dir_i), 32, 0, stream>>>(A, dir_i, in, from_res, out);
    else if (pf_lines[d])
      launch_lines_pf<1>(dir_i, w, in, from_res, out);
    else
      launch_lines_pf<0>(dir_i, w, in, from_res, out);
  }
  template <bool PF>
  void launch_subst_pf(int dir_i, int w, const float4* in, float4* out, int pass) {
    const int nl = LI(dir_i);
    const int nb = (nl + w - 1) / w;
    switch (w) {
      case 1: k_lines_subst<1, PF><<<nb, 32, 0, stream>>>(A, dir_i, in, out, pass); break;
      case 2: k_lines_subst<2, PF><<<nb, 64, 0, stream>>>(A, dir_i, in, out, pass); break;
      case 8: k_lines_subst<8, PF><<<nb, 256, 0, stream>>>(A, dir_i, in, out, pass); break;
      default: k_lines_subst<4, PF><<<nb, 128, 0, stream>>>(A, dir_i, in, out, pass); break;
    }
  }
  void launch_subst(int dir_i, const float4* in, float4* out, int pass) {
    const int d = dir_i ? 1 : 0;
    if (pf_subst[d] == 2 || LI(dir_i) <= staged_lines)
      k_lines_subst_st<<<LI(dir_i), 32, 0, stream>>>(A, dir_i, in, out, pass);
    else if (pf_subst[d])
      launch_subst_pf<true>(dir_i, lw_subst[d], in, out, pass);
    else
      launch_subst_pf<false>(dir_i, lw_subst[d], in, out, pass);
  }
  void launch_turb_lines(int dir_i, cudaStream_t st) {
    const int nl = LI(dir_i), w = lw_turb;
    const int nb = (nl + w - 1) / w;
    switch (w) {
      case 1: k_turb_lines_w<1><<<nb, 32, 0, st>>>(A, dir_i); break;
      case 2: k_turb_lines_w<2><<<nb, 64, 0, st>>>(A, dir_i); break;
      case 8: k_turb_lines_w<8><<<nb, 256, 0, st>>>(A, dir_i); break;
      default: k_turb_lines_w<4><<<nb, 128, 0, st>>>(A, dir_i); break;
    }
  }
  // turbulence.rs:542-581, from this iteration's primitives, mass fluxes, gradients and time step: the SST update up to
  // its final step
  void launch_turb_chain(cudaStream_t st, int slot) {
    launch_turb_terms(st, slot);
    launch_turb_solves(st);
  }
  void launch_turb_terms(cudaStream_t st, int slot) {
    L(G_TURB, [&] { k_turb_grad<<<LT(), TI * TJ, 0, st>>>(A); });
    if (sst_coupled && A.tcpl)
      L(G_TURB, [&] { k_turb_cell<true><<<LT(), TI * TJ, 0, st>>>(A, slot); });
    else
      L(G_TURB, [&] { k_turb_cell<false><<<LT(), TI * TJ, 0, st>>>(A, slot); });
  }
  // the two scalar line systems (with the coupled lines, after k_turb_couple on the mean flow's stream)
  void launch_turb_solves(cudaStream_t st) {
    if (max_line <= 32 * TL_MAXM) {
      L(G_TURB_LINES, [&] { launch_turb_lines(1, st); });
      L(G_TURB_LINES, [&] { launch_turb_lines(0, st); });
    } else {  // thread-per-line kernel: its Thomas coefficients borrow the line records, so it runs after the mean flow
      L(G_TURB, [&] { k_turb_lines<<<(2 * LI(1) + 127) / 128, 128, 0, st>>>(A, 1); });
      L(G_TURB, [&] { k_turb_lines<<<(2 * LI(0) + 127) / 128, 128, 0, st>>>(A, 0); });
    }
  }
  // Autotuner: per direction, lines per block and prefetching of the first pass and of the substitution passes, lines per block of the SST line kernel, and the residual kernel's variant; only variants that compile to the
  // same arithmetic are candidates (ptxas contracts multiply-adds differently under different register budgets, so a
  // launch-bounds variant can round differently; every candidate here was checked bit for bit): each the fastest candidate over
  // one timed iteration of this arena's own cases (after one warm-up iteration, every candidate kernel loaded first). The
  // state, turbulence and counters are kept in a device copy and restored afterwards; the choice does not change any
  // result (every warp solves one line alone, with the same arithmetic).
  int autotune() {
    if (scheme_of_arena() != SCHEME_IMPLICIT) return 0;
    const size_t nc = cases.size();
    // the state the timed iterations advance, kept in a device copy and put back afterwards
    struct Keep {
      void* dst;
      const void* src;
      size_t bytes;
    };
    std::vector<Keep> keep = {{nullptr, A.U, ncell * sizeof(float4)}, {nullptr, A.Ulo, ncell * sizeof(float4)},
                              {nullptr, d_iter, nc * sizeof(int)}, {nullptr, d_ramp, nc * sizeof(int)}};
    if (any_sst) keep.push_back({nullptr, A.turb, ncell * sizeof(float2)}), keep.push_back({nullptr, A.mu_t, ncell * sizeof(float)});
    size_t kb = 0;
    for (auto& q : keep) kb += (q.bytes + 255) & ~(size_t)255;
    char* kbuf = nullptr;
    BK_CUDA(cudaMalloc(&kbuf, kb));
    kb = 0;
    for (auto& q : keep) {
      q.dst = kbuf + kb, kb += (q.bytes + 255) & ~(size_t)255;
      BK_CUDA(cudaMemcpyAsync(q.dst, q.src, q.bytes, cudaMemcpyDeviceToDevice, stream));
    }
    // load every candidate kernel now (lazy module loading would otherwise charge a variant's first launch)
    {
      cudaFuncAttributes fa;
      const void* fns[] = {(const void*)&k_lines<1, 0>, (const void*)&k_lines<2, 0>, (const void*)&k_lines<4, 0>,
                           (const void*)&k_lines<1, 1>, (const void*)&k_lines<2, 1>, (const void*)&k_lines<4, 1>,
                           (const void*)&k_lines_subst<1, false>, (const void*)&k_lines_subst<2, false>,
                           (const void*)&k_lines_subst<4, false>, (const void*)&k_lines_subst<8, false>,
                           (const void*)&k_lines_subst<1, true>, (const void*)&k_lines_subst<2, true>,
                           (const void*)&k_lines_subst<4, true>, (const void*)&k_lines_subst<8, true>,
                           (const void*)&k_turb_lines_w<1>, (const void*)&k_turb_lines_w<2>, (const void*)&k_turb_lines_w<4>,
                           (const void*)&k_turb_lines_w<8>, (const void*)&k_residual<288, 3>, (const void*)&k_residual<TI * TJ, 3>};
      for (const void* f : fns) BK_CUDA(cudaFuncGetAttributes(&fa, f));
    }
    // The smallest segment per lane (Arena::mmin_i / mmin_j) keeps its setting (2 unless pinned): a longer one changes the
    // rounding of the line solves, and on a limit-cycle case of the sweep it moved the window-mean CD by 2e-4.
    const int cand[4] = {1, 2, 4, 8};
    // timed groups: first pass j / i, substitution j / i, SST lines
    const int grp[5] = {G_LINES_J, G_LINES_I, G_SUBST_J, G_SUBST_I, G_TURB_LINES};
    double best[5] = {1e30, 1e30, 1e30, 1e30, 1e30};
    // pick_pf: prefetching of the first pass (q = 0, 1) and of the substitution passes (q = 2, 3)
    int pick_w[5] = {LINE_WARPS, LINE_WARPS, LINE_WARPS, LINE_WARPS, TL_WARPS}, pick_pf[4] = {0, 0, 0, 0};
    int rc = 0;
    // the staged substitution walks are not candidates: they are chosen by the number of lines (staged_lines), and
    // the variants here are timed as requested
    const int staged_keep = staged_lines;
    staged_lines = 0;
    if ((rc = profile(1))) return rc;  // warm-up
    for (int pf = 0; pf < 2; ++pf)
      for (int w : cand) {
        if (pf && w > 4) continue;
        lw_lines[0] = lw_lines[1] = lw_subst[0] = lw_subst[1] = lw_turb = w;
        pf_lines[0] = pf_lines[1] = pf_subst[0] = pf_subst[1] = pf;  // the staged variants (2) are chosen by staged_lines
        if ((rc = profile(1))) return rc;
        for (int q = 0; q < 5; ++q) {
          if (q == 4 && pf) continue;  // the SST line kernel has no prefetching variant
          if (q < 2 && w > 4) continue;
          const double t = prof_ms[grp[q]];
          if (t < best[q]) {
            best[q] = t, pick_w[q] = w;
            if (q < 4) pick_pf[q] = pf;
          }
        }
      }
    lw_lines[0] = pick_w[0], lw_lines[1] = pick_w[1], pf_lines[0] = pick_pf[0], pf_lines[1] = pick_pf[1];
    lw_subst[0] = pick_w[2], lw_subst[1] = pick_w[3], lw_turb = pick_w[4];
    pf_subst[0] = pick_pf[2], pf_subst[1] = pick_pf[3];
    // the residual kernel's variant is not a candidate: with its tile staged by TMA, the 288-thread build rounds
    // differently from the 256-thread one (ptxas fuses multiply-adds by register budget), so it stays at 1 unless pinned
    staged_lines = staged_keep;
    for (auto& q : keep) BK_CUDA(cudaMemcpyAsync(const_cast<void*>(q.src), q.dst, q.bytes, cudaMemcpyDeviceToDevice, stream));
    BK_CUDA(cudaStreamSynchronize(stream));
    BK_CUDA(cudaFree(kbuf));
    if (graph) cudaGraphExecDestroy(graph), graph = nullptr;
    return 0;
  }
  void launch_mean_flow_prep() {
    L(G_PRIMS, [&] { k_prims<<<LP(), 256, 0, stream>>>(A); });
    if (any_viscous) {
      L(G_VISC, [&] { k_visc_cell<<<LT(), TI * TJ, 0, stream>>>(A); });
      L(G_VISC, [&] { k_visc_face<<<LT(), TI * TJ, 0, stream>>>(A); });
    }
  }
  // Switches between the coupled SST lines and the reference's loosely coupled ones (for the next chunk on).
  int set_sst_coupled(bool on) {
    sst_coupled = on;
    if (on && any_sst && !A.tcpl) {
      int rc = dalloc(&A.tcpl, 3 * (size_t)ncell, err);
      if (rc) return rc;
    }
    if (graph) cudaGraphExecDestroy(graph), graph = nullptr;
    return 0;
  }
  int scheme_of_arena() const { return desc.empty() ? 0 : desc[0].scheme; }
  int sub_iters_of_arena() const {
    int s = 1;
    for (auto& d : desc) s = std::max(s, d.sub_iters);
    return s;
  }
  // One line-implicit iteration of every active case (implicit.rs:601-663): primitives, residual and time step, the
  // blocks of both directions, the factorising line solves and sub_iters - 1 defect corrections, the damped update, and
  // the SST update for SST cases.
  void implicit_step(int slot) {
    // the line ends' ghost Jacobians need only the primitives: in a captured iteration they run on the graph's second
    // branch beside the viscous terms, the residual and the assembly
    const int nle = 2 * (LI(1) + LI(0));
    const bool fork_ends = capturing && !profiling;
    L(G_PRIMS, [&] { k_prims<<<LP(), 256, 0, stream>>>(A); });
    if (fork_ends) {
      cudaEventRecord(ev_fork, stream);
      cudaStreamWaitEvent(side, ev_fork, 0);
      k_line_ends_T<<<(nle + 127) / 128, 128, 0, side>>>(A);
      cudaEventRecord(ev_ends, side);
    } else {
      L(G_ASSEMBLE, [&] { k_line_ends_T<<<(nle + 127) / 128, 128, 0, stream>>>(A); });
    }
    if (any_viscous) {
      L(G_VISC, [&] { k_visc_cell<<<LT(), TI * TJ, 0, stream>>>(A); });
      L(G_VISC, [&] { k_visc_face<<<LT(), TI * TJ, 0, stream>>>(A); });
    }
    L(G_RESIDUAL, [&] { launch_residual(2, slot); });
    const int s = sub_iters_of_arena();
    // the SST chain on the graph's second branch (only the warp-per-line SST kernel: the thread-per-line one borrows
    // the line records)
    const bool fork = any_sst && capturing && !profiling && max_line <= 32 * TL_MAXM;
    const bool coupled = any_sst && sst_coupled && A.tcpl;
    if (fork) {
      cudaEventRecord(ev_fork, stream);
      cudaStreamWaitEvent(side, ev_fork, 0);
      if (coupled)  // the line solves need the mean flow's increment: only the terms run beside the mean flow
        launch_turb_terms(side, slot);
      else
        launch_turb_chain(side, slot);
      cudaEventRecord(ev_join, side);
    }
    L(G_ASSEMBLE, [&] {
      k_assemble<<<dim3(LT(), 2), TI * TJ, 0, stream>>>(A);
    });
    if (fork_ends) cudaStreamWaitEvent(stream, ev_ends, 0);
    L(G_ASSEMBLE, [&] { k_line_ends_fold<<<(nle + 127) / 128, 128, 0, stream>>>(A); });
    L(G_LINES_I, [&] { launch_lines(1, A.R, 1, A.X); });
    L(G_LINES_J, [&] { launch_lines(0, A.X, 0, nullptr); });
    for (int p = 1; p < s; ++p) {
      L(G_DEFECT, [&] { k_defect<<<LT(), TI * TJ, 0, stream>>>(A, p); });
      L(G_SUBST_I, [&] { launch_subst(1, A.RR, A.X, p); });
      L(G_SUBST_J, [&] { launch_subst(0, A.X, nullptr, p); });
    }
    if (any_sst) {
      if (fork)
        cudaStreamWaitEvent(stream, ev_join, 0);
      else if (coupled)
        launch_turb_terms(stream, slot);
      else
        launch_turb_chain(stream, slot);
      if (coupled) {
        L(G_TURB, [&] { k_turb_couple<<<LT(), TI * TJ, 0, stream>>>(A); });
        launch_turb_solves(stream);
      }
      L(G_TURB, [&] { k_turb_update<<<LT(), TI * TJ, 0, stream>>>(A); });
    }
  }
  void launch_iteration(int slot) {
    if (scheme_of_arena() == SCHEME_MULTIGRID) {
      mg_level(0, slot);
      set_level(0);
    } else if (scheme_of_arena() == SCHEME_IMPLICIT) {
      implicit_step(slot);
    } else {  // SSP-RK3, with implicit residual smoothing of every stage's residual for Scheme::Smoothed
      launch_mean_flow_prep();
      L(G_RESIDUAL, [&] { k_residual<TI * TJ, 3><<<LT(), TI * TJ, 0, stream>>>(A, 1, slot); });
      launch_irs();
      L(G_STAGE, [&] { k_stage<<<LT(), TI * TJ, 0, stream>>>(A, 1.f, 0.f, 1, 0); });
      launch_mean_flow_prep();
      L(G_RESIDUAL, [&] { k_residual<TI * TJ, 3><<<LT(), TI * TJ, 0, stream>>>(A, 0, -1); });
      launch_irs();
      L(G_STAGE, [&] { k_stage<<<LT(), TI * TJ, 0, stream>>>(A, 0.25f, 0.75f, 0, 0); });
      launch_mean_flow_prep();
      L(G_RESIDUAL, [&] { k_residual<TI * TJ, 3><<<LT(), TI * TJ, 0, stream>>>(A, 0, -1); });
      launch_irs();
      L(G_STAGE, [&] { k_stage<<<LT(), TI * TJ, 0, stream>>>(A, 2.f / 3.f, 1.f / 3.f, 0, 1); });
    }
  }
  // implicit residual smoothing of A.R (solver.rs:722-803): the i factor into X, the j factor back into R; the kernels
  // return at once for cases without smoothing
  bool any_irs() const {
    for (const HostCase& h : cases)
      if ((h.scheme == SCHEME_SMOOTHED || h.scheme == SCHEME_MULTIGRID) && h.cfl_star > 0.0) return true;
    return false;
  }
  void launch_irs() {
    if (!any_irs()) return;
    L(G_STAGE, [&] { k_irs<<<(nil + 127) / 128, 128, 0, stream>>>(A, 1, A.R, A.X); });
    L(G_STAGE, [&] { k_irs<<<(njl + 127) / 128, 128, 0, stream>>>(A, 0, A.X, A.R); });
  }
  // n iterations with CUDA events around every launch (no graph); per-group totals in prof_ms / prof_launches
  int profile(long long n) {
    for (int g = 0; g < G_N; ++g) prof_ms[g] = 0, prof_launches[g] = 0;
    bool g0 = use_graphs;
    use_graphs = false;
    profiling = true;
    int rc = run(n, nullptr);
    profiling = false;
    use_graphs = g0;
    return rc;
  }

  bool use_graphs = true;
  // the stop rules of a solve evaluated on the device after every chunk (runner.cuh: k_run_control); false: on the host
  bool device_run_control = true;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms_per_iter = 0.0;
  // one chunk of `chunk` iterations: captured once into a CUDA graph, replayed afterwards
  int launch_chunk(int chunk) {
    const int nc = (int)cases.size();
    if (!use_graphs) {
      BK_CUDA(cudaMemsetAsync(A.rsum, 0, (size_t)chunk * nc * sizeof(double), stream));
      if (any_sst) BK_CUDA(cudaMemsetAsync(A.tsum, 0, (size_t)chunk * nc * sizeof(double), stream));
      for (int k = 0; k < chunk; ++k) launch_iteration(k);
      BK_CUDA(cudaGetLastError());
      return 0;
    }
    int rc = capture_chunk(chunk);
    if (rc) return rc;
    BK_CUDA(cudaGraphLaunch(graph, stream));
    return 0;
  }
  // The CUDA graph of a chunk of `chunk` iterations, captured and instantiated unless it is the one already held.
  int capture_chunk(int chunk) {
    const int nc = (int)cases.size();
    if (!graph || graph_len != chunk || graph_dirty) {
      cudaGraph_t g;
      BK_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      cudaMemsetAsync(A.rsum, 0, (size_t)chunk * nc * sizeof(double), stream);
      if (any_sst) cudaMemsetAsync(A.tsum, 0, (size_t)chunk * nc * sizeof(double), stream);
      capturing = true;
      if (ngroups > 1) {  // one independent chain of iterations per case group, forked from and joined into `stream`
        cudaEventRecord(ev_split, stream);
        for (int g = 0; g < ngroups; ++g) {
          Group& q = grp[g];
          cudaStreamWaitEvent(q.st, ev_split, 0);
          Arena ga = A;
          ga.active = q.d_act, ga.tile_list = q.d_tl, ga.pblk_list = q.d_pb, ga.iline_list = q.d_il, ga.jline_list = q.d_jl;
          ga.n_tl = q.n_tl, ga.n_pb = q.n_pb, ga.n_il = q.n_il, ga.n_jl = q.n_jl;
          swap_group(q, ga);
          for (int k = 0; k < chunk; ++k) launch_iteration(k);
          swap_group(q, ga);
          cudaEventRecord(q.ev_done, q.st);
          cudaStreamWaitEvent(stream, q.ev_done, 0);
        }
      } else {
        for (int k = 0; k < chunk; ++k) launch_iteration(k);
      }
      capturing = false;
      cudaError_t le = cudaGetLastError();
      BK_CUDA(cudaStreamEndCapture(stream, &g));
      if (le != cudaSuccess) {
        cudaGraphDestroy(g);
        err = std::string("launch during capture: ") + cudaGetErrorString(le);
        return 3;
      }
      if (graph && graph_len == chunk) {  // a change of the active cases: update the instantiated graph in place
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(graph, g, &info) == cudaSuccess) {
          cudaGraphDestroy(g);
          graph_dirty = false;
          return 0;
        }
        cudaGetLastError();  // the update was refused: instantiate anew
      }
      if (graph) cudaGraphExecDestroy(graph), graph = nullptr;
      graph_dirty = false;
      cudaError_t ie = cudaGraphInstantiate(&graph, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        graph = nullptr;
        err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie);
        return 3;
      }
      graph_len = chunk;
    }
    return 0;
  }
  // Build the graph run(n) launches first, without running it (so that a timed run(n) does no capture).
  int prepare(long long n) {
    if (!use_graphs || n <= 0) return 0;
    return capture_chunk((int)std::min<long long>(n, slots));
  }

  // n iterations; residual (n x ncases, iteration-major) may be null
  int run(long long n, double* residual) {
    const int nc = (int)cases.size();
    long long done = 0;
    if (!ev0) {
      BK_CUDA(cudaEventCreate(&ev0));
      BK_CUDA(cudaEventCreate(&ev1));
    }
    double ms_total = 0.0;
    while (done < n) {
      int chunk = (int)std::min<long long>(n - done, slots);
      int rc_ = prepare(chunk);  // graph construction (host work) before the events that time the chunk on the device
      if (rc_) return rc_;
      BK_CUDA(cudaEventRecord(ev0, stream));
      rc_ = launch_chunk(chunk);
      if (rc_) return rc_;
      BK_CUDA(cudaEventRecord(ev1, stream));
      if (residual) {
        h_rsum.resize((size_t)chunk * nc);
        BK_CUDA(cudaMemcpyAsync(h_rsum.data(), A.rsum, h_rsum.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
      }
      std::vector<double> ht;
      if (any_sst) {
        ht.resize(nc);
        BK_CUDA(cudaMemcpyAsync(ht.data(), A.tsum + (size_t)(chunk - 1) * nc, nc * sizeof(double), cudaMemcpyDeviceToHost, stream));
      }
      BK_CUDA(cudaStreamSynchronize(stream));
      float ms = 0.f;
      BK_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
      ms_total += ms;
      if (any_sst) {
        last_turb_residual.resize(nc);
        for (int c = 0; c < nc; ++c) last_turb_residual[c] = std::sqrt(ht[c] / (double)desc[c].n_active);
      }
      if (residual)
        for (int k = 0; k < chunk; ++k)
          for (int c = 0; c < nc; ++c)
            residual[(done + k) * nc + c] = std::sqrt(h_rsum[(size_t)k * nc + c] / (double)desc[c].n_active);
      done += chunk;
    }
    last_ms_per_iter = n > 0 ? ms_total / (double)n : 0.0;
    return 0;
  }

  // Solver::eval_residual of the current state (no update): dt_kind 1 = explicit dt, 2 = implicit dt
  int eval_residual(int dt_kind, std::vector<double>* dens) {
    const int nc = (int)cases.size();
    BK_CUDA(cudaMemsetAsync(A.rsum, 0, nc * sizeof(double), stream));
    launch_mean_flow_prep();
    k_residual<TI * TJ, 3><<<LT(), TI * TJ, 0, stream>>>(A, dt_kind, 0);
    BK_CUDA(cudaGetLastError());
    std::vector<double> h(nc);
    BK_CUDA(cudaMemcpyAsync(h.data(), A.rsum, nc * sizeof(double), cudaMemcpyDeviceToHost, stream));
    BK_CUDA(cudaStreamSynchronize(stream));
    if (dens) {
      dens->resize(nc);
      for (int c = 0; c < nc; ++c) (*dens)[c] = std::sqrt(h[c] / (double)desc[c].n_active);
    }
    return 0;
  }

  template <class T, class D>
  int download_cells(int k, const T* dptr, std::vector<D>& out, int comps) {
    const CaseDev& c = desc[k];
    size_t n = (size_t)c.ni * c.nj;
    std::vector<T> h(n);
    BK_CUDA(cudaStreamSynchronize(stream));
    BK_CUDA(copy_sync(stream, h.data(), dptr + c.cell_off, n * sizeof(T), cudaMemcpyDeviceToHost));
    out.resize(n * comps);
    const float* f = reinterpret_cast<const float*>(h.data());
    for (size_t i = 0; i < n * comps; ++i) out[i] = f[i];
    return 0;
  }
};

}  // namespace bk
