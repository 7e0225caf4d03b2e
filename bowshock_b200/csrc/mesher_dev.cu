// Device mesher: the body-fitted grids of many cases built on the GPU from their body and grid parameters — the 1D
// node distributions (the bisections of geometric_offsets and two_sided_nodes, grid.rs:199-228, body_grid.rs:134-157),
// the nodes of base_domain_grid (body_grid.rs:360-452) and large_domain_grid (body_grid.rs:160-231), and the FP64 metrics
// of every face and cell (grid.rs:65-119). No counterpart in the reference (its mesher runs on the host, one case at a
// time); the host mesher of this library (mesher.cuh) stays the default because it is bit for bit the reference's.
//
// Three launches for a whole batch: k_mesh_lines (one warp per case: the independent 1D distributions on separate lanes,
// then the ones that depend on them), k_mesh_nodes (one thread per node) and k_mesh_metrics (one thread per face or cell).
// This file is compiled on its own without multiply-add contraction (-fmad=false), so its additions, multiplications,
// divisions and square roots round as the host mesher's do, in the same order; the results differ from the host
// mesher's only where CUDA's tanh, tan, pow, acos, sin and hypot round differently from the host C library (an ulp or
// two, checked by the tests against the host mesher).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bowshock_b200.h"
#include "mesher.cuh"
#include "mesher_dev.h"
#include "stream_copy.cuh"

namespace bkmesh {

// One case of a batch in plain data (copied to the device), with its output offsets.
struct DReq {
  int wake, nose, nseg, gap_one_sided;
  double fineness, half_angle, param, sting_radius;
  double seg_len[BOWSHOCK_MAX_SEGMENTS], seg_slope[BOWSHOCK_MAX_SEGMENTS];
  double x_up, x_down, r_far, dx_tip, dr_wall;
  int n_up, n_nose, n_seg[BOWSHOCK_MAX_SEGMENTS], n_wake, n_sting, n_gap, nj_out, n_ext, nj_sting;
  int ni, nj, i_end, j_end, j_sting;
  long long node_off, met_off, line_off;  // offsets into the node, metric and 1D scratch arrays
};

// ------------------------------------------------------------------------------------------ body (device copies)
// The expressions of bk::mesh::Body (body_grid.rs:62-88, 269-311) in the same order.
__device__ double nose_length(const DReq& q) { return q.nose == bk::mesh::NOSE_CONE ? 0.5 / tan(q.half_angle) : q.fineness; }
__device__ double nose_r(const DReq& q, double x) {
  if (x <= 0.0) return 0.0;
  double ln = nose_length(q), R = 0.5;
  if (x >= ln) return R;
  double eta = x / ln;
  switch (q.nose) {
    case bk::mesh::NOSE_TANGENT_OGIVE: {
      double l = q.fineness, rho = (l * l + R * R) / (2.0 * R), xx = fmax(x, 0.0);
      return sqrt(fmax(rho * rho - (l - xx) * (l - xx), 0.0)) - (rho - R);
    }
    case bk::mesh::NOSE_CONE:
      return x * tan(q.half_angle);
    case bk::mesh::NOSE_POWER:
      return R * pow(eta, q.param);
    case bk::mesh::NOSE_PARABOLIC:
      return R * (2.0 * eta - q.param * eta * eta) / (2.0 - q.param);
    default: {
      double t = 1.0 - 2.0 * eta;
      t = t < -1.0 ? -1.0 : (t > 1.0 ? 1.0 : t);
      double th = acos(t), s = sin(th);
      return R * sqrt(fmax((th - 0.5 * sin(2.0 * th) + q.param * s * s * s) / M_PI, 0.0));
    }
  }
}
__device__ void station(const DReq& q, int k, double& x, double& r) {
  x = nose_length(q), r = 0.5;
  for (int t = 0; t < k; ++t) {
    x += q.seg_len[t];
    r += q.seg_len[t] * q.seg_slope[t];
  }
}
__device__ double aft_length(const DReq& q) {
  double a = 0;
  for (int k = 0; k < q.nseg; ++k) a = a + q.seg_len[k];
  return a;
}
__device__ double body_r(const DReq& q, double x) {
  if (x <= nose_length(q)) return nose_r(q, x);
  double x0 = nose_length(q), r0 = 0.5;
  for (int k = 0; k < q.nseg; ++k) {
    double x1 = x0 + q.seg_len[k];
    if (x < x1) return r0 + (x - x0) * q.seg_slope[k];
    x0 = x1;
    r0 += q.seg_len[k] * q.seg_slope[k];
  }
  double xb, rb;
  station(q, q.nseg, xb, rb);
  return rb;
}

// ------------------------------------------------------------------------------------------ 1D distributions
// grid.rs:199-228: n + 1 offsets from 0 to `length`, first spacing `first`, ratio found by 200 bisection steps
__device__ void geometric_offsets(double first, double length, int n, double* out) {
  double lo = 0.2, hi = 4.0;
  for (int k = 0; k < 200; ++k) {
    double mid = 0.5 * (lo + hi);
    double s = 0, d = first;
    for (int t = 0; t < n; ++t) s += d, d *= mid;
    if (s < length)
      lo = mid;
    else
      hi = mid;
  }
  double q = 0.5 * (lo + hi);
  double s = 0, d = first;
  for (int k = 0; k < n; ++k) out[k] = s, s += d, d *= q;
  out[n] = length;
}
// body_grid.rs:134-157: n + 1 tanh-clustered nodes on [0, len], end spacing dx where the uniform one is larger
__device__ double two_sided_node(double len, int n, double delta, int k) {
  double t = (double)k / (double)n;
  if (delta < 1e-9) return len * t;
  return 0.5 * len * (1.0 + tanh(delta * (t - 0.5)) / tanh(0.5 * delta));
}
__device__ void two_sided_nodes(double len, int n, double dx, double* out) {
  double delta = 0.0;
  if (!(dx >= len / (double)n)) {
    double lo = 0.0, hi = 40.0;
    for (int it = 0; it < 200; ++it) {
      double mid = 0.5 * (lo + hi);
      if (two_sided_node(len, n, mid, 1) > dx)
        lo = mid;
      else
        hi = mid;
    }
    delta = 0.5 * (lo + hi);
  }
  for (int k = 0; k <= n; ++k) out[k] = two_sided_node(len, n, delta, k);
}

// Scratch of one case (line_off): xs [ni + 1], the radial distributions [nj + 2], then the nose, upstream, segment and
// downstream distributions (the last also holds the one-sided base-gap offsets before the wake's). A case's offsets:
struct Lines {
  double *xs, *rad, *nose, *up, *seg, *down;
};
__host__ __device__ inline long long line_words(const DReq& q) {
  long long segs = 0;
  for (int k = 0; k < q.nseg; ++k) segs += q.n_seg[k] + 1;
  int down = q.n_wake > q.n_ext ? q.n_wake : q.n_ext;
  if (q.n_gap > down) down = q.n_gap;
  return (q.ni + 1) + (q.nj + 2) + (q.n_nose + 1) + (q.n_up + 1) + segs + (down + 1);
}
__device__ Lines lines_of(const DReq& q, double* scratch) {
  Lines L;
  L.xs = scratch + q.line_off;
  L.rad = L.xs + (q.ni + 1);
  L.nose = L.rad + (q.nj + 2);
  L.up = L.nose + (q.n_nose + 1);
  L.seg = L.up + (q.n_up + 1);
  long long segs = 0;
  for (int k = 0; k < q.nseg; ++k) segs += q.n_seg[k] + 1;
  L.down = L.seg + segs;
  return L;
}
__device__ double* seg_dist(const DReq& q, const Lines& L, int k) {
  double* p = L.seg;
  for (int t = 0; t < k; ++t) p += q.n_seg[t] + 1;
  return p;
}

// One warp per case: xs and the radial distribution. Base grids: lane 0 the nose, lanes 1.. the aft segments, lane 30
// the base-gap distribution, lane 31 the outer one; then lane 0 the upstream offsets and lane 1 the wake offsets (they
// need the nose's and the last segment's end spacings). Sting grids: the segments' distributions depend on each
// other's end spacing (one chain, lane 0), lane 31 the radial distribution.
__global__ void k_mesh_lines(const DReq* __restrict__ reqs, int n, double* __restrict__ scratch) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (c >= n) return;
  const DReq q = reqs[c];
  const Lines L = lines_of(q, scratch);
  const double ln = nose_length(q);
  if (q.wake == BOWSHOCK_WAKE_BASE) {
    double xb, re;
    station(q, q.nseg, xb, re);
    const double rs = q.sting_radius;
    if (lane == 0) two_sided_nodes(ln, q.n_nose, q.dx_tip, L.nose);
    if (lane >= 1 && lane <= q.nseg) two_sided_nodes(q.seg_len[lane - 1], q.n_seg[lane - 1], q.dx_tip, seg_dist(q, L, lane - 1));
    if (lane == 30) {  // rad[0 .. n_gap]: the base gap
      if (q.gap_one_sided) {
        double* off = L.down;  // borrowed until the wake needs it (after the next __syncwarp it is rewritten by lane 1)
        geometric_offsets(q.dr_wall, re - rs, q.n_gap, off);
        for (int k = 0; k <= q.n_gap; ++k) L.rad[k] = (re - rs) - off[q.n_gap - k];
      } else {
        two_sided_nodes(re - rs, q.n_gap, q.dr_wall, L.rad);
      }
    }
    if (lane == 31) geometric_offsets(q.dr_wall / (q.r_far - re), 1.0, q.nj_out, L.rad + q.n_gap + 1);
    __syncwarp();
    // xs: upstream [0, n_up), nose [n_up, n_up + n_nose], segments, wake
    if (lane == 0) geometric_offsets(L.nose[1] - L.nose[0], q.x_up, q.n_up, L.up);
    for (int t = lane; t <= q.n_nose; t += 32) L.xs[q.n_up + t] = L.nose[t];
    int base = q.n_up + q.n_nose;
    for (int k = 0; k < q.nseg; ++k) {
      double x0, r0;
      station(q, k, x0, r0);
      const double* sn = seg_dist(q, L, k);
      for (int i = 1 + lane; i <= q.n_seg[k]; i += 32) L.xs[base + i] = x0 + sn[i];
      base += q.n_seg[k];
    }
    __syncwarp();
    const int i_end = base;
    if (lane == 1) geometric_offsets(L.xs[i_end] - L.xs[i_end - 1], q.x_down, q.n_wake, L.down);
    __syncwarp();
    for (int k = 1 + lane; k <= q.n_wake; k += 32) L.xs[i_end + k] = xb + L.down[k];
    for (int k = lane; k < q.n_up; k += 32) L.xs[k] = -L.up[q.n_up - k];
    return;
  }
  // sting grid
  if (lane == 31) geometric_offsets(q.dr_wall / q.r_far, 1.0, q.nj_sting, L.rad);
  if (lane == 0) {
    two_sided_nodes(ln, q.n_nose, q.dx_tip, L.nose);
    const double d_tip = L.nose[1] - L.nose[0], d_sh = L.nose[q.n_nose] - L.nose[q.n_nose - 1];
    geometric_offsets(d_tip, q.x_up, q.n_up, L.up);
    for (int k = q.n_up; k >= 1; --k) L.xs[q.n_up - k] = -L.up[k];
    for (int t = 0; t <= q.n_nose; ++t) L.xs[q.n_up + t] = L.nose[t];
    int base = q.n_up + q.n_nose;
    double d_prev = d_sh;
    for (int k = 0; k < q.nseg; ++k) {
      const int nk = q.n_seg[k];
      double x0, r0;
      station(q, k, x0, r0);
      const bool geometric_fits = d_prev * (1.0 - pow(0.2, (double)nk)) / 0.8 < q.seg_len[k];
      double* offs = seg_dist(q, L, k);
      if (k == q.nseg - 1 && q.seg_slope[k] == 0.0 && geometric_fits)
        geometric_offsets(d_prev, q.seg_len[k], nk, offs);
      else
        two_sided_nodes(q.seg_len[k], nk, q.dx_tip, offs);
      for (int i = 1; i <= nk; ++i) L.xs[base + i] = x0 + offs[i];
      base += nk;
      d_prev = offs[nk] - offs[nk - 1];
    }
    geometric_offsets(d_prev, q.x_down - aft_length(q), q.n_ext, L.down);
    double xb, rb;
    station(q, q.nseg, xb, rb);
    for (int k = 1; k <= q.n_ext; ++k) L.xs[base + k] = xb + L.down[k];
  }
}

// One thread per node (blockIdx.y = case): the radial coordinate of base_domain_grid / large_domain_grid
__global__ void k_mesh_nodes(const DReq* __restrict__ reqs, const double* __restrict__ scratch, double* __restrict__ x, double* __restrict__ r) {
  const DReq& q = reqs[blockIdx.y];
  const long long nn = (long long)(q.ni + 1) * (q.nj + 1);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nn) return;
  const int i = (int)(t % (q.ni + 1)), j = (int)(t / (q.ni + 1));
  const double* xs = scratch + q.line_off;
  const double* rad = xs + (q.ni + 1);
  const double xi = xs[i];
  double rr;
  if (q.wake == BOWSHOCK_WAKE_BASE) {
    double xb, re;
    station(q, q.nseg, xb, re);
    const double rs = q.sting_radius, rw = body_r(q, xi);
    const double* gap = rad;
    const double* sj = rad + q.n_gap + 1;
    if (i >= q.i_end) {
      if (j <= q.j_sting)
        rr = rs - (double)(q.j_sting - j) * q.dr_wall;
      else if (j <= q.j_end)
        rr = rs + gap[j - q.j_sting];
      else
        rr = re + sj[j - q.j_end] * (q.r_far - re);
    } else if (j <= q.j_end) {
      rr = rw - (double)(q.j_end - j) * q.dr_wall;
    } else {
      rr = rw + sj[j - q.j_end] * (q.r_far - rw);
    }
  } else {
    const double r_in = body_r(q, xi);
    rr = r_in + rad[j] * (q.r_far - r_in);
  }
  x[q.node_off + t] = xi;
  r[q.node_off + t] = rr;
}

// One thread per i face, j face or cell (blockIdx.y = case), grid.rs:65-119 as compute_metrics: per case
// [if_nx, if_nr, if_len, if_rm] ((ni+1) nj each), [jf_nx, jf_nr, jf_len, jf_rm] (ni (nj+1) each), [area, vol, xc, rc]
// (ni nj each). bad[case] = 1 + the first cell index with a non-positive area.
__global__ void k_mesh_metrics(const DReq* __restrict__ reqs, const double* __restrict__ x, const double* __restrict__ r, double* __restrict__ met,
                               long long* __restrict__ bad) {
  const DReq& q = reqs[blockIdx.y];
  const int ni = q.ni, nj = q.nj;
  const long long nif = (long long)(ni + 1) * nj, njf = (long long)ni * (nj + 1), nc = (long long)ni * nj;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nif + njf + nc) return;
  const double* X = x + q.node_off;
  const double* R = r + q.node_off;
  double* m = met + q.met_off;
  auto nn = [&](int i, int j) { return (long long)j * (ni + 1) + i; };
  if (t < nif) {
    const int i = (int)(t % (ni + 1)), j = (int)(t / (ni + 1));
    const long long a = nn(i, j), b = nn(i, j + 1);
    const double dx = X[b] - X[a], dr = R[b] - R[a], len = hypot(dx, dr);
    m[t] = dr / len;
    m[nif + t] = -dx / len;
    m[2 * nif + t] = len;
    m[3 * nif + t] = 0.5 * (R[a] + R[b]);
    return;
  }
  if (t < nif + njf) {
    const long long f = t - nif;
    const int i = (int)(f % ni), j = (int)(f / ni);
    const long long a = nn(i, j), b = nn(i + 1, j);
    const double dx = X[b] - X[a], dr = R[b] - R[a], len = hypot(dx, dr);
    double* mj = m + 4 * nif;
    mj[f] = -dr / len;
    mj[njf + f] = dx / len;
    mj[2 * njf + f] = len;
    mj[3 * njf + f] = 0.5 * (R[a] + R[b]);
    return;
  }
  const long long c = t - nif - njf;
  const int i = (int)(c % ni), j = (int)(c / ni);
  const long long p[4] = {nn(i, j), nn(i + 1, j), nn(i + 1, j + 1), nn(i, j + 1)};
  double ar = 0, v = 0, sx = 0, sr = 0;
  const int tri[2][3] = {{0, 1, 2}, {0, 2, 3}};
  for (int u = 0; u < 2; ++u) {
    const long long k0 = p[tri[u][0]], k1 = p[tri[u][1]], k2 = p[tri[u][2]];
    const double at = 0.5 * ((X[k1] - X[k0]) * (R[k2] - R[k0]) - (X[k2] - X[k0]) * (R[k1] - R[k0]));
    const double cx = (X[k0] + X[k1] + X[k2]) / 3.0, cr = (R[k0] + R[k1] + R[k2]) / 3.0;
    ar += at;
    v += at * cr;
    sx += at * cx;
    sr += at * cr;
  }
  if (!(ar > 0.0)) atomicCAS(reinterpret_cast<unsigned long long*>(bad + blockIdx.y), 0ull, (unsigned long long)(c + 1));
  double* mc = m + 4 * nif + 4 * njf;
  mc[c] = ar;
  mc[nc + c] = v;
  mc[2 * nc + c] = sx / ar;
  mc[3 * nc + c] = sr / ar;
}

// ------------------------------------------------------------------------------------------ host side
static bk::mesh::Body body_of(const bowshock_body& b) {
  bk::mesh::Body mb;
  mb.nose = b.nose_kind, mb.fineness = b.fineness, mb.half_angle = b.half_angle, mb.param = b.param;
  for (int s = 0; s < b.nseg; ++s) mb.seg_len.push_back(b.seg_length[s]), mb.seg_slope.push_back(b.seg_slope[s]);
  mb.sting_radius = b.sting_radius;
  return mb;
}

bool dims(const bowshock_mesh_request& q, Dims& d, std::string& err) {
  const bowshock_body& b = q.body;
  if (b.nseg < 1 || b.nseg > BOWSHOCK_MAX_SEGMENTS) return err = "a body needs 1 to 8 aft segments", false;
  if (b.nose_kind < 0 || b.nose_kind > 4) return err = "unknown nose shape", false;
  const bk::mesh::Body mb = body_of(b);
  long long segs = 0;
  if (q.wake == BOWSHOCK_WAKE_BASE) {
    const bowshock_base_grid& p = q.base;
    bk::mesh::BaseGrid g{p.x_up, p.x_down, p.r_far, p.n_up, p.n_nose, {}, p.n_wake, p.n_sting, p.n_gap, p.nj_out, p.dx_tip, p.dr_wall, p.gap_one_sided != 0};
    for (int k = 0; k < b.nseg; ++k) g.n_seg.push_back(p.n_seg[k]), segs += (long long)p.n_seg[k];
    if (!bk::mesh::base_grid_check(mb, g, err)) return false;
    d.i_end = (long long)p.n_up + p.n_nose + segs;
    d.ni = d.i_end + p.n_wake;
    d.j_sting = p.n_sting;
    d.j_end = p.n_sting + p.n_gap;
    d.nj = d.j_end + p.nj_out;
  } else if (q.wake == BOWSHOCK_WAKE_STING) {
    const bowshock_sting_grid& p = q.sting;
    bk::mesh::StingGrid g{p.x_up, p.x_down, p.r_far, p.n_up, p.n_nose, {}, p.n_ext, p.nj, p.dx_tip, p.dr_wall};
    for (int k = 0; k < b.nseg; ++k) g.n_seg.push_back(p.n_seg[k]), segs += (long long)p.n_seg[k];
    if (!bk::mesh::large_grid_check(mb, g, err)) return false;
    d.ni = (long long)p.n_up + p.n_nose + segs + p.n_ext;
    d.nj = p.nj;
    d.i_end = d.j_end = d.j_sting = 0;
  } else {
    return err = "unknown wake kind", false;
  }
  if (d.ni > (1 << 20) || d.nj > (1 << 20) || (d.ni + 1) * (d.nj + 1) > (1LL << 31)) return err = "grid too large", false;
  return true;
}

int mesh_batch(uint64_t n, const bowshock_mesh_request* q, int device, double* x, double* r, double* metrics, double* device_ms, std::string& err) {
  std::vector<DReq> h(n);
  long long nodes = 0, mets = 0, lines = 0, max_items = 0;
  for (uint64_t k = 0; k < n; ++k) {
    Dims d;
    if (!dims(q[k], d, err)) {
      err = "case " + std::to_string(k) + ": " + err;
      return BOWSHOCK_INVALID;
    }
    DReq& o = h[k];
    std::memset(&o, 0, sizeof(o));
    const bowshock_body& b = q[k].body;
    o.wake = q[k].wake, o.nose = b.nose_kind, o.nseg = b.nseg;
    o.fineness = b.fineness, o.half_angle = b.half_angle, o.param = b.param, o.sting_radius = b.sting_radius;
    for (int s = 0; s < b.nseg; ++s) o.seg_len[s] = b.seg_length[s], o.seg_slope[s] = b.seg_slope[s];
    if (o.wake == BOWSHOCK_WAKE_BASE) {
      const bowshock_base_grid& p = q[k].base;
      o.x_up = p.x_up, o.x_down = p.x_down, o.r_far = p.r_far, o.dx_tip = p.dx_tip, o.dr_wall = p.dr_wall;
      o.n_up = (int)p.n_up, o.n_nose = (int)p.n_nose, o.n_wake = (int)p.n_wake, o.n_sting = (int)p.n_sting, o.n_gap = (int)p.n_gap;
      o.nj_out = (int)p.nj_out, o.gap_one_sided = p.gap_one_sided != 0;
      for (int s = 0; s < b.nseg; ++s) o.n_seg[s] = (int)p.n_seg[s];
    } else {
      const bowshock_sting_grid& p = q[k].sting;
      o.x_up = p.x_up, o.x_down = p.x_down, o.r_far = p.r_far, o.dx_tip = p.dx_tip, o.dr_wall = p.dr_wall;
      o.n_up = (int)p.n_up, o.n_nose = (int)p.n_nose, o.n_ext = (int)p.n_ext, o.nj_sting = (int)p.nj;
      for (int s = 0; s < b.nseg; ++s) o.n_seg[s] = (int)p.n_seg[s];
    }
    o.ni = (int)d.ni, o.nj = (int)d.nj, o.i_end = (int)d.i_end, o.j_end = (int)d.j_end, o.j_sting = (int)d.j_sting;
    o.node_off = nodes, o.met_off = mets, o.line_off = lines;
    nodes += (d.ni + 1) * (d.nj + 1);
    mets += BOWSHOCK_MESH_METRIC_WORDS(d.ni, d.nj);
    lines += line_words(o);
    max_items = std::max(max_items, std::max((d.ni + 1) * (d.nj + 1), (d.ni + 1) * d.nj + d.ni * (d.nj + 1) + d.ni * d.nj));
  }
  if (n == 0) return BOWSHOCK_OK;
  if (n > 65535) return err = "at most 65,535 cases per batch", BOWSHOCK_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return err = "no such CUDA device", BOWSHOCK_CUDA_ERROR;
  cudaSetDevice(device);
  DReq* d_req = nullptr;
  double *d_scr = nullptr, *d_x = nullptr, *d_r = nullptr, *d_m = nullptr;
  long long* d_bad = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = BOWSHOCK_OK;
  auto ck = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == BOWSHOCK_OK) {
      err = std::string(what) + ": " + cudaGetErrorString(e);
      rc = BOWSHOCK_CUDA_ERROR;
    }
    return rc == BOWSHOCK_OK;
  };
  if (ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream") && ck(cudaEventCreate(&e0), "event") && ck(cudaEventCreate(&e1), "event") &&
      ck(cudaMalloc(&d_req, n * sizeof(DReq)), "malloc") && ck(cudaMalloc(&d_scr, lines * sizeof(double)), "malloc") &&
      ck(cudaMalloc(&d_x, nodes * sizeof(double)), "malloc") && ck(cudaMalloc(&d_r, nodes * sizeof(double)), "malloc") &&
      ck(cudaMalloc(&d_bad, n * sizeof(long long)), "malloc") && (!metrics || ck(cudaMalloc(&d_m, mets * sizeof(double)), "malloc")) &&
      ck(copy_sync(st, d_req, h.data(), n * sizeof(DReq), cudaMemcpyHostToDevice), "upload") &&
      ck(cudaMemsetAsync(d_bad, 0, n * sizeof(long long), st), "memset") && ck(cudaEventRecord(e0, st), "event")) {
    k_mesh_lines<<<(unsigned)((n + 3) / 4), 128, 0, st>>>(d_req, (int)n, d_scr);
    const unsigned bx = (unsigned)((max_items + 255) / 256);
    k_mesh_nodes<<<dim3(bx, (unsigned)n), 256, 0, st>>>(d_req, d_scr, d_x, d_r);
    if (metrics) k_mesh_metrics<<<dim3(bx, (unsigned)n), 256, 0, st>>>(d_req, d_x, d_r, d_m, d_bad);
    if (ck(cudaGetLastError(), "launch") && ck(cudaEventRecord(e1, st), "event") && ck(cudaStreamSynchronize(st), "mesher kernels")) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (device_ms) *device_ms = ms;
      std::vector<long long> bad(n);
      if (ck(copy_sync(st, bad.data(), d_bad, n * sizeof(long long), cudaMemcpyDeviceToHost), "download") &&
          (!x || ck(copy_sync(st, x, d_x, nodes * sizeof(double), cudaMemcpyDeviceToHost), "download")) &&
          (!r || ck(copy_sync(st, r, d_r, nodes * sizeof(double), cudaMemcpyDeviceToHost), "download")) &&
          (!metrics || ck(copy_sync(st, metrics, d_m, mets * sizeof(double), cudaMemcpyDeviceToHost), "download"))) {
        for (uint64_t k = 0; k < n; ++k)
          if (bad[k]) {
            const long long c = bad[k] - 1;
            err = "case " + std::to_string(k) + ": non-positive cell area at (" + std::to_string(c % h[k].ni) + "," + std::to_string(c / h[k].ni) + ")";
            rc = BOWSHOCK_INVALID;
            break;
          }
      }
    }
  }
  cudaFree(d_req), cudaFree(d_scr), cudaFree(d_x), cudaFree(d_r), cudaFree(d_m), cudaFree(d_bad);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  return rc;
}

}  // namespace bkmesh

extern "C" {

int bowshock_mesh_dims(const bowshock_mesh_request* q, uint64_t* ni, uint64_t* nj, bowshock_block* block) {
  if (!q || !ni || !nj) return BOWSHOCK_INVALID;
  bkmesh::Dims d;
  std::string err;
  if (!bkmesh::dims(*q, d, err)) return BOWSHOCK_INVALID;
  *ni = (uint64_t)d.ni, *nj = (uint64_t)d.nj;
  if (block) *block = bowshock_block{(uint64_t)d.i_end, (uint64_t)d.j_end, (uint64_t)d.j_sting};
  return BOWSHOCK_OK;
}

int bowshock_mesh_batch(uint64_t n, const bowshock_mesh_request* q, int device, double* x, double* r, double* metrics, double* device_ms) {
  if (!q || n == 0) return BOWSHOCK_INVALID;
  std::string err;
  return bkmesh::mesh_batch(n, q, device, x, r, metrics, device_ms, err);
}

}  // extern "C"
