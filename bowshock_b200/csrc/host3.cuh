// Host side of the 3D batch (euler3.cuh): FP64 grid metrics from the node coordinates (grid3.rs:66-174: faces from their four
// corners, volumes by the divergence theorem over the face centroids, one global handedness sign), the cell across the
// axis (solver3.rs:98-117), device buffers, the iteration launch sequence, and the reference's 3D stop rules
// (run3.rs:220-330) with per-case masks.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "euler3.cuh"
#include "stream_copy.cuh"

namespace bk3 {

struct Grid3H {
  size_t ni = 0, nj = 0, nk = 0;
  std::vector<double> fi, fj, fk;  // 7 per face: n[3], area, c[3]
  std::vector<double> vol, xc;     // xc 3 per cell
};

static inline void face_of(const double* p0, const double* p1, const double* p2, const double* p3, double* out, double* s) {
  double a[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]}, b[3] = {p3[0] - p1[0], p3[1] - p1[1], p3[2] - p1[2]};
  s[0] = 0.5 * (a[1] * b[2] - a[2] * b[1]);
  s[1] = 0.5 * (a[2] * b[0] - a[0] * b[2]);
  s[2] = 0.5 * (a[0] * b[1] - a[1] * b[0]);
  double area = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
  if (area < 1e-300) {
    out[0] = out[1] = out[2] = out[3] = 0.0;
  } else {
    out[0] = s[0] / area, out[1] = s[1] / area, out[2] = s[2] / area, out[3] = area;
  }
  for (int m = 0; m < 3; ++m) out[4 + m] = 0.25 * (p0[m] + p1[m] + p2[m] + p3[m]);
}

// false (with a message) on a negative cell volume
inline bool grid3_metrics(size_t ni, size_t nj, size_t nk, const double* x, const double* y, const double* z, Grid3H& g, std::string& err) {
  g = Grid3H{};
  g.ni = ni, g.nj = nj, g.nk = nk;
  auto pt = [&](size_t i, size_t j, size_t k, double* p) {
    size_t n = (k * (nj + 1) + j) * (ni + 1) + i;
    p[0] = x[n], p[1] = y[n], p[2] = z[n];
  };
  size_t nfi = (ni + 1) * nj * nk, nfj = ni * (nj + 1) * nk, nfk = ni * nj * (nk + 1);
  g.fi.assign(7 * nfi, 0.0), g.fj.assign(7 * nfj, 0.0), g.fk.assign(7 * nfk, 0.0);
  std::vector<double> si(3 * nfi), sj(3 * nfj), sk(3 * nfk);
  double p[4][3];
  for (size_t k = 0; k < nk; ++k)
    for (size_t j = 0; j < nj; ++j)
      for (size_t i = 0; i <= ni; ++i) {
        size_t q = (k * nj + j) * (ni + 1) + i;
        pt(i, j, k, p[0]), pt(i, j + 1, k, p[1]), pt(i, j + 1, k + 1, p[2]), pt(i, j, k + 1, p[3]);
        face_of(p[0], p[1], p[2], p[3], &g.fi[7 * q], &si[3 * q]);
      }
  for (size_t k = 0; k < nk; ++k)
    for (size_t j = 0; j <= nj; ++j)
      for (size_t i = 0; i < ni; ++i) {
        size_t q = (k * (nj + 1) + j) * ni + i;
        pt(i, j, k, p[0]), pt(i, j, k + 1, p[1]), pt(i + 1, j, k + 1, p[2]), pt(i + 1, j, k, p[3]);
        face_of(p[0], p[1], p[2], p[3], &g.fj[7 * q], &sj[3 * q]);
      }
  for (size_t k = 0; k <= nk; ++k)
    for (size_t j = 0; j < nj; ++j)
      for (size_t i = 0; i < ni; ++i) {
        size_t q = (k * nj + j) * ni + i;
        pt(i, j, k, p[0]), pt(i + 1, j, k, p[1]), pt(i + 1, j + 1, k, p[2]), pt(i, j + 1, k, p[3]);
        face_of(p[0], p[1], p[2], p[3], &g.fk[7 * q], &sk[3 * q]);
      }
  size_t nc = ni * nj * nk;
  g.vol.assign(nc, 0.0), g.xc.assign(3 * nc, 0.0);
  auto dotc = [](const double* f, const double* s) { return f[4] * s[0] + f[5] * s[1] + f[6] * s[2]; };
  double tot = 0.0;
  for (size_t k = 0; k < nk; ++k)
    for (size_t j = 0; j < nj; ++j)
      for (size_t i = 0; i < ni; ++i) {
        size_t il = (k * nj + j) * (ni + 1) + i, jl = (k * (nj + 1) + j) * ni + i, kl = (k * nj + j) * ni + i;
        size_t jr = jl + ni, kr = kl + ni * nj;
        double v = 0.0;
        v += dotc(&g.fi[7 * (il + 1)], &si[3 * (il + 1)]);
        v -= dotc(&g.fi[7 * il], &si[3 * il]);
        v += dotc(&g.fj[7 * jr], &sj[3 * jr]);
        v -= dotc(&g.fj[7 * jl], &sj[3 * jl]);
        v += dotc(&g.fk[7 * kr], &sk[3 * kr]);
        v -= dotc(&g.fk[7 * kl], &sk[3 * kl]);
        size_t c = kl;
        g.vol[c] = v / 3.0;
        tot += g.vol[c];
        double m[3] = {0, 0, 0};
        for (int bb = 0; bb < 8; ++bb) {
          double q[3];
          pt(i + (bb & 1), j + (bb >> 1 & 1), k + (bb >> 2 & 1), q);
          for (int a = 0; a < 3; ++a) m[a] += 0.125 * q[a];
        }
        for (int a = 0; a < 3; ++a) g.xc[3 * c + a] = m[a];
      }
  if (tot < 0.0) {
    for (auto* fam : {&g.fi, &g.fj, &g.fk})
      for (size_t q = 0; q < fam->size(); q += 7) (*fam)[q] = -(*fam)[q], (*fam)[q + 1] = -(*fam)[q + 1], (*fam)[q + 2] = -(*fam)[q + 2];
    for (auto& v : g.vol) v = -v;
  }
  double vmax = 0.0;
  for (double v : g.vol) vmax = std::fmax(vmax, std::fabs(v));
  for (size_t c = 0; c < nc; ++c)
    if (g.vol[c] < -1e-12 * vmax || std::isnan(g.vol[c])) {
      err = "negative cell volume at cell " + std::to_string(c);
      return false;
    }
  return true;
}

struct Case3Host {
  double mach = 0.5, alpha = 0.0, cfl = 0.5;
  int limiter = 1, low_mach = 0, implicit = 1;
  long long first_order_iters = 0;
  double cfl0 = 1.0, cfl_max = 30.0, growth = 1.02, eps_fix = 0.1;
  int dt_mode = 0, sub_iters = 2, roe = 1, implicit_bc = 1, lines = 1;
};

#define BK3_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
      return 3;                                                                 \
    }                                                                           \
  } while (0)

struct Batch3 {
  B3 B{};
  Grid3H g;
  std::vector<Case3Host> cases;
  std::vector<int> axis_k;
  std::vector<double> wall;  // WALL3 per wall face (k3_forces)
  int nwall = 0, device = 0, slots = 64;
  std::vector<unsigned char> solid_h;  // per cell, inside a solid box
  long long n_active = 0;              // fluid cells: the density norm's denominator (solver3.rs:97, 152-155)
  unsigned char* d_solid = nullptr;
  size_t wall_cap = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms_per_iter = 0.0;
  std::string err;
  std::vector<void*> owned;
  double *d_wall = nullptr, *d_forces = nullptr, *d_parts = nullptr;
  std::vector<int> h_active;

  ~Batch3() { release(); }
  void release() {
    if (stream) cudaStreamSynchronize(stream);
    for (cudaStream_t st : gst) cudaStreamDestroy(st);
    for (cudaEvent_t ev : gev) cudaEventDestroy(ev);
    gst.clear(), gev.clear();
    if (ev_fork3) cudaEventDestroy(ev_fork3), ev_fork3 = nullptr;
    if (pe0) cudaEventDestroy(pe0), pe0 = nullptr;
    if (pe1) cudaEventDestroy(pe1), pe1 = nullptr;
    for (void* p : owned)
      if (p) cudaFree(p);
    owned.clear();
    if (ev0) cudaEventDestroy(ev0), ev0 = nullptr;
    if (ev1) cudaEventDestroy(ev1), ev1 = nullptr;
    if (stream) cudaStreamDestroy(stream), stream = nullptr;
  }
  template <class T>
  int alloc(T** p, size_t n) {
    *p = nullptr;
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
      err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
      return 3;
    }
    owned.push_back((void*)*p);
    return 0;
  }

  static void to_dev(const Case3Host& h, Case3Dev& d) {
    double a = h.alpha;
    d.fs[0] = 1.0, d.fs[1] = h.mach * std::cos(a), d.fs[2] = 0.0, d.fs[3] = h.mach * std::sin(a), d.fs[4] = 1.0 / 1.4;  // gas3.rs:42-44
    d.cfl = (float)h.cfl, d.cfl0 = (float)h.cfl0, d.cfl_max = (float)h.cfl_max, d.growth = (float)h.growth, d.eps_fix = (float)h.eps_fix;
    d.limiter = h.limiter, d.low_mach = h.low_mach, d.first_order_iters = (int)h.first_order_iters, d.implicit = h.implicit;
    d.dt_mode = h.dt_mode, d.sub_iters = h.sub_iters, d.roe = h.roe, d.implicit_bc = h.implicit_bc, d.lines = h.lines;
  }

  int create(size_t ni, size_t nj, size_t nk, const double* x, const double* y, const double* z, size_t axis_cells,
             const std::vector<Case3Host>& cs, int dev) {
    if (ni < 2 || nj < 2 || nk < 2 || cs.empty() || axis_cells > ni) {
      err = "invalid 3D grid or case list";
      return 2;
    }
    if (!grid3_metrics(ni, nj, nk, x, y, z, g, err)) return 2;
    cases = cs;
    device = dev;
    BK3_CUDA(cudaSetDevice(dev));
    BK3_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    BK3_CUDA(cudaEventCreate(&ev0));
    BK3_CUDA(cudaEventCreate(&ev1));
    const int nb = (int)cs.size();
    B.ni = (int)ni, B.nj = (int)nj, B.nk = (int)nk, B.nb = nb, B.axis_cells = (int)axis_cells;
    B.nc = (long long)ni * nj * nk;
    B.npad = (long long)(ni + 4) * (nj + 4) * (nk + 4);
    B.nfi = (long long)(ni + 1) * nj * nk, B.nfj = (long long)ni * (nj + 1) * nk, B.nfk = (long long)ni * nj * (nk + 1);
    // the cell across the axis: the one whose centroid azimuth is closest to pi - theta (solver3.rs:98-117)
    axis_k.assign(std::max<size_t>(axis_cells * nk, 1), 0);
    auto theta = [&](size_t i, size_t k) {
      const double* c = &g.xc[3 * ((k * nj) * ni + i)];
      return std::atan2(c[1], c[2]);
    };
    for (size_t i = 0; i < axis_cells; ++i)
      for (size_t k = 0; k < nk; ++k) {
        double target = M_PI - theta(i, k), best = INFINITY;
        size_t bk = 0;
        for (size_t kk = 0; kk < nk; ++kk) {
          double d = std::fabs(theta(i, kk) - target);
          if (d < best) best = d, bk = kk;
        }
        axis_k[i * nk + k] = (int)bk;
      }
    solid_h.assign((size_t)B.nc, 0);
    n_active = B.nc;
    build_wall();
    wall_cap = std::max<size_t>(wall.size(), 1);
    int rc;
    float4 *fi, *fj, *fk;
    float2 *ri, *rj, *rk;
    float* vol;
    int* ak;
    Case3Dev* dcs;
    if ((rc = alloc(&fi, B.nfi)) || (rc = alloc(&fj, B.nfj)) || (rc = alloc(&fk, B.nfk)) || (rc = alloc(&ri, B.nfi)) || (rc = alloc(&rj, B.nfj)) ||
        (rc = alloc(&rk, B.nfk)) || (rc = alloc(&vol, B.nc)) || (rc = alloc(&ak, axis_k.size())) || (rc = alloc(&dcs, nb)) ||
        (rc = alloc(&B.iter, nb)) || (rc = alloc(&B.ramp, nb)) || (rc = alloc(&B.active, nb)))
      return rc;
    size_t ns = (size_t)nb * 5 * B.nc;
    if ((rc = alloc(&B.U, ns)) || (rc = alloc(&B.U0, ns)) || (rc = alloc(&B.W, (size_t)nb * 5 * B.npad)) || (rc = alloc(&B.R, ns)) ||
        (rc = alloc(&B.X, ns)) || (rc = alloc(&B.DU, ns)) || (rc = alloc(&B.RR, ns)) || (rc = alloc(&B.dt, (size_t)nb * B.nc)) ||
        (rc = alloc(&B.scr, (size_t)nb * 3 * REC3 * B.nc)) || (rc = alloc(&B.FI, (size_t)nb * 5 * B.nfi)) || (rc = alloc(&B.FJ, (size_t)nb * 5 * B.nfj)) ||
        (rc = alloc(&B.FK, (size_t)nb * 5 * B.nfk)) || (rc = alloc(&B.rsum, (size_t)slots * nb)) || (rc = alloc(&d_wall, wall_cap)) ||
        (rc = alloc(&d_forces, 3 * (size_t)nb)) || (rc = alloc(&d_parts, 15 * (size_t)nb)))
      return rc;
    auto up_faces = [&](const std::vector<double>& f, long long n, float4* d4, float2* d2) -> int {
      std::vector<float4> h4(n);
      std::vector<float2> h2(n);
      for (long long q = 0; q < n; ++q) {
        const double* p = &f[7 * q];
        h4[q] = make_float4((float)p[0], (float)p[1], (float)p[2], (float)p[3]);
        double r = std::hypot(p[5], p[6]);  // face_rot (flux3.rs:11-19)
        h2[q] = r < 1e-300 ? make_float2(0.f, 1.f) : make_float2((float)(p[5] / r), (float)(p[6] / r));
      }
      BK3_CUDA(copy_sync(stream, d4, h4.data(), n * sizeof(float4), cudaMemcpyHostToDevice));
      BK3_CUDA(copy_sync(stream, d2, h2.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
      return 0;
    };
    if ((rc = up_faces(g.fi, B.nfi, fi, ri)) || (rc = up_faces(g.fj, B.nfj, fj, rj)) || (rc = up_faces(g.fk, B.nfk, fk, rk))) return rc;
    std::vector<float> hv(B.nc);
    for (long long c = 0; c < B.nc; ++c) hv[c] = (float)g.vol[c];
    BK3_CUDA(copy_sync(stream, vol, hv.data(), B.nc * sizeof(float), cudaMemcpyHostToDevice));
    BK3_CUDA(copy_sync(stream, ak, axis_k.data(), axis_k.size() * sizeof(int), cudaMemcpyHostToDevice));
    BK3_CUDA(copy_sync(stream, d_wall, wall.data(), wall.size() * sizeof(double), cudaMemcpyHostToDevice));
    B.fi = fi, B.fj = fj, B.fk = fk, B.ri = ri, B.rj = rj, B.rk = rk, B.vol = vol, B.axis_k = ak, B.cs = dcs;
    if ((rc = upload_cases())) return rc;
    h_active.assign(nb, 1);
    BK3_CUDA(copy_sync(stream, B.active, h_active.data(), nb * sizeof(int), cudaMemcpyHostToDevice));
    return reset();
  }
  // run3.rs:130-212: the wall faces that carry forces, WALL3 doubles each (k3_forces): the j = 0 faces of fluid cells with
  // i >= axis_cells, then the faces between a fluid and a solid cell in i, j and k
  void build_wall() {
    const size_t ni = g.ni, nj = g.nj, nk = g.nk;
    auto cell = [&](size_t i, size_t j, size_t k) { return (k * nj + j) * ni + i; };
    auto sol = [&](size_t i, size_t j, size_t k) { return solid_h[cell(i, j, k)] != 0; };
    wall.clear();
    int part = 0;  // run3.rs:130-212: 0 body wall, 2 fin sides (k faces), 3 fin edges (i faces), 4 fin tips (j faces)
    auto add = [&](const double* f, size_t a, long long b, double sign) {
      for (int q = 0; q < 7; ++q) wall.push_back(f[q]);
      for (int q = 0; q < 3; ++q) wall.push_back(g.xc[3 * a + q]);
      for (int q = 0; q < 3; ++q) wall.push_back(b >= 0 ? g.xc[3 * (size_t)b + q] : 0.0);
      wall.push_back((double)a), wall.push_back((double)b), wall.push_back(sign), wall.push_back((double)part);
    };
    for (size_t k = 0; k < nk; ++k)
      for (size_t i = (size_t)B.axis_cells; i < ni; ++i)
        if (!sol(i, 0, k)) add(&g.fj[7 * (k * (nj + 1) * ni + i)], cell(i, 0, k), nj > 1 && !sol(i, 1, k) ? (long long)cell(i, 1, k) : -1, -1.0);
    if (n_active != B.nc) {
      part = 3;
      for (size_t k = 0; k < nk; ++k)
        for (size_t j = 0; j < nj; ++j)
          for (size_t i = 1; i < ni; ++i) {
            const double* f = &g.fi[7 * ((k * nj + j) * (ni + 1) + i)];
            const bool a = sol(i - 1, j, k), b = sol(i, j, k);
            if (!a && b) add(f, cell(i - 1, j, k), i >= 2 && !sol(i - 2, j, k) ? (long long)cell(i - 2, j, k) : -1, 1.0);
            if (a && !b) add(f, cell(i, j, k), i + 1 < ni && !sol(i + 1, j, k) ? (long long)cell(i + 1, j, k) : -1, -1.0);
          }
      part = 4;
      for (size_t k = 0; k < nk; ++k)
        for (size_t j = 1; j < nj; ++j)
          for (size_t i = 0; i < ni; ++i) {
            const double* f = &g.fj[7 * ((k * (nj + 1) + j) * ni + i)];
            const bool a = sol(i, j - 1, k), b = sol(i, j, k);
            if (!a && b) add(f, cell(i, j - 1, k), j >= 2 && !sol(i, j - 2, k) ? (long long)cell(i, j - 2, k) : -1, 1.0);
            if (a && !b) add(f, cell(i, j, k), j + 1 < nj && !sol(i, j + 1, k) ? (long long)cell(i, j + 1, k) : -1, -1.0);
          }
      part = 2;
      for (size_t k = 1; k < nk; ++k)
        for (size_t j = 0; j < nj; ++j)
          for (size_t i = 0; i < ni; ++i) {
            const double* f = &g.fk[7 * ((k * nj + j) * ni + i)];
            const bool a = sol(i, j, k - 1), b = sol(i, j, k);
            if (!a && b) add(f, cell(i, j, k - 1), k >= 2 && !sol(i, j, k - 2) ? (long long)cell(i, j, k - 2) : -1, 1.0);
            if (a && !b) add(f, cell(i, j, k), k + 1 < nk && !sol(i, j, k + 1) ? (long long)cell(i, j, k + 1) : -1, -1.0);
          }
    }
    nwall = (int)(wall.size() / WALL3);
  }
  // Solid boxes (grid3.rs:17-24 SolidBox; 6 per box: i0, i1, j0, j1, k0, k1, half-open cell ranges) of the shared grid:
  // the cell mask, the fluid-cell count, the force faces; every case back to its free stream (solid cells keep it).
  int set_solid(size_t nbox, const uint64_t* boxes) {
    const uint64_t ext[3] = {(uint64_t)B.ni, (uint64_t)B.nj, (uint64_t)B.nk};
    for (size_t q = 0; q < nbox; ++q)
      for (int d = 0; d < 3; ++d)
        if (!(boxes[6 * q + 2 * d] < boxes[6 * q + 2 * d + 1] && boxes[6 * q + 2 * d + 1] <= ext[d])) {
          err = "solid box out of the grid or empty";
          return 2;
        }
    std::vector<unsigned char> mask((size_t)B.nc, 0);
    for (size_t q = 0; q < nbox; ++q) {
      const uint64_t* r = boxes + 6 * q;
      for (uint64_t k = r[4]; k < r[5]; ++k)
        for (uint64_t j = r[2]; j < r[3]; ++j)
          for (uint64_t i = r[0]; i < r[1]; ++i) mask[(k * B.nj + j) * B.ni + i] = 1;
    }
    long long fluid = 0;
    for (unsigned char v : mask) fluid += v ? 0 : 1;
    if (fluid == 0) {  // refused with the batch as it was
      err = "every cell is solid";
      return 2;
    }
    solid_h.swap(mask);
    n_active = fluid;
    int rc;
    if (!d_solid && (rc = alloc(&d_solid, (size_t)B.nc))) return rc;
    BK3_CUDA(copy_sync(stream, d_solid, solid_h.data(), (size_t)B.nc, cudaMemcpyHostToDevice));
    B.solid = n_active != B.nc ? d_solid : nullptr;
    build_wall();
    if (wall.size() > wall_cap) {
      wall_cap = wall.size();
      if ((rc = alloc(&d_wall, wall_cap))) return rc;
    }
    BK3_CUDA(copy_sync(stream, d_wall, wall.data(), wall.size() * sizeof(double), cudaMemcpyHostToDevice));
    return reset();
  }
  // GpuSolver3::set_config (gpu/mod.rs:482-487) for case b: free stream, CFL, limiter, first-order iterations and the
  // low-Mach flag may change between runs, state and geometry untouched; a changed scheme restarts the case's CFL ramp.
  // The batch runs one scheme: the explicit / implicit kind changes only for a batch of one case.
  int set_config(int b, const Case3Host& h) {
    const Case3Host& o = cases[b];
    if (h.implicit != o.implicit && B.nb > 1) {
      err = "one scheme per batch: the explicit / implicit kind changes only for a batch of one case";
      return 1;
    }
    const bool scheme_changed = h.implicit != o.implicit || h.cfl0 != o.cfl0 || h.cfl_max != o.cfl_max || h.growth != o.growth ||
                                h.eps_fix != o.eps_fix || h.dt_mode != o.dt_mode || h.sub_iters != o.sub_iters || h.roe != o.roe ||
                                h.implicit_bc != o.implicit_bc || h.lines != o.lines;
    cases[b] = h;
    int rc;
    if ((rc = upload_cases())) return rc;
    if (scheme_changed) {
      const int zero = 0;
      BK3_CUDA(copy_sync(stream, B.ramp + b, &zero, sizeof(int), cudaMemcpyHostToDevice));
    }
    return 0;
  }
  int upload_cases() {
    std::vector<Case3Dev> h(cases.size());
    for (size_t k = 0; k < cases.size(); ++k) to_dev(cases[k], h[k]);
    BK3_CUDA(copy_sync(stream, const_cast<Case3Dev*>(B.cs), h.data(), h.size() * sizeof(Case3Dev), cudaMemcpyHostToDevice));
    return 0;
  }
  // every case to its free stream, iteration and ramp counters to zero
  int reset() {
    for (int b = 0; b < B.nb; ++b) {
      Case3Dev d;
      to_dev(cases[b], d);
      double q[5] = {d.fs[0], d.fs[0] * d.fs[1], d.fs[0] * d.fs[2], d.fs[0] * d.fs[3],
                     d.fs[4] / 0.4 + 0.5 * d.fs[0] * (d.fs[1] * d.fs[1] + d.fs[2] * d.fs[2] + d.fs[3] * d.fs[3])};
      std::vector<float> h(B.nc);
      for (int v = 0; v < 5; ++v) {
        std::fill(h.begin(), h.end(), (float)q[v]);
        BK3_CUDA(copy_sync(stream, B.U + ((size_t)b * 5 + v) * B.nc, h.data(), B.nc * sizeof(float), cudaMemcpyHostToDevice));
      }
    }
    std::vector<int> z(B.nb, 0);
    BK3_CUDA(copy_sync(stream, B.iter, z.data(), B.nb * sizeof(int), cudaMemcpyHostToDevice));
    BK3_CUDA(copy_sync(stream, B.ramp, z.data(), B.nb * sizeof(int), cudaMemcpyHostToDevice));
    return 0;
  }
  int set_state(int b, const double* u) {  // u: ncell x 5 (Cons3 layout)
    std::vector<float> h(5 * B.nc);
    for (long long c = 0; c < B.nc; ++c)
      for (int v = 0; v < 5; ++v) h[v * B.nc + c] = (float)u[5 * c + v];
    BK3_CUDA(copy_sync(stream, B.U + (size_t)b * 5 * B.nc, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
    return 0;
  }
  int get_state(int b, double* u) {
    std::vector<float> h(5 * B.nc);
    BK3_CUDA(cudaStreamSynchronize(stream));
    BK3_CUDA(copy_sync(stream, h.data(), B.U + (size_t)b * 5 * B.nc, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (long long c = 0; c < B.nc; ++c)
      for (int v = 0; v < 5; ++v) u[5 * c + v] = h[v * B.nc + c];
    return 0;
  }
  int set_counters(int it, int ramp) {
    std::vector<int> a(B.nb, it), r(B.nb, ramp);
    BK3_CUDA(copy_sync(stream, B.iter, a.data(), B.nb * sizeof(int), cudaMemcpyHostToDevice));
    BK3_CUDA(copy_sync(stream, B.ramp, r.data(), B.nb * sizeof(int), cudaMemcpyHostToDevice));
    return 0;
  }
  int set_active(const std::vector<int>& act) {
    h_active = act;
    BK3_CUDA(cudaMemcpyAsync(B.active, h_active.data(), B.nb * sizeof(int), cudaMemcpyHostToDevice, stream));
    BK3_CUDA(cudaStreamSynchronize(stream));
    return 0;
  }

  // Case groups: with groups > 1 the cases are split into that many groups of consecutive cases and each group's
  // iterations of a chunk run on a stream of their own (the launches of a group cover its cases only: B.b0, gnb), so
  // one group's kernels fill the SMs while another's last wave runs. Every kernel touches only its own cases, so the
  // states are those of one group bit for bit (the norms' atomic block sums aside).
  int groups = 1, gnb = 0;
  std::vector<cudaStream_t> gst;
  std::vector<cudaEvent_t> gev;
  cudaEvent_t ev_fork3 = nullptr;
  int set_groups(int n) {
    if (n < 1 || n > 4 || n > B.nb) {
      err = "case groups out of range (1 to 4, at most the case count)";
      return 2;
    }
    while ((int)gst.size() < n) {
      cudaStream_t st;
      cudaEvent_t ev;
      BK3_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      BK3_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      gst.push_back(st), gev.push_back(ev);
    }
    if (!ev_fork3) BK3_CUDA(cudaEventCreateWithFlags(&ev_fork3, cudaEventDisableTiming));
    groups = n;
    return 0;
  }
  dim3 grid_of(long long n, int threads) const { return dim3((unsigned)((n + threads - 1) / threads), (unsigned)(gnb ? gnb : B.nb)); }
  // Per-kernel profile (GpuSolver3::profile_step / profile_replay, gpu/mod.rs:525-535): with `profiling` set every launch
  // is bracketed by CUDA events and its time added to its group.
  enum { P3_PRIMS = 0, P3_FLUX, P3_RESIDUAL, P3_ASSEMBLE, P3_LINES, P3_SUBST, P3_DEFECT, P3_STAGE, P3_N };
  bool profiling = false;
  double prof_ms[P3_N] = {0};
  long long prof_n[P3_N] = {0};
  cudaEvent_t pe0 = nullptr, pe1 = nullptr;
  template <class F>
  void L3(int g, F&& launch) {
    if (!profiling) {
      launch();
      return;
    }
    cudaEventRecord(pe0, stream);
    launch();
    cudaEventRecord(pe1, stream);
    cudaEventSynchronize(pe1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, pe0, pe1);
    prof_ms[g] += ms, prof_n[g] += 1;
  }
  int profile(long long n, double* ms, unsigned long long* launches) {
    if (!pe0) {
      BK3_CUDA(cudaEventCreate(&pe0));
      BK3_CUDA(cudaEventCreate(&pe1));
    }
    for (int g = 0; g < P3_N; ++g) prof_ms[g] = 0.0, prof_n[g] = 0;
    const int g0 = groups;
    groups = 1, profiling = true;
    int rc = run(n, nullptr);
    profiling = false, groups = g0;
    for (int g = 0; g < P3_N; ++g) ms[g] = prof_ms[g], launches[g] = (unsigned long long)prof_n[g];
    return rc;
  }
  // `chunk` iterations of every active case, per group on its own stream between a fork and a join on `stream`
  void launch_chunk(int chunk) {
    if (groups <= 1) {
      for (int k = 0; k < chunk; ++k) launch_iteration(k);
      return;
    }
    const cudaStream_t main = stream;
    cudaEventRecord(ev_fork3, main);
    for (int g = 0; g < groups; ++g) {
      const int lo = (int)((long long)B.nb * g / groups), hi = (int)((long long)B.nb * (g + 1) / groups);
      if (hi <= lo) continue;
      stream = gst[g];
      cudaStreamWaitEvent(stream, ev_fork3, 0);
      B.b0 = lo, gnb = hi - lo;
      for (int k = 0; k < chunk; ++k) launch_iteration(k);
      cudaEventRecord(gev[g], stream);
    }
    stream = main;
    B.b0 = 0, gnb = 0;
    for (int g = 0; g < groups; ++g) cudaStreamWaitEvent(stream, gev[g], 0);
  }
  void launch_prep() {
    L3(P3_PRIMS, [&] { k3_prims<<<grid_of(B.nc, 256), 256, 0, stream>>>(B); });
    long long ng = 2LL * B.nj * B.nk + 2LL * B.ni * B.nk + 2LL * B.ni * B.nj;
    L3(P3_PRIMS, [&] { k3_ghosts<<<grid_of(ng, 128), 128, 0, stream>>>(B); });
    L3(P3_FLUX, [&] { k3_flux<<<grid_of(B.nfi, 128), 128, 0, stream>>>(B, 0); });
    L3(P3_FLUX, [&] { k3_flux<<<grid_of(B.nfj, 128), 128, 0, stream>>>(B, 1); });
    L3(P3_FLUX, [&] { k3_flux<<<grid_of(B.nfk, 128), 128, 0, stream>>>(B, 2); });
  }
  bool implicit() const { return cases[0].implicit != 0; }
  // the staged first pass (k3_lines_st): on unless pinned off; only where a warp's 32 lines are adjacent (i lines: nj a
  // multiple of 32; j and k lines: ni a multiple of 32), which also makes every one of its 16-byte copies aligned
  bool staged = true;
  bool staged_ok(int dir) const { return staged && (dir == 0 ? B.nj % 32 == 0 : B.ni % 32 == 0); }
  void launch_lines(int dir, long long nl, const float* in, int from_res, float* out, int epilogue) {
    L3(P3_LINES, [&] {
      if (staged_ok(dir))
        k3_lines_st<<<grid_of(nl, 32), 32, 0, stream>>>(B, dir, in, from_res, out, epilogue);
      else
        k3_lines<<<grid_of(nl, 64), 64, 0, stream>>>(B, dir, in, from_res, out, epilogue);
    });
  }
  void launch_subst(int dir, long long nl, const float* in, float* out, int epilogue, int pass) {
    L3(P3_SUBST, [&] {
      if (staged_ok(dir))
        k3_lines_subst_st<<<grid_of(nl, 32), 32, 0, stream>>>(B, dir, in, out, epilogue, pass);
      else
        k3_lines_subst<<<grid_of(nl, 128), 128, 0, stream>>>(B, dir, in, out, epilogue, pass);
    });
  }
  int max_sub() const {
    int s = 1;
    for (auto& c : cases) s = std::max(s, c.sub_iters);
    return s;
  }
  void launch_iteration(int slot) {
    if (implicit()) {
      launch_prep();
      L3(P3_RESIDUAL, [&] { k3_residual<<<grid_of(B.nc, 256), 256, 0, stream>>>(B, 2, slot); });
      const long long li = (long long)B.nj * B.nk, lj = (long long)B.ni * B.nk, lk = (long long)B.ni * B.nj;
      L3(P3_ASSEMBLE, [&] { k3_assemble<<<grid_of(B.nc, 128), 128, 0, stream>>>(B, 0); });
      L3(P3_ASSEMBLE, [&] { k3_assemble<<<grid_of(B.nc, 128), 128, 0, stream>>>(B, 1); });
      launch_lines(0, li, B.R, 1, B.X, 0);
      launch_lines(1, lj, B.X, 0, B.X, 0);
      launch_lines(2, lk, B.X, 0, nullptr, 1);
      for (int p = 1; p < max_sub(); ++p) {
        L3(P3_DEFECT, [&] { k3_defect_i<<<grid_of(B.nc, 128), 128, 0, stream>>>(B, p); });
        L3(P3_DEFECT, [&] { k3_defect<<<grid_of(B.nc, 128), 128, 0, stream>>>(B, p); });
        launch_subst(0, li, B.RR, B.X, 0, p);
        launch_subst(1, lj, B.X, B.X, 0, p);
        launch_subst(2, lk, B.X, nullptr, 2, p);
      }
    } else {  // SSP-RK3 (solver3.rs:303-314)
      launch_prep();
      L3(P3_RESIDUAL, [&] { k3_residual<<<grid_of(B.nc, 256), 256, 0, stream>>>(B, 1, slot); });
      L3(P3_STAGE, [&] { k3_stage<<<grid_of(B.nc, 256), 256, 0, stream>>>(B, 1.f, 0.f, 1, 0); });
      launch_prep();
      L3(P3_RESIDUAL, [&] { k3_residual<<<grid_of(B.nc, 256), 256, 0, stream>>>(B, 0, -1); });
      L3(P3_STAGE, [&] { k3_stage<<<grid_of(B.nc, 256), 256, 0, stream>>>(B, 0.25f, 0.75f, 0, 0); });
      launch_prep();
      L3(P3_RESIDUAL, [&] { k3_residual<<<grid_of(B.nc, 256), 256, 0, stream>>>(B, 0, -1); });
      L3(P3_STAGE, [&] { k3_stage<<<grid_of(B.nc, 256), 256, 0, stream>>>(B, 2.f / 3.f, 1.f / 3.f, 0, 1); });
    }
  }
  // n iterations; residual: n x nb (iteration-major), may be null
  int run(long long n, double* residual) {
    const int nb = B.nb;
    std::vector<double> h;
    long long done = 0;
    double ms_total = 0.0;
    while (done < n) {
      int chunk = (int)std::min<long long>(n - done, slots);
      BK3_CUDA(cudaMemsetAsync(B.rsum, 0, (size_t)chunk * nb * sizeof(double), stream));
      BK3_CUDA(cudaEventRecord(ev0, stream));
      launch_chunk(chunk);
      BK3_CUDA(cudaGetLastError());
      BK3_CUDA(cudaEventRecord(ev1, stream));
      h.resize((size_t)chunk * nb);
      BK3_CUDA(cudaMemcpyAsync(h.data(), B.rsum, h.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
      BK3_CUDA(cudaStreamSynchronize(stream));
      float ms = 0.f;
      BK3_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
      ms_total += ms;
      if (residual)
        for (int k = 0; k < chunk; ++k)
          for (int b = 0; b < nb; ++b) residual[(done + k) * nb + b] = std::sqrt(h[(size_t)k * nb + b] / (double)n_active);
      done += chunk;
    }
    last_ms_per_iter = n > 0 ? ms_total / (double)n : 0.0;
    return 0;
  }
  // residual (and implicit time step with the current ramp) of the current state of every active case
  int eval_residual(std::vector<double>& dens) {
    BK3_CUDA(cudaMemsetAsync(B.rsum, 0, B.nb * sizeof(double), stream));
    launch_prep();
    k3_residual<<<grid_of(B.nc, 256), 256, 0, stream>>>(B, implicit() ? 2 : 1, 0);
    BK3_CUDA(cudaGetLastError());
    dens.resize(B.nb);
    BK3_CUDA(cudaMemcpyAsync(dens.data(), B.rsum, B.nb * sizeof(double), cudaMemcpyDeviceToHost, stream));
    BK3_CUDA(cudaStreamSynchronize(stream));
    for (auto& d : dens) d = std::sqrt(d / (double)n_active);
    return 0;
  }
  int read_residual(int b, double* res, double* dt) {
    std::vector<float> h(5 * B.nc), hd(B.nc);
    BK3_CUDA(copy_sync(stream, h.data(), B.R + (size_t)b * 5 * B.nc, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
    BK3_CUDA(copy_sync(stream, hd.data(), B.dt + (size_t)b * B.nc, hd.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (long long c = 0; c < B.nc; ++c) {
      if (res)
        for (int v = 0; v < 5; ++v) res[5 * c + v] = h[v * B.nc + c];
      if (dt) dt[c] = hd[c];
    }
    return 0;
  }
  // GpuSolver3::read_boundary_into (gpu/mod.rs:519-523): the states of case b at the cells the force integration reads
  // (the first fluid cell of every wall face and the one behind it) into u (ncell x 5, Cons3 order); other cells untouched
  int read_boundary(int b, double* u) {
    std::vector<long long> cells;
    for (int q = 0; q < nwall; ++q) {
      const double* w = &wall[(size_t)WALL3 * q];
      cells.push_back((long long)w[13]);
      if (w[14] >= 0) cells.push_back((long long)w[14]);
    }
    std::sort(cells.begin(), cells.end());
    cells.erase(std::unique(cells.begin(), cells.end()), cells.end());
    const int n = (int)cells.size();
    if (n == 0) return 0;
    long long* dc = nullptr;
    double* dv = nullptr;
    BK3_CUDA(cudaMallocAsync(&dc, n * sizeof(long long), stream));
    BK3_CUDA(cudaMallocAsync(&dv, 5 * (size_t)n * sizeof(double), stream));
    BK3_CUDA(cudaMemcpyAsync(dc, cells.data(), n * sizeof(long long), cudaMemcpyHostToDevice, stream));
    k3_gather<<<(n + 255) / 256, 256, 0, stream>>>(B, b, dc, n, dv);
    std::vector<double> hv(5 * (size_t)n);
    BK3_CUDA(cudaMemcpyAsync(hv.data(), dv, hv.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    BK3_CUDA(cudaFreeAsync(dc, stream));
    BK3_CUDA(cudaFreeAsync(dv, stream));
    BK3_CUDA(cudaStreamSynchronize(stream));
    for (int q = 0; q < n; ++q)
      for (int v = 0; v < 5; ++v) u[5 * cells[q] + v] = hv[5 * (size_t)q + v];
    return 0;
  }
  // (cn, ca, x_cp) of the 5 parts of every case (k3_forces_parts)
  int forces_parts(double x_max, double x_nose, std::vector<double>& out) {
    k3_forces_parts<<<B.nb, 128, 0, stream>>>(B, d_wall, nwall, x_max, x_nose, d_parts);
    BK3_CUDA(cudaGetLastError());
    out.resize(15 * (size_t)B.nb);
    BK3_CUDA(cudaMemcpyAsync(out.data(), d_parts, out.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    BK3_CUDA(cudaStreamSynchronize(stream));
    return 0;
  }
  int forces(double x_max, std::vector<double>& out) {
    k3_forces<<<B.nb, 256, 0, stream>>>(B, d_wall, nwall, x_max, d_forces);
    BK3_CUDA(cudaGetLastError());
    out.resize(3 * (size_t)B.nb);
    BK3_CUDA(cudaMemcpyAsync(out.data(), d_forces, out.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
    BK3_CUDA(cudaStreamSynchronize(stream));
    return 0;
  }
};

// run3.rs:253-330 StopRule3
struct StopRule3 {
  size_t skip = 20, nwin = 10, window = 500;
  double rel_tol = 0.002, rmax = 0.0, r = NAN;
  std::vector<double> hist;
  int reason = 0;  // 0 max iterations, 1 residual drop, 2 CN stationary, 5 non-finite
  bool check(size_t it, double res, bool sampled, double cn) {
    r = res;
    if (!std::isfinite(res)) return reason = 5, true;
    if (it >= skip) rmax = std::fmax(rmax, res);
    double drop = rmax > 0.0 ? std::log10(rmax / std::fmax(res, 1e-300)) : 0.0;
    if (drop >= 6.0) return reason = 1, true;
    if (sampled) {
      if (!std::isfinite(cn) || std::fabs(cn) > 1e3) return reason = 5, true;
      hist.push_back(cn);
      if (it + 1 >= std::max<size_t>(window, 1000) && hist.size() >= nwin) {
        const double* w = hist.data() + hist.size() - nwin;
        bool frozen = true;
        for (size_t q = 0; q < nwin; ++q) frozen = frozen && std::memcmp(&w[q], &w[0], sizeof(double)) == 0;
        if (drop < 1.0 && frozen) return reason = 5, true;
        double lo = INFINITY, hi = -INFINITY, sum = 0.0;
        for (size_t q = 0; q < nwin; ++q) lo = std::fmin(lo, w[q]), hi = std::fmax(hi, w[q]), sum += w[q];
        if (hi - lo < rel_tol * std::fabs(sum / (double)nwin)) return reason = 2, true;
      }
    }
    return false;
  }
};

}  // namespace bk3
