// Run control above the arena: the FP64 force pass (forces.cuh) used as the convergence monitor, the stop rules of
// crates/bowshock-core/src/engine/run.rs:105-170, the chunked run of engine/gpu.rs:86-169 (SYNC = 50 iterations per
// device->host exchange, the stop iteration found CPU-equivalently inside a chunk) and, for the batched arena, the
// per-case convergence masks. Each chunk of iterations is captured once into a CUDA graph and replayed.
#pragma once
#include <cstddef>
#include <functional>

#include "forces.cuh"
#include "host_arena.cuh"
#include "stream_copy.cuh"

namespace bk {

constexpr int SYNC = 50;  // engine/gpu.rs:24-25, numerics.rs:236 (MONITOR_EVERY)
constexpr size_t DRAG_REL_WINDOW = 500;

struct RunParams {
  long long max_iter = 10000, min_iter = 0;
  double drop_orders = 6.0;
  long long monitor_window = 2000;
  bool has_monitor_tol = false;
  double monitor_tol = 0;
  bool has_mean_window = false;
  long long mean_window = 0;
  bool has_drag_rel_tol = false;
  double drag_rel_tol = 0;
  int wake = 0;
  bool warm = false;
  double r_ref = -1;
};

struct Forces {
  double f[F_NF];
  double cd_total(int nseg) const {
    double fore = f[F_CD_NOSE];
    for (int k = 0; k < nseg; ++k) fore = fore + f[F_CD_AFT0 + k];
    return fore + f[F_CD_FRICTION] + f[F_CD_BASE];
  }
};

// run.rs:157-170
inline bool mean_stationary(const std::vector<std::pair<long long, double>>& hist, size_t k) {
  size_t from = 0;
  while (from < hist.size() && hist[from].first <= 2000) ++from;
  if (k == 0 || hist.size() - from < 2 * k) return false;
  const auto* w = &hist[hist.size() - 2 * k];
  double m0 = 0, m1 = 0;
  for (size_t t = 0; t < k; ++t) m0 += w[t].second;
  for (size_t t = k; t < 2 * k; ++t) m1 += w[t].second;
  m0 /= (double)k;
  m1 /= (double)k;
  double m = 0.5 * (m0 + m1), lo = INFINITY, hi = -INFINITY;
  for (size_t t = 0; t < 2 * k; ++t) lo = std::fmin(lo, w[t].second), hi = std::fmax(hi, w[t].second);
  double a = w[2 * k - 2].second - m, b = w[2 * k - 1].second - m;
  return std::fabs(m1 - m0) <= 2e-3 * std::fabs(m) && hi - lo <= 0.05 * std::fabs(m) && a * b < 0.0;
}

// run.rs:105-150; returns true with `why` set when iteration `it` (0-based) ends the run
inline bool stop_reason(const RunParams& n, bool viscous, long long it, double r, double reference, long long skip,
                        const std::vector<std::pair<long long, double>>& hist, int& why) {
  if (!std::isfinite(r) || (!hist.empty() && hist.back().first == it + 1 && (!std::isfinite(hist.back().second) || std::fabs(hist.back().second) > 1e3))) {
    why = 5;
    return true;
  }
  if (it + 1 < n.min_iter) return false;
  if (it > skip && reference / r >= std::pow(10.0, n.drop_orders)) {
    why = 1;
    return true;
  }
  if (n.has_drag_rel_tol) {
    size_t k = DRAG_REL_WINDOW / SYNC;
    if (viscous && !hist.empty() && hist.back().first == it + 1 && it + 1 >= (long long)DRAG_REL_WINDOW && reference / r >= 100.0 &&
        hist.size() >= k) {
      double lo = INFINITY, hi = -INFINITY, mean = 0;
      for (size_t t = hist.size() - k; t < hist.size(); ++t) lo = std::fmin(lo, hist[t].second), hi = std::fmax(hi, hist[t].second), mean += hist[t].second;
      mean /= (double)k;
      if (hi - lo < n.drag_rel_tol * std::fabs(mean)) {
        why = 2;
        return true;
      }
    }
  }
  if (n.has_monitor_tol && it % 500 == 499 && it + 1 >= 2 * n.monitor_window && reference / r >= 100.0) {
    size_t k = (size_t)(n.monitor_window / SYNC);
    if (hist.size() >= k) {
      double lo = INFINITY, hi = -INFINITY;
      for (size_t t = hist.size() - k; t < hist.size(); ++t) lo = std::fmin(lo, hist[t].second), hi = std::fmax(hi, hist[t].second);
      if (hi - lo < n.monitor_tol) {
        why = (!viscous && n.wake == 1) ? 3 : 2;
        return true;
      }
    }
  }
  if (viscous && n.has_mean_window && !hist.empty() && hist.back().first == it + 1 && mean_stationary(hist, (size_t)(n.mean_window / SYNC))) {
    why = 4;
    return true;
  }
  return false;
}

// per-case run state of the chunked runner
struct CaseRun {
  RunParams p;
  int nseg = 0;
  long long it = 0, skip = 20;
  double rmax = 0;
  std::vector<double> residual;
  std::vector<std::pair<long long, double>> hist;
  bool done = false;
  int reason = 0;
  double last_monitor = NAN;
  double cd_window = NAN;  // set by the device run control when it stops a case on the mean-stationary rule
};

struct ForcePass {
  double *nx = nullptr, *nr = nullptr, *xc = nullptr, *rc = nullptr, *out = nullptr;
  long long* node_off = nullptr;
  BodyDev* bodies = nullptr;
  std::vector<BodyDev> hb;
  int nc = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double last_ms = 0.0;  // device time of the last pass (kernel + read-back)
  ~ForcePass() {
    for (void* p : {(void*)nx, (void*)nr, (void*)xc, (void*)rc, (void*)out, (void*)node_off, (void*)bodies})
      if (p) cudaFree(p);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
  int setup(ArenaHost& ar) {
    std::string& err = ar.err;
    nc = (int)ar.cases.size();
    long long nn = 0;
    std::vector<long long> off(nc);
    for (int k = 0; k < nc; ++k) off[k] = nn, nn += (long long)(ar.cases[k].ni + 1) * (ar.cases[k].nj + 1);
    int rc_ = 0;
    if ((rc_ = dalloc(&nx, nn, err)) || (rc_ = dalloc(&nr, nn, err)) || (rc_ = dalloc(&xc, ar.ncell, err)) || (rc_ = dalloc(&rc, ar.ncell, err)) ||
        (rc_ = dalloc(&out, (size_t)nc * F_NF, err)) || (rc_ = dalloc(&node_off, nc, err)) || (rc_ = dalloc(&bodies, nc, err)))
      return rc_;
    for (int k = 0; k < nc; ++k) {
      const HostCase& h = ar.cases[k];
      BK_CUDA(copy_sync(ar.stream, nx + off[k], h.x.data(), h.x.size() * sizeof(double), cudaMemcpyHostToDevice));
      BK_CUDA(copy_sync(ar.stream, nr + off[k], h.r.data(), h.r.size() * sizeof(double), cudaMemcpyHostToDevice));
      BK_CUDA(copy_sync(ar.stream, xc + ar.desc[k].cell_off, h.xc.data(), h.xc.size() * sizeof(double), cudaMemcpyHostToDevice));
      BK_CUDA(copy_sync(ar.stream, rc + ar.desc[k].cell_off, h.rc.data(), h.rc.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    BK_CUDA(copy_sync(ar.stream, node_off, off.data(), nc * sizeof(long long), cudaMemcpyHostToDevice));
    hb.assign(nc, BodyDev{});
    return 0;
  }
  int set_body(ArenaHost& ar, int k, const bowshock_body* b) {
    std::string& err = ar.err;
    BodyDev d{};
    mesh::Body mb;
    mb.nose = b->nose_kind;
    mb.fineness = b->fineness;
    mb.half_angle = b->half_angle;
    mb.param = b->param;
    for (int s = 0; s < b->nseg && s < MAX_SEG; ++s) mb.seg_len.push_back(b->seg_length[s]), mb.seg_slope.push_back(b->seg_slope[s]);
    d.nose_length = mb.nose_length();
    d.rb2 = 0.25;
    d.x_base = mb.x_base();
    d.nseg = (int)mb.seg_len.size();
    for (int s = 0; s <= d.nseg; ++s) d.stations[s] = mb.station(s).first;
    d.has_body = 1;
    hb[k] = d;
    BK_CUDA(copy_sync(ar.stream, bodies + k, &d, sizeof(BodyDev), cudaMemcpyHostToDevice));
    return 0;
  }
  int run(ArenaHost& ar, std::vector<Forces>& res) {
    std::string& err = ar.err;
    if (!e0) {
      BK_CUDA(cudaEventCreate(&e0));
      BK_CUDA(cudaEventCreate(&e1));
    }
    BK_CUDA(cudaEventRecord(e0, ar.stream));
    k_forces<<<nc, 256, 0, ar.stream>>>(ar.A, bodies, nx, nr, node_off, xc, rc, out);
    BK_CUDA(cudaGetLastError());
    std::vector<double> h((size_t)nc * F_NF);
    BK_CUDA(cudaMemcpyAsync(h.data(), out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ar.stream));
    BK_CUDA(cudaEventRecord(e1, ar.stream));
    BK_CUDA(cudaStreamSynchronize(ar.stream));
    float ms = 0.f;
    BK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    last_ms = ms;
    res.resize(nc);
    for (int k = 0; k < nc; ++k) std::memcpy(res[k].f, &h[(size_t)k * F_NF], F_NF * sizeof(double));
    return 0;
  }
};

// run.rs:174-185: total CD of a viscous case, else the nose CD (sting) or the area-mean base Cp (base wake)
inline double monitor_of(const HostCase& h, const RunParams& p, const Forces& f, int nseg) {
  if (h.viscous) return f.cd_total(nseg);
  return p.wake == 0 ? f.f[F_CD_NOSE] : f.f[F_CP_BASE];
}

inline void fill_point(const CaseRun& cr, const Forces& f, bowshock_point_result* o) {
  std::memset(o, 0, sizeof(*o));
  o->iters = (uint64_t)cr.residual.size();
  o->residual_peak = cr.rmax;
  double last = cr.residual.empty() ? cr.rmax : cr.residual.back();
  o->drop_orders = (cr.rmax > 0 && last > 0) ? std::log10(cr.rmax / last) : 0.0;
  o->stop_reason = cr.reason;
  o->forces.cd_nose = f.f[F_CD_NOSE];
  o->forces.cd_nose_cell = f.f[F_CD_NOSE_CELL];
  o->forces.cd_base = f.f[F_CD_BASE];
  o->forces.cp_base = f.f[F_CP_BASE];
  o->forces.cp_base_cell = f.f[F_CP_BASE_CELL];
  o->forces.cd_friction = f.f[F_CD_FRICTION];
  o->forces.y_plus_max = f.f[F_YPLUS];
  for (int k = 0; k < MAX_SEG; ++k) o->forces.cd_aft[k] = k < cr.nseg ? f.f[F_CD_AFT0 + k] : 0.0;
  o->forces.cd_total = f.cd_total(cr.nseg);
  o->last_monitor = cr.last_monitor;
  o->cd_window = o->forces.cd_total;
  // mean stationary: the mean of the last window the rule compared (run.rs:157-172); its 120 samples lie on the
  // limit cycle, so the value does not depend on the 50-iteration chunk at which the rule first holds
  if (cr.reason == 4 && !std::isnan(cr.cd_window)) {
    o->cd_window = cr.cd_window;
  } else if (cr.reason == 4 && cr.p.mean_window >= SYNC) {
    size_t k = (size_t)(cr.p.mean_window / SYNC);
    if (cr.hist.size() >= k) {
      double m = 0.0;
      for (size_t t = cr.hist.size() - k; t < cr.hist.size(); ++t) m += cr.hist[t].second;
      o->cd_window = m / (double)k;
    }
  }
}

// ==================================================================================== GPU-resident run control
// The stop rules above evaluated on the device after every chunk (no counterpart in the reference, whose rules run on
// the host, engine/gpu.rs:123-164): one thread per case walks the chunk's iterations with the density residuals of the
// arena's residual sums and the monitor of the FP64 force pass, in the same order and arithmetic as stop_reason (the
// drop threshold 10^drop_orders is computed on the host, so no device pow enters a decision), and keeps the monitor
// samples in a ring of RUN_RING entries. The host reads back only each case's status.
constexpr int RUN_RING = 256;  // monitor samples kept: twice a mean window of 6,400 iterations
struct RunDev {
  long long max_iter, min_iter, monitor_window, mean_window;
  double drop_thresh, monitor_tol, drag_rel_tol, r_ref, n_active;
  int has_monitor_tol, has_mean_window, has_drag_rel_tol, wake, viscous, nseg, cd_of_wake_base;
  // state
  long long it, skip;
  double rmax, last_r, last_monitor, cd_window;
  int done, reason, nh, n_after;  // samples so far, samples past iteration 2000
  long long hit[RUN_RING];
  double hv[RUN_RING];
};

__device__ __forceinline__ double ring(const RunDev& d, int q) { return d.hv[q % RUN_RING]; }

// run.rs:157-170 on the last 2k samples of the ring
__device__ bool mean_stationary_dev(const RunDev& d, int k) {
  if (k == 0 || d.n_after < 2 * k) return false;
  const int b = d.nh - 2 * k;
  double m0 = 0, m1 = 0;
  for (int t = 0; t < k; ++t) m0 += ring(d, b + t);
  for (int t = k; t < 2 * k; ++t) m1 += ring(d, b + t);
  m0 /= (double)k;
  m1 /= (double)k;
  double m = 0.5 * (m0 + m1), lo = INFINITY, hi = -INFINITY;
  for (int t = 0; t < 2 * k; ++t) lo = fmin(lo, ring(d, b + t)), hi = fmax(hi, ring(d, b + t));
  double a = ring(d, b + 2 * k - 2) - m, c = ring(d, b + 2 * k - 1) - m;
  return fabs(m1 - m0) <= 2e-3 * fabs(m) && hi - lo <= 0.05 * fabs(m) && a * c < 0.0;
}

// run.rs:105-150, the device restatement of stop_reason
__device__ bool stop_reason_dev(const RunDev& d, long long it, double r, double reference, int& why) {
  const bool sampled_now = d.nh > 0 && d.hit[(d.nh - 1) % RUN_RING] == it + 1;
  if (!isfinite(r) || (sampled_now && (!isfinite(ring(d, d.nh - 1)) || fabs(ring(d, d.nh - 1)) > 1e3))) {
    why = 5;
    return true;
  }
  if (it + 1 < d.min_iter) return false;
  if (it > d.skip && reference / r >= d.drop_thresh) {
    why = 1;
    return true;
  }
  if (d.has_drag_rel_tol) {
    const int k = (int)(DRAG_REL_WINDOW / SYNC);
    if (d.viscous && sampled_now && it + 1 >= (long long)DRAG_REL_WINDOW && reference / r >= 100.0 && d.nh >= k) {
      double lo = INFINITY, hi = -INFINITY, mean = 0;
      for (int t = d.nh - k; t < d.nh; ++t) lo = fmin(lo, ring(d, t)), hi = fmax(hi, ring(d, t)), mean += ring(d, t);
      mean /= (double)k;
      if (hi - lo < d.drag_rel_tol * fabs(mean)) {
        why = 2;
        return true;
      }
    }
  }
  if (d.has_monitor_tol && it % 500 == 499 && it + 1 >= 2 * d.monitor_window && reference / r >= 100.0) {
    const int k = (int)(d.monitor_window / SYNC);
    if (d.nh >= k) {
      double lo = INFINITY, hi = -INFINITY;
      for (int t = d.nh - k; t < d.nh; ++t) lo = fmin(lo, ring(d, t)), hi = fmax(hi, ring(d, t));
      if (hi - lo < d.monitor_tol) {
        why = (!d.viscous && d.wake == 1) ? 3 : 2;
        return true;
      }
    }
  }
  if (d.viscous && d.has_mean_window && sampled_now && mean_stationary_dev(d, (int)(d.mean_window / SYNC))) {
    why = 4;
    return true;
  }
  return false;
}

// One chunk of `n` iterations for every case still running: residuals from rsum [slot][case], the monitor from the force
// pass output (run.rs:174-185: the total CD of a viscous case, else the nose CD of a sting or the base Cp of a base wake).
__global__ void k_run_control(RunDev* runs, int nruns, const double* __restrict__ rsum, int ncases, const double* __restrict__ forces, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nruns) return;
  RunDev& d = runs[k];
  if (d.done) return;
  const double* f = forces + (size_t)k * F_NF;
  double mon;
  if (d.viscous) {
    double fore = f[F_CD_NOSE];
    for (int s = 0; s < d.nseg; ++s) fore = fore + f[F_CD_AFT0 + s];
    mon = fore + f[F_CD_FRICTION] + f[F_CD_BASE];
  } else {
    mon = d.wake == 0 ? f[F_CD_NOSE] : f[F_CP_BASE];
  }
  const bool sample = d.wake == 1 || d.has_monitor_tol || d.has_drag_rel_tol;
  for (int t = 0; t < n && !d.done; ++t) {
    const long long it = d.it;
    const double r = sqrt(rsum[(size_t)t * ncases + k] / d.n_active);
    d.last_r = r;
    if (it >= d.skip) d.rmax = fmax(d.rmax, r);
    if (sample && it % SYNC == SYNC - 1) {
      d.hit[d.nh % RUN_RING] = it + 1;
      d.hv[d.nh % RUN_RING] = mon;
      d.nh += 1;
      if (it + 1 > 2000) d.n_after += 1;
      d.last_monitor = mon;
    }
    int why = 0;
    if (stop_reason_dev(d, it, r, d.r_ref >= 0 ? d.r_ref : d.rmax, why)) {
      d.done = 1;
      d.reason = why;
      if (why == 4 && d.mean_window >= SYNC) {  // the mean of the last window the rule compared
        const int kk = (int)(d.mean_window / SYNC);
        double m = 0.0;
        for (int q = d.nh - kk; q < d.nh; ++q) m += ring(d, q);
        d.cd_window = m / (double)kk;
      }
    } else if (it + 1 >= d.max_iter) {
      d.done = 1;
      d.reason = 0;
    }
    d.it += 1;
  }
}

// Whether the stop rules of these runs fit the device ring (their windows at most RUN_RING / 2 mean samples)
inline bool device_control_fits(const std::vector<CaseRun>& runs) {
  for (const CaseRun& cr : runs) {
    if (cr.p.has_mean_window && 2 * (cr.p.mean_window / SYNC) > RUN_RING) return false;
    if (cr.p.has_monitor_tol && cr.p.monitor_window / SYNC > RUN_RING) return false;
  }
  return true;
}

// Cold (or warm) start of case k for a run: free stream, turbulence re-initialised, counters reset (run.rs:44-63).
inline int start_case(ArenaHost& ar, int k, const RunParams& p, long long first_order_iters) {
  int rc = 0;
  if (!p.warm) {
    if ((rc = ar.reset_case(k))) return rc;
    if (ar.cases[k].viscous && ar.cases[k].turbulence == 1 && (rc = ar.turb_init(k))) return rc;
  }
  if ((rc = ar.set_counter(ar.d_iter, k, p.warm ? (int)first_order_iters : 0))) return rc;
  return ar.set_counter(ar.d_ramp, k, 0);
}

// Iterate every active case of the arena to its stop rule in chunks of SYNC iterations.
// `device_ms` (optional) receives the device time of the iterations and force passes (CUDA events around each).
inline int solve_arena(ArenaHost& ar, ForcePass& fp, std::vector<CaseRun>& runs,
                       const std::function<bool(int, long long, double, double)>& progress, double* device_ms = nullptr) {
  double dev_ms = 0.0;
  // runs: one per arena case, or, for a single case with a multigrid hierarchy, one for the fine level (the coarse
  // levels, cases 1.., follow its activity)
  const int nc = (int)ar.cases.size(), nr = (int)runs.size();
  std::vector<int> act(nc);
  auto sync_levels = [&] {
    for (int k = nr; k < nc; ++k) act[k] = act[0];
  };
  for (int k = 0; k < nr; ++k) act[k] = runs[k].done ? 0 : 1;
  sync_levels();
  int rc = ar.set_active(act.data());
  if (rc) return rc;
  std::vector<double> res((size_t)SYNC * nc);
  std::vector<Forces> f;
  // the stop rules on the device (the host then reads each case's status) unless switched off or beyond the ring
  const bool dev = ar.device_run_control && device_control_fits(runs);
  std::vector<RunDev> hr(dev ? nr : 0);
  RunDev* d_runs = nullptr;
  struct Free {
    RunDev*& p;
    ~Free() {
      if (p) cudaFree(p);
    }
  } free_runs{d_runs};
  const size_t head = offsetof(RunDev, hit);  // the parameters and the status, without the monitor ring
  if (dev) {
    for (int k = 0; k < nr; ++k) {
      const CaseRun& cr = runs[k];
      RunDev& d = hr[k];
      std::memset(&d, 0, sizeof(RunDev));
      d.max_iter = cr.p.max_iter, d.min_iter = cr.p.min_iter, d.monitor_window = cr.p.monitor_window, d.mean_window = cr.p.mean_window;
      d.drop_thresh = std::pow(10.0, cr.p.drop_orders), d.monitor_tol = cr.p.monitor_tol, d.drag_rel_tol = cr.p.drag_rel_tol;
      d.r_ref = cr.p.r_ref, d.n_active = (double)ar.desc[k].n_active;
      d.has_monitor_tol = cr.p.has_monitor_tol, d.has_mean_window = cr.p.has_mean_window, d.has_drag_rel_tol = cr.p.has_drag_rel_tol;
      d.wake = cr.p.wake, d.viscous = ar.cases[k].viscous ? 1 : 0, d.nseg = cr.nseg;
      d.it = cr.it, d.skip = cr.skip, d.rmax = cr.rmax, d.done = cr.done ? 1 : 0, d.last_monitor = NAN, d.cd_window = NAN;
    }
    std::string& err = ar.err;
    BK_CUDA(cudaMalloc(&d_runs, (size_t)nr * sizeof(RunDev)));
    BK_CUDA(copy_sync(ar.stream, d_runs, hr.data(), (size_t)nr * sizeof(RunDev), cudaMemcpyHostToDevice));
  }
  while (true) {
    int left = 0;
    for (int k = 0; k < nr; ++k) left += !runs[k].done;
    if (!left) break;
    if ((rc = ar.run(SYNC, res.data()))) return rc;
    if ((rc = fp.run(ar, f))) return rc;
    dev_ms += ar.last_ms_per_iter * SYNC + fp.last_ms;
    if (device_ms) *device_ms = dev_ms;
    if (dev) {
      std::string& err = ar.err;
      k_run_control<<<(nr + 127) / 128, 128, 0, ar.stream>>>(d_runs, nr, ar.A.rsum, nc, fp.out, SYNC);
      BK_CUDA(cudaGetLastError());
      BK_CUDA(cudaMemcpy2DAsync(hr.data(), sizeof(RunDev), d_runs, sizeof(RunDev), head, nr, cudaMemcpyDeviceToHost, ar.stream));
      BK_CUDA(cudaStreamSynchronize(ar.stream));
    }
    bool mask_changed = false;
    for (int k = 0; k < nr; ++k) {
      CaseRun& cr = runs[k];
      if (cr.done) continue;
      double mon = monitor_of(ar.cases[k], cr.p, f[k], cr.nseg);
      if (dev) {  // the device's decision; the host keeps the residual history
        const RunDev& d = hr[k];
        for (long long t = 0; cr.it + t < d.it; ++t) cr.residual.push_back(res[(size_t)t * nc + k]);
        cr.it = d.it, cr.rmax = d.rmax, cr.last_monitor = d.last_monitor;
        if (d.done) cr.done = true, cr.reason = d.reason, cr.cd_window = d.cd_window;
      } else {
        bool sample = cr.p.wake == 1 || cr.p.has_monitor_tol || cr.p.has_drag_rel_tol;
        for (int t = 0; t < SYNC && !cr.done; ++t) {
          long long it = cr.it;
          double r = res[(size_t)t * nc + k];
          cr.residual.push_back(r);
          if (it >= cr.skip) cr.rmax = std::fmax(cr.rmax, r);
          if (sample && it % SYNC == SYNC - 1) cr.hist.emplace_back(it + 1, mon), cr.last_monitor = mon;
          int why = 0;
          if (stop_reason(cr.p, ar.cases[k].viscous, it, r, cr.p.r_ref >= 0 ? cr.p.r_ref : cr.rmax, cr.skip, cr.hist, why)) {
            cr.done = true;
            cr.reason = why;
          } else if (it + 1 >= cr.p.max_iter) {
            cr.done = true;
            cr.reason = 0;
          }
          cr.it += 1;
        }
      }
      if (!cr.done && progress && !progress(k, cr.it, cr.residual.back(), mon)) {
        cr.done = true;
        cr.reason = 6;
        if (dev) {  // the device stops iterating this run too
          std::string& err = ar.err;
          const int one = 1;
          BK_CUDA(copy_sync(ar.stream, reinterpret_cast<char*>(d_runs + k) + offsetof(RunDev, done), &one, sizeof(int), cudaMemcpyHostToDevice));
        }
      }
      if (cr.done) act[k] = 0, mask_changed = true;
    }
    sync_levels();
    if (mask_changed && (rc = ar.set_active(act.data()))) return rc;
  }
  return 0;
}

}  // namespace bk
