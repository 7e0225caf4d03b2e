// C ABI of the single-case solver (include/bowshock_b200.h): a GpuSolver (crates/bowshock-cfd/src/gpu/mod.rs:233-414)
// backed by a case arena of one. Unity build: the kernels and the host arena are compiled into this translation unit.
#include <cstdio>
#include <exception>
#include <mutex>

#include "../../include/bowshock_b200.h"
#include "fv_kernels.cu"
#include "turbulence.cuh"
#include "multigrid.cuh"
#include "host_arena.cuh"
#include "mesher.cuh"
#include "host3.cuh"
#include "mesher_dev.h"

using namespace bk;

struct bowshock_solver {
  ArenaHost ar;
  std::string last_error;
};

static int fail(bowshock_solver* s, int code, const std::string& m) {
  if (s) s->last_error = m;
  return code;
}
static int from_arena(bowshock_solver* s, int rc) {
  if (rc) s->last_error = s->ar.err;
  return rc;
}

static bool valid_config(const bowshock_config* c, std::string& m) {
  if (!c) return m = "null config", false;
  if (!(c->cfl > 0)) return m = "cfl must be positive", false;
  if (c->limiter < 0 || c->limiter > 3) return m = "unknown limiter", false;
  for (int k = 0; k < 4; ++k)
    if (c->bc[k] < 0 || c->bc[k] > 4) return m = "unknown boundary condition", false;
  if (!(c->freestream[0] > 0 && c->freestream[3] > 0)) return m = "free stream needs rho > 0 and p > 0", false;
  return true;
}
static void apply_config(HostCase& h, const bowshock_config* c) {
  h.cfl = c->cfl;
  h.limiter = c->limiter;
  for (int k = 0; k < 4; ++k) {
    h.fs[k] = c->freestream[k];
    h.bc[k] = c->bc[k];
  }
  h.first_order_iters = (long long)c->first_order_iters;
}

extern "C" {

int bowshock_solver_create(uint64_t ni, uint64_t nj, const double* x, const double* r, const bowshock_config* cfg, int device,
                           bowshock_solver** out) {
  if (!out) return BOWSHOCK_INVALID;
  *out = nullptr;
  std::string m;
  if (ni < 4 || nj < 2 || !x || !r) return BOWSHOCK_INVALID;
  if (!valid_config(cfg, m)) return BOWSHOCK_INVALID;
  bowshock_solver* s = new (std::nothrow) bowshock_solver();
  if (!s) return BOWSHOCK_INVALID;
  try {
    HostCase h;
    h.ni = (int)ni;
    h.nj = (int)nj;
    h.x.assign(x, x + (ni + 1) * (nj + 1));
    h.r.assign(r, r + (ni + 1) * (nj + 1));
    apply_config(h, cfg);
    std::string e;
    if (!compute_metrics(h, e)) {
      delete s;
      return BOWSHOCK_INVALID;
    }
    s->ar.device = device;
    s->ar.cases.push_back(std::move(h));
    int rc = s->ar.setup();
    if (rc) {
      delete s;
      return BOWSHOCK_CUDA_ERROR;
    }
  } catch (const std::exception& e) {
    delete s;
    return BOWSHOCK_INVALID;
  }
  *out = s;
  return BOWSHOCK_OK;
}

static void solver_forces_drop(bowshock_solver* s);
void bowshock_solver_destroy(bowshock_solver* s) {
  if (s) solver_forces_drop(s);
  delete s;
}

const char* bowshock_solver_last_error(const bowshock_solver* s) { return s ? s->last_error.c_str() : "null handle"; }

int bowshock_solver_dims(const bowshock_solver* s, uint64_t* ni, uint64_t* nj) {
  if (!s || !ni || !nj) return BOWSHOCK_INVALID;
  *ni = s->ar.cases[0].ni;
  *nj = s->ar.cases[0].nj;
  return BOWSHOCK_OK;
}

int bowshock_solver_set_config(bowshock_solver* s, const bowshock_config* cfg) {
  if (!s) return BOWSHOCK_INVALID;
  std::string m;
  if (!valid_config(cfg, m)) return fail(s, BOWSHOCK_INVALID, m);
  HostCase& h = s->ar.cases[0];
  if (h.viscous && (cfg->bc[0] != h.bc[0] || cfg->bc[1] != h.bc[1] || cfg->bc[2] != h.bc[2] || cfg->bc[3] != h.bc[3]))
    return fail(s, BOWSHOCK_UNSUPPORTED, "the boundary conditions of a viscous run (no-slip walls, wall distance) are fixed by set_viscous");
  apply_config(h, cfg);
  return from_arena(s, s->ar.upload_desc());
}

int bowshock_solver_set_low_mach(bowshock_solver* s, int on) {
  if (!s) return BOWSHOCK_INVALID;
  s->ar.cases[0].low_mach = on ? 1 : 0;
  return from_arena(s, s->ar.upload_desc());
}

int bowshock_solver_set_block(bowshock_solver* s, const bowshock_block* b) {
  if (!s) return BOWSHOCK_INVALID;
  HostCase& h = s->ar.cases[0];
  if (h.viscous) return fail(s, BOWSHOCK_UNSUPPORTED, "the solid block must be declared before the viscous terms");
  if (b) {
    // solver.rs:309-317
    bool ok = b->i_end >= 1 && b->i_end + 2 <= (uint64_t)h.ni && b->j_end >= 2 && b->j_end + 2 <= (uint64_t)h.nj && b->j_end > b->j_sting &&
              (b->j_sting == 0 || b->j_sting >= 2);
    if (!ok) return fail(s, BOWSHOCK_INVALID, "block out of range");
    h.has_block = true;
    h.i_end = (long long)b->i_end;
    h.j_end = (long long)b->j_end;
    h.j_sting = (long long)b->j_sting;
  } else {
    h.has_block = false;
    h.has_nozzle = false;
  }
  h.dwall.clear();
  return from_arena(s, s->ar.upload_desc());
}

int bowshock_solver_set_nozzle(bowshock_solver* s, const bowshock_nozzle* n) {
  if (!s) return BOWSHOCK_INVALID;
  HostCase& h = s->ar.cases[0];
  if (h.viscous || (n && !h.has_block)) return fail(s, BOWSHOCK_UNSUPPORTED, "set_nozzle must follow set_block and precede set_viscous");
  if (n) {
    // solver.rs:335-338
    double c = std::sqrt(1.4 * n->state[3] / n->state[0]);
    if (!(h.j_sting == 0 && n->j_end >= 2 && (long long)n->j_end + 2 <= h.j_end && n->j_end % 2 == 0))
      return fail(s, BOWSHOCK_INVALID, "nozzle out of range");
    if (!(n->state[0] > 0 && n->state[3] > 0 && n->state[1] >= c)) return fail(s, BOWSHOCK_INVALID, "nozzle exit must be supersonic");
    h.has_nozzle = true;
    h.nz_j_end = (long long)n->j_end;
    for (int k = 0; k < 4; ++k) h.nz_state[k] = n->state[k];
    h.nz_turb[0] = n->turb[0];
    h.nz_turb[1] = n->turb[1];
  } else {
    h.has_nozzle = false;
  }
  h.dwall.clear();
  return from_arena(s, s->ar.upload_desc());
}

// Rebuild the arena of a solver with its FAS hierarchy (multigrid.rs:29-64): the fine grid, then grids with every second
// node line removed while both dimensions are even and the coarse one stays >= 8, and the block halves; coarse levels are
// first order with the fine level's BCs, free stream and CFL. nlev = 1 removes the hierarchy. The state is kept.
static int rebuild_levels(bowshock_solver* s, int nlev) {
  ArenaHost& ar = s->ar;
  HostCase fine = ar.cases[0];
  std::vector<double> u((size_t)fine.ni * fine.nj * 4);
  int rc = ar.get_state(0, u.data());
  if (rc) return from_arena(s, rc);
  std::vector<HostCase> lv{fine};
  lv[0].level = 0;
  lv[0].fine_case = lv[0].coarse_case = -1;
  while ((int)lv.size() < nlev) {
    const HostCase& f = lv.back();
    if (f.ni % 2 || f.nj % 2 || f.ni / 2 < 8 || f.nj / 2 < 8) break;
    if (f.has_block && (f.i_end % 2 || f.j_end % 2 || f.j_sting % 2)) break;
    HostCase c = f;
    c.ni = f.ni / 2;
    c.nj = f.nj / 2;
    c.x.clear();
    c.r.clear();
    for (int j = 0; j <= c.nj; ++j)
      for (int i = 0; i <= c.ni; ++i) {
        size_t k = (size_t)2 * j * (f.ni + 1) + 2 * i;
        c.x.push_back(f.x[k]);
        c.r.push_back(f.r[k]);
      }
    std::string e;
    if (!compute_metrics(c, e)) return fail(s, BOWSHOCK_INVALID, e);
    if (f.has_block) c.i_end = f.i_end / 2, c.j_end = f.j_end / 2, c.j_sting = f.j_sting / 2;
    c.limiter = 0;
    c.first_order_iters = 0;
    c.level = (int)lv.size();
    c.fine_case = (int)lv.size() - 1;
    c.coarse_case = -1;
    lv.back().coarse_case = (int)lv.size();
    lv.push_back(std::move(c));
  }
  ar.cases = std::move(lv);
  ar.mg_levels = (int)ar.cases.size();
  if ((rc = ar.setup())) return from_arena(s, rc);
  return from_arena(s, ar.set_state(0, u.data()));
}

int bowshock_solver_set_scheme(bowshock_solver* s, const bowshock_scheme* sc) {
  if (!s || !sc) return BOWSHOCK_INVALID;
  if (sc->kind != BOWSHOCK_SCHEME_EXPLICIT && sc->kind != BOWSHOCK_SCHEME_SMOOTHED && sc->kind != BOWSHOCK_SCHEME_IMPLICIT &&
      sc->kind != BOWSHOCK_SCHEME_MULTIGRID)
    return fail(s, BOWSHOCK_UNSUPPORTED, "unknown scheme");
  if (!std::isfinite(sc->cfl_star) || !std::isfinite(sc->mg_cfl_star)) return fail(s, BOWSHOCK_INVALID, "cfl_star must be finite");
  if (sc->kind == BOWSHOCK_SCHEME_MULTIGRID && (!(sc->mg_relax >= 0.0 && sc->mg_relax <= 1.0) || !(sc->mg_cfl_scale >= 0.0 && sc->mg_cfl_scale <= 1.0)))
    return fail(s, BOWSHOCK_INVALID, "mg_relax and mg_cfl_scale must lie in [0, 1] (0: the default 1)");
  const bool implicit_params = sc->kind == BOWSHOCK_SCHEME_IMPLICIT || (sc->kind == BOWSHOCK_SCHEME_MULTIGRID && sc->mg_implicit);
  if (implicit_params && (sc->sub_iters < 1 || sc->sub_iters > 16 || !(sc->cfl0 > 0) || !(sc->cfl_max > 0)))
    return fail(s, BOWSHOCK_INVALID, "implicit parameters out of range");
  if (sc->kind == BOWSHOCK_SCHEME_MULTIGRID) {
    // multigrid.rs:29-31: refused with viscous terms and with a nozzle
    if (s->ar.cases[0].viscous) return fail(s, BOWSHOCK_UNSUPPORTED, "viscous terms need Scheme::Explicit or Scheme::Implicit");
    if (s->ar.cases[0].has_nozzle) return fail(s, BOWSHOCK_UNSUPPORTED, "nozzle needs Scheme::Explicit or Scheme::Implicit");
    if (sc->mg_levels < 1 || sc->mg_levels > 16 || sc->mg_coarsest > 1000 || sc->mg_pre > 100 || sc->mg_post > 100 || sc->mg_gamma > 4)
      return fail(s, BOWSHOCK_INVALID, "multigrid parameters out of range");
  }
  int want_levels = sc->kind == BOWSHOCK_SCHEME_MULTIGRID ? (int)sc->mg_levels : 1;
  if (want_levels != s->ar.mg_levels || (int)s->ar.cases.size() != want_levels) {
    s->ar.cases[0].scheme = sc->kind;
    int rc = rebuild_levels(s, want_levels);
    if (rc) return rc;
  }
  ArenaHost& ar = s->ar;
  ar.mg_pre = (int)sc->mg_pre;
  ar.mg_post = (int)sc->mg_post;
  ar.mg_gamma = (int)sc->mg_gamma;
  ar.mg_coarsest = (int)sc->mg_coarsest;
  ar.mg_implicit = sc->kind == BOWSHOCK_SCHEME_MULTIGRID && sc->mg_implicit != 0;
  ar.mg_relax = sc->kind == BOWSHOCK_SCHEME_MULTIGRID && sc->mg_relax > 0.0 ? sc->mg_relax : 1.0;
  const double cfl_scale = sc->kind == BOWSHOCK_SCHEME_MULTIGRID && sc->mg_cfl_scale > 0.0 ? sc->mg_cfl_scale : 1.0;
  for (auto& hc : ar.cases) {
    if (implicit_params) {  // every level smooths with the same implicit parameters (each with its own CFL ramp), the
                            // CFL numbers of level l scaled by mg_cfl_scale^l
      const double f = std::pow(cfl_scale, (double)hc.level);
      hc.cfl0 = sc->cfl0 * f, hc.cfl_max = sc->cfl_max * f, hc.growth = sc->growth, hc.dt_mode = sc->dt_mode, hc.lines = sc->lines;
      hc.implicit_bc = sc->implicit_bc, hc.sub_iters = (int)sc->sub_iters, hc.roe = sc->roe, hc.eps_fix = sc->eps_fix;
    }
    hc.scheme = sc->kind;
    // Scheme::Smoothed(Irs) smooths the SSP-RK3 stages; the multigrid smoother on every level with MgParams::irs
    hc.cfl_star = sc->kind == BOWSHOCK_SCHEME_SMOOTHED ? sc->cfl_star : sc->kind == BOWSHOCK_SCHEME_MULTIGRID ? sc->mg_cfl_star : 0.0;
  }
  HostCase& h = s->ar.cases[0];
  h.scheme = sc->kind;
  h.cfl0 = sc->cfl0;
  h.cfl_max = sc->cfl_max;
  h.growth = sc->growth;
  h.dt_mode = sc->dt_mode;
  h.lines = sc->lines;
  h.implicit_bc = sc->implicit_bc;
  h.sub_iters = (int)sc->sub_iters;
  h.roe = sc->roe;
  h.eps_fix = sc->eps_fix;
  int rc = s->ar.upload_desc();
  if (rc) return from_arena(s, rc);
  for (int k = 0; k < (int)s->ar.cases.size(); ++k)
    if ((rc = s->ar.set_counter(s->ar.d_ramp, k, 0))) return from_arena(s, rc);
  return BOWSHOCK_OK;
}

int bowshock_solver_set_viscous(bowshock_solver* s, const bowshock_viscous* v) {
  if (!s) return BOWSHOCK_INVALID;
  HostCase& h = s->ar.cases[0];
  if (v) {
    if (!(v->roughness >= 0.0 && std::isfinite(v->roughness))) return fail(s, BOWSHOCK_INVALID, "roughness must be finite and >= 0");
    if (!(v->re_c > 0 && v->sutherland > 0)) return fail(s, BOWSHOCK_INVALID, "re_c and sutherland must be positive");
    if (v->turbulence == BOWSHOCK_TURB_SST && h.scheme != BOWSHOCK_SCHEME_IMPLICIT)
      return fail(s, BOWSHOCK_UNSUPPORTED, "the SST model runs with the implicit scheme on this backend");
    h.viscous = true;
    h.turbulence = v->turbulence;
    h.wall_i_start = (long long)v->wall_i_start;
    h.re_c = v->re_c;
    h.sutherland = v->sutherland;
    h.roughness = v->roughness;
  } else {
    h.viscous = false;
    h.turbulence = 0;
  }
  h.dwall.clear();  // the no-slip faces may have changed
  int rc = s->ar.upload_desc();
  if (rc) return from_arena(s, rc);
  if (h.viscous && h.turbulence == BOWSHOCK_TURB_SST) return from_arena(s, s->ar.turb_init(0));
  return BOWSHOCK_OK;
}

int bowshock_solver_set_state(bowshock_solver* s, const double* u) {
  if (!s || !u) return BOWSHOCK_INVALID;
  return from_arena(s, s->ar.set_state(0, u));
}

int bowshock_solver_reset(bowshock_solver* s) {
  if (!s) return BOWSHOCK_INVALID;
  return from_arena(s, s->ar.reset_case(0));
}

int bowshock_solver_state(const bowshock_solver* s, double* u) {
  if (!s || !u) return BOWSHOCK_INVALID;
  return from_arena(const_cast<bowshock_solver*>(s), const_cast<ArenaHost&>(s->ar).get_state(0, u));
}

int bowshock_solver_turb_state(const bowshock_solver* s, double* turb, double* mu_t) {
  if (!s) return BOWSHOCK_INVALID;
  bowshock_solver* m = const_cast<bowshock_solver*>(s);
  if (!(s->ar.cases[0].viscous && s->ar.cases[0].turbulence == 1)) return fail(m, BOWSHOCK_UNSUPPORTED, "turb_state needs the SST model");
  std::vector<double> t, mt;
  int rc = m->ar.download_cells(0, m->ar.A.turb, t, 2);
  if (!rc) rc = m->ar.download_cells(0, m->ar.A.mu_t, mt, 1);
  if (rc) return from_arena(m, rc);
  if (turb) std::memcpy(turb, t.data(), t.size() * sizeof(double));
  if (mu_t) std::memcpy(mu_t, mt.data(), mt.size() * sizeof(double));
  return BOWSHOCK_OK;
}

int bowshock_solver_set_turb(bowshock_solver* s, const double* turb, const double* mu_t) {
  if (!s) return BOWSHOCK_INVALID;
  if (!(s->ar.cases[0].viscous && s->ar.cases[0].turbulence == 1)) return fail(s, BOWSHOCK_UNSUPPORTED, "set_turb needs the SST model");
  return from_arena(s, s->ar.turb_upload(0, turb, mu_t));
}

int bowshock_solver_iter(const bowshock_solver* s, uint64_t* iter) {
  if (!s || !iter) return BOWSHOCK_INVALID;
  int v = 0;
  int rc = const_cast<ArenaHost&>(s->ar).get_counter(s->ar.d_iter, 0, v);
  *iter = (uint64_t)v;
  return from_arena(const_cast<bowshock_solver*>(s), rc);
}

int bowshock_solver_set_iter(bowshock_solver* s, uint64_t iter) {
  if (!s) return BOWSHOCK_INVALID;
  return from_arena(s, s->ar.set_counter(s->ar.d_iter, 0, (int)std::min<uint64_t>(iter, 1u << 30)));
}

int bowshock_solver_restart_ramp(bowshock_solver* s) {
  if (!s) return BOWSHOCK_INVALID;
  return from_arena(s, s->ar.set_counter(s->ar.d_ramp, 0, 0));
}

int bowshock_solver_run(bowshock_solver* s, uint64_t n, double* residual) {
  if (!s) return BOWSHOCK_INVALID;
  const size_t nc = s->ar.cases.size();  // > 1 with a multigrid hierarchy: report the fine level only
  std::vector<double> all(residual && nc > 1 ? n * nc : 0);
  int rc = s->ar.run((long long)n, nc > 1 ? (residual ? all.data() : nullptr) : residual);
  if (rc) return from_arena(s, rc);
  if (residual && nc > 1)
    for (uint64_t k = 0; k < n; ++k) residual[k] = all[k * nc];
  if (residual)
    for (uint64_t k = 0; k < n; ++k)
      if (!std::isfinite(residual[k])) return fail(s, BOWSHOCK_NONFINITE, "non-finite residual at iteration " + std::to_string(k));
  return BOWSHOCK_OK;
}

int bowshock_solver_eval_residual(bowshock_solver* s, int compute_dt, double* res, double* dt, double* density_residual) {
  if (!s) return BOWSHOCK_INVALID;
  std::vector<double> dens;
  int rc = s->ar.eval_residual(compute_dt ? 1 : 0, &dens);
  if (rc) return from_arena(s, rc);
  if (density_residual) *density_residual = dens[0];
  std::vector<double> tmp;
  if (res) {
    if ((rc = s->ar.download_cells(0, s->ar.A.R, tmp, 4))) return from_arena(s, rc);
    std::memcpy(res, tmp.data(), tmp.size() * sizeof(double));
  }
  if (dt) {
    if ((rc = s->ar.download_cells(0, s->ar.A.dt, tmp, 1))) return from_arena(s, rc);
    std::memcpy(dt, tmp.data(), tmp.size() * sizeof(double));
  }
  return BOWSHOCK_OK;
}

int bowshock_solver_turb_residual(const bowshock_solver* s, double* r) {
  if (!s || !r) return BOWSHOCK_INVALID;
  *r = s->ar.last_turb_residual.empty() ? 0.0 : s->ar.last_turb_residual[0];
  return BOWSHOCK_OK;
}

int bowshock_solver_read_boundary(const bowshock_solver* s, double* u) {
  if (!s || !u) return BOWSHOCK_INVALID;
  bowshock_solver* m = const_cast<bowshock_solver*>(s);
  const HostCase& h = s->ar.cases[0];
  std::vector<double> all((size_t)h.ni * h.nj * 4);
  int rc = m->ar.get_state(0, all.data());
  if (rc) return from_arena(m, rc);
  auto copy = [&](int i, int j) {
    if (i < 0 || j < 0 || i >= h.ni || j >= h.nj) return;
    size_t c = (size_t)j * h.ni + i;
    for (int q = 0; q < 4; ++q) u[4 * c + q] = all[4 * c + q];
  };
  for (int i = 0; i < h.ni; ++i) {
    int j0 = h.has_block ? (i < h.i_end ? (int)h.j_end : (int)h.j_sting) : 0;
    copy(i, j0);
    copy(i, j0 + 1);
    copy(i, h.nj - 1);
    if (h.has_block && h.j_sting > 0) {
      copy(i, (int)h.j_sting);
      copy(i, (int)h.j_sting + 1);
    }
  }
  for (int j = 0; j < h.nj; ++j) {
    copy(0, j);
    copy(h.ni - 1, j);
    if (h.has_block) {
      copy((int)h.i_end, j);
      copy((int)h.i_end + 1, j);
    }
  }
  return BOWSHOCK_OK;
}

int bowshock_solver_base_cells(const bowshock_solver* s, double* out) {
  if (!s || !out) return BOWSHOCK_INVALID;
  bowshock_solver* m = const_cast<bowshock_solver*>(s);
  const HostCase& h = s->ar.cases[0];
  if (!h.has_block) return fail(m, BOWSHOCK_UNSUPPORTED, "base_cells needs a solid block");
  std::vector<double> all((size_t)h.ni * h.nj * 4);
  int rc = m->ar.get_state(0, all.data());
  if (rc) return from_arena(m, rc);
  size_t o = 0;
  for (long long j = h.j_sting; j < h.j_end; ++j)
    for (int d = 0; d < 2; ++d) {
      size_t c = (size_t)j * h.ni + h.i_end + d;
      for (int q = 0; q < 4; ++q) out[o++] = all[4 * c + q];
    }
  return BOWSHOCK_OK;
}

}  // extern "C"

// ==================================================================================== forces, runner, mesher, arena
#include "runner.cuh"

struct bowshock_solver_ext {
  ForcePass fp;
  bool ready = false;
};
static std::vector<std::pair<bowshock_solver*, bowshock_solver_ext*>>& ext_table() {
  static std::vector<std::pair<bowshock_solver*, bowshock_solver_ext*>> t;
  return t;
}

static RunParams to_params(const bowshock_run_params* p) {
  RunParams r;
  r.max_iter = (long long)p->max_iter;
  r.min_iter = (long long)p->min_iter;
  r.drop_orders = p->drop_orders;
  r.monitor_window = (long long)p->monitor_window;
  r.has_monitor_tol = p->has_monitor_tol != 0;
  r.monitor_tol = p->monitor_tol;
  r.has_mean_window = p->has_mean_window != 0;
  r.mean_window = (long long)p->mean_window;
  r.has_drag_rel_tol = p->has_drag_rel_tol != 0;
  r.drag_rel_tol = p->drag_rel_tol;
  r.wake = p->wake;
  r.warm = p->warm != 0;
  r.r_ref = p->r_ref;
  return r;
}

static bool valid_body(const bowshock_body* b, std::string& m) {
  if (!b) return m = "null body", false;
  if (b->nseg < 1 || b->nseg > BOWSHOCK_MAX_SEGMENTS) return m = "a body needs 1 to 8 aft segments", false;
  if (b->nose_kind < 0 || b->nose_kind > 4) return m = "unknown nose shape", false;
  return true;
}

static mesh::Body to_mesh_body(const bowshock_body* b) {
  mesh::Body mb;
  mb.nose = b->nose_kind;
  mb.fineness = b->fineness;
  mb.half_angle = b->half_angle;
  mb.param = b->param;
  for (int s = 0; s < b->nseg; ++s) mb.seg_len.push_back(b->seg_length[s]), mb.seg_slope.push_back(b->seg_slope[s]);
  mb.sting_radius = b->sting_radius;
  return mb;
}

// One ForcePass per solver handle, created on first use.
static ForcePass* solver_forces(bowshock_solver* s, int& rc) {
  rc = 0;
  for (auto& e : ext_table())
    if (e.first == s) return &e.second->fp;
  auto* x = new bowshock_solver_ext();
  rc = x->fp.setup(s->ar);
  if (rc) {
    delete x;
    return nullptr;
  }
  ext_table().push_back({s, x});
  return &x->fp;
}
static void solver_forces_drop(bowshock_solver* s) {
  auto& t = ext_table();
  for (size_t k = 0; k < t.size(); ++k)
    if (t[k].first == s) {
      delete t[k].second;
      t.erase(t.begin() + k);
      return;
    }
}

static void fill_forces(const Forces& f, int nseg, bowshock_forces* o) {
  o->cd_nose = f.f[F_CD_NOSE];
  o->cd_nose_cell = f.f[F_CD_NOSE_CELL];
  o->cd_base = f.f[F_CD_BASE];
  o->cp_base = f.f[F_CP_BASE];
  o->cp_base_cell = f.f[F_CP_BASE_CELL];
  o->cd_friction = f.f[F_CD_FRICTION];
  o->y_plus_max = f.f[F_YPLUS];
  for (int k = 0; k < BOWSHOCK_MAX_SEGMENTS; ++k) o->cd_aft[k] = k < nseg ? f.f[F_CD_AFT0 + k] : 0.0;
  o->cd_total = f.cd_total(nseg);
}

extern "C" {

int bowshock_solver_forces(bowshock_solver* s, const bowshock_body* body, bowshock_forces* out) {
  if (!s || !out) return BOWSHOCK_INVALID;
  std::string m;
  if (!valid_body(body, m)) return fail(s, BOWSHOCK_INVALID, m);
  int rc = 0;
  ForcePass* fp = solver_forces(s, rc);
  if (!fp) return from_arena(s, rc);
  if ((rc = fp->set_body(s->ar, 0, body))) return from_arena(s, rc);
  std::vector<Forces> f;
  if ((rc = fp->run(s->ar, f))) return from_arena(s, rc);
  fill_forces(f[0], body->nseg, out);
  return BOWSHOCK_OK;
}

int bowshock_solver_run_to_stop(bowshock_solver* s, const bowshock_body* body, const bowshock_run_params* p, bowshock_point_result* out,
                                double* residual, uint64_t cap, bowshock_progress_fn progress, void* user) {
  if (!s || !p || !out) return BOWSHOCK_INVALID;
  std::string m;
  if (!valid_body(body, m)) return fail(s, BOWSHOCK_INVALID, m);
  if (s->ar.cases[0].scheme != BOWSHOCK_SCHEME_IMPLICIT && s->ar.cases[0].scheme != BOWSHOCK_SCHEME_EXPLICIT &&
      s->ar.cases[0].scheme != BOWSHOCK_SCHEME_SMOOTHED && s->ar.cases[0].scheme != BOWSHOCK_SCHEME_MULTIGRID)
    return fail(s, BOWSHOCK_UNSUPPORTED, "unknown scheme");
  int rc = 0;
  ForcePass* fp = solver_forces(s, rc);
  if (!fp) return from_arena(s, rc);
  if ((rc = fp->set_body(s->ar, 0, body))) return from_arena(s, rc);
  std::vector<CaseRun> runs(1);
  runs[0].p = to_params(p);
  runs[0].nseg = body->nseg;
  runs[0].skip = runs[0].p.warm ? 0 : 20;
  if ((rc = start_case(s->ar, 0, runs[0].p, s->ar.cases[0].first_order_iters))) return from_arena(s, rc);
  for (int k = 1; k < (int)s->ar.cases.size(); ++k)  // multigrid levels: their counters and CFL ramps restart with the run
    if ((rc = s->ar.set_counter(s->ar.d_iter, k, 0)) || (rc = s->ar.set_counter(s->ar.d_ramp, k, 0))) return from_arena(s, rc);
  std::function<bool(int, long long, double, double)> cb;
  if (progress) cb = [&](int k, long long it, double r, double mon) { return progress(user, (uint64_t)k, (uint64_t)it, r, mon) == 0; };
  if ((rc = solve_arena(s->ar, *fp, runs, cb))) return from_arena(s, rc);
  std::vector<Forces> f;
  if ((rc = fp->run(s->ar, f))) return from_arena(s, rc);
  fill_point(runs[0], f[0], out);
  if (residual)
    for (size_t k = 0; k < runs[0].residual.size() && k < cap; ++k) residual[k] = runs[0].residual[k];
  std::vector<int> all(s->ar.cases.size(), 1);
  s->ar.set_active(all.data());
  return runs[0].reason == 5 ? fail(s, BOWSHOCK_NONFINITE, "non-finite residual or monitor") : BOWSHOCK_OK;
}

int bowshock_base_domain_grid(const bowshock_body* body, const bowshock_base_grid* p, uint64_t* ni, uint64_t* nj, double* x, double* r,
                              bowshock_block* block) {
  std::string m;
  if (!valid_body(body, m) || !p || !ni || !nj) return BOWSHOCK_INVALID;
  mesh::Body mb = to_mesh_body(body);
  mesh::BaseGrid g{p->x_up, p->x_down, p->r_far, p->n_up, p->n_nose, {}, p->n_wake, p->n_sting, p->n_gap, p->nj_out, p->dx_tip, p->dr_wall,
                   p->gap_one_sided != 0};
  for (int k = 0; k < body->nseg; ++k) g.n_seg.push_back(p->n_seg[k]);
  size_t a, b, blk[3];
  std::vector<double> X, R;
  if (!mesh::base_domain_grid(mb, g, a, b, X, R, blk, m)) return BOWSHOCK_INVALID;
  *ni = a;
  *nj = b;
  if (x) std::memcpy(x, X.data(), X.size() * sizeof(double));
  if (r) std::memcpy(r, R.data(), R.size() * sizeof(double));
  if (block) *block = bowshock_block{blk[0], blk[1], blk[2]};
  return BOWSHOCK_OK;
}

int bowshock_large_domain_grid(const bowshock_body* body, const bowshock_sting_grid* p, uint64_t* ni, uint64_t* nj, double* x, double* r) {
  std::string m;
  if (!valid_body(body, m) || !p || !ni || !nj) return BOWSHOCK_INVALID;
  mesh::Body mb = to_mesh_body(body);
  mesh::StingGrid g{p->x_up, p->x_down, p->r_far, p->n_up, p->n_nose, {}, p->n_ext, p->nj, p->dx_tip, p->dr_wall};
  for (int k = 0; k < body->nseg; ++k) g.n_seg.push_back(p->n_seg[k]);
  size_t a, b;
  std::vector<double> X, R;
  if (!mesh::large_domain_grid(mb, g, a, b, X, R, m)) return BOWSHOCK_INVALID;
  *ni = a;
  *nj = b;
  if (x) std::memcpy(x, X.data(), X.size() * sizeof(double));
  if (r) std::memcpy(r, R.data(), R.size() * sizeof(double));
  return BOWSHOCK_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- batched arena
struct bowshock_arena {
  ArenaHost ar;
  ForcePass fp;
  std::vector<bowshock_case_desc> descs;
  std::vector<int> nseg;
  std::string last_error;
  double last_solve_ms = 0.0;
  std::vector<std::vector<double>> hist;  // density residual per iteration of each case's last solve
};

// The host description of one arena case (validated; the metrics are computed separately): false if invalid.
static bool host_case_of(const bowshock_case_desc& d, HostCase& h, std::string& m) {
  if (d.ni < 4 || d.nj < 2 || !d.x || !d.r || !valid_config(&d.cfg, m) || !valid_body(&d.body, m) ||
      d.scheme.kind != BOWSHOCK_SCHEME_IMPLICIT || d.scheme.sub_iters < 1 || d.scheme.sub_iters > 16 ||
      (d.has_viscous && !(d.viscous.roughness >= 0.0 && std::isfinite(d.viscous.roughness)))) {
    return false;
  }
  h.ni = (int)d.ni;
  h.nj = (int)d.nj;
  h.x.assign(d.x, d.x + (d.ni + 1) * (d.nj + 1));
  h.r.assign(d.r, d.r + (d.ni + 1) * (d.nj + 1));
  apply_config(h, &d.cfg);
  h.low_mach = d.low_mach ? 1 : 0;
  h.scheme = BOWSHOCK_SCHEME_IMPLICIT;
  h.cfl0 = d.scheme.cfl0;
  h.cfl_max = d.scheme.cfl_max;
  h.growth = d.scheme.growth;
  h.dt_mode = d.scheme.dt_mode;
  h.lines = d.scheme.lines;
  h.implicit_bc = d.scheme.implicit_bc;
  h.sub_iters = (int)d.scheme.sub_iters;
  h.roe = d.scheme.roe;
  h.eps_fix = d.scheme.eps_fix;
  if (d.has_block) {
    const bowshock_block& b = d.block;
    if (!(b.i_end >= 1 && b.i_end + 2 <= d.ni && b.j_end >= 2 && b.j_end + 2 <= d.nj && b.j_end > b.j_sting && (b.j_sting == 0 || b.j_sting >= 2))) {
      return false;
    }
    h.has_block = true;
    h.i_end = (long long)b.i_end;
    h.j_end = (long long)b.j_end;
    h.j_sting = (long long)b.j_sting;
  }
  if (d.has_viscous) {
    h.viscous = true;
    h.turbulence = d.viscous.turbulence;
    h.wall_i_start = (long long)d.viscous.wall_i_start;
    h.re_c = d.viscous.re_c;
    h.sutherland = d.viscous.sutherland;
    h.roughness = d.viscous.roughness;
  }
  return true;
}

static int afrom(bowshock_arena* a, int rc) {
  if (rc) a->last_error = a->ar.err;
  return rc;
}

extern "C" {

// The arena of ncases descriptors; met[k] (when met is not null): case k's metrics from the device mesher
// (BOWSHOCK_MESH_METRIC_WORDS, in its order), else the FP64 metrics are computed here on the host.
static int arena_build(uint64_t ncases, const bowshock_case_desc* cases, const std::vector<const double*>* met, int device, bowshock_arena** out) {
  bowshock_arena* a = new (std::nothrow) bowshock_arena();
  if (!a) return BOWSHOCK_INVALID;
  std::string m;
  for (uint64_t k = 0; k < ncases; ++k) {
    const bowshock_case_desc& d = cases[k];
    HostCase h;
    if (!host_case_of(d, h, m)) {
      delete a;
      return BOWSHOCK_INVALID;
    }
    a->ar.cases.push_back(std::move(h));
    a->descs.push_back(d);
    a->nseg.push_back(d.body.nseg);
  }
  if (met) {
    for (uint64_t k = 0; k < ncases; ++k) {
      HostCase& h = a->ar.cases[k];
      const size_t nif = (size_t)(h.ni + 1) * h.nj, njf = (size_t)h.ni * (h.nj + 1), nc = (size_t)h.ni * h.nj;
      const double* p = (*met)[k];
      auto take = [&](std::vector<double>& v, size_t n) {
        v.assign(p, p + n);
        p += n;
      };
      take(h.if_nx, nif), take(h.if_nr, nif), take(h.if_len, nif), take(h.if_rm, nif);
      take(h.jf_nx, njf), take(h.jf_nr, njf), take(h.jf_len, njf), take(h.jf_rm, njf);
      take(h.area, nc), take(h.vol, nc), take(h.xc, nc), take(h.rc, nc);
    }
  } else if (!parallel_cases(a->ar.cases.size(), [&](size_t k, std::string& e) { return compute_metrics(a->ar.cases[k], e); }, m)) {
    // the FP64 metrics of each case, the cases spread over the host threads
    delete a;
    return BOWSHOCK_INVALID;
  }
  a->ar.device = device;
  int rc = a->ar.setup();
  if (!rc) rc = a->fp.setup(a->ar);
  for (uint64_t k = 0; !rc && k < ncases; ++k) rc = a->fp.set_body(a->ar, (int)k, &cases[k].body);
  if (!rc) a->ar.wall_distances();
  for (uint64_t k = 0; !rc && k < ncases; ++k)
    if (a->ar.cases[k].viscous && a->ar.cases[k].turbulence == 1) rc = a->ar.turb_init((int)k);
  // lines per block of the line kernels, tuned on the arena's own cases when it is large enough to matter
  if (!rc && a->ar.ncell >= 100000) rc = a->ar.autotune();
  if (rc) {
    delete a;
    return BOWSHOCK_CUDA_ERROR;
  }
  *out = a;
  return BOWSHOCK_OK;
}

int bowshock_arena_create(uint64_t ncases, const bowshock_case_desc* cases, int device, bowshock_arena** out) {
  if (!out || !cases || ncases == 0) return BOWSHOCK_INVALID;
  *out = nullptr;
  return arena_build(ncases, cases, nullptr, device, out);
}

int bowshock_arena_create_meshed(uint64_t ncases, const bowshock_case_desc* cases, const bowshock_mesh_request* meshes, int device,
                                 bowshock_arena** out) {
  if (!out || !cases || !meshes || ncases == 0) return BOWSHOCK_INVALID;
  *out = nullptr;
  std::string m;
  std::vector<size_t> noff(ncases), moff(ncases);
  size_t nodes = 0, mets = 0;
  for (uint64_t k = 0; k < ncases; ++k) {
    bkmesh::Dims d;
    const bowshock_case_desc& c = cases[k];
    if (!bkmesh::dims(meshes[k], d, m) || (long long)c.ni != d.ni || (long long)c.nj != d.nj) return BOWSHOCK_INVALID;
    const bool base = meshes[k].wake == BOWSHOCK_WAKE_BASE;
    if (base != (c.has_block != 0)) return BOWSHOCK_INVALID;
    if (base && ((long long)c.block.i_end != d.i_end || (long long)c.block.j_end != d.j_end || (long long)c.block.j_sting != d.j_sting))
      return BOWSHOCK_INVALID;
    noff[k] = nodes, moff[k] = mets;
    nodes += (size_t)(d.ni + 1) * (d.nj + 1);
    mets += (size_t)BOWSHOCK_MESH_METRIC_WORDS(d.ni, d.nj);
  }
  std::vector<double> X(nodes), R(nodes), M(mets);
  int rc = bkmesh::mesh_batch(ncases, meshes, device, X.data(), R.data(), M.data(), nullptr, m);
  if (rc) return rc;
  std::vector<bowshock_case_desc> ds(cases, cases + ncases);
  std::vector<const double*> met(ncases);
  for (uint64_t k = 0; k < ncases; ++k) {
    ds[k].x = X.data() + noff[k], ds[k].r = R.data() + noff[k];
    met[k] = M.data() + moff[k];
  }
  rc = arena_build(ncases, ds.data(), &met, device, out);
  if (rc == BOWSHOCK_OK) {  // the descriptors keep pointing at the caller's (possibly null) node arrays, as passed
    for (uint64_t k = 0; k < ncases; ++k) (*out)->descs[k].x = cases[k].x, (*out)->descs[k].r = cases[k].r;
  }
  return rc;
}

int bowshock_arena_tuning(const bowshock_arena* a, bowshock_line_tuning* out) {
  if (!a || !out) return BOWSHOCK_INVALID;
  const auto& r = a->ar;
  out->lines_i = r.lw_lines[1] > 4 ? 4 : r.lw_lines[1], out->lines_j = r.lw_lines[0] > 4 ? 4 : r.lw_lines[0];
  out->prefetch_i = r.pf_lines[1], out->prefetch_j = r.pf_lines[0];
  out->subst_i = r.lw_subst[1], out->subst_j = r.lw_subst[0], out->turb_lines = r.lw_turb;
  out->segment_i = r.A.mmin_i, out->segment_j = r.A.mmin_j, out->residual = r.res_variant;
  out->subst_prefetch_i = r.pf_subst[1], out->subst_prefetch_j = r.pf_subst[0];
  out->staged_lines = r.staged_lines;
  return BOWSHOCK_OK;
}

int bowshock_arena_set_case_groups(bowshock_arena* a, int groups) {
  if (!a || groups < 1 || groups > ArenaHost::MAX_GROUPS) return BOWSHOCK_INVALID;
  a->ar.groups_req = groups;
  if (a->ar.compact_lists()) {
    a->last_error = a->ar.err;
    return BOWSHOCK_CUDA_ERROR;
  }
  return BOWSHOCK_OK;
}

int bowshock_arena_set_sst_coupling(bowshock_arena* a, int coupled) {
  if (!a) return BOWSHOCK_INVALID;
  if (a->ar.set_sst_coupled(coupled != 0)) {
    a->last_error = a->ar.err;
    return BOWSHOCK_CUDA_ERROR;
  }
  return BOWSHOCK_OK;
}

int bowshock_arena_set_tuning(bowshock_arena* a, const bowshock_line_tuning* t) {
  if (!a || !t) return BOWSHOCK_INVALID;
  auto w4 = [](int32_t w) { return w == 1 || w == 2 || w == 4; };
  auto w8 = [](int32_t w) { return w == 1 || w == 2 || w == 4 || w == 8; };
  auto m8 = [](int32_t m) { return m == 2 || m == 4 || m == 8; };
  auto b012 = [](int32_t b) { return b >= 0 && b <= 2; };
  if (!(w4(t->lines_i) && w4(t->lines_j) && b012(t->prefetch_i) && b012(t->prefetch_j) && w8(t->subst_i) && w8(t->subst_j) &&
        w8(t->turb_lines) && m8(t->segment_i) && m8(t->segment_j) && (t->residual == 0 || t->residual == 1) &&
        b012(t->subst_prefetch_i) && b012(t->subst_prefetch_j) && t->staged_lines >= 0)) {
    a->last_error = "line tuning out of range";
    return BOWSHOCK_INVALID;
  }
  auto& r = a->ar;
  r.lw_lines[1] = t->lines_i, r.lw_lines[0] = t->lines_j, r.pf_lines[1] = t->prefetch_i, r.pf_lines[0] = t->prefetch_j;
  r.lw_subst[1] = t->subst_i, r.lw_subst[0] = t->subst_j, r.lw_turb = t->turb_lines;
  r.A.mmin_i = t->segment_i, r.A.mmin_j = t->segment_j, r.res_variant = t->residual;
  r.pf_subst[1] = t->subst_prefetch_i, r.pf_subst[0] = t->subst_prefetch_j;
  r.staged_lines = t->staged_lines;
  if (r.graph) cudaGraphExecDestroy(r.graph), r.graph = nullptr;  // the chunk graph holds the old shapes
  return BOWSHOCK_OK;
}

int bowshock_case_wall_distance(const bowshock_case_desc* d, double* out) {
  if (!d || !out) return BOWSHOCK_INVALID;
  HostCase h;
  std::string m;
  if (!host_case_of(*d, h, m) || !compute_metrics(h, m)) return BOWSHOCK_INVALID;
  const std::vector<double> w = wall_distance(h);
  std::copy(w.begin(), w.end(), out);
  return BOWSHOCK_OK;
}

void bowshock_arena_destroy(bowshock_arena* a) { delete a; }
const char* bowshock_arena_last_error(const bowshock_arena* a) { return a ? a->last_error.c_str() : "null handle"; }

int bowshock_arena_cells(const bowshock_arena* a, uint64_t* ncells) {
  if (!a || !ncells) return BOWSHOCK_INVALID;
  *ncells = (uint64_t)a->ar.ncell;
  return BOWSHOCK_OK;
}

int bowshock_arena_run(bowshock_arena* a, uint64_t n, double* residual) {
  if (!a) return BOWSHOCK_INVALID;
  return afrom(a, a->ar.run((long long)n, residual));
}

int bowshock_arena_prepare(bowshock_arena* a, uint64_t n) {
  if (!a) return BOWSHOCK_INVALID;
  return afrom(a, a->ar.prepare((long long)n));
}

int bowshock_arena_solve(bowshock_arena* a, bowshock_point_result* results, bowshock_progress_fn progress, void* user) {
  if (!a || !results) return BOWSHOCK_INVALID;
  const int nc = (int)a->ar.cases.size();
  std::vector<CaseRun> runs(nc);
  int rc = 0;
  for (int k = 0; k < nc; ++k) {
    runs[k].p = to_params(&a->descs[k].run);
    runs[k].nseg = a->nseg[k];
    runs[k].skip = runs[k].p.warm ? 0 : 20;
    if ((rc = start_case(a->ar, k, runs[k].p, a->ar.cases[k].first_order_iters))) return afrom(a, rc);
  }
  std::function<bool(int, long long, double, double)> cb;
  if (progress) cb = [&](int k, long long it, double r, double mon) { return progress(user, (uint64_t)k, (uint64_t)it, r, mon) == 0; };
  a->last_solve_ms = 0.0;
  if ((rc = solve_arena(a->ar, a->fp, runs, cb, &a->last_solve_ms))) return afrom(a, rc);
  std::vector<Forces> f;
  if ((rc = a->fp.run(a->ar, f))) return afrom(a, rc);
  for (int k = 0; k < nc; ++k) fill_point(runs[k], f[k], &results[k]);
  a->hist.resize(nc);
  for (int k = 0; k < nc; ++k) a->hist[k].swap(runs[k].residual);
  std::vector<int> all(nc, 1);
  return afrom(a, a->ar.set_active(all.data()));
}

int bowshock_arena_forces(bowshock_arena* a, bowshock_forces* out) {
  if (!a || !out) return BOWSHOCK_INVALID;
  std::vector<Forces> f;
  int rc = a->fp.run(a->ar, f);
  if (rc) return afrom(a, rc);
  for (size_t k = 0; k < f.size(); ++k) fill_forces(f[k], a->nseg[k], &out[k]);
  return BOWSHOCK_OK;
}

int bowshock_arena_state(const bowshock_arena* a, uint64_t k, double* u) {
  if (!a || !u || k >= a->ar.cases.size()) return BOWSHOCK_INVALID;
  bowshock_arena* m = const_cast<bowshock_arena*>(a);
  return afrom(m, m->ar.get_state((int)k, u));
}

int bowshock_arena_set_state(bowshock_arena* a, uint64_t k, const double* u) {
  if (!a || !u || k >= a->ar.cases.size()) return BOWSHOCK_INVALID;
  return afrom(a, a->ar.set_state((int)k, u));
}

int bowshock_arena_set_run(bowshock_arena* a, uint64_t k, const bowshock_run_params* p) {
  if (!a || !p || k >= a->ar.cases.size()) return BOWSHOCK_INVALID;
  if (p->max_iter == 0 || !(p->drop_orders > 0.0) || (p->has_mean_window && p->mean_window < 50) || p->monitor_window == 0) {
    a->last_error = "run parameters out of range";
    return BOWSHOCK_INVALID;
  }
  a->descs[k].run = *p;
  return BOWSHOCK_OK;
}

int bowshock_arena_turb_state(const bowshock_arena* a, uint64_t k, double* turb, double* mu_t) {
  if (!a || k >= a->ar.cases.size()) return BOWSHOCK_INVALID;
  bowshock_arena* m = const_cast<bowshock_arena*>(a);
  if (!(a->ar.cases[k].viscous && a->ar.cases[k].turbulence == 1)) {
    m->last_error = "turb_state needs an SST case";
    return BOWSHOCK_UNSUPPORTED;
  }
  std::vector<double> t, mt;
  int rc = m->ar.download_cells((int)k, m->ar.A.turb, t, 2);
  if (!rc) rc = m->ar.download_cells((int)k, m->ar.A.mu_t, mt, 1);
  if (rc) return afrom(m, rc);
  if (turb) std::memcpy(turb, t.data(), t.size() * sizeof(double));
  if (mu_t) std::memcpy(mu_t, mt.data(), mt.size() * sizeof(double));
  return BOWSHOCK_OK;
}

int bowshock_arena_set_turb(bowshock_arena* a, uint64_t k, const double* turb, const double* mu_t) {
  if (!a || k >= a->ar.cases.size()) return BOWSHOCK_INVALID;
  if (!(a->ar.cases[k].viscous && a->ar.cases[k].turbulence == 1)) {
    a->last_error = "set_turb needs an SST case";
    return BOWSHOCK_UNSUPPORTED;
  }
  return afrom(a, a->ar.turb_upload((int)k, turb, mu_t));
}

int bowshock_arena_first_residuals(bowshock_arena* a, const int32_t* warm, double* out) {
  if (!a || !out) return BOWSHOCK_INVALID;
  ArenaHost& ar = a->ar;
  const int nc = (int)ar.cases.size();
  int rc = 0;
  for (int k = 0; k < nc; ++k) {
    const int it = (warm && warm[k]) ? (int)ar.cases[k].first_order_iters : 0;
    if ((rc = ar.set_counter(ar.d_iter, k, it))) return afrom(a, rc);
  }
  std::vector<double> dens;
  if ((rc = ar.eval_residual(2, &dens))) return afrom(a, rc);
  for (int k = 0; k < nc; ++k) out[k] = dens[k];
  return BOWSHOCK_OK;
}

int bowshock_arena_residual_history(const bowshock_arena* a, uint64_t k, double* out, uint64_t cap, uint64_t* n) {
  if (!a || !n || k >= a->ar.cases.size()) return BOWSHOCK_INVALID;
  const std::vector<double> empty;
  const std::vector<double>& h = k < a->hist.size() ? a->hist[k] : empty;
  *n = h.size();
  if (out)
    for (size_t q = 0; q < h.size() && q < cap; ++q) out[q] = h[q];
  return BOWSHOCK_OK;
}

int bowshock_arena_set_run_control(bowshock_arena* a, int on_device) {
  if (!a) return BOWSHOCK_INVALID;
  a->ar.device_run_control = on_device != 0;
  return BOWSHOCK_OK;
}

int bowshock_arena_set_active(bowshock_arena* a, const int32_t* active) {
  if (!a || !active) return BOWSHOCK_INVALID;
  std::vector<int> v(active, active + a->ar.cases.size());
  return afrom(a, a->ar.set_active(v.data()));
}

int bowshock_arena_last_ms_per_iter(const bowshock_arena* a, double* ms) {
  if (!a || !ms) return BOWSHOCK_INVALID;
  *ms = a->ar.last_ms_per_iter;
  return BOWSHOCK_OK;
}

int bowshock_arena_last_solve_ms(const bowshock_arena* a, double* ms) {
  if (!a || !ms) return BOWSHOCK_INVALID;
  *ms = a->last_solve_ms;
  return BOWSHOCK_OK;
}

}  // extern "C"

extern "C" int bowshock_arena_profile(bowshock_arena* a, uint64_t n, double* ms, uint64_t* launches) {
  if (!a || !ms || !launches) return BOWSHOCK_INVALID;
  int rc = a->ar.profile((long long)n);
  if (rc) return afrom(a, rc);
  for (int g = 0; g < ArenaHost::G_N; ++g) {
    ms[g] = a->ar.prof_ms[g];
    launches[g] = (uint64_t)a->ar.prof_launches[g];
  }
  return BOWSHOCK_OK;
}

extern "C" int bowshock_solver_profile(bowshock_solver* s, uint64_t n, double* ms, uint64_t* launches) {
  if (!s || !ms || !launches) return BOWSHOCK_INVALID;
  int rc = s->ar.profile((long long)n);
  if (rc) return from_arena(s, rc);
  for (int g = 0; g < ArenaHost::G_N; ++g) {
    ms[g] = s->ar.prof_ms[g];
    launches[g] = (uint64_t)s->ar.prof_launches[g];
  }
  return BOWSHOCK_OK;
}

extern "C" int bowshock_solver_set_run_control(bowshock_solver* s, int on_device) {
  if (!s) return BOWSHOCK_INVALID;
  s->ar.device_run_control = on_device != 0;
  return BOWSHOCK_OK;
}

extern "C" int bowshock_solver_set_mg_fusion(bowshock_solver* s, int on) {
  if (!s) return BOWSHOCK_INVALID;
  s->ar.mg_fused = on != 0;
  if (s->ar.graph) cudaGraphExecDestroy(s->ar.graph), s->ar.graph = nullptr;  // the chunk graph holds the old launches
  return BOWSHOCK_OK;
}

extern "C" int bowshock_solver_set_sst_coupling(bowshock_solver* s, int coupled) {
  if (!s) return BOWSHOCK_INVALID;
  return from_arena(s, s->ar.set_sst_coupled(coupled != 0));
}

extern "C" int bowshock_solver_set_ramp(bowshock_solver* s, uint64_t ramp_k) {
  if (!s) return BOWSHOCK_INVALID;
  return from_arena(s, s->ar.set_counter(s->ar.d_ramp, 0, (int)std::min<uint64_t>(ramp_k, 1u << 30)));
}

// ============================================================================ allocation-free iteration
// bowshock_solver_run_noalloc: the iterations of bowshock_solver_run without a single device allocation. Who needs it:
// a host that sets its solvers up once and then steps them from code that must not allocate device memory, because the
// free memory of the GPU already belongs to that host's own pool (another framework's caching allocator sharing the
// device) or because the step runs in a loop that cannot take the device-wide synchronisation an allocation can bring.
// bowshock_solver_run allocates on its first call (it instantiates a CUDA graph of the iteration chunk and creates timing
// events); this variant launches the same kernels directly on the solver's stream, and the spike storage of its line
// solves (the records of k_lines / k_lines_subst / k_defect: blocks, factors and reduction multipliers) comes from the
// static array below instead of the solver's own buffer.
//
// The array: BOWSHOCK_NOALLOC_SCRATCH_BYTES (64 MiB) in this file's device module, so every GPU that loads the library
// holds it until the process exits. Host code cannot use its name as a device address: the address is looked up once per
// device, with that device current, by the first call on that device (cudaGetSymbolAddress). Every call on a device
// shares the array and it keeps the last call's contents; nothing in it has to start at zero (the first line pass of
// every iteration writes every record entry before any kernel reads it). Calls whose kernels overlap on one GPU (solvers on different streams or host threads)
// race on the array and corrupt each other: the caller must serialise them.
namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
static __device__ __align__(256) float g_noalloc_scratch[BOWSHOCK_NOALLOC_SCRATCH_BYTES / sizeof(float)];
// per device: the looked-up address (null until a lookup succeeded; a failed lookup is not kept, the next call retries)
float* g_noalloc_ptr[NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mu;

// The static array's device address on `device`, looked up with that device current (cudaGetSymbolAddress); the previous
// current device is restored. Returns the CUDA status of the lookup.
cudaError_t noalloc_address(int device, float** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (g_noalloc_ptr[device]) {
    *out = g_noalloc_ptr[device];
    return cudaSuccess;
  }
  int prev = -1;
  cudaError_t e = cudaGetDevice(&prev);
  if (e == cudaSuccess && prev != device) e = cudaSetDevice(device);
  void* p = nullptr;
  if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (prev >= 0 && prev != device) cudaSetDevice(prev);
  if (e == cudaSuccess && !p) e = cudaErrorInvalidSymbol;
  if (e == cudaSuccess) g_noalloc_ptr[device] = static_cast<float*>(p);
  *out = g_noalloc_ptr[device];
  return e;
}

// The solver's own line-record pointer swapped for the static array for the duration of one call, and put back on every
// return path (the kernels take the arena by value at launch, so only launches inside the call see the swap).
struct ScratchSwap {
  ArenaHost& ar;
  float* own;
  ScratchSwap(ArenaHost& a, float* scratch) : ar(a), own(a.A.scratch) { ar.A.scratch = scratch; }
  ~ScratchSwap() { ar.A.scratch = own; }
};

// n iterations of the solver's arena with `scratch` as the line solves' spike storage; errors in ar.err. Like
// ArenaHost::run, the turbulence residual of the last iteration is kept (bowshock_solver_turb_residual); the per-iteration
// device time (bowshock_arena_last_ms_per_iter) is not measured here: that would need timing events.
int noalloc_iterate(ArenaHost& ar, float* scratch, uint64_t n, double* residual) {
  std::string& err = ar.err;
  BK_CUDA(cudaSetDevice(ar.device));
  const int nc = (int)ar.cases.size();  // > 1 with a multigrid hierarchy: the fine level is case 0
  const double n_active = (double)ar.desc[0].n_active;
  ScratchSwap swap(ar, scratch);
  double tsum_last = 0.0;
  uint64_t done = 0;
  while (done < n) {
    const int chunk = (int)std::min<uint64_t>(n - done, (uint64_t)ar.slots);
    BK_CUDA(cudaMemsetAsync(ar.A.rsum, 0, (size_t)chunk * nc * sizeof(double), ar.stream));
    if (ar.any_sst) BK_CUDA(cudaMemsetAsync(ar.A.tsum, 0, (size_t)chunk * nc * sizeof(double), ar.stream));
    for (int k = 0; k < chunk; ++k) ar.launch_iteration(k);
    BK_CUDA(cudaGetLastError());
    if (residual)  // case 0's column of the [slot][case] sums of R_rho^2
      BK_CUDA(cudaMemcpy2DAsync(residual + done, sizeof(double), ar.A.rsum, (size_t)nc * sizeof(double), sizeof(double), chunk,
                                cudaMemcpyDeviceToHost, ar.stream));
    if (ar.any_sst)  // case 0's sum of the turbulence residual in the chunk's last iteration (pageable copy, no allocation)
      BK_CUDA(cudaMemcpyAsync(&tsum_last, ar.A.tsum + (size_t)(chunk - 1) * nc, sizeof(double), cudaMemcpyDeviceToHost, ar.stream));
    BK_CUDA(cudaStreamSynchronize(ar.stream));
    if (residual)
      for (int k = 0; k < chunk; ++k) residual[done + k] = std::sqrt(residual[done + k] / n_active);
    if (ar.any_sst) {
      ar.last_turb_residual.resize(nc);  // host memory only
      ar.last_turb_residual[0] = std::sqrt(tsum_last / n_active);
    }
    done += chunk;
  }
  return 0;
}
}  // namespace

extern "C" int bowshock_solver_run_noalloc(bowshock_solver* s, uint64_t n, double* residual) {
  if (!s) return BOWSHOCK_INVALID;
  ArenaHost& ar = s->ar;
  const int dev = ar.device;
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(s, BOWSHOCK_INVALID, "device index out of range for the static scratch");
  const uint64_t need = (uint64_t)ar.scratch_floats() * sizeof(float);
  if (need > (uint64_t)BOWSHOCK_NOALLOC_SCRATCH_BYTES)
    return fail(s, BOWSHOCK_INVALID,
                "the solver's " + std::to_string((long long)ar.ncell) + " cells and " + std::to_string(ar.nil + ar.njl) + " lines need " +
                    std::to_string(need) + " bytes of line-solve records, more than the static maximum of " +
                    std::to_string(BOWSHOCK_NOALLOC_SCRATCH_BYTES) + " bytes");
  float* scratch = nullptr;
  const cudaError_t e = noalloc_address(dev, &scratch);
  if (e != cudaSuccess || !scratch)
    return fail(s, BOWSHOCK_CUDA_ERROR, std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(e));
  int rc = noalloc_iterate(ar, scratch, n, residual);
  if (rc) return from_arena(s, rc);
  if (residual)
    for (uint64_t k = 0; k < n; ++k)
      if (!std::isfinite(residual[k])) return fail(s, BOWSHOCK_NONFINITE, "non-finite residual at iteration " + std::to_string(k));
  return BOWSHOCK_OK;
}

// ============================================================================ 3D Euler batch
struct bowshock3_batch {
  bk3::Batch3 b;
  std::string last_error;
};
static int b3from(bowshock3_batch* h, int rc) {
  if (rc) h->last_error = h->b.err;
  return rc;
}
extern "C" {
// a bowshock3_config as the batch's case record; BOWSHOCK_OK, UNSUPPORTED (not an explicit / implicit scheme) or INVALID
static int case3_of(const bowshock3_config& c, bk3::Case3Host& h) {
  if (c.scheme.kind != BOWSHOCK_SCHEME_IMPLICIT && c.scheme.kind != BOWSHOCK_SCHEME_EXPLICIT) return BOWSHOCK_UNSUPPORTED;
  if (!(c.mach > 0.0) || c.limiter < 0 || c.limiter > 3) return BOWSHOCK_INVALID;
  h.mach = c.mach, h.alpha = c.alpha, h.cfl = c.cfl, h.limiter = c.limiter, h.low_mach = c.low_mach != 0;
  h.first_order_iters = (long long)c.first_order_iters;
  h.implicit = c.scheme.kind == BOWSHOCK_SCHEME_IMPLICIT;
  h.cfl0 = c.scheme.cfl0, h.cfl_max = c.scheme.cfl_max, h.growth = c.scheme.growth, h.eps_fix = c.scheme.eps_fix;
  h.dt_mode = c.scheme.dt_mode, h.sub_iters = (int)std::max<uint64_t>(c.scheme.sub_iters, 1), h.roe = c.scheme.roe != 0;
  h.implicit_bc = c.scheme.implicit_bc != 0, h.lines = c.scheme.lines != 0;
  return BOWSHOCK_OK;
}
int bowshock3_create(uint64_t ni, uint64_t nj, uint64_t nk, const double* x, const double* y, const double* z, uint64_t axis_cells,
                     uint64_t ncases, const bowshock3_config* cfg, int device, bowshock3_batch** out) {
  if (!x || !y || !z || !cfg || !out || ncases == 0) return BOWSHOCK_INVALID;
  *out = nullptr;
  std::vector<bk3::Case3Host> cs(ncases);
  for (uint64_t k = 0; k < ncases; ++k) {
    if (cfg[k].scheme.kind != cfg[0].scheme.kind) return BOWSHOCK_UNSUPPORTED;  // one scheme per batch
    const int rc = case3_of(cfg[k], cs[k]);
    if (rc) return rc;
  }
  auto* h = new bowshock3_batch();
  int rc = h->b.create(ni, nj, nk, x, y, z, axis_cells, cs, device);
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return BOWSHOCK_OK;
}
void bowshock3_destroy(bowshock3_batch* b) { delete b; }
const char* bowshock3_last_error(const bowshock3_batch* b) { return b ? b->last_error.c_str() : "null handle"; }
int bowshock3_reset(bowshock3_batch* b) { return b ? b3from(b, b->b.reset()) : BOWSHOCK_INVALID; }
int bowshock3_set_solid(bowshock3_batch* b, uint64_t nbox, const uint64_t* boxes) {
  if (!b || (nbox && !boxes)) return BOWSHOCK_INVALID;
  return b3from(b, b->b.set_solid((size_t)nbox, boxes));
}
int bowshock3_set_config(bowshock3_batch* b, uint64_t k, const bowshock3_config* cfg) {
  if (!b || !cfg || k >= (uint64_t)b->b.B.nb) return BOWSHOCK_INVALID;
  bk3::Case3Host h;
  int rc = case3_of(*cfg, h);
  if (rc) return rc;
  rc = b->b.set_config((int)k, h);
  if (rc == 1) {
    b->last_error = b->b.err;
    return BOWSHOCK_UNSUPPORTED;
  }
  return b3from(b, rc);
}
int bowshock3_profile(bowshock3_batch* b, uint64_t n, double* ms, uint64_t* launches) {
  if (!b || !ms || !launches) return BOWSHOCK_INVALID;
  unsigned long long l[bk3::Batch3::P3_N];
  int rc = b->b.profile((long long)n, ms, l);
  for (int g = 0; g < bk3::Batch3::P3_N; ++g) launches[g] = l[g];
  return b3from(b, rc);
}
int bowshock3_set_groups(bowshock3_batch* b, int groups) {
  if (!b) return BOWSHOCK_INVALID;
  return b3from(b, b->b.set_groups(groups));
}
int bowshock3_set_staging(bowshock3_batch* b, int on) {
  if (!b) return BOWSHOCK_INVALID;
  b->b.staged = on != 0;
  return BOWSHOCK_OK;
}
int bowshock3_set_iter(bowshock3_batch* b, uint64_t iter, uint64_t ramp) {
  return b ? b3from(b, b->b.set_counters((int)std::min<uint64_t>(iter, 1u << 30), (int)std::min<uint64_t>(ramp, 1u << 30))) : BOWSHOCK_INVALID;
}
int bowshock3_set_state(bowshock3_batch* b, uint64_t k, const double* u) {
  if (!b || !u || k >= (uint64_t)b->b.B.nb) return BOWSHOCK_INVALID;
  return b3from(b, b->b.set_state((int)k, u));
}
int bowshock3_state(bowshock3_batch* b, uint64_t k, double* u) {
  if (!b || !u || k >= (uint64_t)b->b.B.nb) return BOWSHOCK_INVALID;
  return b3from(b, b->b.get_state((int)k, u));
}
int bowshock3_run(bowshock3_batch* b, uint64_t n, double* residual) {
  if (!b) return BOWSHOCK_INVALID;
  int rc = b->b.run((long long)n, residual);
  if (rc) return b3from(b, rc);
  return BOWSHOCK_OK;
}
int bowshock3_eval_residual(bowshock3_batch* b, uint64_t k, double* res, double* dt, double* density_residual) {
  if (!b || k >= (uint64_t)b->b.B.nb) return BOWSHOCK_INVALID;
  std::vector<double> dens;
  int rc = b->b.eval_residual(dens);
  if (!rc) rc = b->b.read_residual((int)k, res, dt);
  if (rc) return b3from(b, rc);
  if (density_residual) *density_residual = dens[k];
  return BOWSHOCK_OK;
}
int bowshock3_forces(bowshock3_batch* b, double x_max, double* out) {
  if (!b || !out) return BOWSHOCK_INVALID;
  std::vector<double> f;
  int rc = b->b.forces(x_max, f);
  if (rc) return b3from(b, rc);
  std::memcpy(out, f.data(), f.size() * sizeof(double));
  return BOWSHOCK_OK;
}
int bowshock3_read_boundary(bowshock3_batch* b, uint64_t k, double* u) {
  if (!b || !u || k >= (uint64_t)b->b.B.nb) return BOWSHOCK_INVALID;
  return b3from(b, b->b.read_boundary((int)k, u));
}
int bowshock3_forces_parts(bowshock3_batch* b, double x_max, double x_nose, double* out) {
  if (!b || !out) return BOWSHOCK_INVALID;
  std::vector<double> f;
  int rc = b->b.forces_parts(x_max, x_nose, f);
  if (rc) return b3from(b, rc);
  std::memcpy(out, f.data(), f.size() * sizeof(double));
  return BOWSHOCK_OK;
}
int bowshock3_solve(bowshock3_batch* b, const bowshock3_run_params* p, bowshock3_result* out) {
  if (!b || !p || !out) return BOWSHOCK_INVALID;
  bk3::Batch3& B = b->b;
  const int nb = B.B.nb;
  int rc = B.reset();
  if (rc) return b3from(b, rc);
  std::vector<bk3::StopRule3> rules(nb);
  for (auto& r : rules) r.window = p->window, r.nwin = std::max<size_t>(p->window / 50, 1), r.rel_tol = p->rel_tol;
  std::vector<int> act(nb, 1);
  std::vector<uint64_t> its(nb, 0);
  if ((rc = B.set_active(act))) return b3from(b, rc);
  std::vector<double> res(50 * (size_t)nb), f;
  uint64_t done_it = 0;
  while (true) {
    int left = 0;
    for (int k = 0; k < nb; ++k) left += act[k];
    if (!left || done_it >= p->max_iter) break;
    int chunk = (int)std::min<uint64_t>(50, p->max_iter - done_it);
    if ((rc = B.run(chunk, res.data()))) return b3from(b, rc);
    if ((rc = B.forces(p->x_max, f))) return b3from(b, rc);
    bool changed = false;
    for (int k = 0; k < nb; ++k) {
      if (!act[k]) continue;
      for (int t = 0; t < chunk && act[k]; ++t) {
        size_t it = (size_t)(done_it + t);
        bool sampled = (it + 1) % 50 == 0;
        its[k] = it + 1;
        if (rules[k].check(it, res[(size_t)t * nb + k], sampled, f[3 * k])) act[k] = 0, changed = true;
      }
    }
    done_it += chunk;
    if (changed && (rc = B.set_active(act))) return b3from(b, rc);
  }
  if ((rc = B.forces(p->x_max, f))) return b3from(b, rc);
  for (int k = 0; k < nb; ++k) {
    bowshock3_result& o = out[k];
    o.cn = f[3 * k], o.ca = f[3 * k + 1], o.x_cp = f[3 * k + 2];
    o.iterations = its[k];
    o.stop_reason = rules[k].reason;
    o.drop_orders = rules[k].rmax > 0.0 && rules[k].r > 0.0 ? std::log10(rules[k].rmax / rules[k].r) : 0.0;
  }
  std::vector<int> all(nb, 1);
  return b3from(b, B.set_active(all));
}
int bowshock3_last_ms_per_iter(const bowshock3_batch* b, double* ms) {
  if (!b || !ms) return BOWSHOCK_INVALID;
  *ms = b->b.last_ms_per_iter;
  return BOWSHOCK_OK;
}
}  // extern "C"
