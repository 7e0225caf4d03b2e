// C ABI of the single-case solver (include/bowshock_b200.h): a GpuSolver (crates/bowshock-cfd/src/gpu/mod.rs:233-414)
// backed by a case arena of one. Unity build: the kernels and the host arena are compiled into this translation unit.
#include <cstdio>
#include <exception>

#include "../../include/bowshock_b200.h"
#include "fv_kernels.cu"
#include "turbulence.cuh"
#include "host_arena.cuh"

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

void bowshock_solver_destroy(bowshock_solver* s) { delete s; }

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
  return from_arena(s, s->ar.upload_desc());
}

int bowshock_solver_set_scheme(bowshock_solver* s, const bowshock_scheme* sc) {
  if (!s || !sc) return BOWSHOCK_INVALID;
  if (sc->kind != BOWSHOCK_SCHEME_EXPLICIT && sc->kind != BOWSHOCK_SCHEME_IMPLICIT)
    return fail(s, BOWSHOCK_UNSUPPORTED, "only Scheme::Explicit and Scheme::Implicit are implemented on the GPU");
  if (sc->kind == BOWSHOCK_SCHEME_IMPLICIT && (sc->sub_iters < 1 || sc->sub_iters > 16 || !(sc->cfl0 > 0) || !(sc->cfl_max > 0)))
    return fail(s, BOWSHOCK_INVALID, "implicit parameters out of range");
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
  return from_arena(s, s->ar.set_counter(s->ar.d_ramp, 0, 0));
}

int bowshock_solver_set_viscous(bowshock_solver* s, const bowshock_viscous* v) {
  if (!s) return BOWSHOCK_INVALID;
  HostCase& h = s->ar.cases[0];
  if (v) {
    if (v->roughness != 0.0) return fail(s, BOWSHOCK_UNSUPPORTED, "rough walls are not implemented on this backend");
    if (!(v->re_c > 0 && v->sutherland > 0)) return fail(s, BOWSHOCK_INVALID, "re_c and sutherland must be positive");
    if (v->turbulence == BOWSHOCK_TURB_SST && h.scheme != BOWSHOCK_SCHEME_IMPLICIT)
      return fail(s, BOWSHOCK_UNSUPPORTED, "the SST model runs with the implicit scheme on this backend");
    h.viscous = true;
    h.turbulence = v->turbulence;
    h.wall_i_start = (long long)v->wall_i_start;
    h.re_c = v->re_c;
    h.sutherland = v->sutherland;
    h.roughness = 0;
  } else {
    h.viscous = false;
    h.turbulence = 0;
  }
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
  int rc = s->ar.run((long long)n, residual);
  if (rc) return from_arena(s, rc);
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
