"""`GpuSolver` over the B200 backend: the host-side mirror of the reference's GPU solver interface
(crates/bowshock-cfd/src/gpu/mod.rs:233-414), same method names, argument meaning and errors, calling the C ABI.

    s = GpuSolver.new(ni, nj, x, r, Config(...))        # GpuSolver::new
    s.set_block(...); s.set_scheme(...); s.set_viscous(...)
    residuals = s.run(50)                                # GpuSolver::run
    u = s.state_f64()                                    # GpuSolver::state_f64
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _ffi
from ._ffi import BowshockError

GAMMA = 1.4
LIM_FIRST_ORDER, LIM_MINMOD, LIM_VAN_ALBADA, LIM_VENKATAKRISHNAN = 0, 1, 2, 3
BC_FREESTREAM, BC_EXTRAPOLATE, BC_SLIPWALL, BC_CHARACTERISTIC, BC_PRESSURE_OUTFLOW = 0, 1, 2, 3, 4
SCHEME_EXPLICIT, SCHEME_SMOOTHED, SCHEME_MULTIGRID, SCHEME_IMPLICIT = 0, 1, 2, 3
DT_SUM, DT_MIN_DIRECTION = 0, 1
TURB_LAMINAR, TURB_SST = 0, 1


def freestream(mach: float):
    """gas.rs:41-43: rho = 1, c = 1, p = 1/gamma, u = Mach."""
    return (1.0, float(mach), 0.0, 1.0 / GAMMA)


@dataclass
class Config:  # solver.rs:40-48
    cfl: float = 0.5
    limiter: int = LIM_MINMOD
    freestream: tuple = freestream(0.5)
    bc: tuple = (BC_CHARACTERISTIC, BC_CHARACTERISTIC, BC_SLIPWALL, BC_CHARACTERISTIC)
    first_order_iters: int = 0

    def c(self):
        return _ffi.Config(self.cfl, self.limiter, (C.c_double * 4)(*self.freestream), (C.c_int32 * 4)(*self.bc),
                           int(self.first_order_iters))


@dataclass
class ImplicitParams:  # implicit.rs:59-84 (DEFAULT)
    cfl0: float = 1.0
    cfl_max: float = 30.0
    growth: float = 1.02
    dt_mode: int = DT_SUM
    lines: bool = True
    implicit_bc: bool = True
    sub_iters: int = 2
    roe: bool = True
    eps_fix: float = 0.1

    @staticmethod
    def viscous():  # implicit.rs:83
        return ImplicitParams(dt_mode=DT_MIN_DIRECTION, cfl_max=10.0, sub_iters=3)

    @staticmethod
    def rans():  # numerics.rs:245 (RANS_IMPLICIT)
        return ImplicitParams(dt_mode=DT_SUM, cfl_max=50.0, sub_iters=3)


EXPLICIT = "explicit"


@dataclass
class MgParams:  # solver.rs:123-140 (DEFAULT): FAS multigrid with the SSP-RK3 smoother
    levels: int = 6
    pre: int = 1
    post: int = 1
    gamma: int = 1
    coarsest: int = 4
    cfl_star: float = 0.0  # implicit residual smoothing of the smoother (MgParams::irs)
    implicit: "ImplicitParams | None" = None  # the line-implicit smoother (no counterpart in the reference) with these parameters
    relax: float = 1.0  # fraction of the prolongated correction applied
    cfl_scale: float = 1.0  # the implicit smoother's CFL numbers on level l times cfl_scale^l


@dataclass
class Smoothed:  # solver.rs:104-120 `Scheme::Smoothed(Irs)`: SSP-RK3 with implicit residual smoothing
    cfl_star: float = 2.0


@dataclass
class Viscous:  # solver.rs:164-176
    re_c: float
    sutherland: float
    turbulence: int = TURB_LAMINAR
    wall_i_start: int = 0
    roughness: float = 0.0


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class GpuSolver:
    """One case on the B200 backend (a case arena of one)."""

    def __init__(self, handle, ni, nj):
        self._h = handle
        self.ni, self.nj = ni, nj
        self._viscous = None

    # -------------------------------------------------------------- construction
    @classmethod
    def new(cls, ni: int, nj: int, x, r, cfg: Config, device: int = 0) -> "GpuSolver":
        lib = _ffi.load()
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1)
        if x.size != (ni + 1) * (nj + 1) or r.size != x.size:
            raise BowshockError(_ffi.INVALID, "node arrays must hold (ni+1)*(nj+1) entries")
        h = C.c_void_p()
        c = cfg.c()
        rc = lib.bowshock_solver_create(ni, nj, _dp(x), _dp(r), C.byref(c), device, C.byref(h))
        if rc:
            raise BowshockError(rc, "bowshock_solver_create failed (invalid grid / config, or no usable CUDA device)")
        return cls(h, ni, nj)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _ffi.load().bowshock_solver_destroy(h)
            self._h = None

    def _check(self, rc):
        if rc:
            msg = _ffi.load().bowshock_solver_last_error(self._h)
            raise BowshockError(rc, msg.decode() if msg else "")

    # -------------------------------------------------------------- configuration (gpu/mod.rs:279-362)
    def set_config(self, cfg: Config):
        c = cfg.c()
        self._check(_ffi.load().bowshock_solver_set_config(self._h, C.byref(c)))

    def set_low_mach(self, on: bool):
        self._check(_ffi.load().bowshock_solver_set_low_mach(self._h, int(bool(on))))

    def set_mg_fusion(self, on: bool):
        """Multigrid restriction folded into the coarse level's kernels (True, the default) or as separate transfer
        kernels in the reference's order (False); the same states."""
        self._check(_ffi.load().bowshock_solver_set_mg_fusion(self._h, int(bool(on))))

    def set_sst_coupling(self, coupled: bool):
        """False (default): the reference's loosely coupled SST lines; True: the 6x6 block lines (Arena.set_sst_coupling)."""
        self._check(_ffi.load().bowshock_solver_set_sst_coupling(self._h, int(bool(coupled))))

    def set_block(self, block):
        """`block`: None or (i_end, j_end, j_sting)."""
        if block is None:
            self._check(_ffi.load().bowshock_solver_set_block(self._h, None))
        else:
            b = _ffi.Block(*[int(v) for v in block])
            self._check(_ffi.load().bowshock_solver_set_block(self._h, C.byref(b)))

    def set_nozzle(self, nozzle):
        """`nozzle`: None or (j_end, state[4], turb[2])."""
        if nozzle is None:
            self._check(_ffi.load().bowshock_solver_set_nozzle(self._h, None))
        else:
            j_end, state, turb = nozzle
            n = _ffi.Nozzle(int(j_end), (C.c_double * 4)(*state), (C.c_double * 2)(*turb))
            self._check(_ffi.load().bowshock_solver_set_nozzle(self._h, C.byref(n)))

    def set_scheme(self, scheme):
        """`scheme`: EXPLICIT, Smoothed, MgParams or ImplicitParams."""
        if isinstance(scheme, str) and scheme == EXPLICIT:
            s = _ffi.Scheme(kind=SCHEME_EXPLICIT)
        elif isinstance(scheme, Smoothed):
            s = _ffi.Scheme(kind=SCHEME_SMOOTHED, cfl_star=scheme.cfl_star)
        elif isinstance(scheme, MgParams):
            s = _ffi.Scheme(kind=SCHEME_MULTIGRID, mg_levels=scheme.levels, mg_pre=scheme.pre, mg_post=scheme.post, mg_gamma=scheme.gamma,
                            mg_coarsest=scheme.coarsest, mg_cfl_star=scheme.cfl_star, mg_relax=scheme.relax, mg_cfl_scale=scheme.cfl_scale)
            if scheme.implicit is not None:
                p = scheme.implicit
                s.mg_implicit = 1
                s.cfl0, s.cfl_max, s.growth, s.dt_mode, s.lines = p.cfl0, p.cfl_max, p.growth, p.dt_mode, int(p.lines)
                s.implicit_bc, s.sub_iters, s.roe, s.eps_fix = int(p.implicit_bc), int(p.sub_iters), int(p.roe), p.eps_fix
        else:
            p = scheme
            s = _ffi.Scheme(SCHEME_IMPLICIT, p.cfl0, p.cfl_max, p.growth, p.dt_mode, int(p.lines), int(p.implicit_bc),
                            int(p.sub_iters), int(p.roe), p.eps_fix)
        self._check(_ffi.load().bowshock_solver_set_scheme(self._h, C.byref(s)))

    def set_viscous(self, v: Viscous | None):
        if v is None:
            self._check(_ffi.load().bowshock_solver_set_viscous(self._h, None))
        else:
            c = _ffi.Viscous(v.re_c, v.sutherland, v.turbulence, int(v.wall_i_start), v.roughness)
            self._check(_ffi.load().bowshock_solver_set_viscous(self._h, C.byref(c)))
        self._viscous = v

    # -------------------------------------------------------------- state (gpu/mod.rs:365-392)
    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
        if u.size != 4 * self.ni * self.nj:
            raise BowshockError(_ffi.INVALID, "state must hold ni*nj*4 values")
        self._check(_ffi.load().bowshock_solver_set_state(self._h, _dp(u)))

    def reset(self):
        self._check(_ffi.load().bowshock_solver_reset(self._h))

    def state_f64(self) -> np.ndarray:
        u = np.zeros(4 * self.ni * self.nj)
        self._check(_ffi.load().bowshock_solver_state(self._h, _dp(u)))
        return u.reshape(-1, 4)

    def turb_state(self):
        t = np.zeros(2 * self.ni * self.nj)
        m = np.zeros(self.ni * self.nj)
        self._check(_ffi.load().bowshock_solver_turb_state(self._h, _dp(t), _dp(m)))
        return t.reshape(-1, 2), m

    def set_turb(self, turb, mu_t):
        t = np.ascontiguousarray(turb, dtype=np.float64).reshape(-1)
        m = np.ascontiguousarray(mu_t, dtype=np.float64).reshape(-1)
        self._check(_ffi.load().bowshock_solver_set_turb(self._h, _dp(t), _dp(m)))

    @property
    def iter(self) -> int:
        v = C.c_uint64()
        self._check(_ffi.load().bowshock_solver_iter(self._h, C.byref(v)))
        return v.value

    def set_iter(self, it: int):
        self._check(_ffi.load().bowshock_solver_set_iter(self._h, int(it)))

    def restart_ramp(self):
        self._check(_ffi.load().bowshock_solver_restart_ramp(self._h))

    def set_ramp(self, k: int):
        """Continue the implicit CFL ramp from k iterations (state handed over mid-run)."""
        self._check(_ffi.load().bowshock_solver_set_ramp(self._h, int(k)))

    # -------------------------------------------------------------- iteration (gpu/mod.rs:396-413)
    def run(self, n: int) -> np.ndarray:
        out = np.zeros(n)
        self._check(_ffi.load().bowshock_solver_run(self._h, int(n), _dp(out)))
        return out

    def run_noalloc(self, n: int) -> np.ndarray:
        """`run` without device allocation (bowshock_solver_run_noalloc): for stepping from code that may not allocate
        device memory once the solver exists. The line solves keep their records in the library's static 64 MiB array,
        shared by all calls on the device, so calls overlapping on one GPU must be serialised."""
        out = np.zeros(n)
        self._check(_ffi.load().bowshock_solver_run_noalloc(self._h, int(n), _dp(out)))
        return out

    def eval_residual(self, compute_dt: bool = True):
        """`Solver::eval_residual` + `density_residual` of the current state: (res (n,4), dt (n), density residual)."""
        res = np.zeros(4 * self.ni * self.nj)
        dt = np.zeros(self.ni * self.nj)
        d = C.c_double()
        self._check(_ffi.load().bowshock_solver_eval_residual(self._h, int(compute_dt), _dp(res), _dp(dt), C.byref(d)))
        return res.reshape(-1, 4), dt, d.value

    PROFILE_GROUPS = ("prims", "viscous", "residual", "lines_i", "lines_j", "defect", "turbulence", "stage", "subst_i", "subst_j", "assemble",
                      "turb_lines", "transfer")

    def profile(self, n: int):
        """Per-kernel-group device time over n iterations launched one kernel at a time: {group: (ms, launches)}."""
        ms = np.zeros(len(self.PROFILE_GROUPS))
        cnt = (C.c_uint64 * len(self.PROFILE_GROUPS))()
        self._check(_ffi.load().bowshock_solver_profile(self._h, int(n), _dp(ms), cnt))
        return {g: (float(ms[k]), int(cnt[k])) for k, g in enumerate(self.PROFILE_GROUPS)}

    def turb_residual(self) -> float:
        d = C.c_double()
        self._check(_ffi.load().bowshock_solver_turb_residual(self._h, C.byref(d)))
        return d.value

    def read_boundary_into(self, u: np.ndarray):
        buf = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
        self._check(_ffi.load().bowshock_solver_read_boundary(self._h, _dp(buf)))
        u.reshape(-1)[:] = buf

    def base_cells(self, j_rows: int) -> np.ndarray:
        out = np.zeros(8 * j_rows)
        self._check(_ffi.load().bowshock_solver_base_cells(self._h, _dp(out)))
        return out.reshape(j_rows, 2, 4)

    # -------------------------------------------------------------- FP64 forces and the runner (engine/run.rs, gpu.rs)
    def forces(self, body) -> dict:
        """Force integration of the current state (engine/run.rs:188-313), FP64 on the device. `body`: case.Body."""
        f = _ffi.Forces()
        b = body.c()
        self._check(_ffi.load().bowshock_solver_forces(self._h, C.byref(b), C.byref(f)))
        return forces_dict(f, len(body.segments))

    def run_to_stop(self, body, numerics, wake, warm=False, r_ref=None, progress=None):
        """`GpuRunner::run_on` (engine/gpu.rs:86-169): iterate to the stop rules of engine/run.rs:105-170 in chunks of 50,
        then the forces of the final state. `progress(case, iteration, residual, monitor) -> bool` (False cancels)."""
        p = numerics.run_params(wake, warm, r_ref)
        out = _ffi.PointResult()
        hist = np.zeros(int(numerics.max_iter) + 64)
        b = body.c()
        cb = _ffi.PROGRESS_FN(lambda u, k, it, r, m: 0 if progress is None or progress(k, it, r, m) else 1)
        self._check(_ffi.load().bowshock_solver_run_to_stop(self._h, C.byref(b), C.byref(p), C.byref(out), _dp(hist), hist.size,
                                                            cb if progress else _ffi.PROGRESS_FN(0), None))
        return point_dict(out, len(body.segments), hist[: out.iters].copy())


STOP_REASONS = ["max iterations", "residual drop", "CD stationary", "base pressure stationary", "mean stationary",
                "non-finite residual", "cancelled"]


def forces_dict(f, nseg):
    return dict(cd_nose=f.cd_nose, cd_nose_cell=f.cd_nose_cell, cd_aft=list(f.cd_aft)[:nseg], cd_base=f.cd_base, cp_base=f.cp_base,
                cp_base_cell=f.cp_base_cell, cd_friction=f.cd_friction, y_plus_max=f.y_plus_max, cd_total=f.cd_total)


def point_dict(p, nseg, residual=None):
    d = dict(iters=p.iters, residual_peak=p.residual_peak, drop_orders=p.drop_orders, stop_reason=STOP_REASONS[p.stop_reason],
             last_monitor=p.last_monitor, cd_window=p.cd_window)
    d.update(forces_dict(p.forces, nseg))
    if residual is not None:
        d["residual"] = residual
    return d
