"""3D Euler on the B200 (include/bowshock_b200.h, `bowshock3_*`): the stability path of the reference
(crates/bowshock-cfd/src/solver3.rs + implicit3.rs behind `GpuSolver3`, driven by crates/bowshock-core/src/engine/run3.rs),
as a batch of cases (Mach number, incidence) on one shared revolved grid. `Case3` mirrors the reference's case3.rs: the 2D
sting grid of the body revolved over [0, pi] (grid3.rs:189-206), the axis upstream of the nose, `Numerics3::auto`."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _ffi
from ._ffi import BowshockError
from .case import WAKE_STING, Body, Case
from .solver import EXPLICIT, LIM_MINMOD, LIM_VAN_ALBADA, ImplicitParams

STOP3 = {0: "max iterations", 1: "residual drop", 2: "CN stationary", 5: "non-finite residual"}


class Config3C(C.Structure):  # bowshock3_config
    _fields_ = [("mach", C.c_double), ("alpha", C.c_double), ("cfl", C.c_double), ("limiter", C.c_int32), ("low_mach", C.c_int32),
                ("first_order_iters", C.c_uint64), ("scheme", _ffi.Scheme)]


class RunParams3C(C.Structure):  # bowshock3_run_params
    _fields_ = [("max_iter", C.c_uint64), ("rel_tol", C.c_double), ("window", C.c_uint64), ("x_max", C.c_double)]


class Result3C(C.Structure):  # bowshock3_result
    _fields_ = [("cn", C.c_double), ("ca", C.c_double), ("x_cp", C.c_double), ("iterations", C.c_uint64), ("stop_reason", C.c_int32),
                ("drop_orders", C.c_double)]


_P, _D, _U, _I = C.c_void_p, C.c_double, C.c_uint64, C.c_int
_dp = C.POINTER(C.c_double)
SIGNATURES3 = {
    "bowshock3_create": (_I, [_U, _U, _U, _dp, _dp, _dp, _U, _U, C.POINTER(Config3C), _I, C.POINTER(_P)]),
    "bowshock3_destroy": (None, [_P]),
    "bowshock3_last_error": (C.c_char_p, [_P]),
    "bowshock3_reset": (_I, [_P]),
    "bowshock3_set_solid": (_I, [_P, _U, C.POINTER(_U)]),
    "bowshock3_set_staging": (_I, [_P, _I]),
    "bowshock3_set_groups": (_I, [_P, _I]),
    "bowshock3_set_config": (_I, [_P, _U, C.POINTER(Config3C)]),
    "bowshock3_read_boundary": (_I, [_P, _U, _dp]),
    "bowshock3_profile": (_I, [_P, _U, _dp, C.POINTER(_U)]),
    "bowshock3_set_iter": (_I, [_P, _U, _U]),
    "bowshock3_set_state": (_I, [_P, _U, _dp]),
    "bowshock3_state": (_I, [_P, _U, _dp]),
    "bowshock3_run": (_I, [_P, _U, _dp]),
    "bowshock3_eval_residual": (_I, [_P, _U, _dp, _dp, _dp]),
    "bowshock3_forces": (_I, [_P, _D, _dp]),
    "bowshock3_forces_parts": (_I, [_P, _D, _D, _dp]),
    "bowshock3_solve": (_I, [_P, C.POINTER(RunParams3C), C.POINTER(Result3C)]),
    "bowshock3_last_ms_per_iter": (_I, [_P, _dp]),
}
_ready = False


def lib():
    global _ready
    L = _ffi.load()
    if not _ready:
        for name, (res, args) in SIGNATURES3.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _ready = True
    return L


def _p(a):
    return a.ctypes.data_as(_dp)


@dataclass
class Config3:
    """`Config3` (solver3.rs:44-55) of one case: free stream at (mach, alpha [rad]), explicit CFL, limiter, first-order
    start-up, low-Mach correction, scheme (EXPLICIT or an ImplicitParams)."""
    mach: float
    alpha: float = 0.0
    cfl: float = 0.5
    limiter: int = LIM_MINMOD
    first_order_iters: int = 0
    low_mach: bool = False
    scheme: object = field(default_factory=ImplicitParams)

    def c(self):
        s = self.scheme
        if s == EXPLICIT:
            sc = _ffi.Scheme(kind=0)
        else:
            sc = _ffi.Scheme(3, s.cfl0, s.cfl_max, s.growth, s.dt_mode, int(s.lines), int(s.implicit_bc), int(s.sub_iters), int(s.roe), s.eps_fix)
        return Config3C(self.mach, self.alpha, self.cfl, int(self.limiter), int(self.low_mach), int(self.first_order_iters), sc)


def revolve(x2, r2, nk, theta=None):
    """Nodes of the 2D grid (x, r) revolved about the x axis: (x, r sin theta_k, r cos theta_k), theta over [0, pi]
    (grid3.rs:189-206). Returns x, y, z of (nk+1)(nj+1)(ni+1) nodes."""
    x2 = np.asarray(x2, dtype=np.float64).reshape(-1)
    r2 = np.asarray(r2, dtype=np.float64).reshape(-1)
    th = np.pi * np.arange(nk + 1) / nk if theta is None else np.asarray(theta, dtype=np.float64)
    x = np.tile(x2, nk + 1)
    y = (np.sin(th)[:, None] * r2[None, :]).reshape(-1)
    z = (np.cos(th)[:, None] * r2[None, :]).reshape(-1)
    return x, y, z


class Batch3:
    """Cases on one shared 3D grid; each case its own free stream and numerics (one scheme per batch)."""

    def __init__(self, ni, nj, nk, x, y, z, axis_cells, configs, device=0):
        L = lib()
        self.ni, self.nj, self.nk = ni, nj, nk
        self.configs = list(configs)
        self._x, self._y, self._z = (np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (x, y, z))
        cfg = (Config3C * len(self.configs))(*[c.c() for c in self.configs])
        h = C.c_void_p()
        rc = L.bowshock3_create(ni, nj, nk, _p(self._x), _p(self._y), _p(self._z), axis_cells, len(self.configs), cfg, device, C.byref(h))
        if rc:
            raise BowshockError(rc, "bowshock3_create failed (invalid grid / configs, or no usable CUDA device)")
        self._h = h
        self.nb = len(self.configs)
        self.nc = ni * nj * nk

    def __del__(self):
        if getattr(self, "_h", None):
            lib().bowshock3_destroy(self._h)
            self._h = None

    def _check(self, rc):
        if rc:
            m = lib().bowshock3_last_error(self._h)
            raise BowshockError(rc, m.decode() if m else "")

    def reset(self):
        self._check(lib().bowshock3_reset(self._h))

    def set_solid(self, boxes):
        """Solid boxes of the shared grid (the fins; grid3.rs `SolidBox`): ((i0, i1), (j0, j1), (k0, k1)) half-open cell
        ranges each; resets every case to its free stream."""
        a = np.ascontiguousarray([v for bx in boxes for r in bx for v in r], dtype=np.uint64)
        self._check(lib().bowshock3_set_solid(self._h, len(boxes), a.ctypes.data_as(C.POINTER(_U)) if len(boxes) else None))

    def set_staging(self, on):
        """The first line pass staged through shared memory where the grid allows it (default on); same results."""
        self._check(lib().bowshock3_set_staging(self._h, int(bool(on))))

    def set_config(self, k, config):
        """GpuSolver3::set_config for case k (a Config3): the state is kept; a changed scheme restarts its CFL ramp."""
        c = config.c()
        self._check(lib().bowshock3_set_config(self._h, int(k), C.byref(c)))
        self.configs[k] = config

    PROFILE_GROUPS = ("prims", "flux", "residual", "assemble", "lines", "subst", "defect", "stage")

    def profile(self, n):
        """Per-kernel-group device time over n iterations launched one kernel at a time: {group: (ms, launches)}."""
        ms = np.zeros(len(self.PROFILE_GROUPS))
        cnt = (_U * len(self.PROFILE_GROUPS))()
        self._check(lib().bowshock3_profile(self._h, int(n), _p(ms), cnt))
        return {g: (float(ms[q]), int(cnt[q])) for q, g in enumerate(self.PROFILE_GROUPS)}

    def set_groups(self, groups):
        """Split the cases into 1 to 4 groups whose iterations run on streams of their own (the same states)."""
        self._check(lib().bowshock3_set_groups(self._h, int(groups)))

    def set_iter(self, it, ramp=None):
        self._check(lib().bowshock3_set_iter(self._h, int(it), int(it if ramp is None else ramp)))

    def set_state(self, k, u):
        a = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
        self._check(lib().bowshock3_set_state(self._h, int(k), _p(a)))

    def state(self, k):
        u = np.zeros(5 * self.nc)
        self._check(lib().bowshock3_state(self._h, int(k), _p(u)))
        return u.reshape(-1, 5)

    def read_boundary_into(self, k, u):
        """GpuSolver3::read_boundary_into: the force integration's cells of case k into u (ncell x 5), the rest untouched."""
        if u.shape != (self.nc, 5) or u.dtype != np.float64 or not u.flags.c_contiguous:
            raise ValueError("u must be a C-contiguous float64 array of shape (ncell, 5)")
        self._check(lib().bowshock3_read_boundary(self._h, int(k), _p(u)))

    def run(self, n):
        out = np.zeros(n * self.nb)
        self._check(lib().bowshock3_run(self._h, int(n), _p(out)))
        return out.reshape(n, self.nb)

    def eval_residual(self, k=0):
        res, dt, d = np.zeros(5 * self.nc), np.zeros(self.nc), C.c_double()
        self._check(lib().bowshock3_eval_residual(self._h, int(k), _p(res), _p(dt), C.byref(d)))
        return res.reshape(-1, 5), dt, d.value

    def forces(self, x_max):
        out = np.zeros(3 * self.nb)
        self._check(lib().bowshock3_forces(self._h, float(x_max), _p(out)))
        return [dict(cn=out[3 * k], ca=out[3 * k + 1], x_cp=out[3 * k + 2]) for k in range(self.nb)]

    PARTS = ("nose", "afterbody", "fin_sides", "fin_edges", "fin_tips")

    def forces_parts(self, x_max, x_nose):
        """run3.rs `breakdown_on`: per case {part: dict(cn, ca, x_cp)} for the parts of PARTS."""
        out = np.zeros(15 * self.nb)
        self._check(lib().bowshock3_forces_parts(self._h, float(x_max), float(x_nose), _p(out)))
        return [{p: dict(cn=out[15 * k + 3 * q], ca=out[15 * k + 3 * q + 1], x_cp=out[15 * k + 3 * q + 2]) for q, p in enumerate(self.PARTS)}
                for k in range(self.nb)]

    def solve(self, x_max, max_iter=8000, rel_tol=0.002, window=500):
        p = RunParams3C(int(max_iter), float(rel_tol), int(window), float(x_max))
        out = (Result3C * self.nb)()
        self._check(lib().bowshock3_solve(self._h, C.byref(p), out))
        return [dict(cn=r.cn, ca=r.ca, x_cp=r.x_cp, iterations=r.iterations, stop_reason=STOP3.get(r.stop_reason, "?"),
                     drop_orders=r.drop_orders) for r in out]

    def ms_per_iter(self):
        d = C.c_double()
        self._check(lib().bowshock3_last_ms_per_iter(self._h, C.byref(d)))
        return d.value


@dataclass
class Numerics3:
    """case3.rs:28-46 `Numerics3::auto`: van Albada + low-Mach below Mach 0.85, minmod above; the implicit defaults with
    cfl_max 10; 100 first-order iterations; 8000 << level iterations at most; CN stationary within 0.2 % over 500."""
    limiter: int
    low_mach: bool
    implicit: ImplicitParams
    first_order_iters: int = 100
    max_iter: int = 8000
    rel_tol: float = 0.002
    window: int = 500

    @staticmethod
    def auto(mach, level=0):
        sub = mach < 0.85
        return Numerics3(LIM_VAN_ALBADA if sub else LIM_MINMOD, sub, ImplicitParams(cfl_max=10.0), 100, 8000 << level)


@dataclass
class Case3:
    """case3.rs:50-82: one (Mach number, incidence [rad]) on a body, the 2D sting grid of `Case::new(.., Wake::Sting)`
    revolved with nk = 24 << level azimuthal cells."""
    mach: float
    alpha: float
    body: Body
    case2: Case
    nk: int
    numerics: Numerics3

    @staticmethod
    def new(mach, alpha, body: Body, level=0):
        c2 = Case.new(mach, body, level, WAKE_STING)
        return Case3(mach, alpha, body, c2, 24 << level, Numerics3.auto(mach, level))

    def config(self):
        n = self.numerics
        return Config3(self.mach, self.alpha, 0.5, n.limiter, n.first_order_iters, n.low_mach, n.implicit)

    def grid(self):
        """(ni, nj, nk, x, y, z, axis_cells, x_base)."""
        ni, nj, x2, r2, _ = self.case2.grid()
        x, y, z = revolve(x2, r2, self.nk)
        return ni, nj, self.nk, x, y, z, self.case2.grid_sting.n_up, self.body.x_base()


def batch_of(cases, device=0):
    """One Batch3 over cases that share their grid (same body and counts)."""
    ni, nj, nk, x, y, z, axis, x_base = cases[0].grid()
    return Batch3(ni, nj, nk, x, y, z, axis, [c.config() for c in cases], device), x_base


def lift_sweep_cases(alphas_deg=(0.0, 2.0, 4.0, 6.0, 8.0), machs=(0.8, 1.2, 2.5), ni=192, nj=64, nk=64):
    """The 3D normal-force sweep: the body of the SST workload (tangent-ogive nose 0.30 m x 0.10 m, 0.60 m cylinder,
    0.10 m boattail to 0.08 m), every incidence crossed with every Mach number, one shared revolved sting grid with its axial
    counts scaled to ni and nj radial cells, nk azimuthal cells over the half body."""
    from .sweep import _scale_counts
    body = Body(0, fineness=3.0, segments=((6.0, 0.0), (1.0, -0.1)))
    out = []
    for m in machs:
        for a in alphas_deg:
            c = Case3.new(m, math.radians(a), body)
            g = c.case2.grid_sting
            counts = _scale_counts([g.n_up, g.n_nose] + list(g.n_seg) + [g.n_ext], ni, 4)
            g.n_up, g.n_nose, g.n_seg, g.n_ext = counts[0], counts[1], counts[2:-1], counts[-1]
            g.nj = nj
            c.nk = nk
            out.append(c)
    return out
