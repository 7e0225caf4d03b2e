"""TEST INFRASTRUCTURE — ctypes binding of the oracle (oracle/_build/liboracle.so).

The oracle is an f64 C++ restatement of the reference CPU solver (crates/bowshock-cfd) and its engine layer
(crates/bowshock-core/src/engine). It is the checker of the CUDA backend and the timed CPU baseline; nothing in the
product imports this module. Its API mirrors the reference's `Solver` (crates/bowshock-cfd/src/solver.rs:197-676) and
`Case` / `run_on` (crates/bowshock-core/src/engine/case.rs, run.rs).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

# enums (oracle.hpp)
FIRST_ORDER, MINMOD, VAN_ALBADA, VENKATAKRISHNAN = 0, 1, 2, 3
BC_FREESTREAM, BC_EXTRAPOLATE, BC_SLIPWALL, BC_CHARACTERISTIC, BC_PRESSURE_OUTFLOW = 0, 1, 2, 3, 4
SCHEME_EXPLICIT, SCHEME_SMOOTHED, SCHEME_MULTIGRID, SCHEME_IMPLICIT = 0, 1, 2, 3
DT_SUM, DT_MIN_DIRECTION = 0, 1
TURB_LAMINAR, TURB_SST = 0, 1
NOSE_TANGENT_OGIVE, NOSE_CONE, NOSE_POWER, NOSE_PARABOLIC, NOSE_HAACK = 0, 1, 2, 3, 4
WAKE_STING, WAKE_BASE = 0, 1
STOP_REASONS = ["max iterations", "residual drop", "CD stationary", "base pressure stationary", "mean stationary",
                "non-finite residual", "cancelled"]
GAMMA = 1.4

F_U, F_RES, F_DT, F_W, F_FI, F_FJ, F_TURB, F_MUT, F_DWALL, F_MU, F_GRAD, F_X, F_R, F_VOL, F_AREA, F_XC, F_RC, F_FVI, F_FVJ = range(19)


class OrcConfig(C.Structure):
    _fields_ = [("cfl", C.c_double), ("limiter", C.c_int), ("fs", C.c_double * 4), ("bc", C.c_int * 4),
                ("first_order_iters", C.c_size_t)]


class OrcScheme(C.Structure):
    _fields_ = [("kind", C.c_int), ("cfl_star", C.c_double), ("mg_levels", C.c_size_t), ("mg_pre", C.c_size_t),
                ("mg_post", C.c_size_t), ("mg_gamma", C.c_size_t), ("mg_coarsest", C.c_size_t),
                ("mg_cfl_star", C.c_double), ("cfl0", C.c_double), ("cfl_max", C.c_double), ("growth", C.c_double),
                ("dt_mode", C.c_int), ("lines", C.c_int), ("implicit_bc", C.c_int), ("sub_iters", C.c_size_t),
                ("roe", C.c_int), ("eps_fix", C.c_double)]


class OrcBody(C.Structure):
    _fields_ = [("nose_kind", C.c_int), ("fineness", C.c_double), ("half_angle", C.c_double), ("param", C.c_double),
                ("nseg", C.c_int), ("seg_length", C.c_double * 8), ("seg_slope", C.c_double * 8),
                ("sting_radius", C.c_double)]


class OrcBaseGrid(C.Structure):
    _fields_ = [("x_up", C.c_double), ("x_down", C.c_double), ("r_far", C.c_double), ("n_up", C.c_size_t),
                ("n_nose", C.c_size_t), ("n_seg", C.c_size_t * 8), ("n_wake", C.c_size_t), ("n_sting", C.c_size_t),
                ("n_gap", C.c_size_t), ("nj_out", C.c_size_t), ("dx_tip", C.c_double), ("dr_wall", C.c_double),
                ("gap_one_sided", C.c_int)]


class OrcStingGrid(C.Structure):
    _fields_ = [("x_up", C.c_double), ("x_down", C.c_double), ("r_far", C.c_double), ("n_up", C.c_size_t),
                ("n_nose", C.c_size_t), ("n_seg", C.c_size_t * 8), ("n_ext", C.c_size_t), ("nj", C.c_size_t),
                ("dx_tip", C.c_double), ("dr_wall", C.c_double)]


class OrcNumerics(C.Structure):
    _fields_ = [("cfl", C.c_double), ("limiter", C.c_int), ("low_mach", C.c_int), ("scheme", OrcScheme),
                ("first_order_iters", C.c_size_t), ("max_iter", C.c_size_t), ("min_iter", C.c_size_t),
                ("drop_orders", C.c_double), ("outflow", C.c_int), ("monitor_window", C.c_size_t),
                ("has_monitor_tol", C.c_int), ("monitor_tol", C.c_double), ("has_mean_window", C.c_int),
                ("mean_window", C.c_size_t), ("has_drag_rel_tol", C.c_int), ("drag_rel_tol", C.c_double)]


class OrcCase(C.Structure):
    _fields_ = [("mach", C.c_double), ("body", OrcBody), ("wake", C.c_int), ("grid_base", OrcBaseGrid),
                ("grid_sting", OrcStingGrid), ("numerics", OrcNumerics), ("has_viscous", C.c_int),
                ("re_c", C.c_double), ("sutherland", C.c_double), ("turbulence", C.c_int),
                ("wall_i_start", C.c_size_t), ("roughness", C.c_double)]


class OrcPointResult(C.Structure):
    _fields_ = [("iters", C.c_size_t), ("residual_peak", C.c_double), ("drop_orders", C.c_double),
                ("stop_reason", C.c_int), ("cd_nose", C.c_double), ("cd_nose_cell", C.c_double),
                ("cd_aft", C.c_double * 8), ("cd_base", C.c_double), ("cd_friction", C.c_double),
                ("cd_total", C.c_double), ("cp_base", C.c_double), ("cp_base_cell", C.c_double),
                ("y_plus_max", C.c_double), ("farfield_dp", C.c_double), ("min_rho", C.c_double),
                ("min_p", C.c_double), ("m_max", C.c_double), ("m_wall_max", C.c_double), ("cd_window", C.c_double)]


def build():
    """Compile the oracle with its Makefile (oracle/_build)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        D, P, S, I = C.c_double, C.c_void_p, C.c_size_t, C.c_int
        dp = C.POINTER(C.c_double)
        sig = {
            "orc_physical_flux": (None, [dp, D, D, dp]),
            "orc_hllc": (None, [dp, dp, D, D, dp]),
            "orc_rusanov": (None, [dp, dp, D, D, dp]),
            "orc_shock_weight": (D, [D, D]),
            "orc_limited_slope": (D, [D, D, I]),
            "orc_face_flux_lm": (None, [dp, dp, dp, dp, I, D, D, I, dp]),
            "orc_face_flux": (None, [dp, dp, dp, dp, I, D, D, dp]),
            "orc_low_mach_states": (None, [dp, dp, D, D, dp, dp]),
            "orc_regime": (I, [dp, D, D]),
            "orc_characteristic_ghost": (I, [dp, dp, D, D, dp]),
            "orc_pressure_outflow_ghost": (None, [D, dp, D, D, dp]),
            "orc_flux_jacobian": (None, [dp, D, D, dp]),
            "orc_abs_jacobian": (None, [dp, dp, D, D, D, dp]),
            "orc_inv4": (None, [dp, dp]),
            "orc_mm4": (None, [dp, dp, dp]),
            "orc_block_thomas": (None, [S, dp, dp, dp, dp]),
            "orc_aupoix_wall": (None, [D, D, D, D, dp]),
            "orc_geometric_offsets": (None, [D, D, S, dp]),
            "orc_two_sided_nodes": (None, [D, S, D, dp]),
            "orc_isa": (I, [D, dp]),
            "orc_solver_new": (P, [S, S, dp, dp, C.POINTER(OrcConfig), C.c_char_p, S]),
            "orc_solver_free": (None, [P]),
            "orc_solver_get_config": (None, [P, C.POINTER(OrcConfig)]),
            "orc_solver_set_config": (None, [P, C.POINTER(OrcConfig)]),
            "orc_solver_set_block": (I, [P, I, S, S, S, C.c_char_p, S]),
            "orc_solver_get_block": (I, [P, C.POINTER(C.c_size_t)]),
            "orc_solver_set_low_mach": (None, [P, I]),
            "orc_solver_set_scheme": (I, [P, C.POINTER(OrcScheme), C.c_char_p, S]),
            "orc_solver_mg_levels": (S, [P]),
            "orc_solver_set_viscous": (I, [P, I, D, D, I, S, D, C.c_char_p, S]),
            "orc_solver_set_nozzle": (I, [P, I, S, dp, dp, C.c_char_p, S]),
            "orc_solver_step": (D, [P]),
            "orc_solver_steps": (None, [P, S, dp]),
            "orc_solver_eval_residual": (None, [P, I]),
            "orc_solver_density_residual": (D, [P]),
            "orc_solver_dims": (None, [P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
            "orc_solver_iter": (S, [P]),
            "orc_solver_set_iter": (None, [P, S]),
            "orc_solver_restart_ramp": (None, [P]),
            "orc_solver_n_active": (S, [P]),
            "orc_solver_turb_residual": (D, [P]),
            "orc_solver_field_len": (S, [P, I]),
            "orc_solver_get": (None, [P, I, dp]),
            "orc_solver_set": (None, [P, I, dp]),
            "orc_case_new": (I, [D, C.POINTER(OrcBody), C.c_uint, I, C.POINTER(OrcCase)]),
            "orc_case_viscous": (I, [D, C.POINTER(OrcBody), C.c_uint, I, D, D, D, C.POINTER(OrcCase)]),
            "orc_numerics_preset": (None, [I, D, C.c_uint, I, C.POINTER(OrcNumerics)]),
            "orc_case_build_solver": (P, [C.POINTER(OrcCase), C.c_char_p, S]),
            "orc_run_on": (I, [C.POINTER(OrcCase), P, I, D, C.POINTER(OrcPointResult), dp, S]),
            "orc_finish": (None, [C.POINTER(OrcCase), P, C.POINTER(OrcPointResult)]),
            "orc_monitor": (D, [C.POINTER(OrcCase), P]),
            "orc_sizeof_case": (S, []),
            "orc_sizeof_result": (S, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        assert L.orc_sizeof_case() == C.sizeof(OrcCase), "OrcCase layout mismatch"
        assert L.orc_sizeof_result() == C.sizeof(OrcPointResult), "OrcPointResult layout mismatch"
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _vec(v, n=4) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(n))


# ------------------------------------------------------------------ point kernels
def physical_flux(w, nx, nr):
    o = np.zeros(4)
    lib().orc_physical_flux(_dp(_vec(w)), nx, nr, _dp(o))
    return o


def hllc(wl, wr, nx, nr):
    o = np.zeros(4)
    lib().orc_hllc(_dp(_vec(wl)), _dp(_vec(wr)), nx, nr, _dp(o))
    return o


def rusanov(wl, wr, nx, nr):
    o = np.zeros(4)
    lib().orc_rusanov(_dp(_vec(wl)), _dp(_vec(wr)), nx, nr, _dp(o))
    return o


def shock_weight(pl, pr):
    return lib().orc_shock_weight(pl, pr)


def limited_slope(a, b, lim):
    return lib().orc_limited_slope(a, b, lim)


def face_flux(m2, m1, p0, p1, lim, nx, nr):
    o = np.zeros(4)
    lib().orc_face_flux(_dp(_vec(m2)), _dp(_vec(m1)), _dp(_vec(p0)), _dp(_vec(p1)), lim, nx, nr, _dp(o))
    return o


def face_flux_lm(m2, m1, p0, p1, lim, nx, nr, low_mach):
    o = np.zeros(4)
    lib().orc_face_flux_lm(_dp(_vec(m2)), _dp(_vec(m1)), _dp(_vec(p0)), _dp(_vec(p1)), lim, nx, nr, int(low_mach), _dp(o))
    return o


def low_mach_states(l, r, nx, nr):
    a, b = np.zeros(4), np.zeros(4)
    lib().orc_low_mach_states(_dp(_vec(l)), _dp(_vec(r)), nx, nr, _dp(a), _dp(b))
    return a, b


def regime(w, nx, nr):
    return lib().orc_regime(_dp(_vec(w)), nx, nr)


def characteristic_ghost(fs, interior, nx, nr):
    o = np.zeros(4)
    reg = lib().orc_characteristic_ghost(_dp(_vec(fs)), _dp(_vec(interior)), nx, nr, _dp(o))
    return o, reg


def pressure_outflow_ghost(p_back, interior, nx, nr):
    o = np.zeros(4)
    lib().orc_pressure_outflow_ghost(p_back, _dp(_vec(interior)), nx, nr, _dp(o))
    return o


def flux_jacobian(w, nx, nr):
    o = np.zeros(16)
    lib().orc_flux_jacobian(_dp(_vec(w)), nx, nr, _dp(o))
    return o.reshape(4, 4)


def abs_jacobian(wl, wr, nx, nr, eps_fix):
    o = np.zeros(16)
    lib().orc_abs_jacobian(_dp(_vec(wl)), _dp(_vec(wr)), nx, nr, eps_fix, _dp(o))
    return o.reshape(4, 4)


def inv4(m):
    o = np.zeros(16)
    lib().orc_inv4(_dp(_vec(m, 16)), _dp(o))
    return o.reshape(4, 4)


def block_thomas(lo, d, up, rhs):
    lo, d, up = (np.ascontiguousarray(a, dtype=np.float64) for a in (lo, d, up))
    x = np.ascontiguousarray(rhs, dtype=np.float64).copy()
    lib().orc_block_thomas(x.shape[0], _dp(lo), _dp(d), _dp(up), _dp(x))
    return x


def aupoix_wall(nu, speed, d, ks):
    o = np.zeros(3)
    lib().orc_aupoix_wall(nu, speed, d, ks, _dp(o))
    return o


def geometric_offsets(first, length, n):
    o = np.zeros(n + 1)
    lib().orc_geometric_offsets(first, length, n, _dp(o))
    return o


def two_sided_nodes(length, n, dx):
    o = np.zeros(n + 1)
    lib().orc_two_sided_nodes(length, n, dx, _dp(o))
    return o


def isa(altitude_m):
    o = np.zeros(5)
    if lib().orc_isa(altitude_m, _dp(o)):
        raise ValueError(f"altitude {altitude_m} m outside the ISA range")
    return dict(temperature_k=o[0], pressure_pa=o[1], density=o[2], sound_speed=o[3], viscosity=o[4])


def freestream(mach):
    return np.array([1.0, mach, 0.0, 1.0 / GAMMA])


def prim_to_cons(w):
    w = np.asarray(w, dtype=np.float64)
    rho, u, v, p = w[..., 0], w[..., 1], w[..., 2], w[..., 3]
    return np.stack([rho, rho * u, rho * v, p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v)], axis=-1)


def cons_to_prim(q):
    q = np.asarray(q, dtype=np.float64)
    rho = q[..., 0]
    u = q[..., 1] / rho
    v = q[..., 2] / rho
    p = (GAMMA - 1.0) * (q[..., 3] - 0.5 * rho * (u * u + v * v))
    return np.stack([rho, u, v, p], axis=-1)


# ------------------------------------------------------------------ schemes
def implicit_params(**kw) -> OrcScheme:
    """`Scheme::Implicit(ImplicitParams { .. })`, defaults from implicit.rs:79-80."""
    s = OrcScheme(kind=SCHEME_IMPLICIT, cfl0=1.0, cfl_max=30.0, growth=1.02, dt_mode=DT_SUM, lines=1, implicit_bc=1,
                  sub_iters=2, roe=1, eps_fix=0.1, mg_levels=6, mg_pre=1, mg_post=1, mg_gamma=1, mg_coarsest=4)
    for k, v in kw.items():
        setattr(s, k, int(v) if isinstance(v, bool) else v)
    return s


def implicit_viscous(**kw) -> OrcScheme:
    """`ImplicitParams::VISCOUS` (implicit.rs:83)."""
    base = dict(dt_mode=DT_MIN_DIRECTION, cfl_max=10.0, sub_iters=3)
    base.update(kw)
    return implicit_params(**base)


def explicit_scheme() -> OrcScheme:
    return OrcScheme(kind=SCHEME_EXPLICIT)


def multigrid_scheme(levels=6, pre=1, post=1, gamma=1, coarsest=4, cfl_star=0.0) -> OrcScheme:
    return OrcScheme(kind=SCHEME_MULTIGRID, mg_levels=levels, mg_pre=pre, mg_post=post, mg_gamma=gamma,
                     mg_coarsest=coarsest, mg_cfl_star=cfl_star)


# ------------------------------------------------------------------ solver
class Solver:
    """The reference's `Solver` (solver.rs:197-676) over the oracle."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_nodes(cls, ni, nj, x, r, cfl=0.5, limiter=MINMOD, freestream_=None, bc=(3, 3, 2, 3), first_order_iters=0):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1)
        assert x.size == (ni + 1) * (nj + 1)
        cfg = OrcConfig(cfl=cfl, limiter=limiter, fs=(C.c_double * 4)(*(freestream_ if freestream_ is not None else freestream(0.5))),
                        bc=(C.c_int * 4)(*bc), first_order_iters=first_order_iters)
        err = C.create_string_buffer(256)
        h = lib().orc_solver_new(ni, nj, _dp(x), _dp(r), C.byref(cfg), err, 256)
        if not h:
            raise ValueError(err.value.decode())
        return cls(h)

    @classmethod
    def from_case(cls, case: OrcCase):
        err = C.create_string_buffer(256)
        h = lib().orc_case_build_solver(C.byref(case), err, 256)
        if not h:
            raise ValueError(err.value.decode())
        return cls(h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_solver_free(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @property
    def dims(self):
        ni, nj = C.c_size_t(), C.c_size_t()
        lib().orc_solver_dims(self._h, C.byref(ni), C.byref(nj))
        return ni.value, nj.value

    @property
    def config(self) -> OrcConfig:
        c = OrcConfig()
        lib().orc_solver_get_config(self._h, C.byref(c))
        return c

    def set_config(self, c: OrcConfig):
        lib().orc_solver_set_config(self._h, C.byref(c))

    def set_block(self, block):
        err = C.create_string_buffer(256)
        if block is None:
            rc = lib().orc_solver_set_block(self._h, 0, 0, 0, 0, err, 256)
        else:
            rc = lib().orc_solver_set_block(self._h, 1, *block, err, 256)
        if rc:
            raise ValueError(err.value.decode())

    @property
    def block(self):
        b = (C.c_size_t * 3)()
        return tuple(b) if lib().orc_solver_get_block(self._h, b) else None

    def set_low_mach(self, on=True):
        lib().orc_solver_set_low_mach(self._h, int(on))

    def set_scheme(self, s: OrcScheme) -> int:
        err = C.create_string_buffer(256)
        rc = lib().orc_solver_set_scheme(self._h, C.byref(s), err, 256)
        if rc < 0:
            raise ValueError(err.value.decode())
        return lib().orc_solver_mg_levels(self._h)

    def set_viscous(self, v):
        """`v`: None or dict(re_c, sutherland, turbulence, wall_i_start, roughness)."""
        err = C.create_string_buffer(256)
        if v is None:
            rc = lib().orc_solver_set_viscous(self._h, 0, 0, 0, 0, 0, 0, err, 256)
        else:
            rc = lib().orc_solver_set_viscous(self._h, 1, v["re_c"], v["sutherland"], v.get("turbulence", TURB_LAMINAR),
                                              v.get("wall_i_start", 0), v.get("roughness", 0.0), err, 256)
        if rc:
            raise ValueError(err.value.decode())

    def set_nozzle(self, j_end, state, turb):
        err = C.create_string_buffer(256)
        st, tb = _vec(state), _vec(turb, 2)
        if lib().orc_solver_set_nozzle(self._h, 1, j_end, _dp(st), _dp(tb), err, 256):
            raise ValueError(err.value.decode())

    def step(self) -> float:
        return lib().orc_solver_step(self._h)

    def steps(self, n) -> np.ndarray:
        o = np.zeros(n)
        lib().orc_solver_steps(self._h, n, _dp(o))
        return o

    def eval_residual(self, compute_dt=True):
        lib().orc_solver_eval_residual(self._h, int(compute_dt))

    def density_residual(self):
        return lib().orc_solver_density_residual(self._h)

    @property
    def iter(self):
        return lib().orc_solver_iter(self._h)

    @iter.setter
    def iter(self, v):
        lib().orc_solver_set_iter(self._h, v)

    def restart_ramp(self):
        lib().orc_solver_restart_ramp(self._h)

    @property
    def n_active(self):
        return lib().orc_solver_n_active(self._h)

    @property
    def turb_residual(self):
        return lib().orc_solver_turb_residual(self._h)

    def get(self, field) -> np.ndarray:
        n = lib().orc_solver_field_len(self._h, field)
        o = np.zeros(n)
        if n:
            lib().orc_solver_get(self._h, field, _dp(o))
        return o

    def set(self, field, values):
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        assert v.size == lib().orc_solver_field_len(self._h, field)
        lib().orc_solver_set(self._h, field, _dp(v))

    # convenience views
    @property
    def u(self):
        return self.get(F_U).reshape(-1, 4)

    @u.setter
    def u(self, v):
        self.set(F_U, v)

    @property
    def res(self):
        return self.get(F_RES).reshape(-1, 4)

    @property
    def dt(self):
        return self.get(F_DT)

    @property
    def turb(self):
        return self.get(F_TURB).reshape(-1, 2)

    @turb.setter
    def turb(self, v):
        self.set(F_TURB, v)

    @property
    def mu_t(self):
        return self.get(F_MUT)

    @mu_t.setter
    def mu_t(self, v):
        self.set(F_MUT, v)

    @property
    def dwall(self):
        return self.get(F_DWALL)

    @property
    def nodes(self):
        return self.get(F_X), self.get(F_R)


# ------------------------------------------------------------------ case layer
def body(nose_kind=NOSE_TANGENT_OGIVE, fineness=3.0, half_angle=0.0, param=0.0, segments=((6.0, 0.0),), sting_radius=0.0):
    b = OrcBody(nose_kind=nose_kind, fineness=fineness, half_angle=half_angle, param=param, nseg=len(segments),
                sting_radius=sting_radius)
    for k, (length, slope) in enumerate(segments):
        b.seg_length[k] = length
        b.seg_slope[k] = slope
    return b


def case_new(mach, b: OrcBody, level=0, wake=WAKE_STING) -> OrcCase:
    c = OrcCase()
    lib().orc_case_new(mach, C.byref(b), level, wake, C.byref(c))
    return c


def case_viscous(mach, b: OrcBody, level, wake, re_c, sutherland, mach_max) -> OrcCase:
    c = OrcCase()
    lib().orc_case_viscous(mach, C.byref(b), level, wake, re_c, sutherland, mach_max, C.byref(c))
    return c


def numerics_preset(which: str, mach=0.5, level=0, wake=WAKE_STING) -> OrcNumerics:
    n = OrcNumerics()
    lib().orc_numerics_preset({"subsonic": 0, "transonic": 1, "auto": 2, "viscous": 3}[which], mach, level, wake, C.byref(n))
    return n


@dataclass
class PointResult:
    iters: int
    residual: np.ndarray
    residual_peak: float
    drop_orders: float
    stop_reason: str
    cd_nose: float
    cd_aft: list
    cd_base: float
    cd_friction: float
    cd_total: float
    cp_base: float
    y_plus_max: float
    farfield_dp: float
    min_rho: float
    min_p: float
    m_max: float
    cd_window: float = float("nan")


def _result(p: OrcPointResult, residual, nseg):
    return PointResult(iters=p.iters, residual=residual, residual_peak=p.residual_peak, drop_orders=p.drop_orders,
                       stop_reason=STOP_REASONS[p.stop_reason], cd_nose=p.cd_nose, cd_aft=list(p.cd_aft)[:nseg],
                       cd_base=p.cd_base, cd_friction=p.cd_friction, cd_total=p.cd_total, cp_base=p.cp_base,
                       y_plus_max=p.y_plus_max, farfield_dp=p.farfield_dp, min_rho=p.min_rho, min_p=p.min_p,
                       m_max=p.m_max, cd_window=p.cd_window)


def run_on(case: OrcCase, s: Solver, warm=False, r_ref=None) -> PointResult:
    """`run_on` (run.rs:44-89): iterate to the stop rule, post-process."""
    cap = case.numerics.max_iter
    hist = np.zeros(cap)
    p = OrcPointResult()
    lib().orc_run_on(C.byref(case), s.handle, int(warm), -1.0 if r_ref is None else r_ref, C.byref(p), _dp(hist), cap)
    return _result(p, hist[: p.iters].copy(), case.body.nseg)


def finish(case: OrcCase, s: Solver) -> PointResult:
    """Post-processing of the current state (run.rs:316-419)."""
    p = OrcPointResult()
    lib().orc_finish(C.byref(case), s.handle, C.byref(p))
    return _result(p, np.zeros(0), case.body.nseg)


def monitor(case: OrcCase, s: Solver) -> float:
    return lib().orc_monitor(C.byref(case), s.handle)


# ------------------------------------------------------------------ 3D Euler (solver3.cpp)
class OrcImplicitParams(C.Structure):  # orc::ImplicitParams
    _fields_ = [("cfl0", C.c_double), ("cfl_max", C.c_double), ("growth", C.c_double), ("dt_mode", C.c_int), ("lines", C.c_bool),
                ("implicit_bc", C.c_bool), ("sub_iters", C.c_size_t), ("roe", C.c_bool), ("eps_fix", C.c_double)]


class Orc3Result(C.Structure):
    _fields_ = [("cn", C.c_double), ("ca", C.c_double), ("x_cp", C.c_double), ("iterations", C.c_uint64), ("stop_reason", C.c_int32),
                ("drop_orders", C.c_double)]


STOP3 = {0: "max iterations", 1: "residual drop", 2: "CN stationary", 5: "non-finite residual"}
_lib3_ready = False


def lib3():
    global _lib3_ready
    L = lib()
    if not _lib3_ready:
        D, P, S, I, U = C.c_double, C.c_void_p, C.c_size_t, C.c_int, C.c_uint64
        dp = C.POINTER(C.c_double)
        sig = {
            "orc3_new": (P, [U, U, dp, dp, U, dp, U, D, D, I, U, I, I, C.POINTER(OrcImplicitParams), D, C.c_char_p, U]),
            "orc3_free": (None, [P]),
            "orc3_dims": (None, [P, C.POINTER(U), C.POINTER(U), C.POINTER(U)]),
            "orc3_get": (U, [P, I, dp]),
            "orc3_set_state": (None, [P, dp]),
            "orc3_set_iter": (None, [P, U, U]),
            "orc3_eval_residual": (D, [P, D]),
            "orc3_steps": (None, [P, U, dp]),
            "orc3_forces": (None, [P, D, D, dp]),
            "orc3_run": (None, [P, D, D, U, D, U, C.POINTER(Orc3Result)]),
            "orc3_face_flux": (None, [dp, dp, dp, dp, I, dp, dp, I, dp]),
            "orc3_hllc": (None, [dp, dp, dp, dp]),
            "orc3_physical_flux": (None, [dp, dp, dp]),
            "orc3_char_ghost": (None, [dp, dp, dp, dp]),
            "orc3_flux_jacobian": (None, [dp, dp, dp]),
            "orc3_abs_jacobian": (None, [dp, dp, dp, D, dp]),
            "orc3_inv5": (None, [dp, dp]),
            "orc3_block_thomas5": (None, [U, dp, dp, dp, dp]),
            "orc3_reflection": (None, [dp, dp]),
            "orc3_set_solid": (None, [P, U, C.POINTER(U)]),
            "orc3_face_fluxes": (U, [P, I, dp]),
            "orc3_forces_parts": (None, [P, D, D, D, dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib3_ready = True
    return L


def face_flux3(m2, m1, p0, p1, lim, n, rot, low_mach=False):
    out = np.zeros(5)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (m2, m1, p0, p1, n, rot)]
    lib3().orc3_face_flux(_dp(a[0]), _dp(a[1]), _dp(a[2]), _dp(a[3]), int(lim), _dp(a[4]), _dp(a[5]), int(low_mach), _dp(out))
    return out


def hllc3(wl, wr, n):
    out = np.zeros(5)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (wl, wr, n)]
    lib3().orc3_hllc(_dp(a[0]), _dp(a[1]), _dp(a[2]), _dp(out))
    return out


def physical_flux3(w, n):
    out = np.zeros(5)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (w, n)]
    lib3().orc3_physical_flux(_dp(a[0]), _dp(a[1]), _dp(out))
    return out


def characteristic_ghost3(fs, interior, n):
    out = np.zeros(5)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (fs, interior, n)]
    lib3().orc3_char_ghost(_dp(a[0]), _dp(a[1]), _dp(a[2]), _dp(out))
    return out


def flux_jacobian3(w, n):
    out = np.zeros(25)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (w, n)]
    lib3().orc3_flux_jacobian(_dp(a[0]), _dp(a[1]), _dp(out))
    return out.reshape(5, 5)


def abs_jacobian3(wl, wr, n, eps_fix):
    out = np.zeros(25)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (wl, wr, n)]
    lib3().orc3_abs_jacobian(_dp(a[0]), _dp(a[1]), _dp(a[2]), eps_fix, _dp(out))
    return out.reshape(5, 5)


def inv5(m):
    out = np.zeros(25)
    a = np.ascontiguousarray(m, dtype=np.float64)
    lib3().orc3_inv5(_dp(a), _dp(out))
    return out.reshape(5, 5)


def reflection3(n):
    out = np.zeros(25)
    a = np.ascontiguousarray(n, dtype=np.float64)
    lib3().orc3_reflection(_dp(a), _dp(out))
    return out.reshape(5, 5)


def block_thomas5(lo, d, up, rhs):
    lo, d, up = (np.ascontiguousarray(a, dtype=np.float64) for a in (lo, d, up))
    x = np.ascontiguousarray(rhs, dtype=np.float64).copy()
    lib3().orc3_block_thomas5(x.shape[0], _dp(lo), _dp(d), _dp(up), _dp(x))
    return x


def prim_to_cons3(w):
    w = np.asarray(w, dtype=np.float64)
    rho, u, v, ww, p = (w[..., k] for k in range(5))
    return np.stack([rho, rho * u, rho * v, rho * ww, p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v + ww * ww)], axis=-1)


def cons_to_prim3(q):
    q = np.asarray(q, dtype=np.float64)
    rho = q[..., 0]
    u, v, ww = q[..., 1] / rho, q[..., 2] / rho, q[..., 3] / rho
    p = (GAMMA - 1.0) * (q[..., 4] - 0.5 * rho * (u * u + v * v + ww * ww))
    return np.stack([rho, u, v, ww, p], axis=-1)


def freestream3(mach, alpha):
    return np.array([1.0, mach * np.cos(alpha), 0.0, mach * np.sin(alpha), 1.0 / GAMMA])


def implicit3_params(**kw):
    """`ImplicitParams::DEFAULT` (implicit.rs:79-80) with overrides."""
    p = OrcImplicitParams(cfl0=1.0, cfl_max=30.0, growth=1.02, dt_mode=DT_SUM, lines=True, implicit_bc=True, sub_iters=2, roe=True, eps_fix=0.1)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Solver3:
    """`Solver3` on a revolved 2D grid (grid3.rs:189-206): nodes (ni+1)(nj+1) of x, r; theta: nk+1 angles in [0, pi]."""

    def __init__(self, ni, nj, x2, r2, nk, theta, axis_cells, mach, alpha, limiter=MINMOD, first_order_iters=0, low_mach=False,
                 implicit=True, params=None, cfl=0.5):
        x2 = np.ascontiguousarray(x2, dtype=np.float64).reshape(-1)
        r2 = np.ascontiguousarray(r2, dtype=np.float64).reshape(-1)
        th = np.ascontiguousarray(theta, dtype=np.float64)
        err = C.create_string_buffer(256)
        p = params if params is not None else implicit3_params()
        self._h = lib3().orc3_new(ni, nj, _dp(x2), _dp(r2), nk, _dp(th), axis_cells, mach, alpha, int(limiter), first_order_iters,
                                  int(low_mach), int(implicit), C.byref(p), cfl, err, 256)
        if not self._h:
            raise ValueError(err.value.decode())
        self.mach, self.alpha = mach, alpha
        self.dims = (ni, nj, nk)

    def __del__(self):
        if getattr(self, "_h", None):
            lib3().orc3_free(self._h)
            self._h = None

    def _get(self, field):
        n = lib3().orc3_get(self._h, field, None)
        out = np.zeros(n)
        lib3().orc3_get(self._h, field, _dp(out))
        return out

    @property
    def u(self):
        return self._get(0).reshape(-1, 5)

    @u.setter
    def u(self, v):
        a = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        lib3().orc3_set_state(self._h, _dp(a))

    @property
    def res(self):
        return self._get(1).reshape(-1, 5)

    @property
    def dt(self):
        return self._get(2)

    @property
    def vol(self):
        return self._get(3)

    @property
    def xc(self):
        return self._get(4).reshape(-1, 3)

    def faces(self, fam):
        """(n, area, centroid) per face of family 0 / 1 / 2 (i / j / k)."""
        f = self._get(5 + fam).reshape(-1, 7)
        return f[:, :3], f[:, 3], f[:, 4:]

    def set_iter(self, it, ramp=None):
        lib3().orc3_set_iter(self._h, it, it if ramp is None else ramp)

    def set_solid(self, boxes):
        """Solid boxes (grid3.rs:17-24 `SolidBox`): ((i0, i1), (j0, j1), (k0, k1)) half-open cell ranges each."""
        a = np.ascontiguousarray([v for b in boxes for r in b for v in r], dtype=np.uint64)
        lib3().orc3_set_solid(self._h, len(boxes), a.ctypes.data_as(C.POINTER(C.c_uint64)))

    def face_fluxes(self, fam):
        """Face fluxes (per unit area, 5 per face) of family 0 / 1 / 2 from the last residual evaluation."""
        n = lib3().orc3_face_fluxes(self._h, fam, None)
        out = np.zeros(n)
        lib3().orc3_face_fluxes(self._h, fam, _dp(out))
        return out.reshape(-1, 5)

    def eval_residual(self, cfl=0.5):
        return lib3().orc3_eval_residual(self._h, cfl)

    def steps(self, n):
        r = np.zeros(n)
        lib3().orc3_steps(self._h, n, _dp(r))
        return r

    def forces(self, x_max):
        out = np.zeros(3)
        lib3().orc3_forces(self._h, self.mach, x_max, _dp(out))
        return dict(cn=out[0], ca=out[1], x_cp=out[2])

    PARTS = ("nose", "afterbody", "fin_sides", "fin_edges", "fin_tips")

    def forces_parts(self, x_max, x_nose):
        """run3.rs `breakdown_on`: {part: dict(cn, ca, x_cp)}."""
        out = np.zeros(15)
        lib3().orc3_forces_parts(self._h, self.mach, x_max, x_nose, _dp(out))
        return {p: dict(cn=out[3 * q], ca=out[3 * q + 1], x_cp=out[3 * q + 2]) for q, p in enumerate(self.PARTS)}

    def run(self, x_max, max_iter=8000, rel_tol=0.002, window=500):
        r = Orc3Result()
        lib3().orc3_run(self._h, self.mach, x_max, max_iter, rel_tol, window, C.byref(r))
        return dict(cn=r.cn, ca=r.ca, x_cp=r.x_cp, iterations=r.iterations, stop_reason=STOP3.get(r.stop_reason, "?"), drop_orders=r.drop_orders)
