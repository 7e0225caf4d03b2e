"""Case layer: one Mach number on one body — its grid (meshed by the library's C++ mesher, body_grid.rs:134-452), its
numerics preset and stop rules (numerics.rs:261-362), and the sweep case assembly of the facade (case.rs:51-102,
analysis.rs:447-469, atmosphere.rs:84-112). Mirrors the reference's `Case`, `Numerics` and `BaseBody`."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, replace

import numpy as np

from . import _ffi
from ._ffi import BowshockError
from .solver import (BC_CHARACTERISTIC, BC_SLIPWALL, LIM_MINMOD, LIM_VAN_ALBADA, TURB_SST, Config, GpuSolver, ImplicitParams,
                     Viscous, freestream)

NOSE_TANGENT_OGIVE, NOSE_CONE, NOSE_POWER, NOSE_PARABOLIC, NOSE_HAACK = 0, 1, 2, 3, 4
WAKE_STING, WAKE_BASE = 0, 1
STOP_REASONS = ["max iterations", "residual drop", "CD stationary", "base pressure stationary", "mean stationary",
                "non-finite residual", "cancelled"]
REGIME_SPLIT_MACH = 0.85  # numerics.rs:240
SUTHERLAND_S = 110.4


@dataclass
class Body:
    """`BaseBody` (body_grid.rs:246-319): nose + aft segments (length, dr/dx), lengths in nose diameters."""
    nose_kind: int = NOSE_TANGENT_OGIVE
    fineness: float = 3.0
    half_angle: float = 0.0
    param: float = 0.0
    segments: tuple = ((6.0, 0.0),)
    sting_radius: float = 0.0

    def c(self):
        b = _ffi.BowshockBody(self.nose_kind, self.fineness, self.half_angle, self.param, len(self.segments))
        for k, (length, slope) in enumerate(self.segments):
            b.seg_length[k] = length
            b.seg_slope[k] = slope
        b.sting_radius = self.sting_radius
        return b

    def nose_length(self):
        return 0.5 / math.tan(self.half_angle) if self.nose_kind == NOSE_CONE else self.fineness

    def station(self, k):
        x, r = self.nose_length(), 0.5
        for length, slope in self.segments[:k]:
            x += length
            r += length * slope
        return x, r

    def x_base(self):
        return self.station(len(self.segments))[0]

    def base_radius(self):
        return self.station(len(self.segments))[1]


@dataclass
class Numerics:
    """numerics.rs:261-287 (scheme is always the line-implicit scheme on this backend)."""
    cfl: float = 0.5
    limiter: int = LIM_VAN_ALBADA
    low_mach: bool = True
    scheme: ImplicitParams = field(default_factory=ImplicitParams)
    first_order_iters: int = 100
    max_iter: int = 10000
    min_iter: int = 0
    drop_orders: float = 6.0
    outflow: int = BC_CHARACTERISTIC
    monitor_window: int = 2000
    monitor_tol: float | None = None
    mean_window: int | None = None
    drag_rel_tol: float | None = None

    @staticmethod
    def subsonic(level, wake):  # numerics.rs:291-310
        return Numerics(max_iter=10000 << level, monitor_tol=1e-3 if wake == WAKE_BASE else None)

    @staticmethod
    def transonic():
        """numerics.rs:313-329 with the line-implicit scheme in place of SSP-RK3 (the same spatial operator, so the same
        fixed point). The implicit scheme converges the 300-iteration first-order phase by itself, which SSP-RK3 at CFL 0.5
        never does, so the stop rules are held until the first second-order residual (min_iter = first_order_iters + 1):
        otherwise a run would stop on the first-order solution."""
        return Numerics(limiter=LIM_MINMOD, low_mach=False, first_order_iters=300, max_iter=60000, min_iter=301, monitor_tol=2e-4)

    @staticmethod
    def auto(mach, level, wake):  # numerics.rs:332-339
        n = Numerics.subsonic(level, wake) if mach < REGIME_SPLIT_MACH else Numerics.transonic()
        n.monitor_tol = 1e-3 if wake == WAKE_BASE else 2e-4
        return n

    @staticmethod
    def viscous(mach, level):  # numerics.rs:345-362
        sub = mach < REGIME_SPLIT_MACH
        scheme = ImplicitParams.rans() if mach < 1.0 else replace(ImplicitParams.rans(), cfl_max=20.0)
        return Numerics(limiter=LIM_VAN_ALBADA if sub else LIM_MINMOD, low_mach=sub, scheme=scheme, first_order_iters=200,
                        max_iter=80000 << level, drop_orders=5.0, monitor_tol=1e-4, mean_window=6000)

    def run_params(self, wake, warm=False, r_ref=None):
        p = _ffi.RunParams()
        p.max_iter, p.min_iter, p.drop_orders, p.monitor_window = self.max_iter, self.min_iter, self.drop_orders, self.monitor_window
        p.has_monitor_tol, p.monitor_tol = int(self.monitor_tol is not None), self.monitor_tol or 0.0
        p.has_mean_window, p.mean_window = int(self.mean_window is not None), self.mean_window or 0
        p.has_drag_rel_tol, p.drag_rel_tol = int(self.drag_rel_tol is not None), self.drag_rel_tol or 0.0
        p.wake, p.warm, p.r_ref = wake, int(warm), -1.0 if r_ref is None else r_ref
        return p


def _even_ceil(x):  # case.rs:179-182
    n = math.ceil(x)
    return n + n % 2


def layer_count(h, y1):  # case.rs:185-187
    return _even_ceil(math.log(1.0 + 0.2 * h / y1) / math.log(1.2))


@dataclass
class BaseGrid:  # body_grid.rs:330-355
    x_up: float
    x_down: float
    r_far: float
    n_up: int
    n_nose: int
    n_seg: list
    n_wake: int
    n_sting: int
    n_gap: int
    nj_out: int
    dx_tip: float
    dr_wall: float
    gap_one_sided: bool = False


@dataclass
class StingGrid:  # body_grid.rs:112-131
    x_up: float
    x_down: float
    r_far: float
    n_up: int
    n_nose: int
    n_seg: list
    n_ext: int
    nj: int
    dx_tip: float
    dr_wall: float


@dataclass
class Case:
    """case.rs:33-46 (power-off)."""
    mach: float
    body: Body
    wake: int
    grid_base: BaseGrid
    grid_sting: StingGrid
    numerics: Numerics
    viscous: Viscous | None = None

    @staticmethod
    def new(mach, body: Body, level: int, wake: int, numerics: Numerics | None = None):  # case.rs:51-78
        f = 1 << level
        dx_tip = 0.03 / f
        l_body = body.x_base()
        n_sting = 4 * f if body.sting_radius > 0.0 else 0
        count = lambda per, length: max(min(per, _even_ceil(length / dx_tip)), 4)
        gb = BaseGrid(10 * l_body, 5 * l_body, 10 * l_body, 28 * f, 48 * f,
                      [count(40 * f if s == 0.0 else 24 * f, ln) for ln, s in body.segments], 40 * f, n_sting, 12 * f, 64 * f, dx_tip,
                      0.03 / f)
        nseg = len(body.segments)
        gs = StingGrid(10 * l_body, 5 * l_body, 10 * l_body, 30 * f, 48 * f,
                       [count(24 * f if s != 0.0 else (36 * f if k + 1 == nseg else 40 * f), ln) for k, (ln, s) in enumerate(body.segments)],
                       30 * f, 70 * f, dx_tip, 0.03 / f)
        return Case(mach, body, wake, gb, gs, numerics if numerics is not None else Numerics.auto(mach, level, wake))

    @staticmethod
    def viscous_case(mach, body: Body, level, wake, re_c, sutherland, mach_max):  # case.rs:84-102
        c = Case.new(mach, body, level, wake, Numerics.viscous(mach, level))
        cf = 0.027 * (re_c * mach_max * body.x_base()) ** (-1.0 / 7.0)
        y1 = 1.0 / (re_c * mach_max * math.sqrt(0.5 * cf))
        re, rs = body.base_radius(), body.sting_radius
        c.grid_base.dr_wall = y1
        c.grid_base.nj_out = layer_count(c.grid_base.r_far - re, y1)
        c.grid_base.n_gap = layer_count(re - rs, y1)
        c.grid_base.gap_one_sided = True
        c.grid_sting.dr_wall = y1
        c.grid_sting.nj = layer_count(c.grid_sting.r_far, y1)
        wall_i_start = c.grid_base.n_up if wake == WAKE_BASE else c.grid_sting.n_up
        c.viscous = Viscous(re_c, sutherland, TURB_SST, wall_i_start, 0.0)
        return c

    def cells(self):  # case.rs:132-139
        if self.wake == WAKE_BASE:
            b = self.grid_base
            return b.n_up + b.n_nose + sum(b.n_seg) + b.n_wake, b.n_sting + b.n_gap + b.nj_out
        g = self.grid_sting
        return g.n_up + g.n_nose + sum(g.n_seg) + g.n_ext, g.nj

    def grid(self):
        """(ni, nj, x, r, block) from the C++ mesher."""
        lib = _ffi.load()
        b = self.body.c()
        ni, nj = C.c_uint64(), C.c_uint64()
        if self.wake == WAKE_BASE:
            g = self.grid_base
            p = _ffi.BaseGridC(g.x_up, g.x_down, g.r_far, g.n_up, g.n_nose, (C.c_uint64 * 8)(*g.n_seg), g.n_wake, g.n_sting, g.n_gap,
                               g.nj_out, g.dx_tip, g.dr_wall, int(g.gap_one_sided))
            rc = lib.bowshock_base_domain_grid(C.byref(b), C.byref(p), C.byref(ni), C.byref(nj), None, None, None)
            if rc:
                raise BowshockError(rc, "invalid base-grid parameters")
            n = (ni.value + 1) * (nj.value + 1)
            x, r = np.zeros(n), np.zeros(n)
            blk = _ffi.Block()
            lib.bowshock_base_domain_grid(C.byref(b), C.byref(p), C.byref(ni), C.byref(nj), _ffi.dptr(x), _ffi.dptr(r), C.byref(blk))
            return ni.value, nj.value, x, r, (blk.i_end, blk.j_end, blk.j_sting)
        g = self.grid_sting
        p = _ffi.StingGridC(g.x_up, g.x_down, g.r_far, g.n_up, g.n_nose, (C.c_uint64 * 8)(*g.n_seg), g.n_ext, g.nj, g.dx_tip, g.dr_wall)
        rc = lib.bowshock_large_domain_grid(C.byref(b), C.byref(p), C.byref(ni), C.byref(nj), None, None)
        if rc:
            raise BowshockError(rc, "invalid sting-grid parameters")
        n = (ni.value + 1) * (nj.value + 1)
        x, r = np.zeros(n), np.zeros(n)
        lib.bowshock_large_domain_grid(C.byref(b), C.byref(p), C.byref(ni), C.byref(nj), _ffi.dptr(x), _ffi.dptr(r))
        return ni.value, nj.value, x, r, None

    def mesh_request(self):
        """bowshock_mesh_request of this case's grid (the device mesher's input: body and grid parameters)."""
        q = _ffi.MeshRequest()
        q.wake = self.wake
        q.body = self.body.c()
        if self.wake == WAKE_BASE:
            g = self.grid_base
            q.base = _ffi.BaseGridC(g.x_up, g.x_down, g.r_far, g.n_up, g.n_nose, (C.c_uint64 * 8)(*g.n_seg), g.n_wake, g.n_sting, g.n_gap,
                                    g.nj_out, g.dx_tip, g.dr_wall, int(g.gap_one_sided))
        else:
            g = self.grid_sting
            q.sting = _ffi.StingGridC(g.x_up, g.x_down, g.r_far, g.n_up, g.n_nose, (C.c_uint64 * 8)(*g.n_seg), g.n_ext, g.nj, g.dx_tip,
                                      g.dr_wall)
        return q

    def mesh_dims(self):
        """(ni, nj, block or None) of this case's grid, from the cell counts (no meshing)."""
        q = self.mesh_request()
        ni, nj, blk = C.c_uint64(), C.c_uint64(), _ffi.Block()
        rc = _ffi.load().bowshock_mesh_dims(C.byref(q), C.byref(ni), C.byref(nj), C.byref(blk))
        if rc:
            raise BowshockError(rc, "invalid grid parameters")
        return ni.value, nj.value, ((blk.i_end, blk.j_end, blk.j_sting) if self.wake == WAKE_BASE else None)

    def config(self) -> Config:  # case.rs:148-155
        n = self.numerics
        return Config(n.cfl, n.limiter, freestream(self.mach), (BC_CHARACTERISTIC, n.outflow, BC_SLIPWALL, BC_CHARACTERISTIC),
                      n.first_order_iters)

    def build_solver(self, device=0, grid=None) -> GpuSolver:  # case.rs:147-176
        ni, nj, x, r, blk = grid if grid is not None else self.grid()
        s = GpuSolver.new(ni, nj, x, r, self.config(), device)
        if blk is not None:
            s.set_block(blk)
        s.set_low_mach(self.numerics.low_mach)
        s.set_scheme(self.numerics.scheme)
        s.set_viscous(self.viscous)
        return s

    def case_desc(self, grid=None):
        """bowshock_case_desc of this case for the batched arena (the node arrays are kept alive on the struct)."""
        ni, nj, x, r, blk = grid if grid is not None else self.grid()
        d = _ffi.CaseDesc()
        d.ni, d.nj = ni, nj
        d._x, d._r = np.ascontiguousarray(x), np.ascontiguousarray(r)
        d.x, d.r = _ffi.dptr(d._x), _ffi.dptr(d._r)
        d.cfg = self.config().c()
        d.low_mach = int(self.numerics.low_mach)
        if blk is not None:
            d.has_block = 1
            d.block = _ffi.Block(*blk)
        p = self.numerics.scheme
        d.scheme = _ffi.Scheme(3, p.cfl0, p.cfl_max, p.growth, p.dt_mode, int(p.lines), int(p.implicit_bc), int(p.sub_iters), int(p.roe),
                               p.eps_fix)
        if self.viscous is not None:
            v = self.viscous
            d.has_viscous = 1
            d.viscous = _ffi.Viscous(v.re_c, v.sutherland, v.turbulence, int(v.wall_i_start), v.roughness)
        d.body = self.body.c()
        d.run = self.numerics.run_params(self.wake)
        return d

    def wall_distance(self, grid=None):
        """Distance of every cell centroid to the nearest no-slip wall face (turbulence.rs:91-125), computed on the host:
        an (nj, ni) array, +inf on solid cells and where the case has no wall."""
        d = self.case_desc(grid)
        out = np.zeros(d.ni * d.nj)
        rc = _ffi.load().bowshock_case_wall_distance(C.byref(d), _ffi.dptr(out))
        if rc:
            raise BowshockError(rc, "invalid case")
        return out.reshape(d.nj, d.ni)


def isa(altitude_m):
    """atmosphere.rs:84-112: (T, p, rho, c, mu)."""
    R, G, T0, P0, LAPSE = 287.05287, 1.4, 288.15, 101325.0, 0.0065
    if 0.0 <= altitude_m <= 11000.0:
        t = T0 - LAPSE * altitude_m
        p = P0 * (t / T0) ** 5.255877
    elif 11000.0 < altitude_m <= 20000.0:
        t = 216.65
        p = 22632.06 * math.exp(-(altitude_m - 11000.0) / 6341.62)
    else:
        raise BowshockError(_ffi.INVALID, f"altitude {altitude_m} m outside 0 to 20 000 m")
    mu = 1.716e-5 * (t / 273.15) ** 1.5 * (273.15 + SUTHERLAND_S) / (t + SUTHERLAND_S)
    return dict(temperature_k=t, pressure_pa=p, density=p / (R * t), sound_speed=math.sqrt(G * R * t), viscosity=mu)


def rans_params(altitude_m, d_nose):
    """analysis.rs:447-469: re_c = rho c d / mu and the Sutherland constant of the free stream."""
    a = isa(altitude_m)
    return a["density"] * a["sound_speed"] * d_nose / a["viscosity"], SUTHERLAND_S / a["temperature_k"]


METRIC_NAMES = ("if_nx", "if_nr", "if_len", "if_rm", "jf_nx", "jf_nr", "jf_len", "jf_rm", "area", "vol", "xc", "rc")


def mesh_batch(cases, device=0, metrics=True):
    """The grids of `cases` built on the device (bowshock_mesh_batch): a list of (ni, nj, x, r, block) like Case.grid(),
    the metrics of each case (a dict of METRIC_NAMES arrays, i faces (nj, ni+1), j faces (nj+1, ni), cells (nj, ni)) when
    `metrics`, and the device time in ms."""
    lib = _ffi.load()
    qs = (_ffi.MeshRequest * len(cases))()
    dims = []
    for k, c in enumerate(cases):
        qs[k] = c.mesh_request()
        dims.append(c.mesh_dims())
    nodes = sum((ni + 1) * (nj + 1) for ni, nj, _ in dims)
    words = sum(4 * ((ni + 1) * nj + ni * (nj + 1) + ni * nj) for ni, nj, _ in dims)
    x, r = np.zeros(nodes), np.zeros(nodes)
    m = np.zeros(words) if metrics else None
    ms = C.c_double()
    rc = lib.bowshock_mesh_batch(len(cases), qs, int(device), _ffi.dptr(x), _ffi.dptr(r), _ffi.dptr(m) if metrics else None, C.byref(ms))
    if rc:
        raise BowshockError(rc, "bowshock_mesh_batch failed (invalid request, non-positive cell area, or no CUDA device)")
    grids, mets, o, mo = [], [], 0, 0
    for ni, nj, blk in dims:
        n = (ni + 1) * (nj + 1)
        grids.append((ni, nj, x[o:o + n].copy(), r[o:o + n].copy(), blk))
        o += n
        if metrics:
            d = {}
            for name, shape in zip(METRIC_NAMES, [(nj, ni + 1)] * 4 + [(nj + 1, ni)] * 4 + [(nj, ni)] * 4):
                sz = shape[0] * shape[1]
                d[name] = m[mo:mo + sz].reshape(shape).copy()
                mo += sz
            mets.append(d)
    return grids, (mets if metrics else None), ms.value
