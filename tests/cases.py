"""Test fixtures shared by the parity tests: each builds the same grid nodes, configuration, block, scheme and start state
for the oracle (`oracle_ffi.Solver`) and the B200 backend (`bowshock_b200.GpuSolver`), following the reference's GPU-vs-CPU
protocol (crates/bowshock-gpu-cases/tests/common/mod.rs): identical start state, N iterations, then
`state = max |dU| / (1 + |U_cpu|)` and `residual = max |r_gpu - r_cpu| / r_cpu`."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

import oracle_ffi as o


@dataclass
class Spec:
    ni: int
    nj: int
    x: np.ndarray
    r: np.ndarray
    cfl: float
    limiter: int
    fs: tuple
    bc: tuple
    first_order_iters: int
    low_mach: bool = False
    block: tuple | None = None
    scheme: dict | None = None  # None = explicit; else implicit params
    viscous: dict | None = None
    u0: np.ndarray | None = None
    nozzle: tuple | None = None  # (j_end, state[4], turb[2]) of the base-face jet
    label: str = ""


def far_field_box(mach, outflow=o.BC_CHARACTERISTIC):  # common/mod.rs:11-29
    ni, nj = 40, 20
    ii, jj = np.meshgrid(np.arange(ni + 1), np.arange(nj + 1))
    x = 4.0 * (ii / ni) ** 1.15
    r = 2.0 * (jj / nj) ** 1.1
    return Spec(ni, nj, x, r, 0.5, o.MINMOD, tuple(o.freestream(mach)), (o.BC_CHARACTERISTIC, outflow, o.BC_SLIPWALL, o.BC_CHARACTERISTIC),
                5, label=f"far-field box M{mach}")


def perturbed_state(spec: Spec):  # common/mod.rs:33-42
    s = oracle_solver(spec)
    xc, rc = s.get(o.F_XC), s.get(o.F_RC)
    fs = spec.fs
    g = np.exp(-((xc - 3.0) ** 2 + (rc - 1.4) ** 2) / 0.8) + 0.5 * np.exp(-((xc - 0.6) ** 2 + (rc - 1.6) ** 2) / 0.5)
    w = np.stack([fs[0] * (1 + 0.25 * g), fs[1] + 0.2 * g, 0.3 * g * np.sin(0.5 * xc), fs[3] * (1 + 0.4 * g)], axis=-1)
    return o.prim_to_cons(w)


def from_case(case: o.OrcCase, label: str) -> Spec:
    """A Spec from an engine case (the grid, block and numerics `Case::try_build_solver` would use, case.rs:147-176)."""
    s = o.Solver.from_case(case)
    ni, nj = s.dims
    x, r = s.nodes
    n = case.numerics
    sch = n.scheme
    scheme = None
    if sch.kind == o.SCHEME_IMPLICIT:
        scheme = dict(cfl0=sch.cfl0, cfl_max=sch.cfl_max, growth=sch.growth, dt_mode=sch.dt_mode, lines=bool(sch.lines),
                      implicit_bc=bool(sch.implicit_bc), sub_iters=sch.sub_iters, roe=bool(sch.roe), eps_fix=sch.eps_fix)
    visc = None
    if case.has_viscous:
        visc = dict(re_c=case.re_c, sutherland=case.sutherland, turbulence=case.turbulence, wall_i_start=case.wall_i_start,
                    roughness=case.roughness)
    cfg = s.config
    return Spec(ni, nj, x.reshape(nj + 1, ni + 1), r.reshape(nj + 1, ni + 1), cfg.cfl, cfg.limiter, tuple(cfg.fs), tuple(cfg.bc),
                cfg.first_order_iters, bool(n.low_mach), s.block, scheme, visc, label=label)


def subsonic_sting(mach=0.5, level=0):
    """Ogive (fineness 3) + 6-diameter tube on the sting grid, `Numerics::auto` (line-implicit, van Albada, low Mach)."""
    b = o.body(o.NOSE_TANGENT_OGIVE, fineness=3.0, segments=((6.0, 0.0),))
    return from_case(o.case_new(mach, b, level, o.WAKE_STING), f"ogive sting M{mach}")


def subsonic_base(mach=0.5, level=0):
    """The same body with a flat base and a wake behind it (solid block, j_sting = 0)."""
    b = o.body(o.NOSE_TANGENT_OGIVE, fineness=3.0, segments=((6.0, 0.0),))
    return from_case(o.case_new(mach, b, level, o.WAKE_BASE), f"ogive base M{mach}")


def g3_body():
    """The reference's G3 body (viscous.rs gate): SST, base wake, 156 x 122."""
    from tests.golden.g3_case import g3_case
    return from_case(g3_case(), "G3 body SST")


def oracle_solver(spec: Spec) -> o.Solver:
    s = o.Solver.from_nodes(spec.ni, spec.nj, spec.x, spec.r, cfl=spec.cfl, limiter=spec.limiter, freestream_=np.array(spec.fs),
                            bc=spec.bc, first_order_iters=spec.first_order_iters)
    s.set_low_mach(spec.low_mach)
    if spec.block is not None:
        s.set_block(spec.block)
    if spec.scheme is not None:
        s.set_scheme(o.implicit_params(**spec.scheme))
    if spec.nozzle is not None:  # the jet rows before the viscous walls (solver.rs:333-347)
        s.set_nozzle(*spec.nozzle)
    if spec.viscous is not None:
        s.set_viscous(spec.viscous)
    if spec.u0 is not None:
        s.u = spec.u0
    return s


def gpu_solver(spec: Spec):
    import bowshock_b200 as bk
    cfg = bk.Config(spec.cfl, spec.limiter, tuple(spec.fs), tuple(spec.bc), spec.first_order_iters)
    s = bk.GpuSolver.new(spec.ni, spec.nj, spec.x, spec.r, cfg)
    s.set_low_mach(spec.low_mach)
    if spec.block is not None:
        s.set_block(spec.block)
    if spec.scheme is not None:
        s.set_scheme(bk.ImplicitParams(**spec.scheme))
    else:
        s.set_scheme(bk.EXPLICIT)
    if spec.nozzle is not None:
        s.set_nozzle(spec.nozzle)
    if spec.viscous is not None:
        s.set_viscous(bk.Viscous(**spec.viscous))
    if spec.u0 is not None:
        s.set_state(spec.u0)
    return s


def state_diff(a, b):
    """max |a - b| / (1 + |b|) over cells and components (common/mod.rs:45-47)."""
    a, b = np.asarray(a).reshape(-1, 4), np.asarray(b).reshape(-1, 4)
    return float(np.max(np.abs(a - b) / (1.0 + np.abs(b))))


def residual_diff(a, b):
    """max |a - b| / b over a residual history (common/mod.rs:50-52)."""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / b))
