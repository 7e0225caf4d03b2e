"""Pins of the oracle's solver: ports of the reference's own solver-level unit tests (crates/bowshock-cfd/src/
{solver,implicit,multigrid,viscous,turbulence}.rs), same grids, iteration counts and tolerances."""
import math

import numpy as np
import pytest

import oracle_ffi as o


def curved_grid(ni, nj):  # solver.rs:811-823 (also implicit.rs:783-794)
    x = np.zeros((nj + 1, ni + 1))
    r = np.zeros((nj + 1, ni + 1))
    for j in range(nj + 1):
        for i in range(ni + 1):
            s, t = i / ni, j / nj
            x[j, i] = 2.0 * s + 0.15 * math.sin(3.0 * t) * math.cos(2.0 * s) + 0.1 * t * t
            r[j, i] = t * (1.0 + 0.3 * s) * (1.0 + 0.2 * t) + 0.05 * math.sin(4.0 * s) * t * (1.0 - t)
    return x, r


def mg_grid(ni, nj):  # multigrid.rs:227-237
    x = np.zeros((nj + 1, ni + 1))
    r = np.zeros((nj + 1, ni + 1))
    for j in range(nj + 1):
        for i in range(ni + 1):
            s, t = i / ni, j / nj
            x[j, i] = 4.0 * s + 0.1 * math.sin(3.0 * t)
            r[j, i] = 3.0 * t * (1.0 + 0.2 * s)
    return x, r


def drift(s, fs):
    q0 = o.prim_to_cons(fs)
    return np.max(np.abs(s.u - q0) / np.maximum(np.abs(q0), 1.0))


@pytest.mark.parametrize("limiter", [o.MINMOD, o.VAN_ALBADA])
def test_freestream_preserved_on_curved_axisymmetric_grid(limiter):  # solver.rs:847-872
    fs = o.freestream(2.0)
    x, r = curved_grid(24, 16)
    s = o.Solver.from_nodes(24, 16, x, r, cfl=0.5, limiter=limiter, freestream_=fs,
                            bc=(o.BC_FREESTREAM, o.BC_EXTRAPOLATE, o.BC_SLIPWALL, o.BC_FREESTREAM))
    s.steps(50)
    assert drift(s, fs) < 1e-12


def test_freestream_residual_is_roundoff_with_all_dirichlet_boundaries():  # solver.rs:875-893
    fs = o.freestream(3.0)
    ni, nj = 20, 12
    x = np.zeros((nj + 1, ni + 1))
    r = np.zeros((nj + 1, ni + 1))
    for j in range(nj + 1):
        for i in range(ni + 1):
            s_, t = i / ni, j / nj
            x[j, i] = s_ + 0.05 * math.sin(5.0 * t)
            r[j, i] = 0.5 + t + 0.1 * math.sin(6.0 * s_) * (1.0 + t)
    s = o.Solver.from_nodes(ni, nj, x, r, cfl=0.5, limiter=o.VAN_ALBADA, freestream_=fs, bc=(0, 0, 0, 0))
    s.eval_residual(True)
    assert np.max(np.abs(s.res)) < 1e-12


@pytest.mark.parametrize("mach", [0.1, 0.5, 0.9])
@pytest.mark.parametrize("outflow", [o.BC_CHARACTERISTIC, o.BC_PRESSURE_OUTFLOW])
def test_implicit_scheme_preserves_the_free_stream(mach, outflow):  # implicit.rs:797-822
    fs = o.freestream(mach)
    x, r = curved_grid(24, 16)
    s = o.Solver.from_nodes(24, 16, x, r, cfl=0.5, limiter=o.VAN_ALBADA, freestream_=fs,
                            bc=(o.BC_CHARACTERISTIC, outflow, o.BC_SLIPWALL, o.BC_CHARACTERISTIC))
    s.set_low_mach(True)
    s.set_scheme(o.implicit_params(cfl_max=40.0, growth=1.2))
    s.steps(40)
    assert drift(s, fs) < 1e-11


def test_multigrid_hierarchy_is_built_and_the_free_stream_is_preserved():  # multigrid.rs:239-258
    fs = o.freestream(0.5)
    x, r = mg_grid(64, 32)
    s = o.Solver.from_nodes(64, 32, x, r, cfl=0.5, limiter=o.VAN_ALBADA, freestream_=fs,
                            bc=(o.BC_CHARACTERISTIC, o.BC_CHARACTERISTIC, o.BC_SLIPWALL, o.BC_CHARACTERISTIC))
    assert s.set_scheme(o.multigrid_scheme()) == 3
    s.steps(30)
    assert np.max(np.abs(s.u - o.prim_to_cons(fs))) < 1e-11


def test_multigrid_reaches_the_explicit_fixed_point():  # multigrid.rs:260-291
    fs = o.freestream(0.4)

    def mk(scheme):
        x, r = mg_grid(32, 16)
        s = o.Solver.from_nodes(32, 16, x, r, cfl=0.8, limiter=o.FIRST_ORDER, freestream_=fs,
                                bc=(o.BC_CHARACTERISTIC, o.BC_CHARACTERISTIC, o.BC_SLIPWALL, o.BC_CHARACTERISTIC))
        s.set_scheme(scheme)
        w = np.array([fs[0] * 1.02, fs[1], fs[2], fs[3] * 1.03])
        s.u = np.tile(o.prim_to_cons(w), (32 * 16, 1))
        last = 1.0
        for _ in range(4000):
            last = s.step()
            if last < 1e-11:
                break
        return s, last

    a, ra = mk(o.explicit_scheme())
    b, rb = mk(o.multigrid_scheme())
    assert ra < 1e-9 and rb < 1e-9
    assert np.max(np.abs(a.u - b.u)) < 1e-7


def test_uniform_flow_is_preserved_with_viscous_terms():  # viscous.rs:465-481
    fs = o.freestream(0.5)
    x, r = curved_grid(24, 16)
    s = o.Solver.from_nodes(24, 16, x, r, cfl=0.5, limiter=o.VAN_ALBADA, freestream_=fs,
                            bc=(o.BC_FREESTREAM, o.BC_EXTRAPOLATE, o.BC_SLIPWALL, o.BC_FREESTREAM))
    s.set_viscous(dict(re_c=1e4, sutherland=0.368, turbulence=o.TURB_LAMINAR, wall_i_start=24))
    s.eval_residual(True)
    assert np.max(np.abs(s.res)) < 1e-12


def plate_grid(r0, x_up, length, height, n_up, n_plate, nj, dx_le, dr_wall):  # grid.rs:255-274
    up = o.geometric_offsets(dx_le, x_up, n_up)
    plate = o.geometric_offsets(dx_le, length, n_plate)
    xs = [-up[k] for k in range(n_up, 0, -1)] + list(plate)
    ni = n_up + n_plate
    rs = o.geometric_offsets(dr_wall, height, nj)
    x = np.tile(np.array(xs), (nj + 1, 1))
    r = np.tile((r0 + rs)[:, None], (1, ni + 1))
    return ni, nj, x, r


def test_sst_flat_plate_smoke():  # turbulence.rs:664-691
    ni, nj, x, r = plate_grid(20.0, 0.33, 2.0, 1.0, 24, 112, 72, 0.002, 4e-6)
    s = o.Solver.from_nodes(ni, nj, x, r, cfl=0.5, limiter=o.VAN_ALBADA, freestream_=o.freestream(0.2),
                            bc=(o.BC_CHARACTERISTIC, o.BC_PRESSURE_OUTFLOW, o.BC_SLIPWALL, o.BC_CHARACTERISTIC),
                            first_order_iters=50)
    s.set_low_mach(True)
    s.set_scheme(o.implicit_viscous())
    s.set_viscous(dict(re_c=2.5e7, sutherland=0.368, turbulence=o.TURB_SST, wall_i_start=24))
    s.steps(300)
    assert np.all(np.isfinite(s.u))
    t = s.turb
    assert np.all(np.isfinite(t)) and np.all(t > 0.0)
    assert np.all(np.isfinite(s.mu_t)) and np.all(s.mu_t >= 0.0)
    assert math.isfinite(s.turb_residual)


BLOCK = (12, 8, 0)


def jet():  # solver.rs:903-907
    p = 1.0 / o.GAMMA
    c = math.sqrt(o.GAMMA * p / 0.5)
    return 4, [0.5, 2.5 * c, 0.0, p], [1e-4, 50.0]


def test_nozzle_jet_flux_is_the_jet_flux():  # solver.rs:919-937
    ni, nj = 24, 16
    x, r = curved_grid(ni, nj)
    s = o.Solver.from_nodes(ni, nj, x, r, cfl=0.5, limiter=o.VAN_ALBADA, freestream_=o.freestream(2.0),
                            bc=(o.BC_FREESTREAM, o.BC_EXTRAPOLATE, o.BC_SLIPWALL, o.BC_FREESTREAM))
    s.set_block(BLOCK)
    j_end, state, turb = jet()
    s.set_nozzle(j_end, state, turb)
    s.eval_residual(False)
    fi = s.get(o.F_FI).reshape(nj, ni + 1, 4)
    # face normals of the base face from the nodes (grid.rs:71-77)
    for j in range(BLOCK[1]):
        a, b = (x[j, BLOCK[0]], r[j, BLOCK[0]]), (x[j + 1, BLOCK[0]], r[j + 1, BLOCK[0]])
        dx, dr = b[0] - a[0], b[1] - a[1]
        ln = math.hypot(dx, dr)
        nx, nr = dr / ln, -dx / ln
        mass = fi[j, BLOCK[0], 0]
        if j < j_end:
            want = state[0] * (state[1] * nx + state[2] * nr)
            assert abs(mass - want) <= 1e-12 * abs(want)
        else:
            assert abs(mass) < 1e-12


def test_g1_uniform_sst_init_eddy_viscosity():  # turbulence.rs:128-138
    x, r = curved_grid(24, 16)
    s = o.Solver.from_nodes(24, 16, x, r, freestream_=o.freestream(0.5))
    s.set_scheme(o.implicit_params())
    s.set_viscous(dict(re_c=1e6, sutherland=0.368, turbulence=o.TURB_SST, wall_i_start=0))
    assert np.allclose(s.turb[:, 0], 9e-9) and np.allclose(s.turb[:, 1], 1.0)
    assert np.allclose(s.mu_t, 9e-9 / 1.0)
