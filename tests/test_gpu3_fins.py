"""3D fins as solid boxes (bowshock3_set_solid; crates/bowshock-cfd/src/solver3.rs:13, 362-405, implicit3.rs:14-16,
engine/run3.rs:130-212) on the B200 against the 3D oracle with the same boxes: the per-cell residual of one evaluation,
the explicit (1e-5) and implicit (1e-3) protocols, the forces with the fin faces on the same state, and the reference's
own fin test (solver3.rs:606-670: 200 implicit iterations at M 2 drop the residual 2 orders, the solid cells keep their
state)."""
import math

import numpy as np
import pytest

import oracle_ffi as o
from tests.test_oracle3 import fin_grid

pytestmark = pytest.mark.gpu


def _mask(ni, nj, nk, boxes):
    m = np.zeros((nk, nj, ni), bool)
    for (i0, i1), (j0, j1), (k0, k1) in boxes:
        m[k0:k1, j0:j1, i0:i1] = True
    return m.reshape(-1)


def _fin_pair(implicit=True, first_order=50, limiter=o.VAN_ALBADA, cfl_max=20.0):
    """The reference's fin_grid (solver3.rs:589-604) at M 2, on the oracle and on the B200."""
    import bowshock_b200.euler3 as e3
    ni, nj, nk, x, r, theta, box = fin_grid()
    p = o.implicit3_params(cfl_max=cfl_max)
    cpu = o.Solver3(ni, nj, x, r, nk, theta, ni, 2.0, 0.0, limiter=limiter, first_order_iters=first_order, implicit=implicit, params=p)
    cpu.set_solid([box])
    cfg = e3.Config3(2.0, 0.0, 0.5, limiter, first_order, False, e3.ImplicitParams(cfl_max=cfl_max) if implicit else e3.EXPLICIT)
    gx, gy, gz = e3.revolve(x, r, nk, theta)
    gpu = e3.Batch3(ni, nj, nk, gx, gy, gz, ni, [cfg])
    gpu.set_solid([box])
    return cpu, gpu, (ni, nj, nk), [box]


def _body_pair(mach, alpha_deg, implicit=True, first_order=5):
    """The lift-sweep body at 48 x 16 x 8 with a fin box on the afterbody wall (4 cells long, 3 cells high, 2 cells
    thick), on the oracle and on the B200."""
    import bowshock_b200.euler3 as e3
    from tests.test_gpu3 import _grid
    c, ni2, nj2, x2, r2 = _grid(48, 16, 8, mach, alpha_deg)
    nk = 8
    theta = np.pi * np.arange(nk + 1) / nk
    axis = c.case2.grid_sting.n_up
    i0 = axis + (ni2 - axis) // 2
    box = ((i0, i0 + 4), (0, 3), (3, 5))
    alpha = math.radians(alpha_deg)
    p = o.implicit3_params(cfl_max=10.0)
    cpu = o.Solver3(ni2, nj2, x2, r2, nk, theta, axis, mach, alpha, first_order_iters=first_order, implicit=implicit, params=p)
    cpu.set_solid([box])
    cfg = e3.Config3(mach, alpha, 0.5, o.MINMOD, first_order, False, e3.ImplicitParams(cfl_max=10.0) if implicit else e3.EXPLICIT)
    x, y, z = e3.revolve(x2, r2, nk)
    gpu = e3.Batch3(ni2, nj2, nk, x, y, z, axis, [cfg])
    gpu.set_solid([box])
    return cpu, gpu, (ni2, nj2, nk), [box], c


def _perturb(u, solid, seed, amp=0.02):
    rng = np.random.default_rng(seed)
    w = o.cons_to_prim3(u)
    n = len(w)
    w[:, 0] *= 1 + amp * rng.standard_normal(n)
    w[:, 1:4] += amp * rng.standard_normal((n, 3))
    w[:, 4] *= 1 + amp * rng.standard_normal(n)
    q = o.prim_to_cons3(w)
    q[solid] = u[solid]
    return q


@pytest.mark.parametrize("where", ["fin_grid", "body"])
def test_residual_per_cell_with_solid_boxes(where):
    if where == "fin_grid":
        cpu, gpu, dims, boxes = _fin_pair()
    else:
        cpu, gpu, dims, boxes, _ = _body_pair(1.2, 4.0)
    solid = _mask(*dims, boxes)
    u0 = _perturb(cpu.u, solid, 3)
    cpu.u = u0
    gpu.set_state(0, u0)
    dc = cpu.eval_residual(1.0)
    rg, dtg, dg = gpu.eval_residual(0)
    rc = cpu.res
    assert np.all(rg[solid] == 0.0) and np.all(dtg[solid] == 0.0)
    for k in range(5):
        scale = np.max(np.abs(rc[:, k])) + 1e-30
        err = np.max(np.abs(rg[:, k] - rc[:, k])) / scale
        assert err < 1e-5, f"component {k}: max rel err {err:.3e}"
    assert abs(dg - dc) / dc < 1e-5  # the norm over the fluid cells
    f = ~solid
    assert np.max(np.abs(dtg[f] - cpu.dt[f]) / cpu.dt[f]) < 1e-5


def test_explicit_state_with_fin_matches_oracle():
    cpu, gpu, dims, boxes, _ = _body_pair(2.5, 6.0, implicit=False, first_order=0)
    solid = _mask(*dims, boxes)
    u0 = _perturb(cpu.u, solid, 5, 0.01)
    cpu.u = u0
    gpu.set_state(0, u0)
    rc = cpu.steps(20)
    rg = gpu.run(20)[:, 0]
    ug = gpu.state(0)
    assert np.array_equal(ug[solid], u0[solid].astype(np.float32).astype(np.float64))
    d = np.max(np.abs(ug - cpu.u) / (1 + np.abs(cpu.u)))
    assert d < 1e-5, d
    assert np.max(np.abs(rg - rc) / rc) < 1e-4


@pytest.mark.parametrize("mach,alpha", [(0.8, 4.0), (2.5, 8.0)])
def test_implicit_state_with_fin_matches_oracle(mach, alpha):
    cpu, gpu, dims, boxes, c = _body_pair(mach, alpha, implicit=True, first_order=5)
    rc = cpu.steps(30)
    rg = gpu.run(30)[:, 0]
    ug = gpu.state(0)
    d = np.max(np.abs(ug - cpu.u) / (1 + np.abs(cpu.u)))
    assert d < 1e-3, d
    assert np.all(np.isfinite(rg))
    assert np.max(np.abs(rg[:5] - rc[:5]) / rc[:5]) < 1e-3
    # forces with the fin faces, evaluated on the GPU's state by both sides (FP64 on both)
    cpu.u = ug
    x_base = c.body.x_base()
    fc = cpu.forces(x_base)
    fg = gpu.forces(x_base)[0]
    assert abs(fg["cn"] - fc["cn"]) <= 1e-9 * max(1.0, abs(fc["cn"])), (fg, fc)
    assert abs(fg["ca"] - fc["ca"]) <= 1e-9 * max(1.0, abs(fc["ca"])), (fg, fc)
    assert abs(fg["x_cp"] - fc["x_cp"]) <= 1e-7 * max(1.0, abs(fc["x_cp"])), (fg, fc)


def test_fin_wall_run_converges_on_the_gpu():  # solver3.rs:606-670, with the oracle beside it
    cpu, gpu, dims, boxes = _fin_pair()
    solid = _mask(*dims, boxes)
    q0 = gpu.state(0)[solid].copy()
    rg = gpu.run(200)[:, 0]
    rc = cpu.steps(200)
    ug = gpu.state(0)
    assert np.all(np.isfinite(ug))
    assert rg[-1] <= 1e-2 * rg.max(), (rg.max(), rg[-1])
    assert np.array_equal(ug[solid], q0)  # solid cells untouched
    fs = o.prim_to_cons3(o.freestream3(2.0, 0.0))
    assert np.allclose(q0, fs, rtol=0, atol=1e-6)
    d = np.max(np.abs(ug - cpu.u) / (1 + np.abs(cpu.u)))
    print("fin grid: drop GPU", math.log10(rg.max() / rg[-1]), "oracle", math.log10(rc.max() / rc[-1]), "state diff", d)
    assert d < 1e-3, d


def test_removing_the_boxes_restores_the_finless_batch():
    cpu, gpu, dims, boxes, _ = _body_pair(1.2, 4.0)
    import bowshock_b200.euler3 as e3
    gpu.set_solid([])
    ref = _body_pair(1.2, 4.0)[1]
    ref.set_solid([])
    r1, r2 = gpu.run(5), ref.run(5)
    assert np.array_equal(gpu.state(0), ref.state(0))
    assert np.max(np.abs(r1 - r2) / r2) < 1e-12  # the norm's block sums are added atomically in no fixed order
    with pytest.raises(e3.BowshockError):
        gpu.set_solid([((0, 0), (0, 1), (0, 1))])  # empty
    with pytest.raises(e3.BowshockError):
        gpu.set_solid([((0, 1), (0, 1), (0, dims[2] + 1))])  # outside the grid
    with pytest.raises(e3.BowshockError):
        gpu.set_solid([((0, dims[0]), (0, dims[1]), (0, dims[2]))])  # every cell: refused, the batch as it was
    r3 = gpu.run(2)
    assert np.all(np.isfinite(r3)) and np.all(r3 > 0)


def test_fin_body_converged_forces_match_oracle():
    """The afterbody fin box at M 2.5, 4 degrees, both sides run to run3.rs's stop rules (the density norm over the fluid
    cells, CN sampled with the fin faces): the converged CN within 0.2 % and the centre of pressure within 2e-2 (the
    tolerances of the finless case, the CN-stationary rule holding CN to 0.2 % over its window)."""
    cpu, gpu, dims, boxes, c = _body_pair(2.5, 4.0, implicit=True, first_order=100)
    x_base = c.body.x_base()
    rc = cpu.run(x_base, max_iter=4000)
    rg = gpu.solve(x_base, max_iter=4000)[0]
    print("fin body", rc, rg)
    assert rc["stop_reason"] in ("residual drop", "CN stationary"), rc
    assert rg["stop_reason"] in ("residual drop", "CN stationary"), rg
    assert abs(rg["cn"] - rc["cn"]) <= 2e-3 * abs(rc["cn"]) + 1e-4, (rg, rc)
    assert abs(rg["x_cp"] - rc["x_cp"]) <= 2e-2, (rg, rc)


def test_force_parts_match_oracle():
    """run3.rs `breakdown_on` (bowshock3_forces_parts) on the afterbody fin box after 30 implicit iterations, evaluated on
    the GPU's state by both sides: every part's CN and CA to 1e-9, and the parts add up to the totals."""
    cpu, gpu, dims, boxes, c = _body_pair(2.5, 8.0, implicit=True, first_order=5)
    gpu.run(30)
    cpu.u = gpu.state(0)
    x_base, x_nose = c.body.x_base(), c.body.nose_length()
    pc = cpu.forces_parts(x_base, x_nose)
    pg = gpu.forces_parts(x_base, x_nose)[0]
    tot = gpu.forces(x_base)[0]
    for part in pc:
        for key in ("cn", "ca"):
            assert abs(pg[part][key] - pc[part][key]) <= 1e-9 * max(1.0, abs(pc[part][key])), (part, key, pg[part], pc[part])
    for key in ("cn", "ca"):
        assert abs(sum(p[key] for p in pg.values()) - tot[key]) <= 1e-10 * max(1.0, abs(tot[key]))
    assert abs(pg["fin_sides"]["cn"]) > 1e-6  # the fin box carries normal force at 8 degrees


def test_read_boundary_holds_what_the_forces_read():
    """bowshock3_read_boundary (GpuSolver3::read_boundary_into): after 20 iterations of the fin body, the cells it fills
    equal the state's, every other entry keeps its value (NaN here), and the oracle's forces (body wall and fin faces)
    computed from that sparse state alone equal the GPU's to 1e-9."""
    cpu, gpu, dims, boxes, c = _body_pair(2.5, 8.0, implicit=True, first_order=5)
    gpu.run(20)
    full = gpu.state(0)
    u = np.full_like(full, np.nan)
    gpu.read_boundary_into(0, u)
    got = ~np.isnan(u[:, 0])
    assert 0 < got.sum() < len(u)
    assert np.array_equal(u[got], full[got])
    cpu.u = u
    x_base = c.body.x_base()
    fc, fg = cpu.forces(x_base), gpu.forces(x_base)[0]
    for key in ("cn", "ca"):
        assert np.isfinite(fc[key]) and abs(fg[key] - fc[key]) <= 1e-9 * max(1.0, abs(fc[key])), (key, fg, fc)
