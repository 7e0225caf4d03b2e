"""B200 backend against the oracle, through the C ABI, with the reference's GPU-vs-CPU protocol and tolerances
(crates/bowshock-gpu-cases/tests/{explicit,implicit,viscous}.rs): the same start state, N iterations, state and residual
history compared. The FP32 tolerances are the reference's own for its f32 GPU path: explicit state 1e-5 / residual 1e-4
(explicit.rs:10-12), implicit state 1e-3 (implicit.rs:6-8, viscous.rs body check)."""
import numpy as np
import pytest

import oracle_ffi as o
from tests import cases

pytestmark = pytest.mark.gpu


def _per_cell_residual_check(spec, tol):
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    cpu.eval_residual(True)
    rc, dc = cpu.res, cpu.dt
    rg, dg, dens = gpu.eval_residual(True)
    # per component, relative to the component's largest magnitude over the grid (FP32 flux differences)
    for k in range(4):
        scale = np.max(np.abs(rc[:, k])) + 1e-30
        err = np.max(np.abs(rg[:, k] - rc[:, k])) / scale
        assert err < tol, f"{spec.label}: residual component {k} max rel err {err:.3e}"
    fluid = dc > 0
    assert np.max(np.abs(dg[fluid] - dc[fluid]) / dc[fluid]) < 1e-5
    assert abs(dens - cpu.density_residual()) / cpu.density_residual() < 1e-4


def test_residual_per_cell_far_field_box():
    spec = cases.far_field_box(0.5)
    spec.u0 = cases.perturbed_state(spec)
    spec.first_order_iters = 0
    _per_cell_residual_check(spec, 1e-5)


def test_residual_per_cell_base_block():
    spec = cases.subsonic_base(0.5)
    rng = np.random.default_rng(7)
    u = np.tile(o.prim_to_cons(np.array(spec.fs)), (spec.ni * spec.nj, 1))
    w = o.cons_to_prim(u)
    w[:, 0] *= 1 + 0.05 * rng.standard_normal(len(w))
    w[:, 1] += 0.05 * rng.standard_normal(len(w))
    w[:, 2] += 0.05 * rng.standard_normal(len(w))
    w[:, 3] *= 1 + 0.05 * rng.standard_normal(len(w))
    spec.u0 = o.prim_to_cons(w)
    spec.first_order_iters = 0
    _per_cell_residual_check(spec, 2e-5)


@pytest.mark.parametrize("mach,outflow", [(0.5, o.BC_CHARACTERISTIC), (1.3, o.BC_CHARACTERISTIC), (0.5, o.BC_PRESSURE_OUTFLOW)])
def test_explicit_state_matches_oracle(mach, outflow):  # explicit.rs protocol, f32 tolerances
    spec = cases.far_field_box(mach, outflow)
    spec.u0 = cases.perturbed_state(spec)
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    rc = cpu.steps(30)
    rg = gpu.run(30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-5
    assert cases.residual_diff(rg, rc) < 1e-4


@pytest.mark.parametrize("maker", [cases.subsonic_sting, cases.subsonic_base])
def test_implicit_state_matches_oracle(maker):  # implicit.rs:11-35 protocol
    spec = maker(0.5)
    spec.first_order_iters = 5
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    rc = cpu.steps(30)
    rg = gpu.run(30)
    d = cases.state_diff(gpu.state_f64(), cpu.u)
    assert d < 1e-3, f"{spec.label}: state diff {d:.3e}"
    assert np.all(np.isfinite(rg))
    assert cases.residual_diff(rg[:5], rc[:5]) < 1e-3


def test_implicit_box_with_perturbation_matches_oracle():
    spec = cases.far_field_box(0.5)
    spec.u0 = cases.perturbed_state(spec)
    spec.scheme = dict(cfl0=1.0, cfl_max=30.0, growth=1.02, dt_mode=0, lines=True, implicit_bc=True, sub_iters=2, roe=True, eps_fix=0.1)
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    rc = cpu.steps(30)
    rg = gpu.run(30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-3
    assert cases.residual_diff(rg, rc) < 1e-2


def test_g3_body_sst_matches_oracle():  # viscous.rs body check: 30 implicit iterations, first 5 first order
    spec = cases.g3_body()
    spec.first_order_iters = 5
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    rc = cpu.steps(30)
    rg = gpu.run(30)
    d = cases.state_diff(gpu.state_f64(), cpu.u)
    assert d < 1e-3, f"G3 state diff {d:.3e}"
    t_g, m_g = gpu.turb_state()
    t_c = cpu.turb
    fluid = t_c[:, 0] > 0
    for e, name in ((0, "k"), (1, "omega")):
        err = np.max(np.abs(t_g[fluid, e] - t_c[fluid, e]) / np.abs(t_c[fluid, e]))
        assert err < 1e-2, f"G3 {name} max rel diff {err:.3e}"
    assert np.max(np.abs(m_g[fluid] - cpu.mu_t[fluid]) / np.abs(cpu.mu_t[fluid])) < 1e-2


def _mg_spec(ni, nj, mach, limiter, cfl, u_scale=None):
    from tests.test_oracle_solver import mg_grid
    x, r = mg_grid(ni, nj)
    spec = cases.Spec(ni, nj, x, r, cfl, limiter, tuple(o.freestream(mach)),
                      (o.BC_CHARACTERISTIC, o.BC_CHARACTERISTIC, o.BC_SLIPWALL, o.BC_CHARACTERISTIC), 0, label="mg grid")
    if u_scale is not None:
        fs = o.freestream(mach)
        w = np.array([fs[0] * u_scale[0], fs[1], fs[2], fs[3] * u_scale[1]])
        spec.u0 = np.tile(o.prim_to_cons(w), (ni * nj, 1))
    return spec


def _mg_pair(spec):
    import bowshock_b200 as bk
    cpu = cases.oracle_solver(spec)
    levels = cpu.set_scheme(o.multigrid_scheme())
    gpu = cases.gpu_solver(spec)
    gpu.set_scheme(bk.solver.MgParams())
    if spec.u0 is not None:
        gpu.set_state(spec.u0)
    return cpu, gpu, levels


def test_multigrid_hierarchy_preserves_the_free_stream():  # multigrid.rs:239-258
    spec = _mg_spec(64, 32, 0.5, o.VAN_ALBADA, 0.5)
    cpu, gpu, levels = _mg_pair(spec)
    assert levels == 3
    gpu.run(30)
    # FP32 round-off: a few ulps of E ~ 1.9 (the reference's f32 explicit state tolerance is 1e-5)
    assert np.max(np.abs(gpu.state_f64() - o.prim_to_cons(o.freestream(0.5)))) < 1e-5


def test_multigrid_cycles_match_the_oracle():  # cycle-by-cycle FAS state, perturbed start of multigrid.rs:274-276
    spec = _mg_spec(32, 16, 0.4, o.FIRST_ORDER, 0.8, u_scale=(1.02, 1.03))
    cpu, gpu, _ = _mg_pair(spec)
    rc = cpu.steps(30)
    rg = gpu.run(30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-5
    assert cases.residual_diff(rg[:10], rc[:10]) < 1e-3


def test_multigrid_reaches_the_explicit_fixed_point():  # multigrid.rs:260-291, to FP32 round-off
    spec = _mg_spec(32, 16, 0.4, o.FIRST_ORDER, 0.8, u_scale=(1.02, 1.03))
    cpu = cases.oracle_solver(spec)
    for _ in range(4000):
        if cpu.step() < 1e-11:
            break
    import bowshock_b200 as bk
    gpu = cases.gpu_solver(spec)
    gpu.set_scheme(bk.solver.MgParams())
    gpu.set_state(spec.u0)
    r = gpu.run(1500)
    # an FP32 state stalls about 4-5 orders down (the reference's f32 runs: crates/bowshock-cfd/src/gpu/mod.rs:61-62)
    assert r[-1] < 1e-4 * r[0]
    assert np.max(np.abs(gpu.state_f64() - cpu.u)) < 1e-5


# Per-cell residual on the two single-case workloads' own grids (config 0: Euler, 128 x 64, M 1.5 with its bow shock;
# config 1: RANS SST, 256 x 128, y+ ~ 1 wall cells, M 0.9), from a developed state: 40 oracle iterations of the case's
# own numerics from the free stream, handed to both sides (mean flow and, for SST, k, omega and mu_t), then one residual
# evaluation with the second-order reconstruction. Tolerance relative to each component's largest magnitude: 2e-5 for
# the inviscid residual, 1e-4 with the viscous and SST terms (gradients and eddy viscosity read the FP32 state).
@pytest.mark.parametrize("name,tol", [("config0", 2e-5), ("config1", 1e-4)])
def test_residual_per_cell_on_config_grids(name, tol):
    from tests.golden.configs import CONFIGS
    from tests.golden.sweep_oracle import oracle_case
    c = CONFIGS[name]()
    spec = cases.from_case(oracle_case(c), name)
    dev = cases.oracle_solver(spec)
    dev.steps(40)
    spec.u0 = dev.u.copy()
    spec.first_order_iters = 0
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    if spec.viscous is not None:
        cpu.turb, cpu.mu_t = dev.turb.copy(), dev.mu_t.copy()
        gpu.set_turb(dev.turb, dev.mu_t)
    cpu.eval_residual(True)
    rc, dc = cpu.res, cpu.dt
    rg, dg, dens = gpu.eval_residual(True)
    errs = []
    for k in range(4):
        scale = np.max(np.abs(rc[:, k])) + 1e-30
        errs.append(np.max(np.abs(rg[:, k] - rc[:, k])) / scale)
    print(name, "per-component max rel residual error", [f"{e:.2e}" for e in errs])
    assert max(errs) < tol, f"{name}: residual max rel err {max(errs):.3e}"
    fluid = dc > 0
    assert np.max(np.abs(dg[fluid] - dc[fluid]) / dc[fluid]) < 1e-5
    assert abs(dens - cpu.density_residual()) / cpu.density_residual() < 1e-4


# Implicit residual smoothing (Scheme::Smoothed, solver.rs:104-120, 722-803): SSP-RK3 at CFL 1.5 with every direction
# whose CFL number exceeds 0.5 smoothed, on the far-field box and on the base-block grid (smoothing coefficients zero
# next to solid cells); the explicit protocol's tolerances (the smoothing's Thomas sweeps run in FP32).
@pytest.mark.parametrize("maker", ["box", "base"])
def test_smoothed_scheme_matches_oracle(maker):
    import bowshock_b200 as bk
    if maker == "box":
        spec = cases.far_field_box(0.5)
        spec.u0 = cases.perturbed_state(spec)
    else:
        spec = cases.subsonic_base(0.5)
        spec.scheme = None
        spec.first_order_iters = 5
    spec.cfl = 1.5
    cpu = cases.oracle_solver(spec)
    cpu.set_scheme(o.OrcScheme(kind=1, cfl_star=0.5))
    gpu = cases.gpu_solver(spec)
    gpu.set_scheme(bk.solver.Smoothed(0.5))
    if spec.u0 is not None:
        gpu.set_state(spec.u0)
    rc = cpu.steps(30)
    rg = gpu.run(30)
    d = cases.state_diff(gpu.state_f64(), cpu.u)
    assert np.all(np.isfinite(rg)) and d < 1e-5, f"{maker}: state diff {d:.3e}"
    assert cases.residual_diff(rg, rc) < 1e-4


def test_multigrid_with_smoothed_smoother_matches_oracle():  # MgParams::irs: the smoother's stages smoothed on every level
    import bowshock_b200 as bk
    spec = _mg_spec(32, 16, 0.4, o.FIRST_ORDER, 1.2, u_scale=(1.02, 1.03))
    cpu = cases.oracle_solver(spec)
    cpu.set_scheme(o.multigrid_scheme(cfl_star=0.5))
    gpu = cases.gpu_solver(spec)
    gpu.set_scheme(bk.solver.MgParams(cfl_star=0.5))
    gpu.set_state(spec.u0)
    rc = cpu.steps(30)
    rg = gpu.run(30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-5
    assert cases.residual_diff(rg[:10], rc[:10]) < 1e-3


# The same check on every grid of the 32-case sweep (96 x 48 to 320 x 160 cells; cone, ogive and von Karman noses,
# boattails, sting and base wakes, Euler and RANS SST, M 0.36 to 2.91), from 40 oracle iterations of each case's own
# numerics (the oracle case of the sweep census, tests/golden/sweep_oracle.py).
@pytest.mark.parametrize("k", range(32))
def test_residual_per_cell_on_sweep_grids(k):
    from bowshock_b200.sweep import sweep_cases
    from tests.golden.sweep_oracle import oracle_case
    c = sweep_cases()[k]
    tol = 2e-5 if c.viscous is None else 1e-4
    spec = cases.from_case(oracle_case(c), f"sweep case {k}")
    dev = cases.oracle_solver(spec)
    dev.steps(40)
    spec.u0 = dev.u.copy()
    spec.first_order_iters = 0
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    if spec.viscous is not None:
        cpu.turb, cpu.mu_t = dev.turb.copy(), dev.mu_t.copy()
        gpu.set_turb(dev.turb, dev.mu_t)
    cpu.eval_residual(True)
    rc, dc = cpu.res, cpu.dt
    rg, dg, dens = gpu.eval_residual(True)
    errs = [np.max(np.abs(rg[:, q] - rc[:, q])) / (np.max(np.abs(rc[:, q])) + 1e-30) for q in range(4)]
    assert max(errs) < tol, f"sweep case {k}: residual max rel err {max(errs):.3e}"
    fluid = dc > 0
    assert np.max(np.abs(dg[fluid] - dc[fluid]) / dc[fluid]) < 1e-5
    assert abs(dens - cpu.density_residual()) / cpu.density_residual() < 1e-4


# The reference's implicit GPU-vs-CPU protocol (implicit.rs:11-35; viscous.rs body check for the SST cases) on sweep
# grids: each case's own numerics from the free stream, 5 first-order iterations, 30 iterations, the state within 1e-3
# and the first 5 residuals within 1e-3. Euler and SST, sting and base wakes, sub- and supersonic.
@pytest.mark.parametrize("k", [0, 1, 2, 7, 13, 18, 21, 24])
def test_implicit_protocol_on_sweep_grids(k):
    from bowshock_b200.sweep import sweep_cases
    from tests.golden.sweep_oracle import oracle_case
    spec = cases.from_case(oracle_case(sweep_cases()[k]), f"sweep case {k}")
    spec.first_order_iters = 5
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    rc = cpu.steps(30)
    rg = gpu.run(30)
    d = cases.state_diff(gpu.state_f64(), cpu.u)
    assert np.all(np.isfinite(rg))
    assert d < 1e-3, f"{spec.label}: state diff {d:.3e}"
    assert cases.residual_diff(rg[:5], rc[:5]) < 1e-3
