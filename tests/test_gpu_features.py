"""B200 backend against the oracle on the solver options the sweep workloads leave out, with the reference's GPU-vs-CPU
protocol (crates/bowshock-gpu-cases/tests/common/mod.rs) and its f32 tolerances: the nozzle jet on the base face
(solver.rs:333-347, the jet of solver.rs:903-907), the Venkatakrishnan and first-order limiters, the implicit scheme's
options one at a time (point-implicit, Rusanov Jacobian, explicit boundary rows, the min-direction time step, one
sub-iteration; implicit.rs:59-84), laminar viscosity, and SST with wall roughness and with the jet's k and omega."""
import numpy as np
import pytest

import oracle_ffi as o
from tests import cases
from tests.test_oracle_solver import BLOCK, curved_grid, jet

pytestmark = pytest.mark.gpu

IMPLICIT = dict(cfl0=1.0, cfl_max=30.0, growth=1.02, dt_mode=0, lines=True, implicit_bc=True, sub_iters=2, roe=True, eps_fix=0.1)


def _nozzle_spec(scheme=None, viscous=None):
    ni, nj = 24, 16
    x, r = curved_grid(ni, nj)
    spec = cases.Spec(ni, nj, x, r, 0.5, o.VAN_ALBADA, tuple(o.freestream(2.0)),
                      (o.BC_FREESTREAM, o.BC_EXTRAPOLATE, o.BC_SLIPWALL, o.BC_FREESTREAM), 0, block=BLOCK, scheme=scheme,
                      viscous=viscous, nozzle=jet(), label="curved grid, base block, nozzle jet M2")
    return spec


def _run_pair(spec, n):
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    rc = cpu.steps(n)
    rg = gpu.run(n)
    return cpu, gpu, rc, rg


def test_nozzle_jet_residual_per_cell():  # the jet's face flux enters the residual of the cells behind the base
    spec = _nozzle_spec()
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    cpu.eval_residual(False)
    rg, _, _ = gpu.eval_residual(False)
    rc = cpu.res
    for k in range(4):
        scale = np.max(np.abs(rc[:, k])) + 1e-30
        assert np.max(np.abs(rg[:, k] - rc[:, k])) / scale < 1e-5, k


def test_nozzle_jet_explicit_state_matches_oracle():  # explicit.rs protocol: 1e-5 state, 1e-4 residual history
    cpu, gpu, rc, rg = _run_pair(_nozzle_spec(), 30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-5
    assert cases.residual_diff(rg, rc) < 1e-4


def test_nozzle_jet_implicit_state_matches_oracle():  # implicit.rs protocol: 1e-3
    spec = _nozzle_spec(scheme=dict(IMPLICIT))
    spec.first_order_iters = 5
    cpu, gpu, rc, rg = _run_pair(spec, 30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-3
    assert cases.residual_diff(rg[:5], rc[:5]) < 1e-3


def test_nozzle_jet_sst_matches_oracle():  # the jet's k and omega in the SST ghosts of the nozzle rows
    spec = _nozzle_spec(scheme=dict(IMPLICIT, dt_mode=1, cfl_max=10.0, sub_iters=3),
                        viscous=dict(re_c=1e6, sutherland=0.368, turbulence=o.TURB_SST, wall_i_start=0, roughness=0.0))
    spec.first_order_iters = 5
    cpu, gpu, rc, rg = _run_pair(spec, 20)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-3
    t_g, _ = gpu.turb_state()
    fluid = cpu.turb[:, 0] > 0
    for e in range(2):
        err = np.max(np.abs(t_g[fluid, e] - cpu.turb[fluid, e]) / np.abs(cpu.turb[fluid, e]))
        assert err < 1e-2, (e, err)


@pytest.mark.parametrize("limiter", [o.VENKATAKRISHNAN, o.FIRST_ORDER])
@pytest.mark.parametrize("mach", [0.5, 1.3])
def test_limiters_explicit_state_matches_oracle(limiter, mach):
    spec = cases.far_field_box(mach)
    spec.limiter = limiter
    spec.u0 = cases.perturbed_state(spec)
    cpu, gpu, rc, rg = _run_pair(spec, 30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-5
    assert cases.residual_diff(rg, rc) < 1e-4


@pytest.mark.parametrize("option", [dict(lines=False), dict(roe=False), dict(implicit_bc=False), dict(dt_mode=1),
                                    dict(sub_iters=1), dict(sub_iters=4)], ids=lambda d: next(iter(d)) + "=" + str(next(iter(d.values()))))
def test_implicit_options_match_oracle(option):  # one option of implicit.rs:59-84 changed from the default
    spec = cases.far_field_box(0.5)
    spec.u0 = cases.perturbed_state(spec)
    spec.scheme = dict(IMPLICIT, **option)
    cpu, gpu, rc, rg = _run_pair(spec, 30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-3
    assert cases.residual_diff(rg, rc) < 1e-2


def test_venkatakrishnan_implicit_sting_matches_oracle():
    spec = cases.subsonic_sting(0.5)
    spec.limiter = o.VENKATAKRISHNAN
    spec.first_order_iters = 5
    cpu, gpu, rc, rg = _run_pair(spec, 30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-3
    assert cases.residual_diff(rg[:5], rc[:5]) < 1e-3


def test_g3_body_laminar_matches_oracle():  # the G3 grid with laminar viscosity only (no turbulence model)
    spec = cases.g3_body()
    spec.viscous = dict(spec.viscous, turbulence=o.TURB_LAMINAR)
    spec.first_order_iters = 5
    cpu, gpu, rc, rg = _run_pair(spec, 30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-3
    assert cases.residual_diff(rg[:5], rc[:5]) < 1e-3


def test_g3_body_rough_wall_sst_matches_oracle():  # SST with a sand-grain roughness on the body (the rough-wall omega)
    spec = cases.g3_body()
    spec.viscous = dict(spec.viscous, roughness=2e-4)
    spec.first_order_iters = 5
    cpu, gpu, rc, rg = _run_pair(spec, 30)
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-3
    t_g, m_g = gpu.turb_state()
    fluid = cpu.turb[:, 0] > 0
    for e in range(2):
        err = np.max(np.abs(t_g[fluid, e] - cpu.turb[fluid, e]) / np.abs(cpu.turb[fluid, e]))
        assert err < 1e-2, (e, err)
    assert np.max(np.abs(m_g[fluid] - cpu.mu_t[fluid]) / np.abs(cpu.mu_t[fluid])) < 1e-2
