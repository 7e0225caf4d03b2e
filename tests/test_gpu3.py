"""3D Euler on the B200 (bowshock3_* through the C ABI) against the 3D oracle (oracle/solver3.cpp), with the reference's
GPU-vs-CPU protocol: the same start state, the per-cell residual of one evaluation, N iterations of the explicit (1e-5) and
implicit (1e-3) schemes, the batch against single cases, and a converged small case's normal force; at the full sweep grid
(192 x 64 x 64) the per-cell residual of one evaluation."""
import math

import numpy as np
import pytest

import oracle_ffi as o

pytestmark = pytest.mark.gpu


def _grid(ni, nj, nk, mach=1.2, alpha_deg=4.0):
    from bowshock_b200.euler3 import lift_sweep_cases
    c = lift_sweep_cases((alpha_deg,), (mach,), ni=ni, nj=nj, nk=nk)[0]
    ni2, nj2, x2, r2, _ = c.case2.grid()
    return c, ni2, nj2, np.asarray(x2), np.asarray(r2)


def _pair(ni, nj, nk, mach, alpha_deg, implicit=True, first_order=0, limiter=o.MINMOD):
    import bowshock_b200.euler3 as e3
    c, ni2, nj2, x2, r2 = _grid(ni, nj, nk, mach, alpha_deg)
    theta = np.pi * np.arange(nk + 1) / nk
    axis = c.case2.grid_sting.n_up
    alpha = math.radians(alpha_deg)
    p = o.implicit3_params(cfl_max=10.0)
    cpu = o.Solver3(ni2, nj2, x2, r2, nk, theta, axis, mach, alpha, limiter=limiter, first_order_iters=first_order, implicit=implicit,
                    params=p)
    cfg = e3.Config3(mach, alpha, 0.5, limiter, first_order, False, e3.ImplicitParams(cfl_max=10.0) if implicit else e3.EXPLICIT)
    x, y, z = e3.revolve(x2, r2, nk)
    gpu = e3.Batch3(ni2, nj2, nk, x, y, z, axis, [cfg])
    return cpu, gpu, c


def _perturb(cpu, seed, amp=0.02):
    rng = np.random.default_rng(seed)
    w = o.cons_to_prim3(cpu.u)
    w[:, 0] *= 1 + amp * rng.standard_normal(len(w))
    w[:, 1:4] += amp * rng.standard_normal((len(w), 3))
    w[:, 4] *= 1 + amp * rng.standard_normal(len(w))
    return o.prim_to_cons3(w)


def _residual_check(ni, nj, nk, tol):
    cpu, gpu, _ = _pair(ni, nj, nk, 1.2, 4.0)
    u0 = _perturb(cpu, 3)
    cpu.u = u0
    gpu.set_state(0, u0)
    dc = cpu.eval_residual(1.0)  # implicit dt at the first ramp step: cfl0 = 1
    rg, dtg, dg = gpu.eval_residual(0)
    rc = cpu.res
    for k in range(5):
        scale = np.max(np.abs(rc[:, k])) + 1e-30
        err = np.max(np.abs(rg[:, k] - rc[:, k])) / scale
        assert err < tol, f"component {k}: max rel err {err:.3e}"
    assert abs(dg - dc) / dc < 1e-5
    assert np.max(np.abs(dtg - cpu.dt) / cpu.dt) < 1e-5


def test_residual_per_cell_small():
    _residual_check(48, 16, 8, 1e-5)


def test_residual_per_cell_at_the_sweep_grid():  # 192 x 64 x 64 = 786,432 cells
    _residual_check(192, 64, 64, 1e-5)


def test_explicit_state_matches_oracle():  # explicit.rs protocol, f32 tolerance
    cpu, gpu, _ = _pair(48, 16, 8, 2.5, 6.0, implicit=False, limiter=o.MINMOD)
    u0 = _perturb(cpu, 5, 0.01)
    cpu.u = u0
    gpu.set_state(0, u0)
    rc = cpu.steps(20)
    rg = gpu.run(20)[:, 0]
    d = np.max(np.abs(gpu.state(0) - cpu.u) / (1 + np.abs(cpu.u)))
    assert d < 1e-5, d
    assert np.max(np.abs(rg - rc) / rc) < 1e-4


@pytest.mark.parametrize("mach,alpha", [(0.8, 4.0), (2.5, 8.0)])
def test_implicit_state_matches_oracle(mach, alpha):  # implicit.rs protocol (f32 left-hand side): 1e-3
    cpu, gpu, _ = _pair(48, 16, 8, mach, alpha, implicit=True, first_order=5)
    rc = cpu.steps(30)
    rg = gpu.run(30)[:, 0]
    d = np.max(np.abs(gpu.state(0) - cpu.u) / (1 + np.abs(cpu.u)))
    assert d < 1e-3, d
    assert np.all(np.isfinite(rg))
    assert np.max(np.abs(rg[:5] - rc[:5]) / rc[:5]) < 1e-3


def test_batch_matches_single_cases():
    import bowshock_b200.euler3 as e3
    cases = e3.lift_sweep_cases((0.0, 4.0), (0.8, 2.5), ni=48, nj=16, nk=8)
    batch, _ = e3.batch_of(cases)
    rb = batch.run(25)
    for k, c in enumerate(cases):
        single, _ = e3.batch_of([c])
        rs = single.run(25)[:, 0]
        assert np.array_equal(single.state(0), batch.state(k))
        # the norm's FP64 block sums are added atomically in no fixed order: equal to round-off
        assert np.max(np.abs(rs - rb[:, k]) / rb[:, k]) < 1e-12


def test_converged_normal_force_matches_oracle():  # run3.rs stop rules on both, CN and centre of pressure
    cpu, gpu, c = _pair(48, 16, 8, 2.5, 4.0, implicit=True, first_order=100)
    x_base = c.body.x_base()
    rc = cpu.run(x_base, max_iter=4000)
    rg = gpu.solve(x_base, max_iter=4000)[0]
    assert rc["stop_reason"] in ("residual drop", "CN stationary"), rc
    assert rg["stop_reason"] in ("residual drop", "CN stationary"), rg
    assert abs(rg["cn"] - rc["cn"]) <= 2e-3 * abs(rc["cn"]) + 1e-4, (rg, rc)
    assert abs(rg["x_cp"] - rc["x_cp"]) <= 2e-2, (rg, rc)


def test_converged_normal_force_matches_oracle_at_96x32x32():
    """The lift-sweep body at 96 x 32 x 32 cells (98,304; the largest the 3D oracle finishes in minutes on the host) at
    M 1.2 and M 2.5, 4 degrees: the batch's converged CN and centre of pressure against the oracle's
    (tests/golden/lift3_oracle.json, make_lift3_fixture.py), both to run3.rs's stop rules. Tolerances as for the small
    case: the CN-stationary rule holds CN to 0.2 % over its window on either side."""
    import json
    import os
    import bowshock_b200.euler3 as e3
    fx = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lift3_oracle.json")))
    ni, nj, nk = fx["grid"]
    cfgs, x_base = [], None
    machs = sorted(fx["cases"], key=float)
    grid = None
    for m in machs:
        c, ni2, nj2, x2, r2 = _grid(ni, nj, nk, float(m), fx["alpha_deg"])
        cfgs.append(e3.Config3(float(m), math.radians(fx["alpha_deg"]), 0.5, o.MINMOD, fx["first_order"], False, e3.ImplicitParams(cfl_max=10.0)))
        grid = (ni2, nj2, x2, r2, c.case2.grid_sting.n_up)
        x_base = c.body.x_base()
    ni2, nj2, x2, r2, axis = grid
    x, y, z = e3.revolve(x2, r2, nk)
    gpu = e3.Batch3(ni2, nj2, nk, x, y, z, axis, cfgs)
    res = gpu.solve(x_base, max_iter=fx["max_iter"])
    for m, rg in zip(machs, res):
        rc = fx["cases"][m]
        print(m, rg["iterations"], rg["stop_reason"], rg["cn"], rc["cn"], rg["x_cp"], rc["x_cp"])
        assert rg["stop_reason"] in ("residual drop", "CN stationary"), rg
        assert abs(rg["cn"] - rc["cn"]) <= 2e-3 * abs(rc["cn"]) + 1e-4, (m, rg, rc)
        assert abs(rg["x_cp"] - rc["x_cp"]) <= 2e-2, (m, rg, rc)


@pytest.mark.parametrize("dims", [(96, 32, 32), (192, 64, 64)])
def test_staged_first_pass_is_bit_identical(dims):
    """The first line pass staged through shared memory (bowshock3_set_staging, on where a warp's 32 lines are adjacent:
    all three directions on these grids) against the unstaged walk: the same arithmetic, so the same states bit for bit
    after 6 implicit iterations of a batch at two Mach numbers, with and without a fin box; the residual norms to the
    round-off of their atomic block sums."""
    import bowshock_b200.euler3 as e3
    ni, nj, nk = dims
    cases = e3.lift_sweep_cases((4.0,), (0.8, 2.5), ni=ni, nj=nj, nk=nk)
    for boxes in ([], [((ni // 2, ni // 2 + 8), (0, 4), (nk // 2 - 1, nk // 2 + 1))]):
        runs = []
        for staged in (True, False):
            b, _ = e3.batch_of(cases)
            if boxes:
                b.set_solid(boxes)
            b.set_staging(staged)
            r = b.run(6)
            runs.append((r, [b.state(k) for k in range(len(cases))]))
            del b
        (r1, s1), (r0, s0) = runs
        for a, c in zip(s1, s0):
            assert np.array_equal(a, c)
        assert np.max(np.abs(r1 - r0) / r0) < 1e-12


def test_case_groups_are_bit_identical():
    """bowshock3_set_groups: the batch's cases split into 2 or 3 groups whose iterations run on streams of their own give
    the states of one group bit for bit (every kernel touches only its own cases) after 6 implicit iterations."""
    import bowshock_b200.euler3 as e3
    cases = e3.lift_sweep_cases((0.0, 4.0, 8.0), (0.8, 2.5), ni=96, nj=32, nk=32)
    ref = None
    for groups in (1, 2, 3):
        b, _ = e3.batch_of(cases)
        b.set_groups(groups)
        r = b.run(6)
        st = [b.state(k) for k in range(len(cases))]
        del b
        if ref is None:
            ref = (r, st)
            continue
        for a, c in zip(st, ref[1]):
            assert np.array_equal(a, c)
        assert np.max(np.abs(r - ref[0]) / ref[0]) < 1e-12
    b, _ = e3.batch_of(cases)
    with pytest.raises(e3.BowshockError):
        b.set_groups(5)


def test_set_config_changes_the_free_stream_between_runs():
    """bowshock3_set_config (GpuSolver3::set_config): case 0's Mach number changed after 10 iterations, state and
    counters kept; the next 10 iterations equal, bit for bit, those of a batch created with the new configuration from
    the same state and counters."""
    import bowshock_b200.euler3 as e3
    cases = e3.lift_sweep_cases((4.0,), (0.8, 2.5), ni=48, nj=16, nk=8)
    b, _ = e3.batch_of(cases)
    b.run(10)
    u0, u1 = b.state(0), b.state(1)
    new = e3.lift_sweep_cases((4.0,), (1.2,), ni=48, nj=16, nk=8)[0].config()
    b.set_config(0, new)
    b.run(10)
    ref, _ = e3.batch_of(e3.lift_sweep_cases((4.0,), (1.2,), ni=48, nj=16, nk=8) + cases[1:])
    ref.set_state(0, u0)
    ref.set_state(1, u1)
    ref.set_iter(10, 10)
    ref.run(10)
    assert np.array_equal(b.state(0), ref.state(0))
    assert np.array_equal(b.state(1), ref.state(1))


def test_profile_groups():
    """bowshock3_profile: every kernel group of the implicit iteration timed (the RK3 stage not launched), with the launch
    counts of the three-factor scheme at sub_iters 2."""
    import bowshock_b200.euler3 as e3
    b, _ = e3.batch_of(e3.lift_sweep_cases((4.0,), (0.8, 2.5), ni=48, nj=16, nk=8))
    b.run(3)
    p = b.profile(4)
    counts = {g: n for g, (ms, n) in p.items()}
    assert counts == {"prims": 8, "flux": 12, "residual": 4, "assemble": 8, "lines": 12, "subst": 12, "defect": 8, "stage": 0}, counts
    assert all(ms > 0 for g, (ms, n) in p.items() if n), p
