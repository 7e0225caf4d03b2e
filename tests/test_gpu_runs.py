"""Whole runs on the B200 backend: the FP64 device force pass against the oracle's post-processing of the same state,
converged drag of the reference's G3 body against the FP64 oracle (|dCD| <= 1e-4, the target of the sweep metric), and
the batched arena against single-case solvers."""
import json
import os

import numpy as np
import pytest

import oracle_ffi as o

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def g3_cases():
    from bowshock_b200.case import Body, Case, WAKE_BASE, rans_params
    from tests.golden.g3_case import g3_case
    re_c, suth = rans_params(0.0, 0.1)
    pc = Case.viscous_case(0.5, Body(0, fineness=3.0, segments=((6.0, 0.0),)), 0, WAKE_BASE, re_c, suth, 0.5)
    return pc, g3_case()


@pytest.mark.parametrize("roughness", [0.0, 2e-5])
def test_device_forces_match_the_oracle_post_processing(roughness):  # engine/run.rs:188-313 on the same state
    pc, oc = g3_cases()
    pc.viscous.roughness = roughness  # rough: the friction adds the Aupoix mu_t,w (run.rs:241)
    oc.roughness = roughness
    s = pc.build_solver()
    s.run(300)
    f = s.forces(pc.body)
    cpu = o.Solver.from_case(oc)
    cpu.u = s.state_f64()
    r = o.finish(oc, cpu)
    for k in ("cd_nose", "cd_base", "cd_friction", "cp_base", "y_plus_max", "cd_total"):
        a, b = f[k], getattr(r, k)
        assert abs(a - b) <= 1e-10 * max(1.0, abs(b)), (k, a, b)


def test_g3_converged_drag_matches_the_fp64_oracle():
    pc, _ = g3_cases()
    ref = json.load(open(os.path.join(HERE, "golden", "g3_oracle.json")))
    s = pc.build_solver()
    r = s.run_to_stop(pc.body, pc.numerics, pc.wake)
    print("G3 on B200:", {k: r[k] for k in ("iters", "stop_reason", "cd_total", "cd_friction", "cd_base", "cp_base", "y_plus_max")})
    assert r["stop_reason"] in ("CD stationary", "residual drop", "mean stationary")
    for k in ("cd_total", "cd_friction", "cd_base"):
        assert abs(r[k] - ref[k]) <= 1e-4, (k, r[k], ref[k])


def test_arena_cases_match_single_case_solvers():
    from bowshock_b200.arena import Arena
    from bowshock_b200.case import Body, Case, WAKE_BASE, WAKE_STING
    pc, _ = g3_cases()
    cases = [Case.new(0.5, Body(0, 3.0, segments=((6.0, 0.0),)), 0, WAKE_STING), Case.new(1.5, Body(0, 3.0, segments=((6.0, 0.0),)), 0, WAKE_BASE), pc]
    for c in cases:
        c.numerics.first_order_iters = 5
    a = Arena(cases)
    ra = a.run(40)
    for k, c in enumerate(cases):
        s = c.build_solver()
        rs = s.run(40)
        assert np.array_equal(a.state(k), s.state_f64()), f"case {k} differs from its single-case solver"
        assert np.allclose(ra[:, k], rs, rtol=1e-12)


def test_captured_chunks_match_kernel_by_kernel_launches():
    """run() replays 50-iteration chunks captured as CUDA graphs; profile() launches the same kernels one at a time
    (SST case). The states agree bit for bit."""
    from bowshock_b200.arena import Arena
    pc, _ = g3_cases()
    pc.numerics.first_order_iters = 5
    a, b = Arena([pc]), Arena([pc])
    a.run(30)
    b.profile(30)
    assert np.array_equal(a.state(0), b.state(0))


@pytest.mark.parametrize("segment", [4, 8])
def test_longer_line_segments_match_the_oracle(segment):
    """Line solves with at least `segment` cells per lane (fewer separators on short lines, a shape the autotuner may
    pick): the viscous.rs body protocol against the oracle, 30 implicit iterations, state within 1e-3."""
    from bowshock_b200.arena import Arena
    from tests import cases
    pc, oc = g3_cases()
    pc.numerics.first_order_iters = 5
    a = Arena([pc])
    a.set_tuning(segment_i=segment, segment_j=segment)
    assert a.tuning()["segment_i"] == segment
    a.run(30)
    spec = cases.from_case(oc, "G3")
    spec.first_order_iters = 5
    cpu = cases.oracle_solver(spec)
    cpu.steps(30)
    assert cases.state_diff(a.state(0), cpu.u) < 1e-3


def test_autotuner_candidates_give_bit_identical_states():
    """Every launch shape the autotuner may pick (lines per block and prefetching of the first pass and of the
    substitution passes, the walks of both passes staged through shared memory, lines per block of the SST line kernel;
    not the residual kernel's threads per tile, which the autotuner no longer varies) compiles to the same
    arithmetic, so the state after a run does not depend on the tuning: checked bit for bit on a mixed Euler / SST arena."""
    from bowshock_b200.arena import Arena
    from bowshock_b200.sweep import sweep_cases
    sel = [sweep_cases()[k] for k in (0, 9)]  # an Euler sting case and an SST limit-cycle case
    base = dict(lines_i=4, lines_j=4, prefetch_i=0, prefetch_j=0, subst_i=4, subst_j=4, turb_lines=4, segment_i=2, segment_j=2,
                residual=1, subst_prefetch_i=0, subst_prefetch_j=0, staged_lines=0)
    variants = [dict(lines_i=1, lines_j=2, prefetch_i=1, prefetch_j=1), dict(subst_i=1, subst_j=8),
                dict(subst_prefetch_i=1, subst_prefetch_j=1), dict(subst_i=1, subst_j=8, subst_prefetch_i=1, subst_prefetch_j=1),
                dict(subst_prefetch_i=2, subst_prefetch_j=2), dict(subst_prefetch_i=2), dict(prefetch_i=2, prefetch_j=2),
                dict(staged_lines=1 << 20),
                dict(turb_lines=1), dict(turb_lines=8)]
    ref = None
    for v in [dict()] + variants:
        a = Arena(sel)
        a.set_tuning(**{**base, **v})
        a.run(60)
        st = [a.state(k) for k in range(len(sel))]
        if ref is None:
            ref = st
        else:
            assert all(np.array_equal(x, y) for x, y in zip(st, ref)), f"tuning {v} changed the state"
