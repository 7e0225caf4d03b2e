"""Failure paths of the run control, made on the host (no GPU fault): a non-finite state handed to the solver through
set_state must come back as BOWSHOCK_NONFINITE (the reference's NonFinite stop, engine/run.rs:105-109), a
negative-pressure cell is handled as the reference handles it (finite, positivity fallbacks),
and a progress callback that asks to stop ends the run at the next report with the Cancelled stop reason
(crates/bowshock-core/src/progress.rs:1-8, engine/run.rs:82-85). The solver kernels have no data-dependent loops or
indices, so a NaN only propagates through the arithmetic."""
import numpy as np
import pytest

from bowshock_b200 import _ffi
from bowshock_b200._ffi import BowshockError
from tests import cases

pytestmark = pytest.mark.gpu


def _implicit_base_solver():
    spec = cases.subsonic_base(0.5)
    return spec, cases.gpu_solver(spec)


def test_nan_state_gives_nonfinite_status():
    spec, s = _implicit_base_solver()
    u = s.state_f64().reshape(-1, 4).copy()
    u[spec.ni * (spec.nj // 2) + spec.ni // 3, 3] = np.nan
    s.set_state(u)
    with pytest.raises(BowshockError) as e:
        s.run(3)
    assert e.value.status == _ffi.NONFINITE


def test_negative_pressure_cell_is_handled_like_the_reference():
    """A cell whose energy is below its kinetic energy (p < 0) is not a non-finite state for the reference: its
    reconstruction falls back to first order next to the cell and the update is positivity-damped (flux.rs:56-72,
    implicit.rs:641-660), so the oracle iterates on with finite residuals. The B200 path does the same, to the
    implicit protocol's tolerance."""
    spec, s = _implicit_base_solver()
    u = s.state_f64().reshape(-1, 4).copy()
    c = spec.ni * (spec.nj // 2) + spec.ni // 3
    u[c, 3] = 0.5 * (u[c, 1] ** 2 + u[c, 2] ** 2) / u[c, 0] - 0.5  # rho E below the kinetic energy: p < 0
    spec.u0 = u
    cpu = cases.oracle_solver(spec)
    gpu = cases.gpu_solver(spec)
    rc = cpu.steps(3)
    rg = gpu.run(3)
    assert np.all(np.isfinite(rc)) and np.all(np.isfinite(rg))
    assert cases.residual_diff(rg, rc) < 1e-3
    assert cases.state_diff(gpu.state_f64(), cpu.u) < 1e-3


def test_warm_run_from_a_nan_state_stops_nonfinite():
    """run_to_stop from a kept (warm) state with a NaN in it: NonFinite at the first iteration, status NONFINITE."""
    from bowshock_b200.case import Case, Numerics, WAKE_BASE, Body, NOSE_TANGENT_OGIVE
    body = Body(NOSE_TANGENT_OGIVE, fineness=3.0, segments=((6.0, 0.0),))
    c = Case.new(0.5, body, 0, WAKE_BASE, Numerics.auto(0.5, 0, WAKE_BASE))
    s = c.build_solver(0)
    ni, nj = c.cells()
    u = s.state_f64().reshape(-1, 4).copy()
    u[ni * (nj // 2) + ni // 3, 0] = np.nan
    s.set_state(u)
    with pytest.raises(BowshockError) as e:
        s.run_to_stop(c.body, c.numerics, c.wake, warm=True, r_ref=1.0)
    assert e.value.status == _ffi.NONFINITE


def test_progress_callback_cancels_the_run():
    from bowshock_b200.case import Case, Numerics, WAKE_BASE, Body, NOSE_TANGENT_OGIVE
    body = Body(NOSE_TANGENT_OGIVE, fineness=3.0, segments=((6.0, 0.0),))
    c = Case.new(0.5, body, 0, WAKE_BASE, Numerics.auto(0.5, 0, WAKE_BASE))
    s = c.build_solver(0)
    seen = []

    def progress(case, it, r, mon):
        seen.append((case, it, r))
        return it < 100  # stop at the second report

    r = s.run_to_stop(c.body, c.numerics, c.wake, progress=progress)
    assert r["stop_reason"] == "cancelled"
    assert r["iters"] == 100 and [it for _, it, _ in seen] == [50, 100]
    assert all(np.isfinite(x) and x > 0 for _, _, x in seen)


def test_arena_cancel_stops_only_that_case():
    """In a batched arena the callback cancels one case; the other runs on to its own stop rule."""
    from bowshock_b200.arena import Arena
    from bowshock_b200.sweep import sweep_cases
    cs = [sweep_cases(32)[k] for k in (2, 6)]  # two Euler cases that stop on the residual drop (485 / 507 iterations)
    a = Arena(cs)
    res = a.solve(progress=lambda k, it, r, m: not (k == 0 and it >= 150))
    assert res[0]["stop_reason"] == "cancelled" and res[0]["iters"] == 150
    assert res[1]["stop_reason"] == "residual drop"
