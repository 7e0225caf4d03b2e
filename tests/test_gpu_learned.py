"""The warm-start path of the batched arena on the B200: per-case residual histories of a solve, warm runs (state and
turbulence handed in, no first-order phase, the drop measured from a given reference; engine/run.rs:54-63) and the
first-residual probe the fallback rule uses; and, with the committed trained network, the learned warm start on held-out
SST cases against their cold starts."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cd(r):
    return r["cd_window"] if r["stop_reason"] == "mean stationary" else r["cd_total"]


def test_warm_restart_from_a_converged_state_stops_at_once():
    from bowshock_b200.arena import Arena
    from bowshock_b200.sweep import sweep_cases
    cs = [sweep_cases(32)[k] for k in (2, 6)]  # Euler cases that stop on the residual drop
    a = Arena(cs)
    cold = a.solve()
    for k in range(2):
        h = a.residual_history(k)
        assert len(h) == cold[k]["iters"] and np.all(np.isfinite(h)) and cold[k]["stop_reason"] == "residual drop"
        assert cold[k]["residual_peak"] == pytest.approx(h[20:].max(), rel=1e-12)  # the peak after the 20 skipped iterations
    states = [a.state(k) for k in range(2)]
    b = Arena(cs)
    for k in range(2):
        b.set_state(k, states[k])
        b.set_run(k, cs[k].numerics, warm=True, r_ref=cold[k]["residual_peak"])
    first_warm = b.first_residuals([1, 1])
    warm = b.solve()
    for k in range(2):
        assert warm[k]["stop_reason"] == "residual drop" and warm[k]["iters"] <= 50, warm[k]
        assert abs(_cd(warm[k]) - _cd(cold[k])) < 1e-6
    # the cold start's first residual (the free stream, first order) is orders above the converged state's
    cold_first = np.array([a.residual_history(k)[0] for k in range(2)])
    assert np.all(first_warm < 1e-3 * cold_first)


def test_sst_turbulence_state_round_trip():
    from bowshock_b200.arena import Arena
    from bowshock_b200.sweep import sweep_cases
    c = sweep_cases(32)[1]
    a = Arena([c])
    a.run(20)
    t, m = a.turb_state(0)
    assert np.all(np.isfinite(t)) and t.shape[1] == 2
    t2 = t * 1.5
    a.set_turb(0, t2, m)
    t3, m3 = a.turb_state(0)
    assert np.allclose(t3, t2.astype(np.float32), rtol=1e-6) and np.allclose(m3, m, rtol=1e-6)


WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bowshock_b200", "data", "warmstart_sst.npz")


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained warm-start network committed")
def test_learned_warm_start_on_held_out_cases():
    """16 held-out SST cases (the held-out stream), cold and warm in one arena. The predicted fields start far closer to
    the converged state than the free stream (median first residual below a tenth of the cold start's) and reach the
    first order of residual drop sooner on average; at most a quarter of the predictions need the fallback; and the
    cases both runs converge agree on CD within 1e-4 (one case may sit just above: the reference's CD-stationary rule
    stops each run inside its own 1e-4 band). The later orders are not faster: the reference's stationarity windows,
    not the start field, set when an SST run stops."""
    from bowshock_b200 import learned as lw
    model = lw.WarmStart.load(lw.WEIGHTS)
    rep = lw.evaluate(model, 16, lw.HELD_OUT_SEED, 6000, log=lambda *a: None)
    print({k: rep[k] for k in ("first_residual_ratio_median", "fallbacks", "converged_both", "within_1e-4", "dcd_max")}, rep["drop"]["1"])
    assert rep["first_residual_ratio_median"] < 0.1, rep["first_residual_ratio_median"]
    d1 = rep["drop"]["1"]
    assert d1["mean_ratio_warm_over_cold"] is not None and d1["mean_ratio_warm_over_cold"] < 1.0, rep["drop"]
    assert rep["fallbacks"] <= 4
    assert rep["converged_both"] >= 6 and rep["within_1e-4"] >= rep["converged_both"] - 1, rep
