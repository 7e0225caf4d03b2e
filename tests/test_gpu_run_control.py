"""GPU-resident run control: the stop rules (engine/run.rs:105-170) evaluated on the device after every chunk give the
same decisions as the host's evaluation of the same residuals and monitors, on sweep cases that stop on each rule
(residual drop, CD stationary, and the mean-stationary limit cycle after 14,000 iterations): identical iteration counts
and stop reasons, residual histories and CDs equal to round-off."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_stop_rules_match_host_rules():
    from bowshock_b200.arena import Arena
    from bowshock_b200.sweep import sweep_cases
    picks = (2, 18, 7, 9)  # Euler residual drop (subsonic, transonic), SST CD stationary, SST limit cycle (mean stationary)
    cs = [sweep_cases(32)[k] for k in picks]
    out = []
    for on_device in (True, False):
        a = Arena(cs)
        a.set_run_control(on_device)
        res = a.solve()
        out.append((res, [a.residual_history(k) for k in range(len(cs))]))
        del a
    (rd, hd), (rh, hh) = out
    reasons = set()
    for k in range(len(cs)):
        assert rd[k]["iters"] == rh[k]["iters"] and rd[k]["stop_reason"] == rh[k]["stop_reason"], (picks[k], rd[k], rh[k])
        # the states are the same; the FP64 force and norm sums add per-block partials atomically, in whatever order
        # the blocks finish, so CDs and residuals compare to round-off
        assert abs(rd[k]["cd_total"] - rh[k]["cd_total"]) <= 1e-12 * abs(rh[k]["cd_total"])
        assert abs(rd[k]["cd_window"] - rh[k]["cd_window"]) <= 1e-12 * abs(rh[k]["cd_window"])
        assert np.allclose(hd[k], hh[k], rtol=1e-12, atol=0.0)
        reasons.add(rd[k]["stop_reason"])
    assert {"residual drop", "mean stationary"} <= reasons
