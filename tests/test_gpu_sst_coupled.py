"""Coupled 6x6 SST lines (Arena / GpuSolver.set_sst_coupling), the option beside the reference's loose coupling
(crates/bowshock-cfd/src/turbulence.rs:542-611). The mean-flow operator freezes mu_t, so each 6x6 block of (dU, dk,
domega) is lower block-triangular: the mean flow of an iteration is that of the loose scheme bit for bit, and only the
turbulence rows see the coupling. The residuals are the reference's, so the converged CDs are the loose scheme's and the
oracle's (1e-4 absolute, per case)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-4


def test_coupled_lines_change_the_turbulence_rows_only():
    from bowshock_b200.configs import CONFIGS
    c = CONFIGS["config1"]()
    loose, cpl = c.build_solver(0), c.build_solver(0)
    cpl.set_sst_coupling(True)
    loose.run(1)
    cpl.run(1)
    assert np.array_equal(loose.state_f64(), cpl.state_f64())
    (k0, w0), (k1, w1) = loose.turb_state(), cpl.turb_state()
    for a in (k1, w1):
        assert np.all(np.isfinite(a))
    # the coupling moves omega most (its production and destruction scale with rho): 1.3e-3 measured
    dw = np.max(np.abs(w1 - w0)) / np.max(np.abs(w0))
    assert 1e-6 < dw < 1e-1, dw
    cpl.set_sst_coupling(False)  # and back: the next iteration runs the loose lines again
    loose.run(1)
    cpl.run(1)
    assert np.all(np.isfinite(cpl.state_f64()))


def test_coupled_config1_converges_to_the_oracle_cd():
    from bowshock_b200.configs import CONFIGS
    ref = json.load(open(os.path.join(HERE, "golden", "configs_oracle.json")))["config1"]
    out = {}
    for coupled in (False, True):
        c = CONFIGS["config1"]()
        s = c.build_solver(0)
        s.set_sst_coupling(coupled)
        out[coupled] = s.run_to_stop(c.body, c.numerics, c.wake)
    r, r0 = out[True], out[False]
    fore = r["cd_nose"] + sum(r["cd_aft"])
    errs = {"forebody pressure": fore - ref["cd_forebody_pressure"], "friction": r["cd_friction"] - ref["cd_friction"],
            "base": r["cd_base"] - ref["cd_base"], "total": r["cd_total"] - ref["cd_total"]}
    print("coupled", r["iters"], r["stop_reason"], {k: f"{v:.2e}" for k, v in errs.items()},
          "loose", r0["iters"], f"{r['cd_total'] - r0['cd_total']:.2e}")
    for k, v in errs.items():
        assert abs(v) <= TOL, f"{k}: {v:.2e}"
    assert r["stop_reason"] == ref["stop"]
    assert abs(r["cd_total"] - r0["cd_total"]) <= 1e-6  # measured 4e-9


def test_coupled_sst_sweep_cases_match_the_oracle():
    """The ten SST sweep cases that stop on the CD-stationary window, in one arena with coupled and with loose lines:
    the same stop rule and iteration as the oracle's census (tests/golden/sweep_census.json), CD within 1e-4 of the
    oracle (measured 6.8e-5 at most, the loose scheme 6.3e-5) and within 1e-5 of the loose scheme (measured 4.7e-6).
    The six limit-cycle cases (mean-stationary stop) are left out: their window-mean CD moves with the rounding of the
    launch shapes by more than 1e-4 under either scheme."""
    from bowshock_b200.arena import Arena
    from bowshock_b200.sweep import sweep_cases
    cen = json.load(open(os.path.join(HERE, "golden", "sweep_census.json")))["cases"]
    picks = sorted(int(k) for k, v in cen.items() if v["viscous"] and v["stop"] == "CD stationary")
    assert len(picks) == 10
    cs = [sweep_cases()[k] for k in picks]
    res = {}
    for coupled in (False, True):
        a = Arena(cs)
        a.set_sst_coupling(coupled)
        res[coupled] = a.solve()
        del a
    for k, r, r0 in zip(picks, res[True], res[False]):
        ref = cen[str(k)]
        print(k, r["iters"], ref["iters"], r["stop_reason"], f"{r['cd_total'] - ref['cd_total']:+.2e}",
              f"{r['cd_total'] - r0['cd_total']:+.2e}")
        assert r["stop_reason"] == ref["stop"], k
        assert r["iters"] == ref["iters"], k
        assert abs(r["cd_total"] - ref["cd_total"]) <= TOL, k
        assert abs(r["cd_total"] - r0["cd_total"]) <= 1e-5, k


def test_coupling_touches_the_sst_cases_only():
    """The 32-case sweep arena (16 Euler, 16 SST cases) for 200 iterations with coupled and with loose SST lines: every
    Euler case's state is the same bit for bit (the coupling kernel and the SST line systems touch only SST cases), and
    every SST case's mean flow differs (its turbulence rows, and through mu_t its later iterations, changed)."""
    from bowshock_b200.arena import Arena
    from bowshock_b200.sweep import sweep_cases
    cs = sweep_cases()
    states = {}
    for coupled in (False, True):
        a = Arena(cs)
        a.set_sst_coupling(coupled)
        a.run(200)
        states[coupled] = [a.state(k) for k in range(len(cs))]
        del a
    n_sst = 0
    for k, c in enumerate(cs):
        same = np.array_equal(states[True][k], states[False][k])
        assert np.all(np.isfinite(states[True][k]))
        if c.viscous is None:  # Euler
            assert same, k
        else:
            n_sst += 1
            assert not same, k
    assert n_sst == 16
