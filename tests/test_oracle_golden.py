"""The oracle against the reference's published converged values of its G3 body (crates/bowshock-cfd/README.md:795-797:
total CD 0.21300, friction 0.09003, base 0.12257, Cp_b -0.1226, y+ max 0.648, `CD stationary` after 4000 iterations).
The run takes about a minute on 8 cores, so it is opt-in (BOWSHOCK_SLOW=1); its last output is committed in
tests/golden/g3_oracle.json and checked here on every run."""
import json
import os

import pytest

import oracle_ffi as o

HERE = os.path.dirname(os.path.abspath(__file__))


def _check(r):
    from tests.golden.g3_case import REFERENCE
    assert r["iters"] == REFERENCE["iters"] and r["stop"] == REFERENCE["stop_reason"]
    assert round(r["cd_total"], 5) == REFERENCE["cd_total"]
    assert round(r["cd_friction"], 5) == REFERENCE["cd_friction"]
    assert round(r["cd_base"], 5) == REFERENCE["cd_base"]
    assert round(r["cp_base"], 4) == REFERENCE["cp_base"]
    assert round(r["y_plus_max"], 3) == REFERENCE["y_plus_max"]


def test_committed_g3_oracle_run_matches_the_reference_digits():
    with open(os.path.join(HERE, "golden", "g3_oracle.json")) as f:
        _check(json.load(f))


@pytest.mark.slow
def test_g3_oracle_run_matches_the_reference_digits():
    from tests.golden.g3_case import g3_case
    c = g3_case()
    s = o.Solver.from_case(c)
    assert s.dims == (156, 122)
    r = o.run_on(c, s)
    _check(dict(iters=r.iters, stop=r.stop_reason, cd_total=r.cd_total, cd_friction=r.cd_friction, cd_base=r.cd_base,
                cp_base=r.cp_base, y_plus_max=r.y_plus_max))


def test_limit_cycle_spread_fixture():
    """The oracle is deterministic (the unperturbed run of the spread fixture is the census's run of the same case, to the
    last bit), and a limit-cycle SST case's window-mean CD, the quantity the mean-stationary rule reports
    (engine/run.rs:150-170), moves by more than the 1e-4 parity bar when only the free-stream Mach number moves by
    1e-12 (tests/golden/limit_cycle_spread.json, made by make_limit_cycle_spread.py): the bar sits inside the case's
    own rounding sensitivity."""
    import json
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spread = json.load(open(os.path.join(here, "limit_cycle_spread.json")))["cases"]
    census = json.load(open(os.path.join(here, "sweep_census.json")))["cases"]
    for k, s in spread.items():
        base = [r for r in s["runs"] if r["eps"] == 0.0][0]
        assert base["cd_window"] == census[k]["cd_window"] and base["iters"] == census[k]["iters"]
        cds = [r["cd_window"] if r["stop"] == "mean stationary" else r["cd_total"] for r in s["runs"]]
        assert abs(s["spread"] - (max(cds) - min(cds))) < 1e-15
    assert spread["9"]["spread"] > 1e-4
