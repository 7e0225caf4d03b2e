"""The two single-case workloads (tests/golden/configs.py) run to the reference's stop rules on the B200 through
GpuSolver.run_to_stop, against the oracle's converged run (tests/golden/configs_oracle.json): forebody-pressure, friction
and base CD within 1e-4 absolute, per case (the converged-force parity bar of the path)."""
import json
import os

import pytest

from tests.golden.configs import CONFIGS

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = json.load(open(os.path.join(HERE, "golden", "configs_oracle.json")))
TOL = 1e-4


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_config_converged_cd_matches_oracle(name):
    c = CONFIGS[name]()
    ref = FIXTURE[name]
    s = c.build_solver(0)
    r = s.run_to_stop(c.body, c.numerics, c.wake)
    fore = r["cd_nose"] + sum(r["cd_aft"])
    errs = {"forebody pressure": fore - ref["cd_forebody_pressure"], "friction": r["cd_friction"] - ref["cd_friction"],
            "base": r["cd_base"] - ref["cd_base"], "total": r["cd_total"] - ref["cd_total"]}
    print(name, r["iters"], r["stop_reason"], {k: f"{v:.2e}" for k, v in errs.items()})
    for k, v in errs.items():
        assert abs(v) <= TOL, f"{name}: {k} CD differs by {v:.2e} (ours {r['stop_reason']} after {r['iters']}, oracle {ref['stop']} after {ref['iters']})"
