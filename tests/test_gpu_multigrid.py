"""FAS multigrid with the line-implicit smoother on the B200 (the reference's FAS transfers, multigrid.rs:115-218, with one
line-implicit iteration per smoothing step in place of its SSP-RK3 smoother; no counterpart in the reference). Checks:
the three-level hierarchy keeps the free stream, and config 0 (Euler, 128 x 64 -> 64 x 32 -> 32 x 16, M 1.5) converges
to the fine-grid fixed point: forebody, base and total CD within 1e-4 of the FP64 oracle's converged run
(tests/golden/configs_oracle.json), the same bar as the single-grid scheme."""
import json
import os

import numpy as np
import pytest

import oracle_ffi as o
from tests import cases

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_implicit_multigrid_preserves_the_free_stream():
    import bowshock_b200 as bk
    from tests.test_oracle_solver import mg_grid
    x, r = mg_grid(64, 32)
    spec = cases.Spec(64, 32, x, r, 0.5, o.VAN_ALBADA, tuple(o.freestream(0.5)),
                      (o.BC_CHARACTERISTIC, o.BC_CHARACTERISTIC, o.BC_SLIPWALL, o.BC_CHARACTERISTIC), 0, label="mg grid")
    gpu = cases.gpu_solver(spec)
    gpu.set_scheme(bk.solver.MgParams(levels=3, implicit=bk.ImplicitParams()))
    rg = gpu.run(30)
    assert np.all(np.isfinite(rg))
    assert np.max(np.abs(gpu.state_f64() - o.prim_to_cons(o.freestream(0.5)))) < 1e-5


def test_config0_implicit_multigrid_reaches_the_oracle_fixed_point():
    import bowshock_b200 as bk
    from tests.golden.configs import config0_case
    ref = json.load(open(os.path.join(HERE, "golden", "configs_oracle.json")))["config0"]
    c = config0_case()
    s = c.build_solver(0)
    s.set_scheme(bk.solver.MgParams(levels=3, pre=1, post=1, implicit=c.numerics.scheme))
    r = s.run_to_stop(c.body, c.numerics, c.wake)
    fore = r["cd_nose"] + sum(r["cd_aft"])
    errs = {"forebody pressure": fore - ref["cd_forebody_pressure"], "base": r["cd_base"] - ref["cd_base"],
            "total": r["cd_total"] - ref["cd_total"]}
    print("config0 multigrid", r["iters"], r["stop_reason"], {k: f"{v:.2e}" for k, v in errs.items()})
    assert r["stop_reason"] != "non-finite residual"
    for k, v in errs.items():
        assert abs(v) <= 1e-4, f"{k} CD differs by {v:.2e} after {r['iters']} cycles ({r['stop_reason']})"
