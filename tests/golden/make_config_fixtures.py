"""Regenerates tests/golden/configs_oracle.json: the oracle's run of the two single-case workloads (tests/golden/configs.py)
to the reference's stop rules, with the converged forebody-pressure, friction and base CD. Config 1 takes minutes."""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, HERE)
import numpy as np  # noqa: E402
import oracle_ffi as o  # noqa: E402
from configs import CONFIGS  # noqa: E402
from sweep_oracle import oracle_case  # noqa: E402

OUT = os.path.join(HERE, "configs_oracle.json")
data = {}
for name, make in CONFIGS.items():
    c = make()
    oc = oracle_case(c)
    s = o.Solver.from_case(oc)
    gni, gnj, x, r, _ = c.grid()
    xo, ro = s.nodes
    assert (gni, gnj) == s.dims and np.array_equal(np.ravel(xo), x) and np.array_equal(np.ravel(ro), r), name
    t0 = time.time()
    res = o.run_on(oc, s)
    fore = res.cd_nose + sum(res.cd_aft)
    data[name] = dict(ni=gni, nj=gnj, mach=c.mach, viscous=c.viscous is not None, iters=res.iters, stop=res.stop_reason,
                      drop=res.drop_orders, cd_total=res.cd_total, cd_forebody_pressure=fore, cd_nose=res.cd_nose,
                      cd_friction=res.cd_friction, cd_base=res.cd_base, cp_base=res.cp_base, cd_window=res.cd_window,
                      y_plus_max=res.y_plus_max, seconds=round(time.time() - t0, 1),
                      threads=int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())))
    print(name, data[name], flush=True)
data["made_by"] = "tests/golden/make_config_fixtures.py"
json.dump(data, open(OUT, "w"), indent=1)
