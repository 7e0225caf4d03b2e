"""Regenerates tests/golden/g3_oracle.json: the oracle's G3 run to the reference's stop rule (about a minute)."""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, HERE)
import oracle_ffi as o  # noqa: E402
from g3_case import g3_case  # noqa: E402

c = g3_case()
s = o.Solver.from_case(c)
t0 = time.time()
r = o.run_on(c, s)
d = dict(iters=r.iters, stop=r.stop_reason, drop=r.drop_orders, cd_total=r.cd_total, cd_friction=r.cd_friction,
         cd_base=r.cd_base, cp_base=r.cp_base, y_plus_max=r.y_plus_max, cd_nose=r.cd_nose, grid=list(s.dims),
         seconds_8_threads=round(time.time() - t0, 1), made_by="tests/golden/make_g3_fixture.py")
json.dump(d, open(os.path.join(HERE, "g3_oracle.json"), "w"), indent=1)
print(json.dumps(d, indent=1))
