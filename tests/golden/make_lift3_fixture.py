"""Regenerates tests/golden/lift3_oracle.json: the 3D oracle (oracle/solver3.cpp, the reference's Solver3 and run3.rs
stop rules restated in FP64) run to its stop rules on a lift-sweep body at 96 x 32 x 32 cells (98,304; the largest the
oracle finishes in minutes on the host), line-implicit (cfl_max 10), 100 first-order iterations, at M 1.2 and M 2.5 and
4 degrees incidence: the converged normal force CN and centre of pressure x_cp that tests/test_gpu3.py compares the
B200 batch with.

Usage: python tests/golden/make_lift3_fixture.py"""
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
import oracle_ffi as o  # noqa: E402
from bowshock_b200.euler3 import lift_sweep_cases  # noqa: E402

OUT = os.path.join(HERE, "lift3_oracle.json")
NI, NJ, NK, ALPHA, MAX_ITER = 96, 32, 32, 4.0, 4000


def main():
    data = dict(made_by="tests/golden/make_lift3_fixture.py", grid=[NI, NJ, NK], alpha_deg=ALPHA, max_iter=MAX_ITER, first_order=100,
                cases={})
    for mach in (1.2, 2.5):
        c = lift_sweep_cases((ALPHA,), (mach,), ni=NI, nj=NJ, nk=NK)[0]
        ni2, nj2, x2, r2, _ = c.case2.grid()
        theta = np.pi * np.arange(NK + 1) / NK
        cpu = o.Solver3(ni2, nj2, np.asarray(x2), np.asarray(r2), NK, theta, c.case2.grid_sting.n_up, mach, math.radians(ALPHA), limiter=o.MINMOD,
                        first_order_iters=100, implicit=True, params=o.implicit3_params(cfl_max=10.0))
        t0 = time.time()
        r = cpu.run(c.body.x_base(), max_iter=MAX_ITER)
        data["cases"][f"{mach}"] = dict(ni=ni2, nj=nj2, nk=NK, cn=r["cn"], x_cp=r["x_cp"], iters=r["iterations"], stop=r["stop_reason"], drop=r["drop_orders"],
                                        seconds=round(time.time() - t0, 1))
        print(mach, data["cases"][f"{mach}"], flush=True)
        json.dump(data, open(OUT + ".tmp", "w"), indent=1)
        os.replace(OUT + ".tmp", OUT)


if __name__ == "__main__":
    main()
