"""Regenerates tests/golden/sweep_census.json: the oracle's run of every case of the seeded 32-case sweep to the
reference's stop rule (run.rs:44-170), with its converged CD components, iteration count and wall time.

Usage: python tests/golden/make_sweep_census.py [case indices...]   (default: the cases not yet in the JSON, cheapest first)
Results are merged into the existing JSON after each case, so an interrupted run keeps what finished. The oracle's
OpenMP thread count (OMP_NUM_THREADS) is recorded beside each time. Several hours of CPU time for all 32 cases."""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
import numpy as np  # noqa: E402
import oracle_ffi as o  # noqa: E402
from bowshock_b200.sweep import sweep_cases  # noqa: E402
from sweep_oracle import oracle_case  # noqa: E402

OUT = os.path.join(HERE, "sweep_census.json")


def main():
    cases = sweep_cases()
    data = json.load(open(OUT)) if os.path.exists(OUT) else dict(made_by="tests/golden/make_sweep_census.py", cases={})
    # explicit indices are (re)run; by default the cases not yet in the JSON, cheapest first
    idx = [int(a) for a in sys.argv[1:]] or sorted((k for k in range(len(cases)) if str(k) not in data["cases"]),
                                                   key=lambda k: (cases[k].viscous is not None, np.prod(cases[k].cells())))
    for k in idx:
        c = cases[k]
        oc = oracle_case(c)
        s = o.Solver.from_case(oc)
        ni, nj = s.dims
        # the oracle meshes the case itself; its nodes must be the CUDA library's mesher's, bit for bit
        gni, gnj, x, r, _ = c.grid()
        xo, ro = s.nodes
        assert (gni, gnj) == (ni, nj) and np.array_equal(np.ravel(xo), x) and np.array_equal(np.ravel(ro), r), f"case {k}: grids differ"
        t0 = time.time()
        res = o.run_on(oc, s)
        sec = time.time() - t0
        data["cases"][str(k)] = dict(ni=ni, nj=nj, viscous=c.viscous is not None, mach=c.mach, iters=res.iters, stop=res.stop_reason,
                                     drop=res.drop_orders, cd_total=res.cd_total, cd_nose=res.cd_nose, cd_aft=res.cd_aft,
                                     cd_friction=res.cd_friction, cd_base=res.cd_base, cp_base=res.cp_base, cd_window=res.cd_window,
                                     seconds=round(sec, 2),
                                     threads=int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())))
        json.dump(data, open(OUT + ".tmp", "w"), indent=1)
        os.replace(OUT + ".tmp", OUT)
        print(k, data["cases"][str(k)], flush=True)


if __name__ == "__main__":
    main()
