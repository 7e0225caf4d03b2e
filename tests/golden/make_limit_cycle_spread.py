"""Regenerates tests/golden/limit_cycle_spread.json: how far the oracle's own converged CD of a limit-cycle SST sweep case
moves when the free-stream Mach number is perturbed at round-off level (times 1 + eps, eps ~ 1e-12; the grid is the
same). The reference's mean-stationary rule (engine/run.rs:150-170) reports the mean CD over the last window; on a limit
cycle whose phase is sensitive to rounding, that mean is reproducible only to the spread measured here, which bounds how
closely any other implementation (the B200 path included) can be expected to match it.

Usage: python tests/golden/make_limit_cycle_spread.py [case indices...]   (default: 9)"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
import oracle_ffi as o  # noqa: E402
from bowshock_b200.sweep import sweep_cases  # noqa: E402
from sweep_oracle import oracle_case  # noqa: E402

OUT = os.path.join(HERE, "limit_cycle_spread.json")
EPS = (0.0, 1e-12, -1e-12, 1e-9)


def main():
    cases = sweep_cases()
    data = json.load(open(OUT)) if os.path.exists(OUT) else dict(made_by="tests/golden/make_limit_cycle_spread.py", cases={})
    for k in [int(a) for a in sys.argv[1:]] or [9]:
        runs = []
        for eps in EPS:
            oc = oracle_case(cases[k])
            oc.mach = oc.mach * (1.0 + eps)  # the free stream only: the grid parameters are already fixed in oc
            s = o.Solver.from_case(oc)
            t0 = time.time()
            r = o.run_on(oc, s)
            runs.append(dict(eps=eps, iters=r.iters, stop=r.stop_reason, cd_total=r.cd_total, cd_window=r.cd_window,
                             seconds=round(time.time() - t0, 1)))
            print(k, runs[-1], flush=True)
        cd = [x["cd_window"] if x["stop"] == "mean stationary" else x["cd_total"] for x in runs]
        data["cases"][str(k)] = dict(mach=cases[k].mach, runs=runs, spread=max(cd) - min(cd))
        json.dump(data, open(OUT + ".tmp", "w"), indent=1)
        os.replace(OUT + ".tmp", OUT)


if __name__ == "__main__":
    main()
