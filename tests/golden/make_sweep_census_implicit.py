"""Regenerates tests/golden/sweep_census_implicit.json: the oracle's run of the sweep's Euler cases at M >= 0.85 with the
numerics the B200 path runs them with (the line-implicit scheme, ImplicitParams::DEFAULT of implicit.rs:79-80, in place
of the reference preset's explicit SSP-RK3, and the stop rules held until the first second-order residual, min_iter =
first_order_iters + 1 = 301), to the reference's stop rules. The default census (make_sweep_census.py) runs the reference
presets; this second fixture compares the GPU with the oracle under the same scheme and stop rule, so that a CD
difference of the preset census can be attributed to the different convergence of the two schemes or to the kernels.

Usage: python tests/golden/make_sweep_census_implicit.py [case indices...]   (default: every Euler case at M >= 0.85)"""
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

OUT = os.path.join(HERE, "sweep_census_implicit.json")


def implicit_oracle_case(c):
    """The oracle case of sweep case c with the B200 path's numerics for a transonic Euler case."""
    oc = oracle_case(c)
    n, g = oc.numerics, c.numerics
    n.scheme = o.implicit_params(cfl0=g.scheme.cfl0, cfl_max=g.scheme.cfl_max, growth=g.scheme.growth, dt_mode=g.scheme.dt_mode,
                                 lines=g.scheme.lines, implicit_bc=g.scheme.implicit_bc, sub_iters=g.scheme.sub_iters, roe=g.scheme.roe,
                                 eps_fix=g.scheme.eps_fix)
    n.min_iter = g.min_iter
    assert (n.first_order_iters, n.limiter, bool(n.low_mach), n.max_iter) == (g.first_order_iters, g.limiter, bool(g.low_mach), g.max_iter)
    return oc


def main():
    cases = sweep_cases()
    data = json.load(open(OUT)) if os.path.exists(OUT) else dict(made_by="tests/golden/make_sweep_census_implicit.py", cases={})
    idx = [int(a) for a in sys.argv[1:]] or [k for k, c in enumerate(cases) if c.viscous is None and c.mach >= 0.85]
    for k in idx:
        c = cases[k]
        oc = implicit_oracle_case(c)
        s = o.Solver.from_case(oc)
        t0 = time.time()
        res = o.run_on(oc, s)
        sec = time.time() - t0
        ni, nj = s.dims
        data["cases"][str(k)] = dict(ni=ni, nj=nj, mach=c.mach, iters=res.iters, stop=res.stop_reason, drop=res.drop_orders,
                                     cd_total=res.cd_total, cd_nose=res.cd_nose, cd_aft=res.cd_aft, cd_base=res.cd_base,
                                     cd_window=res.cd_window, seconds=round(sec, 2), threads=int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())))
        json.dump(data, open(OUT + ".tmp", "w"), indent=1)
        os.replace(OUT + ".tmp", OUT)
        print(k, data["cases"][str(k)], flush=True)


if __name__ == "__main__":
    main()
