"""Benchmark of the B200 backend on the seeded 32-case mixed sweep (Euler + RANS SST, grids 96x48 to 320x160).

Metric: converged cases per hour on one B200 at |dCD| <= 1e-4 against the FP64 oracle's converged CD of the same case
(tests/golden/sweep_census.json, made by tests/golden/make_sweep_census.py).

  timed region  K line-implicit iterations of the whole 32-case arena (every case active), replayed from CUDA graphs,
                CUDA events on the launching stream: `ms_per_step`, the roofline of the dominant kernel group, the launch
                count. 760,692 cells x ~0.5-1.6 KB per cell-update is far above the 126 MB L2, so no flush is needed.
  value         the census: every case cold-started from the free stream and iterated to the reference's stop rules in one
                arena (converged cases masked out), the device time of all its iterations and FP64 force passes (CUDA
                events): value = 3600 * (cases within |dCD| <= 1e-4) / census device seconds.
  e2e           the same census through the public API by the wall clock: meshing, arena creation with the host->device
                copies, the solve with its chunked read-backs, the forces.
  plain         the plain single-case backend: each case alone through GpuSolver.run_to_stop (same kernels, one case per
                launch), wall clock, reported as config.plain_single_case_cases_per_hr.
  cpu_baseline  the oracle (f64 C++ restatement of the reference CPU path, all host threads) timed on a bounded sample of
                iterations of every case, times the oracle's own iteration counts to its stop rules (one GPU only).
  secondary     (one GPU) in config: the census with the learned warm start, the census with the coupled 6x6 SST lines,
                the 3D lift batch, multigrid against the single grid, the device mesher.
  --gpus N      one process per GPU (started here through torch.distributed.run unless launched by it): the 32 cases are
                partitioned over the ranks (longest processing time on cells x expected iterations, bowshock_b200.shard),
                each rank runs its share in its own arena, the point results are gathered (gloo, host objects); times
                are the max over ranks, `scaling` "strong" (the sweep is fixed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged cases/hr at |dCD|<=1e-4: learned+batched vs plain CUDA, 1 B200"
UNIT = "converged cases/hr"
# algorithmic words per cell of one line sweep (3 nv + g + v + 1; nv = 4, g = 10 Euler / 13 viscous, v = 0 / 8)
SWEEP_WORDS = {False: 23, True: 34}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def bf16_peak():
    """(dense BF16 TFLOP/s burst peak, 'measured' | 'fallback')."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1].split()[0]))
                smax.append(float(p[2].split()[0]))
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_cases():
    """The 32-case sweep (the same seeded draw on every rank; each rank solves its own share of it)."""
    from bowshock_b200.sweep import SEED, sweep_cases
    return sweep_cases(32, SEED)


def shard(cases, grids, rank, world):
    """This rank's case indices: the longest-processing-time partition of the sweep over the ranks by cells x expected
    iterations (bowshock_b200.shard); every rank computes the same partition."""
    from bowshock_b200.shard import case_cost, lpt_partition
    return lpt_partition([case_cost(c, g) for c, g in zip(cases, grids)], world)[rank]


def reduce_scalars(dist, values, op):
    """(max or sum over ranks of each value); identity with one process."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t]


def h2d_bytes(cases, grids):
    """Bytes the census copies host->device per case: face metrics (float4 + centres float2, + FP64-derived face stencils for
    viscous cases), cell geometry, the FP64 nodes and cell centres of the force pass, wall distance and turbulence start for
    SST, and the free-stream start state (float pair)."""
    total = 0
    for c, g in zip(cases, grids):
        ni, nj = g[0], g[1]
        fi, fj, nc, nn = (ni + 1) * nj, ni * (nj + 1), ni * nj, (ni + 1) * (nj + 1)
        b = 24 * (fi + fj) + 16 * nc + 16 * nn + 16 * nc + 32 * nc
        if c.viscous is not None:
            b += 16 * (fi + fj) + 4 * nc + 8 * nc
        total += b
    return total


def d2h_bytes(ncases, iters):
    """Bytes read back per 50-iteration chunk (density residuals, turbulence residual, FP64 forces), over the census."""
    chunks = (max(iters) + 49) // 50
    return int(chunks * (50 * ncases * 8 + ncases * 8 + ncases * 15 * 8))


def census_fixture_implicit():
    """The oracle's census of the sweep's Euler cases at M >= 0.85 with the B200 path's line-implicit scheme and stop rules
    (tests/golden/sweep_census_implicit.json): {case index: {...}}."""
    p = os.path.join(ROOT, "tests", "golden", "sweep_census_implicit.json")
    if os.path.exists(p):
        with open(p) as f:
            return {int(k): v for k, v in json.load(f)["cases"].items()}
    return {}


def census_fixture():
    """The oracle's census of the sweep: {case index: {iters, cd_total, ...}} (cases it has not finished are absent)."""
    p = os.path.join(ROOT, "tests", "golden", "sweep_census.json")
    if os.path.exists(p):
        with open(p) as f:
            return {int(k): v for k, v in json.load(f)["cases"].items()}
    return {}


class OracleSample:
    """The oracle solver of every case of the sweep, built once; `step(k)` times one iteration of case k."""

    def __init__(self, cases):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
        import oracle_ffi as o
        from sweep_oracle import oracle_case
        self.o = o
        self.solvers = []
        for c in cases:
            oc = oracle_case(c)
            s = o.Solver.from_case(oc)
            cfg = s.config
            cfg.cfl, cfg.limiter, cfg.first_order_iters = oc.numerics.cfl, oc.numerics.limiter, oc.numerics.first_order_iters
            s.set_config(cfg)
            s.set_low_mach(bool(oc.numerics.low_mach))
            s.set_scheme(oc.numerics.scheme)
            self.solvers.append(s)
        self.t = [[] for _ in cases]

    def step(self, k):
        t0 = time.perf_counter()
        self.solvers[k].step()
        self.t[k].append(time.perf_counter() - t0)

    def cases_per_hr(self, iters):
        """3600 n / sum_k (seconds per iteration of case k x its iterations to the stop rule)."""
        total = sum(float(np.mean(self.t[k])) * iters[k] for k in range(len(self.solvers)))
        return 3600.0 * len(self.solvers) / total


def cd_error(ours, oracle):
    """CD error of a case against the oracle: the final total CD; for a run that both stopped on a limit cycle (mean
    stationary), the mean CD over the last window the rule compared, since the instantaneous CD depends on the phase."""
    if ours["stop_reason"] == "mean stationary" and oracle["stop"] == "mean stationary" and "cd_window" in oracle:
        return ours["cd_window"] - oracle["cd_window"]
    return ours["cd_total"] - oracle["cd_total"]


def oracle_iters(fx, cases):
    """The oracle's iterations to its stop rule per case; a case it has not finished takes the mean of its kind."""
    out, filled = [], []
    for k, c in enumerate(cases):
        if k in fx:
            out.append(fx[k]["iters"])
        else:
            same = [v["iters"] for v in fx.values() if v["viscous"] == (c.viscous is not None)]
            out.append(int(np.mean(same)) if same else int(c.numerics.max_iter))
            filled.append(k)
    return out, filled


def run_reference(args, rank, world):
    """The reference arm: the reference CPU path (its f64 restatement, the oracle) on the same workload and metric. One step
    = one iteration of one case, rotating through the 32 cases; cases/hr from the mean seconds per iteration of each case
    and the oracle's own iteration counts to its stop rules."""
    if rank != 0:
        return None
    cases = build_cases()
    fx = census_fixture()
    iters, filled = oracle_iters(fx, cases)
    smp = OracleSample(cases)
    for s in range(max(args.warmup, len(cases))):  # at least one untimed iteration of every case
        smp.solvers[s % len(cases)].step()
    steps = max(args.steps, len(cases))
    t0 = time.perf_counter()
    for s in range(steps):
        smp.step(s % len(cases))
    wall = time.perf_counter() - t0
    value = smp.cases_per_hr(iters)
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count()))
    sample = f"{steps} oracle iterations, one case per step rotating through the 32 cases, x the oracle's iterations to its stop rules"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * wall / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 32-case sweep, SplitMix64 seed 0x0B05C0C2)",
            "config": {"workload": "32-case mixed Euler/RANS-SST sweep, grids 96x48..320x160, reference CPU path (f64 C++ restatement "
                                   "of crates/bowshock-cfd, OpenMP over lines), reference numerics presets",
                       "cases": len(cases), "oracle_iters": iters, "iters_estimated_for_cases": filled},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def run_ours(args, rank, world, dist):
    import bowshock_b200  # noqa: F401
    from bowshock_b200.arena import Arena
    from bowshock_b200.shard import gather_results
    device = int(os.environ.get("LOCAL_RANK", "0"))
    all_cases = build_cases()
    all_grids = [c.grid() for c in all_cases]
    mine = shard(all_cases, all_grids, rank, world)  # this rank's share of the sweep (all of it on one GPU)
    cases = [all_cases[k] for k in mine]
    grids = [all_grids[k] for k in mine]
    cells = np.array([g[0] * g[1] for g in grids], dtype=float)
    arena = Arena(cases, device=device, grids=grids)
    ncell = arena.cells
    # warm-up, then the CUDA graph of the timed chunk built ahead (graph construction is host work, not a step)
    arena.run(max(args.warmup, 3))
    arena.prepare(args.steps)
    if dist:
        dist.barrier()
    clocks = Clocks(device)
    clocks.start()
    arena.run(args.steps)
    ms_local = arena.ms_per_iter()
    # census: this rank's cases to their stop rules, through the public API (wall clock = e2e; device time = value)
    cen_cases = [build_cases()[k] for k in mine]
    t1 = time.perf_counter()
    cen_grids = [c.grid() for c in cen_cases]
    cen = Arena(cen_cases, device=device, grids=cen_grids)
    results_local = cen.solve()
    wall_census = time.perf_counter() - t1
    clk = clocks.stop()
    census_dev_s = cen.last_solve_ms() / 1000.0
    del cen
    results = gather_results(dist, mine, [{k: v for k, v in r.items() if k != "residual"} for r in results_local], len(all_cases))
    iters_local = np.array([r["iters"] for r in results_local], dtype=float)
    fx = census_fixture()
    dcd = {k: cd_error(results[k], fx[k]) for k in range(len(all_cases)) if k in fx}
    fxi = census_fixture_implicit()
    dcd_same = {k: results[k]["cd_total"] - fxi[k]["cd_total"] for k in range(len(all_cases)) if k in fxi}
    ok = [k for k, d in dcd.items() if abs(d) <= 1e-4]
    n_ok = len(ok)
    steady_local = 3600.0 * len(cases) * cells.sum() / ((ms_local / 1000.0) * float(np.sum(cells * iters_local)))
    # per-kernel profile (CUDA events around every launch) for the roofline of the dominant kernel group
    prof = arena.profile(5)
    tuning = arena.tuning()
    del arena
    hbm, peak_kind = peaks()
    # plain single-case backend: each of this rank's cases alone, to its stop rule, wall clock
    t_plain = 0.0
    plain_ok = 0
    for q, c in enumerate(cases):
        k = mine[q]
        s1 = c.build_solver(device, grid=grids[q])
        t0 = time.perf_counter()
        r1 = s1.run_to_stop(c.body, c.numerics, c.wake)
        t_plain += time.perf_counter() - t0
        if k in fx and abs(cd_error(r1, fx[k])) <= 1e-4:
            plain_ok += 1
        del s1
    ms_step, census_dev_max, wall_max, plain_max = reduce_scalars(dist, [ms_local, census_dev_s, wall_census, t_plain], "max")
    ncell_all, plain_ok_all, steady_all = reduce_scalars(dist, [float(ncell), float(plain_ok), steady_local], "sum")
    total_value = 3600.0 * n_ok / census_dev_max
    e2e_value = 3600.0 * n_ok / wall_max
    plain_cases_per_hr = 3600.0 * plain_ok_all / plain_max
    # roofline of the dominant kernel group: the block line sweeps (k_lines, the factorising first pass of each direction,
    # and k_lines_subst, the defect-correction passes), half of an iteration in the launch list
    groups = {g: v for g, v in prof.items() if v[1] > 0}
    sweep_groups = [g for g in ("lines_i", "lines_j", "subst_i", "subst_j") if g in groups]
    top = "line sweeps (k_lines + k_lines_subst)"
    ms_sweeps = sum(groups[g][0] for g in sweep_groups) / 5.0  # per iteration (profile over 5 iterations)
    launches_iter = sum(groups[g][1] for g in sweep_groups) / 5.0
    viscous = np.array([c.viscous is not None for c in cases])
    words = np.where(viscous, SWEEP_WORDS[True], SWEEP_WORDS[False])
    sub = np.array([c.numerics.scheme.sub_iters for c in cases])
    bytes_sweeps = float(np.sum(cells * words * 4 * 2 * sub))  # 3 nv + g + v + 1 words per cell, 2 directions x sub_iters passes
    bytes_iter = bytes_sweeps / launches_iter
    ms_launch = ms_sweeps / launches_iter
    achieved = bytes_iter / (ms_launch / 1000.0) / 1e9
    launches_per_iter = sum(v[1] for v in prof.values()) / 5.0
    (launches_all,) = reduce_scalars(dist, [launches_per_iter * args.steps], "sum")
    if rank != 0:
        return None
    traffic = line_sweep_traffic()
    learned = secondary(learned_census, all_cases, all_grids, fx, plain_cases_per_hr, device) if world == 1 else None
    lift3 = secondary(measure_lift3, args, device) if world == 1 else None
    coupled = secondary(sst_coupled_census, all_cases, all_grids, fx, results, census_dev_s, device) if world == 1 else None
    mg0 = secondary(measure_multigrid, device) if world == 1 else None
    mesh = secondary(measure_mesher, device) if world == 1 else None
    cpu_base = None
    if world == 1:  # the CPU baseline: the oracle on a bounded sample (3 iterations of every case), x its own iteration counts
        smp = OracleSample(all_cases)
        for k in range(len(all_cases)):
            smp.solvers[k].step()
        for _ in range(3):
            for k in range(len(all_cases)):
                smp.step(k)
        o_iters, filled = oracle_iters(fx, all_cases)
        cpu_base = {"value": smp.cases_per_hr(o_iters), "unit": UNIT, "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())),
                    "kind": "port",
                    "sample": "3 oracle iterations of each of the 32 cases (all host threads) x the oracle's iterations to its stop rules"
                              + (f" (cases {filled} not in the census fixture: mean of their kind)" if filled else "")}
    stops = {}
    for r in results:
        stops[r["stop_reason"]] = stops.get(r["stop_reason"], 0) + 1
    iters = [r["iters"] for r in results]
    h2d = h2d_bytes(all_cases, all_grids)
    d2h = d2h_bytes(len(all_cases), iters)
    line = {
        "metric": METRIC, "value": total_value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
        "dtype": "fp32+fp64",
        "data": "synthetic (seeded 32-case sweep, SplitMix64 seed 0x0B05C0C2, partitioned over the GPUs)",
        "config": {
            "workload": "32-case mixed Euler/RANS-SST sweep, grids 96x48..320x160, line-implicit, batched arena (one launch per kernel "
                        "for all cases), CUDA graph per 50-iteration chunk; state FP32 pair, lines FP32, residual/forces/norms FP64",
            "cases": len(all_cases), "cells": int(ncell_all), "cell_updates_per_s": float(ncell_all / (ms_step / 1000.0)),
            "l2": "no flush: the step's working set (~%.0f MB) is larger than the 126 MB L2" % (ncell * 600 / 1e6),
            "converged_within_1e-4": n_ok, "checked_against_oracle": len(dcd),
            "dcd": {str(k): float(f"{d:.3e}") for k, d in dcd.items()},
            "dcd_euler_transonic_same_scheme": {str(k): float(f"{d:.3e}") for k, d in dcd_same.items()},
            "census_device_s": census_dev_max, "census_wall_s": wall_max, "census_iters": iters, "census_stop_reasons": stops,
            "steady_state_cases_per_hr": steady_all,
            "plain_single_case_cases_per_hr": plain_cases_per_hr, "plain_wall_s": plain_max, "plain_converged_within_1e-4": int(plain_ok_all),
            "batched_vs_plain_e2e": e2e_value / plain_cases_per_hr if plain_cases_per_hr else None,
            "learned_warm_start": learned,
            "learned_plus_batched_vs_plain": (learned or {}).get("learned_plus_batched_vs_plain"),
            "kernel_profile_ms_per_launch": {g: v[0] / v[1] for g, v in groups.items()},
            "autotuned_lines_per_block": tuning,
            "lift3": lift3,
            "sst_coupled": coupled,
            "device_mesher": mesh,
            "multigrid": mg0,
            "parallelism": (f"cases partitioned over {world} GPUs (longest-processing-time on cells x expected iterations), results "
                            "gathered" if world > 1 else "one GPU, one batched arena"),
        },
        "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_launch": bytes_iter, "ms_per_launch": ms_launch,
                     "traffic": traffic},
        "cpu_baseline": cpu_base,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "what": "census by the wall clock through the public API: meshing, arena creation (host->device), solve with chunked "
                        "read-backs (device->host), forces"},
        "clocks": clk,
        "gpu_launches": int(round(launches_all)),
    }
    return line


# algorithmic bytes per cell-update of the 3D Euler line-implicit iteration (nv = 5, 16 geometry words, 3 directions,
# 2 sweeps each: 271 words; the per-kernel model of the 2D path applied to 3D)
WORDS_3D = 271


def secondary(fn, *a):
    """A secondary figure of the bench line: its dict, or the error that kept it from being measured."""
    try:
        return fn(*a)
    except Exception as e:  # reported in the line, not fatal to the headline measurement
        return {"error": f"{type(e).__name__}: {e}"}


def sst_coupled_census(cases, grids, fx, loose, loose_dev_s, device):
    """The census again with the coupled 6x6 SST lines (Arena.set_sst_coupling; the default and the headline run the
    reference's loose coupling): device time, stop iterations and CDs against the loose census and the oracle. The Euler
    cases are untouched by the option; the CD-stationary SST cases reach the same CDs; the mean-stationary (limit-cycle)
    SST cases' window means move with any change of the iteration path."""
    from bowshock_b200.arena import Arena
    a = Arena(cases, device=device, grids=grids)
    a.set_sst_coupling(True)
    res = a.solve()
    dev_s = a.last_solve_ms() / 1000.0
    del a
    sst = [k for k, c in enumerate(cases) if c.viscous is not None]
    cds = [k for k in sst if loose[k]["stop_reason"] == "CD stationary"]
    euler = [k for k in range(len(cases)) if k not in sst]
    dcd = {k: cd_error(res[k], fx[k]) for k in range(len(cases)) if k in fx}
    return {"census_device_s": dev_s, "loose_census_device_s": loose_dev_s,
            "converged_within_1e-4": sum(abs(d) <= 1e-4 for d in dcd.values()), "checked_against_oracle": len(dcd),
            # the option touches no Euler case (their states are the same bit for bit over fixed iteration counts); a
            # census stops on FP64 norms summed by atomics in no fixed order, so two solves can differ in the last bits
            "max_dcd_vs_loose_euler": max(abs(res[k]["cd_total"] - loose[k]["cd_total"]) for k in euler) if euler else None,
            "sst_same_stop_iterations": sum(res[k]["iters"] == loose[k]["iters"] for k in sst), "sst_cases": len(sst),
            "max_dcd_vs_loose_cd_stationary": max(abs(res[k]["cd_total"] - loose[k]["cd_total"]) for k in cds) if cds else None,
            "dcd_vs_loose_limit_cycle": {str(k): float(f"{res[k]['cd_total'] - loose[k]['cd_total']:.3e}") for k in sst if k not in cds},
            "dcd": {str(k): float(f"{d:.3e}") for k, d in dcd.items()}}


def learned_census(cases, grids, fx, plain_cases_per_hr, device):
    """The census again with the learned warm start (bowshock_b200.learned, the committed trained network): a 50-iteration
    cold probe of every case (its first residual is the fallback rule's base, its peak after iteration 20 the warm runs'
    drop reference), then every SST case restarted from the network's predicted field (unless its first residual exceeds
    10x the cold one), the Euler cases cold (the network models the SST base-wake flows), all to the reference's stop
    rules, a warm run that ends neither converged nor stationary solved again cold; device time of the probe and the
    solves; CDs against the oracle."""
    from bowshock_b200 import learned as lw
    from bowshock_b200.arena import Arena
    if not os.path.exists(lw.WEIGHTS):
        return {"status": "no trained network committed"}
    model = lw.WarmStart.load(lw.WEIGHTS, device=device)
    t0 = time.perf_counter()
    a = Arena(cases, device=device, grids=grids)
    probe = a.run(50)
    probe_ms = a.ms_per_iter() * 50
    sst = [k for k, c in enumerate(cases) if c.viscous is not None]
    fields = model.start_fields([cases[k] for k in sst])
    for q, k in enumerate(sst):
        u, t, mt = fields[q]
        a.set_state(k, u)
        a.set_turb(k, t, mt)
    first = a.first_residuals([1 if k in sst else 0 for k in range(len(cases))])
    fallback = []
    for k, c in enumerate(cases):
        warm = k in sst and np.isfinite(first[k]) and first[k] <= lw.FALLBACK_RATIO * probe[0, k]
        if k in sst and not warm:
            fallback.append(k)
        a.set_run(k, c.numerics, warm=bool(warm), r_ref=float(probe[20:, k].max()) if warm else None)
    res = a.solve()
    dev_s = (probe_ms + a.last_solve_ms()) / 1000.0
    # the reference keeps a warm result only when it converged or became stationary (analysis.rs:744-771): the rest
    # are solved again from the free stream
    redo = [k for k in sst if k not in fallback and res[k]["stop_reason"] not in lw.ACCEPTED]
    if redo:
        b = Arena([cases[k] for k in redo], device=device, grids=[grids[k] for k in redo])
        rr = b.solve()
        dev_s += b.last_solve_ms() / 1000.0
        for q, k in enumerate(redo):
            res[k] = rr[q]
        del b
    wall = time.perf_counter() - t0
    del a
    dcd = {k: cd_error(res[k], fx[k]) for k in range(len(cases)) if k in fx}
    n_ok = sum(abs(d) <= 1e-4 for d in dcd.values())
    value = 3600.0 * n_ok / dev_s
    e2e = 3600.0 * n_ok / wall
    return {"census_device_s": dev_s, "census_wall_s": wall, "converged_within_1e-4": n_ok, "checked_against_oracle": len(dcd),
            "cases_per_hr": value, "e2e_cases_per_hr": e2e, "warm_cases": [k for k in sst if k not in fallback], "fallbacks": fallback,
            "warm_resolved_cold": redo,
            "iters": [r["iters"] for r in res], "dcd": {str(k): float(f"{d:.3e}") for k, d in dcd.items()},
            "learned_plus_batched_vs_plain": e2e / plain_cases_per_hr if plain_cases_per_hr else None}


def measure_lift3(args, device):
    """Secondary figure: the 3D Euler lift sweep (15 cases, Mach x incidence, on one 192 x 64 x 64 revolved grid) as one
    batch, CUDA events over K line-implicit iterations after warm-up: ms per iteration, cell-updates/s, and the model's
    bytes per cell-update over the time against the measured HBM copy bandwidth."""
    import bowshock_b200.euler3 as e3
    t0 = time.perf_counter()
    b, _ = e3.batch_of(e3.lift_sweep_cases(), device=device)
    setup_s = time.perf_counter() - t0
    b.run(max(args.warmup, 3))
    n = max(5, min(args.steps, 20))
    b.run(n)
    ms = b.ms_per_iter()
    cells = b.nc * b.nb
    hbm, kind = peaks()
    gbs = cells * WORDS_3D * 4 / (ms / 1000.0) / 1e9
    del b
    return {"workload": "15-case 3D Euler lift sweep (alpha 0-8 deg x Mach 0.8/1.2/2.5), 192 x 64 x 64 cells each, one batch",
            "cells": int(cells), "iterations_timed": n, "ms_per_iter": ms, "cell_updates_per_s": cells / (ms / 1000.0),
            "model_bytes_per_cell_update": WORDS_3D * 4, "achieved_gbs": gbs, "hbm_frac": gbs / hbm, "peak_kind": kind,
            "setup_s": setup_s}


# algorithmic words of the FAS transfers per coarse cell (nv = 4): the restriction reads 4 fine cells x (state, defect,
# volume) and writes the coarse state and forcing, the prolongation reads the coarse state and its start value and
# reads and writes the 4 fine states. The profile's transfer group times the restriction folded into the coarse level's
# primitives (k_prims_restrict, which also converts the coarse states) and the prolongation; the forcing is written by the
# coarse residual launch (timed with the residuals), so the figure is a lower bound.
TRANSFER_WORDS = 4 * 9 + 8 + 8 + 4 * 8


def measure_multigrid(device):
    """Single-grid line-implicit against 3-level FAS with the line-implicit smoother, each to the reference's stop rules
    (wall clock of GpuSolver.run_to_stop): a sting-mounted ogive + cylinder at M 2.0 (attached flow, the coarse-grid
    correction under-relaxed by 0.5, coarse CFL halved per level) and config 0 (Euler, 128 x 64, M 1.5, separated base
    flow, correction under-relaxed by 0.5, capped at 4,000 cycles: it does not converge there; CD against the FP64
    oracle's converged run); and the transfer kernels' model
    bytes over their CUDA-event time (grids this small stay in the L2 cache)."""
    import bowshock_b200 as bk
    from bowshock_b200.case import Body, Case, NOSE_TANGENT_OGIVE, WAKE_STING
    from bowshock_b200.configs import config0_case
    with open(os.path.join(ROOT, "tests", "golden", "configs_oracle.json")) as f:
        ref = json.load(f)["config0"]
    body = Body(NOSE_TANGENT_OGIVE, fineness=3.0, segments=((6.0, 0.0),))
    work = {"sting_m2": ("sting-mounted tangent ogive + cylinder, Euler, M 2.0, level 0", lambda: Case.new(2.0, body, 0, WAKE_STING), 0.5, 0.5),
            "config0": ("config 0: Euler, tangent ogive + cylinder, base wake, M 1.5, 128 x 64", config0_case, 0.5, 1.0)}
    out = {}
    for key, (label, make, relax, scale) in work.items():
        o = out[key] = {"workload": label, "relax": relax, "cfl_scale": scale}
        for name, levels in (("single_grid", 1), ("multigrid3", 3)):
            c = make()
            s = c.build_solver(device)
            numerics = c.numerics
            if levels > 1:
                s.set_scheme(bk.solver.MgParams(levels=levels, pre=1, post=1, implicit=c.numerics.scheme, relax=relax, cfl_scale=scale))
                if key == "config0":  # it does not converge there (a bounded limit cycle): capped at 4,000 cycles
                    numerics = dataclasses.replace(numerics, max_iter=4000)
            t0 = time.perf_counter()
            r = s.run_to_stop(c.body, numerics, c.wake)
            wall = time.perf_counter() - t0
            o[name] = {"iters": r["iters"], "stop": r["stop_reason"], "wall_s": wall, "cd_total": r["cd_total"]}
            if key == "config0":
                o[name]["dcd_total_vs_oracle"] = r["cd_total"] - ref["cd_total"]
            if levels > 1 and key == "config0":
                prof = s.profile(10)
                ms, n = prof["transfer"]
                coarse = (64 * 32 + 32 * 16)  # coarse cells of one cycle's transfers (pre = post = 1, gamma = 1)
                if ms > 0:
                    gbs = coarse * TRANSFER_WORDS * 4 * 10 / (ms / 1000.0) / 1e9
                    o[name]["transfer_ms_per_cycle"] = ms / 10
                    o[name]["transfer_launches_per_cycle"] = n / 10
                    o[name]["transfer_model_gbs"] = gbs
                    o[name]["transfer_hbm_frac"] = gbs / peaks()[0]
            del s
        o["dcd_multigrid_vs_single"] = o["multigrid3"]["cd_total"] - o["single_grid"]["cd_total"]
    return out


def measure_mesher(device):
    """The grids of 2,000 SST cases of the sweep's distribution (the learned warm start's training set, seed 0x0B05_7EA1)
    built by the device mesher (nodes and FP64 metrics, bowshock_mesh_batch: device time of its launches, and wall
    clock with the copies back) against the host mesher (nodes only, one case at a time through the C ABI)."""
    from bowshock_b200 import learned as lw
    from bowshock_b200.case import mesh_batch
    cs = [lw.sweep_case(p) for p in lw.draw_sst(2000, lw.TRAIN_SEED)]
    mesh_batch(cs[:8], device=device)  # module load
    t0 = time.perf_counter()
    grids, _, dev_ms = mesh_batch(cs, device=device)
    wall = time.perf_counter() - t0
    t0 = time.perf_counter()
    for c in cs:
        c.grid()
    host = time.perf_counter() - t0
    nodes = sum((g[0] + 1) * (g[1] + 1) for g in grids)
    return {"cases": len(cs), "nodes": int(nodes), "device_ms": dev_ms, "device_wall_s": wall, "host_nodes_only_s": host}


def line_sweep_traffic():
    """DRAM bytes per line-sweep launch from the committed ncu summary of the line kernels (profiles/line_sweeps_sweep32.md:
    the `traffic_per_launch_bytes` line, written from dram__bytes_read.sum + dram__bytes_write.sum of that capture)."""
    p = os.path.join(ROOT, "profiles", "line_sweeps_sweep32.md")
    try:
        for l in open(p):
            if l.startswith("traffic_per_launch_bytes:"):
                return float(l.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# The sweep's cases that stop on the mean-stationary rule after 14,000-14,050 iterations (limit-cycle SST cases): the
# only ones left in the last ~8,650 iterations of the census.
TAIL6 = (1, 3, 5, 9, 15, 23)


def run_kernels(args):
    """The timed region alone (arena, warm-up, K iterations): the command the ncu captures of the kernels run. With
    --workload tail6: the same arena with only the TAIL6 cases active; with --workload lift3: the 15-case 3D Euler batch
    (192 x 64 x 64 cells per case) instead. The K timed iterations are
    bracketed by cudaProfilerStart / Stop, so that `ncu --profile-from-start off` captures exactly their launches."""
    import torch

    import bowshock_b200  # noqa: F401
    if args.workload == "net":  # training steps of the warm-start network (batch 64): its tensor-core GEMMs
        from bowshock_b200 import learned as lw
        from bowshock_b200.net import Net, flops_per_sample
        net = Net(max_batch=64)
        net.set_params(lw.init_params(0, net.layout(), net.nparams))
        rng = np.random.default_rng(0)
        net.set_dataset(rng.standard_normal((256, 16)).astype(np.float32), rng.standard_normal((256, 2048 * 6)).astype(np.float32))
        fl = 3.0 * flops_per_sample(net.layout()) * 64
        out = {"kernels_only": True, "workload": "net", "steps": args.steps}
        # the default (TMA-fed implicit GEMMs) last: the profiled pass
        for key, mode in (("im2col", Net.CONV_IM2COL), ("gather", Net.CONV_GATHER), ("tma", Net.CONV_TMA)):
            net.set_conv_mode(mode)
            net.train(max(args.warmup, 3), 64, 1e-4)
            if key == "tma":
                torch.cuda.profiler.start()
            net.train(args.steps, 64, 1e-4)
            if key == "tma":
                torch.cuda.profiler.stop()
            ms = net.last_train_ms() / args.steps
            tf = fl / (ms / 1000.0) / 1e12
            out[key] = {"ms_per_step": ms, "tflops": tf, "frac_of_bf16_peak": tf / bf16_peak()[0]}
        out["ms_per_step"] = out["tma"]["ms_per_step"]
        out["bf16_peak_kind"] = bf16_peak()[1]
        return out
    if args.workload in ("lift3", "lift3s"):  # lift3s: 3 of the 15 cases (4 deg at each Mach), for full ncu captures
        import bowshock_b200.euler3 as e3
        b, _ = e3.batch_of(e3.lift_sweep_cases((4.0,)) if args.workload == "lift3s" else e3.lift_sweep_cases())
        b.run(max(args.warmup, 1))
        torch.cuda.profiler.start()
        b.run(args.steps)
        torch.cuda.profiler.stop()
        return {"kernels_only": True, "workload": args.workload, "cells": b.nc * b.nb, "steps": args.steps, "ms_per_step": b.ms_per_iter()}
    from bowshock_b200.arena import Arena
    cases = build_cases()
    arena = Arena(cases, device=int(os.environ.get("LOCAL_RANK", "0")))
    if args.sst_coupled:  # the coupled 6x6 SST lines instead of the reference's loose coupling
        arena.set_sst_coupling(True)
    arena.run(max(args.warmup, 3))
    if args.workload == "tail6":  # the census's last ~8,650 iterations: only the 6 mean-stationary SST cases left
        arena.set_active([1 if k in TAIL6 else 0 for k in range(len(cases))])
        arena.run(max(args.warmup, 3))
    if args.groups > 1:
        arena.set_case_groups(args.groups)
        arena.run(max(args.warmup, 3))
    arena.prepare(args.steps)
    torch.cuda.profiler.start()
    arena.run(args.steps)
    torch.cuda.profiler.stop()
    ms = arena.ms_per_iter()
    prof = {g: round(v[0] / v[1], 4) for g, v in arena.profile(3).items() if v[1]} if args.steps >= 10 else None
    return {"kernels_only": True, "workload": args.workload, "cells": arena.cells, "steps": args.steps, "ms_per_step": ms, "ms_per_launch": prof,
            "autotuned_lines_per_block": arena.tuning(), "case_groups": args.groups, "sst_coupled": args.sst_coupled}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--kernels-only", action="store_true", help="only the timed arena iterations (for ncu captures)")
    ap.add_argument("--workload", default="sweep32", choices=["sweep32", "tail6", "lift3", "lift3s", "net"], help="workload of --kernels-only")
    ap.add_argument("--groups", type=int, default=1, help="case groups of the arena's graph in --kernels-only (1-4)")
    ap.add_argument("--sst-coupled", action="store_true", help="coupled SST lines in the --kernels-only arena")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: start the ranks here when the command was not launched by torchrun
        import socket
        sk = socket.socket()
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
        sk.close()
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1",
               f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as td
        td.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        dist = td
    if args.kernels_only:
        line = run_kernels(args)
    elif args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, dist)
    if line is not None and rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
