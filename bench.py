"""Benchmark of the B200 backend on the seeded 32-case mixed sweep (Euler + RANS SST, grids 96x48 to 320x160).

Metric: converged cases per hour on one B200 for the batched line-implicit backend. One step = one line-implicit iteration
of the whole 32-case arena (all cases active). `value` is the steady-state throughput of a persistent arena that is kept
full (converged cases replaced by new ones):

    cases/s = n_cases * sum_k cells_k / (t_step * sum_k cells_k * N_k)

with t_step the device time of one arena iteration (CUDA events, the timed region: K steps replayed from CUDA graphs) and
N_k the iterations case k needs to reach its stop rule, measured in the same run by the census (every case cold-started and
iterated to the reference's stop rules, converged cases masked out). `e2e` is the census itself measured by the wall clock
through the public API (meshing, arena creation with the host->device copies, the solve, the device->host read-back of
residual histories and forces). `cpu_baseline` times the oracle (the f64 C++ restatement of the reference CPU solver, all
host threads) on a bounded sample of iterations of every case and applies the same N_k. The plain single-case backend is
timed the same way (one case per arena, one after another) and reported as `config.plain_single_case_cases_per_hr`.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
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


def build_cases(rank=0):
    from bowshock_b200.sweep import SEED, sweep_cases
    return sweep_cases(32, SEED + rank)


def combine_ranks(dist, ms_step, value, e2e):
    """Cases-per-GPU replicas: the step time is the max over ranks, the throughputs add up (scalars only, no data-path
    collective)."""
    if dist is None:
        return ms_step, value, e2e
    import torch
    t = torch.tensor([ms_step], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    s = torch.tensor([value, e2e], dtype=torch.float64)
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    return float(t.item()), float(s[0]), float(s[1])


def cpu_sample(cases, grids, n_iter, census):
    """The oracle on `n_iter` iterations of every case (all host threads): cases/hr with the census iteration counts."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_ffi as o
    from tests import cases as tc
    t_case = []
    for k, c in enumerate(cases):
        ni, nj, x, r, blk = grids[k]
        cfg = c.config()
        spec = tc.Spec(ni, nj, np.asarray(x).reshape(nj + 1, ni + 1), np.asarray(r).reshape(nj + 1, ni + 1), cfg.cfl, cfg.limiter,
                       tuple(cfg.freestream), tuple(cfg.bc), cfg.first_order_iters, c.numerics.low_mach, blk,
                       dict(cfl0=c.numerics.scheme.cfl0, cfl_max=c.numerics.scheme.cfl_max, growth=c.numerics.scheme.growth,
                            dt_mode=c.numerics.scheme.dt_mode, lines=True, implicit_bc=True, sub_iters=c.numerics.scheme.sub_iters,
                            roe=True, eps_fix=0.1),
                       None if c.viscous is None else dict(re_c=c.viscous.re_c, sutherland=c.viscous.sutherland, turbulence=1,
                                                           wall_i_start=c.viscous.wall_i_start, roughness=0.0))
        s = tc.oracle_solver(spec)
        s.step()  # warm-up
        t0 = time.perf_counter()
        s.steps(n_iter)
        t_case.append((time.perf_counter() - t0) / n_iter)
    n = np.array([census[k] for k in range(len(cases))], dtype=float)
    total_s = float(np.sum(np.array(t_case) * n))
    return 3600.0 * len(cases) / total_s, t_case


def census_fixture():
    p = os.path.join(ROOT, "tests", "golden", "sweep_census.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def run_reference(args, rank, world):
    """The reference arm: the reference CPU path (its f64 restatement, the oracle) on the same workload and metric."""
    if rank != 0:
        return None
    cases = build_cases(0)
    grids = [c.grid() for c in cases]
    fx = census_fixture()
    census = fx["iters"] if fx else [4000] * len(cases)
    n_iter = 2
    vals, t_case = [], None
    for _ in range(args.warmup):
        cpu_sample(cases[:2], grids[:2], 1, census)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, t_case = cpu_sample(cases, grids, n_iter, census)
        vals.append(v)
    wall = time.perf_counter() - t0
    value = float(np.mean(vals))
    threads = os.cpu_count()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * wall / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 32-case sweep, SplitMix64 seed 0x0B05C0C2)",
            "config": {"workload": "32-case mixed Euler/SST sweep, reference CPU path (f64 restatement), line-implicit",
                       "cases": len(cases), "census": "tests/golden/sweep_census.json" if fx else "4000 iterations per case (no census)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{n_iter} iterations of each of the 32 cases per step, x the census iterations to converge"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def run_ours(args, rank, world, dist):
    import bowshock_b200  # noqa: F401
    from bowshock_b200.arena import Arena
    device = int(os.environ.get("LOCAL_RANK", "0"))
    cases = build_cases(rank)
    grids = [c.grid() for c in cases]
    cells = np.array([g[0] * g[1] for g in grids], dtype=float)
    arena = Arena(cases, device=device, grids=grids)
    ncell = arena.cells
    # warm-up (also builds and instantiates the CUDA graph of the step chunk)
    arena.run(max(args.warmup, 1))
    if dist:
        dist.barrier()
    clocks = Clocks(device)
    clocks.start()
    t0 = time.perf_counter()
    arena.run(args.steps)
    wall_timed = time.perf_counter() - t0
    ms_step = arena.ms_per_iter()
    clk = clocks.stop()
    ms_local = ms_step
    # per-kernel profile (CUDA events around every launch) for the roofline of the dominant kernel
    prof = arena.profile(5)
    hbm, peak_kind = peaks()
    # census: every case to its stop rule, through the public API, timed by the wall clock (e2e)
    cen_cases = build_cases(rank)
    t1 = time.perf_counter()
    cen_grids = [c.grid() for c in cen_cases]
    cen = Arena(cen_cases, device=device, grids=cen_grids)
    results = cen.solve()
    wall_census = time.perf_counter() - t1
    iters = [r["iters"] for r in results]
    n_k = np.array(iters, dtype=float)
    cases_per_s = len(cases) * cells.sum() / ((ms_local / 1000.0) * float(np.sum(cells * n_k)))
    value_rank = 3600.0 * cases_per_s
    # plain single-case backend: one case per arena, one after another, same iteration counts
    t_plain = []
    for k, c in enumerate(cases):
        a1 = Arena([c], device=device, grids=[grids[k]])
        a1.run(3)
        a1.run(20)
        t_plain.append(a1.ms_per_iter() / 1000.0)
        del a1
    plain_cases_per_hr = 3600.0 * len(cases) / float(np.sum(np.array(t_plain) * n_k))
    ms_step, total_value, e2e_value = combine_ranks(dist, ms_local, value_rank, 3600.0 * len(cases) / wall_census)
    if rank != 0:
        return None
    # roofline of the dominant kernel group
    groups = {g: v for g, v in prof.items() if v[1] > 0}
    top = max(groups, key=lambda g: groups[g][0])
    ms_top, launches_top = groups[top]
    viscous = np.array([c.viscous is not None for c in cases])
    if top in ("lines_i", "lines_j"):
        words = np.where(viscous, SWEEP_WORDS[True], SWEEP_WORDS[False])
        sub = np.array([c.numerics.scheme.sub_iters for c in cases])
        # one launch sweeps every case that has a pass at that position; average over the passes of an iteration
        passes = sub.max()
        bytes_iter = float(np.sum(cells * words * 4 * sub)) / passes
    else:
        bytes_iter = float(np.sum(cells * (42 + np.where(viscous, 21, 0)) * 4))  # residual pass: 2 nv + g + v + 1 words
    ms_launch = ms_top / launches_top
    achieved = bytes_iter / (ms_launch / 1000.0) / 1e9
    fx_traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            fx_traffic = json.load(open(tpath)).get(top)
        except Exception:
            fx_traffic = None
    # CPU baseline: the oracle on a bounded sample with the same census iteration counts
    cpu_val, t_cpu = cpu_sample(cases, grids, 2, iters) if rank == 0 else (None, None)
    stops = {}
    for r in results:
        stops[r["stop_reason"]] = stops.get(r["stop_reason"], 0) + 1
    launches_per_iter = sum(v[1] for v in prof.values()) / 5.0
    h2d = int(sum(16 * (g[0] + 1) * (g[1] + 1) + 32 * g[0] * g[1] for g in cen_grids))
    d2h = int(len(cases) * (8 * 50 + 8 * 16))
    line = {
        "metric": METRIC, "value": total_value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic (seeded 32-case sweep per GPU, SplitMix64 seed 0x0B05C0C2 + rank)",
        "config": {
            "workload": "32-case mixed Euler/RANS-SST sweep, grids 96x48..320x160, line-implicit, batched arena (one launch per kernel "
                        "for all cases), CUDA graph per chunk",
            "cases": len(cases), "cells": int(ncell), "cell_updates_per_s": float(ncell / (ms_step / 1000.0)),
            "l2": "working set larger than L2 (no flush needed): ~%.0f MB per iteration" % (ncell * 420 / 1e6),
            "census_iters_mean": float(n_k.mean()), "census_iters": iters, "census_stop_reasons": stops,
            "census_wall_s": wall_census, "value_rule": "n * sum(cells) / (t_step * sum(cells * N_k))",
            "plain_single_case_cases_per_hr": plain_cases_per_hr, "batched_vs_plain": total_value / world / plain_cases_per_hr,
            "learned_warm_start": "not built: cold (free-stream) starts",
            "kernel_profile_ms_per_launch": {g: v[0] / v[1] for g, v in groups.items()},
            "parallelism": f"cases-per-GPU replicas x{world}",
        },
        "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_launch": bytes_iter, "ms_per_launch": ms_launch,
                     "traffic": fx_traffic},
        "cpu_baseline": {"value": cpu_val, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                         "sample": "2 iterations of each of the 32 cases (oracle, all host threads) x the census iterations to converge"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "what": "wall clock of meshing + arena creation + solve to the stop rules + read-back, through the public API"},
        "clocks": clk,
        "gpu_launches": int(round(launches_per_iter * args.steps)),
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as td
        td.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        dist = td
    if args.impl == "reference":
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
