"""The multi-GPU story of the path: the cases of a sweep are partitioned over the ranks (one process per GPU, no
data-path collective) and only the per-case results are gathered (crates/bowshock-core/src/analysis.rs:746-795 solves
its cases independently). Checked on the CPU: the longest-processing-time partition covers every case exactly once and
balances the estimated cost; with two gloo ranks, each solving only its own share (the oracle's first iterations of
each case stand in for the GPU solve here), the gathered results equal a one-rank run of the whole sweep, and the
max / sum reductions of bench.py hold."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bowshock_b200.shard import case_cost, expected_iters, gather_results, lpt_partition


def test_lpt_partition_covers_each_case_once_and_balances():
    from bowshock_b200.sweep import sweep_cases
    cs = sweep_cases(32)
    costs = [case_cost(c) for c in cs]
    for n in (1, 2, 3, 4, 8):
        parts = lpt_partition(costs, n)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(32)), f"{n} ranks: not a partition"
        loads = [sum(costs[k] for k in p) for p in parts]
        # LPT bound: no rank above the mean by more than the largest single item
        assert max(loads) <= sum(costs) / n + max(costs) + 1e-9
        assert lpt_partition(costs, n) == parts  # deterministic
    assert expected_iters(cs[1]) > expected_iters(cs[0])  # SST above Euler


def test_lpt_partition_edge_cases():
    assert lpt_partition([], 3) == [[], [], []]
    assert lpt_partition([5.0], 2) == [[0], []]
    assert lpt_partition([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        lpt_partition([1.0], 0)


def test_gather_results_single_process_and_errors():
    assert gather_results(None, [1, 0], ["b", "a"], 2) == ["a", "b"]
    with pytest.raises(RuntimeError):
        gather_results(None, [0], ["a"], 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _solve_share(indices):
    """CPU stand-in for a rank's arena solve: 3 oracle iterations of each of its cases (their density residuals and the
    final state's checksum), deterministic per case."""
    import oracle_ffi as o
    from tests.golden.sweep_oracle import oracle_case
    from bowshock_b200.sweep import sweep_cases
    cs = sweep_cases(32)
    out = []
    for k in indices:
        s = o.Solver.from_case(oracle_case(cs[k]))
        r = s.steps(3)
        out.append({"case": k, "residual": [float(x) for x in r], "checksum": float(np.sum(s.u))})
    return out


SHARE_CASES = list(range(8))  # a sub-sweep keeps the CPU cost to seconds


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from bowshock_b200.sweep import sweep_cases
    cs = sweep_cases(32)
    costs = [case_cost(cs[k]) for k in SHARE_CASES]
    mine = lpt_partition(costs, world)[rank]
    res = gather_results(dist, mine, _solve_share([SHARE_CASES[q] for q in mine]), len(SHARE_CASES))
    mx = bench.reduce_scalars(dist, [10.0 + rank, 1.0 * rank], "max")
    sm = bench.reduce_scalars(dist, [100.0 * (rank + 1)], "sum")
    out[rank] = (mine, res, mx, sm)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_partition_solve_and_gather():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    (m0, r0, mx0, sm0), (m1, r1, mx1, sm1) = out[0], out[1]
    assert sorted(m0 + m1) == list(range(len(SHARE_CASES))) and not set(m0) & set(m1), "ranks must split the cases"
    assert r0 == r1, "every rank holds the gathered results"
    single = _solve_share(SHARE_CASES)
    assert r0 == single, "the gathered results differ from a one-rank run"
    assert mx0 == mx1 == [11.0, 1.0]
    assert sm0 == sm1 == [300.0]
