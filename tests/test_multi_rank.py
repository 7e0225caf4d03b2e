"""The multi-GPU story of the path is cases-per-GPU replicas (no data-path collective): each rank meshes and solves its
own seeded set of cases, and only scalars (the max step time, the summed throughputs) cross ranks. Checked here with two
gloo ranks on the CPU: the ranks' case sets are disjoint draws and the reduction is max / sum."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from bowshock_b200.sweep import SEED, draw
    machs = [p["mach"] for p in draw(32, SEED + rank)]
    ms, value, e2e = bench.combine_ranks(dist, 10.0 + rank, 100.0 * (rank + 1), 1.0)
    out[rank] = (machs[:4], ms, value, e2e)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_cases_and_reduce_scalars():
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    (m0, ms0, v0, e0), (m1, ms1, v1, e1) = out[0], out[1]
    assert m0 != m1, "each rank draws its own cases"
    assert ms0 == ms1 == 11.0  # max over ranks
    assert v0 == v1 == 300.0 and e0 == e1 == 2.0  # sums over ranks
