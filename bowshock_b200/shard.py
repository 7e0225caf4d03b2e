"""Cases across GPUs: the path shards by case, never inside one. The cases of a sweep are independent (the reference
solves its Mach points one after another, crates/bowshock-core/src/analysis.rs:746-795), while a single case's line
solves span its whole grid. So each GPU (one process per GPU) takes a disjoint subset of the sweep, solves it in its own
batched arena, and the only exchange is a gather of the per-case results (host objects over the process group, no
data-path collective).

The subsets are a longest-processing-time partition: cases sorted by their estimated cost (cells x expected iterations to
the stop rule), each given to the rank with the least estimated work so far. The expected iterations follow the stop rules
(engine/run.rs:105-170): a viscous case runs at least 2 monitor windows before its CD-stationary rule can hold and most
of them run longer; an Euler case stops on its residual drop after about 1,000 line-implicit iterations."""
from __future__ import annotations

EULER_ITERS = 1000  # typical residual-drop stop of a line-implicit Euler case (485-2,386 on the seeded sweep)


def expected_iters(case) -> int:
    """Estimated iterations of `case` to its stop rule (the partition's cost model, not a prediction of the result)."""
    n = case.numerics
    if case.viscous is not None:
        return max(2 * int(n.monitor_window), 4000) + (int(n.mean_window) // 2 if n.mean_window else 0)
    return max(EULER_ITERS, int(n.min_iter))


def case_cost(case, grid=None) -> float:
    ni, nj = (grid[0], grid[1]) if grid is not None else case.cells()
    return float(ni * nj) * float(expected_iters(case))


def lpt_partition(costs, n_ranks):
    """Longest-processing-time partition of items with `costs` over `n_ranks` ranks: item indices per rank, each list in
    ascending index order. Deterministic (ties go to the lower index / lower rank), so every rank computes the same one."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    load = [0.0] * n_ranks
    parts = [[] for _ in range(n_ranks)]
    for k in order:
        r = min(range(n_ranks), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += float(costs[k])
    return [sorted(p) for p in parts]


def gather_results(dist, local_indices, local_results, n_items):
    """Every rank's (index, result) pairs gathered to every rank and put back in item order; with `dist` None (one
    process) the local results are the whole list. Raises if an item is missing or given twice."""
    pairs = list(zip(local_indices, local_results))
    if dist is None:
        gathered = [pairs]
    else:
        gathered = [None] * dist.get_world_size()
        dist.all_gather_object(gathered, pairs)
    out = [None] * n_items
    seen = [0] * n_items
    for part in gathered:
        for k, r in part:
            out[k] = r
            seen[k] += 1
    bad = [k for k in range(n_items) if seen[k] != 1]
    if bad:
        raise RuntimeError(f"items not gathered exactly once: {bad}")
    return out
