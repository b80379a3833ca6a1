"""Multi-GPU plumbing: one process per GPU, independent solver instances.

A single nozzle grid does not shard (its halo exchange would cost more than
its compute at these sizes), so N GPUs run N independent instances: replicas
of one workload, or disjoint shares of a batch of instances. There is no
data-path collective; ranks only agree on timing (max over ranks) and on the
totals of work done.
"""


def partition(n_items, rank, world):
    """Contiguous share of ``n_items`` for ``rank`` of ``world`` (sizes differ by at most one)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def partition_by_cost(costs, rank, world):
    """Indices of the items ``rank`` takes when items of the given costs (e.g.
    grid cells) are spread over ``world`` ranks by longest-processing-time:
    largest first, each to the least-loaded rank (ties to the lower rank).
    Deterministic, so every rank computes the same assignment on its own."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    load = [0] * world
    owner = [0] * len(costs)
    for k in sorted(range(len(costs)), key=lambda q: (-costs[q], q)):
        r = min(range(world), key=lambda w: (load[w], w))
        owner[k] = r
        load[r] += costs[k]
    return [k for k in range(len(costs)) if owner[k] == rank]


def max_over_ranks(value, device="cpu"):
    """Max of a float over all ranks of the default process group (identity when not distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device="cpu"):
    """Sum of a float over all ranks (identity when not distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
