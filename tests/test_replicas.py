"""The N > 1 path on CPU: two gloo ranks agree on max-over-ranks timing and on
the partition of a batch of instances (what bench.py --gpus N uses)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def worker(rank, world, port, q):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    import __graft_entry__ as ge
    rn = ge.load_package()
    from rocket_nozzle_cfd_solver_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mx = replicas.max_over_ranks(1.5 + rank)
        sm = replicas.sum_over_ranks(10 * (rank + 1))
        share = list(replicas.partition(64, rank, world))
        q.put((rank, mx, sm, share))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.5, 2.5]
    assert [r[2] for r in res] == [30.0, 30.0]
    shares = [r[3] for r in res]
    assert shares[0] + shares[1] == list(range(64)) and len(shares[0]) == 32


def test_partition_covers_uneven_batches(rn):
    from rocket_nozzle_cfd_solver_b200 import replicas
    for n in (0, 1, 7, 64, 65):
        for world in (1, 2, 3, 8):
            parts = [list(replicas.partition(n, r, world)) for r in range(world)]
            assert sum(parts, []) == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        replicas.partition(4, 2, 2)


def test_partition_by_cost_balances_uneven_instances(rn):
    """Longest-processing-time split of the batched workload's grids: every
    instance lands on exactly one rank and the largest load is within one
    largest item of the mean."""
    from rocket_nozzle_cfd_solver_b200 import configs, replicas
    cfgs = configs.batched(64, seed=2024)
    cost = [c["Nx"] * round(c["aspect"] * c["Nx"]) for c in cfgs]
    for world in (1, 2, 3, 4, 8):
        parts = [replicas.partition_by_cost(cost, r, world) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(64))
        loads = [sum(cost[k] for k in p) for p in parts]
        assert max(loads) - sum(cost) / world <= max(cost)
    with pytest.raises(ValueError):
        replicas.partition_by_cost(cost, 2, 2)
