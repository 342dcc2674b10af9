"""Host logic of the multi-GPU path (replicas of independent RVE solves): the
footprint partition and the result gather, run as two gloo ranks on CPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mat3d_b200.shard import partition_by_footprint


def test_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.choice([32 ** 3, 48 ** 3, 64 ** 3, 96 ** 3], size=200))
    for world in (1, 2, 3, 8):
        parts = partition_by_footprint(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # largest-first greedy: the spread is at most the largest item
        assert max(loads) - min(loads) <= max(costs)
    assert partition_by_footprint([5.0, 5.0], 2) == [[0], [1]]
    with pytest.raises(ValueError):
        partition_by_footprint([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, n, out_q):
    import torch.distributed as dist

    from mat3d_b200.shard import gather_tensors

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [(i % 4 + 1) ** 3 for i in range(n)]
        mine = partition_by_footprint(costs, world)[rank]
        # stand-in for each rank's homogenization: a tensor that encodes the RVE index
        tensors = [np.eye(6) * (i + 1) for i in mine]
        full = gather_tensors(mine, tensors, n)
        out_q.put((rank, full))
    finally:
        dist.destroy_process_group()


def test_gather_two_gloo_ranks():
    n, world = 11, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, full in res:
        for i in range(n):
            assert np.array_equal(full[i], np.eye(6) * (i + 1))
