"""Multi-GPU host logic on CPU: instance partitioning and the statistics gather over a
world-size-2 gloo process group (the N > 1 path without GPUs)."""
import os
import socket

import pytest

from coffee_sim_b200.shard import gather_statistics, local_instances, partition_instances


def test_partition_covers_every_instance_once_and_balances():
    counts = [20_000 + (i * 37_919) % 280_000 for i in range(64)]
    for world in (1, 2, 3, 8):
        parts = partition_instances(counts, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(counts[i] for i in p) for p in parts]
        # greedy LPT: the heaviest rank exceeds the mean by less than one instance
        assert max(loads) - sum(loads) / world <= max(counts)
    assert partition_instances([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    assert partition_instances([], 2) == [[], []]
    with pytest.raises(ValueError):
        partition_instances([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, counts, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = local_instances(counts, rank, world)
        # a stand-in for per-instance statistics (emitted ml, residual)
        stats = {i: [float(counts[i]) * 0.5, 1e-6 * (i + 1)] for i in mine}
        every = gather_statistics(stats)
        q.put((rank, mine, sorted(every), every[0]))
    finally:
        dist.destroy_process_group()


def test_gather_statistics_over_gloo():
    import torch.multiprocessing as mp

    counts = [300_000, 20_000, 150_000, 90_000, 60_000]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, counts, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    (r0, mine0, all0, s0), (r1, mine1, all1, s1) = results
    assert sorted(mine0 + mine1) == list(range(5))
    assert all0 == all1 == list(range(5))
    assert s0 == s1 == [150_000.0, 1e-6]


def test_gather_statistics_without_process_group():
    assert gather_statistics({3: [1.0]}) == {3: [1.0]}
