"""The multi-GPU host logic with two gloo ranks on CPU: batches split into
contiguous, balanced, disjoint blocks of systems; the job's device time as the
slowest rank's; per-system results gathered back in system order."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cudaring_b200 import replicas


def test_shards_cover_every_system_once_and_balance_vertices():
    rng = np.random.default_rng(3)
    sizes = rng.integers(16 * 16, 512 * 22, size=256)
    for world in (1, 2, 3, 4, 8):
        blocks = [replicas.shard_systems(sizes, world, r) for r in range(world)]
        covered = [i for b in blocks for i in b]
        assert covered == list(range(len(sizes)))
        loads = [int(sizes[list(b)].sum()) for b in blocks]
        assert max(loads) - min(loads) <= 2 * int(sizes.max())
    # more ranks than systems: the extra ranks get empty blocks
    assert [len(replicas.shard_systems([5, 5], 3, r)) for r in range(3)] == [1, 1, 0]
    with pytest.raises(ValueError):
        replicas.shard_systems([1], 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        block = replicas.shard_systems(sizes, world, rank)
        # per-system "results" computed by the owning rank only
        local = [(i, float(sizes[i]) * 0.5) for i in block]
        gathered = replicas.gather_per_system(local, world)
        t_max = replicas.max_over_ranks(10.0 + rank, world)
        units = replicas.sum_over_ranks(float(sum(sizes[i] for i in block)), world)
        out.put((rank, gathered, t_max, units))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    sizes = [int(x) for x in np.random.default_rng(5).integers(300, 3000, size=37)]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, t_max, units in res:
        assert [i for i, _ in gathered] == list(range(len(sizes)))
        assert [v for _, v in gathered] == [0.5 * s for s in sizes]
        assert t_max == 11.0
        assert units == float(sum(sizes))
