"""Replicas across ranks (no GPU): the map assignment is a balanced partition
that every rank computes alike, and the timing reductions agree across ranks
(torch.distributed over gloo, world size 2, on the CPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from curvelet_construction_on_gpu_b200.replicas import assign_maps


def test_assign_maps_is_a_balanced_partition():
    rng = np.random.default_rng(3)
    sizes = rng.integers(2_000, 3_800_000, 64)
    for world in (1, 2, 3, 4, 8):
        parts = assign_maps(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [int(sum(sizes[i] for i in p)) for p in parts]
        # largest-first greedy: no rank exceeds the mean by more than the largest map
        assert max(loads) - sum(loads) / world <= int(sizes.max())
    assert assign_maps([5, 5], 4) == [[0], [1], [], []]
    with pytest.raises(ValueError):
        assign_maps([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, sizes, q):
    import datetime

    import torch.distributed as dist

    from curvelet_construction_on_gpu_b200.replicas import assign_maps, reduce_max, reduce_sum
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = assign_maps(sizes, world)[rank]
        edges = float(sum(sizes[i] for i in mine))
        tot = reduce_sum(dist, edges)
        mx = reduce_max(dist, 10.0 + rank)
        got = [None] * world
        dist.all_gather_object(got, mine)
        dist.barrier()
        q.put((rank, tot, mx, got))
    finally:
        dist.destroy_process_group()


def test_replica_reductions_over_gloo():
    world = 2
    sizes = [int(x) for x in np.random.default_rng(5).integers(1_000, 500_000, 20)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, tot, mx, got in outs:
        assert tot == float(sum(sizes))
        assert mx == 10.0 + world - 1
        assert sorted(i for part in got for i in part) == list(range(len(sizes)))
        assert got == assign_maps(sizes, world)
