"""Replicas across GPUs: one process and one engine per GPU, whole maps per rank.

The path has no exchange step (anchors and maps are independent), so several
GPUs are used as replicas: each rank runs its own maps and no data-path
collective exists. torch.distributed carries only the plumbing: a barrier, and
the max/sum of the ranks' timings and counts.

``assign_maps`` splits one set of maps over the ranks, balanced by edges
(largest first, each to the least-loaded rank). ``reduce_max``/``reduce_sum``
work over NCCL (CUDA tensors) and gloo (CPU tensors) alike.
"""
from __future__ import annotations

import heapq


def assign_maps(sizes, world: int) -> list[list[int]]:
    """Map indices per rank; every map goes to exactly one rank. Ties go to the
    lower rank, so every rank computes the same assignment on its own."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    for r in out:
        r.sort()
    return out


def _tensor(dist, v: float):
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    return torch.tensor([float(v)], dtype=torch.float64, device=dev)


def reduce_max(dist, v: float) -> float:
    """The maximum of v over the ranks (v itself without a process group)."""
    if dist is None:
        return v
    t = _tensor(dist, v)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(dist, v: float) -> float:
    if dist is None:
        return v
    t = _tensor(dist, v)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
