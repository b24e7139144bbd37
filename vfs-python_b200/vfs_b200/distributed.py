"""Multi-GPU plumbing for independent stereo pairs (one process per GPU).

Pairs are independent, so a batch is split across ranks with no collective on
the data path; the only collectives are a max of device times (measurement)
and a sum of the few learned-parameter gradients (parameter learning).  The
reference has no multi-GPU path: it runs on one GPU, on the default stream, and
synchronises after every launch (e.g. Python/vfs.py:107-113).
"""
from __future__ import annotations

import heapq

import torch
import torch.distributed as dist


def pair_cost(h: int, w: int, n_level: int, f_scale: float, n_warp: int, n_iter: int) -> float:
    """Pixel-iterations of one solve, the work the TGV kernels do."""
    total = 0.0
    for _ in range(n_level):
        total += h * w
        h, w = int(h / f_scale), int(w / f_scale)
    return total * n_warp * max(n_iter, 1)


def shard(costs, world: int, rank: int) -> list[int]:
    """Indices of the items rank `rank` solves: longest-processing-time-first
    greedy assignment of `costs` to `world` ranks (deterministic, so every
    rank computes the same partition without communicating)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    owner = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + costs[i], r))
    return [i for i in range(len(costs)) if owner[i] == rank]


def _device():
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """Max of a scalar over the default process group (time-like metrics)."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_gradients(grads: dict) -> dict:
    """Sum of per-rank parameter gradients (one all-reduce of one flat tensor)."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(grads)
    keys = sorted(grads)
    flat = torch.tensor([float(grads[k]) for k in keys], dtype=torch.float64, device=_device())
    dist.all_reduce(flat, op=dist.ReduceOp.SUM)
    return {k: float(v) for k, v in zip(keys, flat.tolist())}
