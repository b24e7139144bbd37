"""Per-level choice of the fused TGV kernel (tile shape, iterations per launch,
threads per block, or the cluster-resident kernel).

Every candidate computes bit-identical results, so the choice is about speed
only.  One timed solve per candidate applies that candidate to every level at
once; the plan's CUDA-event timing splits the TGV time by level, and each
level keeps its fastest candidate.  Large levels favour big tiles with deep
temporal blocking (fewer halo pixels per useful pixel); small levels favour
small tiles or the cluster kernel, which spread a few thousand pixels over
more SMs.
"""
from __future__ import annotations

import ctypes
import json
import os

import torch

from . import _lib

CLUSTER = 1000  # VFS_TGV_CLUSTER

_CACHE: dict = {}


def variants() -> list[int]:
    n = _lib.lib().vfs_tgv_variants(None, 0, None)
    ids = (ctypes.c_int * n)()
    n = min(n, _lib.lib().vfs_tgv_variants(ids, n, None))
    return [ids[i] for i in range(n)]


def _key(vfs) -> tuple:
    p = vfs.param
    return (torch.cuda.get_device_name(), p.width, p.height, p.fScale, p.nLevel, p.nWarpIters, p.nSolverIters)


def autotune(vfs, img_ref, img_other, candidates=None, repeats: int = 2, cache_file: str | None = None) -> list[int]:
    """Returns (and installs on ``vfs``) the per-level kernel choice, finest first."""
    key = _key(vfs)
    if key in _CACHE:
        vfs.set_level_variants(_CACHE[key]["choice"])
        return _CACHE[key]["choice"]
    if cache_file and os.path.exists(cache_file):
        with open(cache_file) as f:
            saved = json.load(f)
        if saved.get("key") == list(key):
            _CACHE[key] = saved
            vfs.set_level_variants(saved["choice"])
            return saved["choice"]
    nlev = vfs.param.nLevel
    cands = list(candidates) if candidates is not None else variants() + [CLUSTER]
    prev = (vfs.use_graph, vfs.timing)
    vfs.configure(use_graph=True, timing=True)
    plan = vfs._sync_plan_inputs()
    fits = [_lib.lib().vfs_plan_level_cluster(plan, l) > 0 for l in range(nlev)]
    best = [(float("inf"), 0)] * nlev
    table = {}
    for c in cands:
        if c == CLUSTER and not any(fits):
            continue
        vfs.set_level_variants([c if (c != CLUSTER or fits[l]) else 0 for l in range(nlev)])
        times = None
        for _ in range(repeats + 1):  # the first solve captures the graph
            vfs.solve_stereo(img_ref, img_other)
            lv = vfs.solve_stats()["tgv_ms_level"]
            times = lv if times is None else [min(a, b) for a, b in zip(times, lv)]
        table[c] = times
        for l in range(nlev):
            if c == CLUSTER and not fits[l]:
                continue
            if times[l] < best[l][0]:
                best[l] = (times[l], c)
    choice = [c for _, c in best]
    vfs.set_level_variants(choice)
    vfs.configure(use_graph=prev[0], timing=prev[1])
    entry = {"key": list(key), "choice": choice, "ms": [t for t, _ in best],
             "table": {str(k): v for k, v in table.items()}}
    _CACHE[key] = entry
    if cache_file:
        with open(cache_file, "w") as f:
            json.dump(entry, f, indent=1)
    return choice


def last_table(vfs) -> dict | None:
    return _CACHE.get(_key(vfs))
