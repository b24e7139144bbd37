"""GPU: the batched multi-pair solve is bit-identical, pair by pair, to the
single-pair solve and to the reference kernels."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import bench_params, pair

pytestmark = pytest.mark.gpu


def _fields(p):
    from vfs_b200 import EquidistantCam
    from vfs_b200.vector_field import get_vector_fields, get_grid_zero
    cam = EquidistantCam(p.intrinsics)
    cam.setup_module()
    return get_vector_fields(get_grid_zero(p.img_ref.shape), cam, cam, p.R, p.t, 1) + (cam,)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_batched_solve_matches_single_pair_and_reference(gpu):
    from vfs_b200 import VFS
    from vfs_b200.batch import VFSBatch
    from oracle.refgpu import refpath
    sizes = [(96, 128), (64, 80), (80, 80), (72, 96)]
    ts = [(0.12, 0.01, 0.0), (0.05, -0.08, 0.02), (0.1, 0.0, 0.0), (-0.07, 0.06, 0.01)]
    pairs = [pair(w, height=h, t=t, seed=20 + i, n_level=3) for i, ((h, w), t) in enumerate(zip(sizes, ts))]
    prm = bench_params(96, 128, n_level=3, n_warp=2, n_iter=11)
    fields = [_fields(p) for p in pairs]
    batch = VFSBatch(prm, sizes)
    for i, (p, (tvf, cvf, _)) in enumerate(zip(pairs, fields)):
        batch.set_pair(i, p.mask, tvf, cvf)
    refs = [p.img_ref for p in pairs]
    oths = [p.img_other for p in pairs]
    for graph in (False, True):
        batch.configure(use_graph=graph)
        warps = [w.cpu().numpy() for w in batch.solve(refs, oths)]
        for i, (p, (tvf, cvf, cam)) in enumerate(zip(pairs, fields)):
            prm_i = bench_params(*sizes[i], n_level=3, n_warp=2, n_iter=11)
            v = VFS(prm_i)
            v.compute_pyramid_sizes()
            v.create_mask_pyramid(p.mask)
            v.create_vector_field_pyramid(tvf, cvf)
            single = v.solve_stereo(p.img_ref, p.img_other).cpu().numpy()
            assert np.array_equal(_bits(single), _bits(warps[i])), f"pair {i} (graph {graph})"
            for method in ("reference", "lsq"):
                xb = batch.triangulate(i, cam, p.t, method=method).cpu().numpy()
                xs = v.triangulate_flow(cam, p.t, method=method).cpu().numpy()
                assert np.array_equal(_bits(xb), _bits(xs)), f"pair {i} xyz ({method})"
    # the launch grouping changes the order of launches only: one pair per
    # group and groups of a budget agree with one group per level
    for gb in (1, 96 << 20):
        batch.configure(group_bytes=gb)
        regrouped = [w.cpu().numpy() for w in batch.solve(refs, oths)]
        for i in range(len(pairs)):
            assert np.array_equal(_bits(regrouped[i]), _bits(warps[i])), f"pair {i} with group budget {gb}"
    batch.configure(group_bytes=0)
    # one pair against the reference's own kernels
    r = refpath.RefVFS(bench_params(*sizes[1], n_level=3, n_warp=2, n_iter=11), "bench")
    r.compute_pyramid_sizes()
    r.create_mask_pyramid(pairs[1].mask)
    r.create_vector_field_pyramid(fields[1][0], fields[1][1])
    rw = r.solve_stereo(pairs[1].img_ref, pairs[1].img_other).cpu().numpy()
    assert np.array_equal(_bits(rw), _bits(warps[1]))
    # the batch autotuner changes speed only
    choice = batch.autotune(refs, oths, candidates=[134, 162, 192], repeats=1)
    assert len(choice) == prm.nLevel
    again = [w.cpu().numpy() for w in batch.solve(refs, oths)]
    for i in range(len(pairs)):
        assert np.array_equal(_bits(again[i]), _bits(warps[i])), f"pair {i} after autotune {choice}"
