"""GPU parity at the benchmark configurations, against the reference's own kernels.

The reference side runs the reference's CUDA kernels (built from its sources
into oracle/_ref) under the reference's host loop (oracle/refgpu/refpath.py,
Python/vfs.py:460-559); the B200 side runs the drop-in VFS (fused plan, CUDA
graph replay) or the batched solver.  Both get the same images, mask,
fields (vfs_b200.synthetic.vector_fields) and parameters.  The comparison is
bit-exact on the flow (warpUV) and on xyz; the tolerance the method is quoted
at, median relative depth error <= 1e-4 over mask != 0 with finite reference
depth in (0, 100] m, is checked as well.

* 512x512, 4 levels x 10 warps x 50 iterations, t = (0.1, 0, 0) m;
* 800x800, 5 levels x 10 warps x 100 iterations, t = (0.12, 0.01, 0) m, with
  the per-level kernels [221, 134, 222, 213, 207] and with the autotuner's
  choice;
* four pairs of the batched uneven workload (sides from {480, 640, 800, 1024},
  random translation directions), 4 levels x 10 warps x 50 iterations, solved
  as one batch.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import bench_params

pytestmark = pytest.mark.gpu

DEPTH_TOL = 1e-4  # median relative depth error against the reference


def _reference(prm, p, tvf, cvf):
    from oracle.refgpu import refpath
    r = refpath.RefVFS(prm, "bench")
    r.compute_pyramid_sizes()
    r.create_mask_pyramid(p.mask)
    r.create_vector_field_pyramid(tvf, cvf)
    cam = refpath.RefEquidistantCam(p.intrinsics, "bench")
    cam.setup_module()
    flow = r.solve_stereo(p.img_ref, p.img_other).cpu().numpy()
    xyz = r.triangulate_flow(cam, p.t).cpu().numpy()
    return flow, xyz


def _check(p, want, got, what):
    (rf, rx), (of, ox) = want, got
    assert rf.shape == of.shape and rx.shape == ox.shape
    df = np.count_nonzero(np.ascontiguousarray(rf).view(np.uint32) != np.ascontiguousarray(of).view(np.uint32))
    dx = np.count_nonzero(np.ascontiguousarray(rx).view(np.uint32) != np.ascontiguousarray(ox).view(np.uint32))
    zr, zo = rx[..., 2].astype(np.float64), ox[..., 2].astype(np.float64)
    assert df == 0, f"{what}: {df} of {rf.size} flow values differ from the reference kernels"
    assert dx == 0, f"{what}: {dx} of {rx.size} xyz values differ from the reference kernels"
    # at Lambda 50 the method drifts from the true depth, so only part of the
    # mask has a plausible reference depth (29-41 % at 800^2 and 512^2)
    sel = (p.mask != 0) & np.isfinite(zr) & (zr > 0) & (zr <= 100)
    if sel.any():
        err = np.median(np.abs(zo[sel] - zr[sel]) / zr[sel])
        assert err <= DEPTH_TOL, f"{what}: median relative depth error {err}"


def _drop_in(prm, p, tvf, cvf):
    from vfs_b200 import VFS, EquidistantCam
    o = VFS(prm)
    o.setup_module()
    o.compute_pyramid_sizes()
    o.create_mask_pyramid(p.mask)
    o.create_vector_field_pyramid(tvf, cvf)
    cam = EquidistantCam(p.intrinsics)
    cam.setup_module()
    return o, cam


def _solve(o, cam, p):
    flow = o.solve_stereo(p.img_ref, p.img_other).cpu().numpy()
    xyz = o.triangulate_flow(cam, p.t).cpu().numpy()
    return flow, xyz


def test_parity_512_4x10x50(gpu):
    from vfs_b200.synthetic import make_pair, vector_fields
    p = make_pair(512, (0.1, 0.0, 0.0), seed=0, n_level=4)
    assert np.isclose(p.intrinsics[0], 256 / (np.pi / 2))
    prm = bench_params(512, 512, n_level=4, n_warp=10, n_iter=50)
    tvf, cvf = vector_fields(p)
    want = _reference(prm, p, tvf, cvf)
    o, cam = _drop_in(prm, p, tvf, cvf)
    o.configure(use_graph=True)
    _check(p, want, _solve(o, cam, p), "default kernels, graph")
    choice = o.autotune(torch.as_tensor(p.img_ref).cuda(), torch.as_tensor(p.img_other).cuda(), repeats=1)
    _check(p, want, _solve(o, cam, p), f"autotuned {choice}, graph")
    _check(p, want, _solve(o, cam, p), f"autotuned {choice}, graph replayed")


def test_parity_800_5x10x100(gpu):
    from vfs_b200.synthetic import make_pair, vector_fields
    p = make_pair(800, (0.12, 0.01, 0.0), seed=0, n_level=5)
    assert np.isclose(p.intrinsics[0], 400 / (np.pi / 2))
    prm = bench_params(800, 800, n_level=5, n_warp=10, n_iter=100)
    tvf, cvf = vector_fields(p)
    want = _reference(prm, p, tvf, cvf)
    o, cam = _drop_in(prm, p, tvf, cvf)
    o.configure(use_graph=True)
    o.set_level_variants([221, 134, 222, 213, 207])
    _check(p, want, _solve(o, cam, p), "variants [221, 134, 222, 213, 207], graph")
    _check(p, want, _solve(o, cam, p), "variants [221, 134, 222, 213, 207], graph replayed")
    choice = o.autotune(torch.as_tensor(p.img_ref).cuda(), torch.as_tensor(p.img_other).cuda(), repeats=1)
    _check(p, want, _solve(o, cam, p), f"autotuned {choice}, graph")


def test_parity_uneven_batch_subset(gpu):
    from vfs_b200.batch import VFSBatch
    from vfs_b200 import EquidistantCam
    from vfs_b200.synthetic import make_pair, uneven_workload, vector_fields
    work = uneven_workload()[:4]
    pairs = [make_pair(s, t, seed=seed, n_level=4) for s, t, seed in work]
    fields = [vector_fields(p) for p in pairs]
    prm = bench_params(1024, 1024, n_level=4, n_warp=10, n_iter=50)
    batch = VFSBatch(prm, [p.img_ref.shape for p in pairs])
    for i, (p, (tvf, cvf)) in enumerate(zip(pairs, fields)):
        batch.set_pair(i, p.mask, tvf, cvf)
    batch.configure(use_graph=True)
    flows = [f.cpu().numpy() for f in batch.solve([p.img_ref for p in pairs], [p.img_other for p in pairs])]
    for i, (p, (tvf, cvf)) in enumerate(zip(pairs, fields)):
        cam = EquidistantCam(p.intrinsics)
        cam.setup_module()
        xyz = batch.triangulate(i, cam, p.t).cpu().numpy()
        side = p.img_ref.shape[0]
        want = _reference(bench_params(side, side, n_level=4, n_warp=10, n_iter=50), p, tvf, cvf)
        _check(p, want, (flows[i], xyz), f"batched pair {i} ({side}x{side}, t {np.round(work[i][1], 3)})")
