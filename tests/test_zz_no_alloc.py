"""The allocation-free whole solve (vfs_solve_stereo_static) against the plan path.

vfs_solve_stereo_static is for callers that cannot call cudaMalloc (a
real-time loop with a fixed memory budget, a host callback, a foreign runtime
that hands over device pointers but owns no CUDA allocator): it takes its
workspace from a scratch array compiled into the library instead of from the
caller.  Here it is called through the C ABI and every result must be
bit-identical to the workspace-based plan path (vfs_plan_solve through
VFS.solve_stereo) on the same inputs:

* twice in a row with the same inputs and parameters;
* back to back on one non-blocking stream with no host synchronisation in
  between, while the image size and the iteration count change from call to
  call (each change rebuilds the plan over the shared scratch);

and a size whose workspace exceeds the scratch must be rejected with
VFS_ERR_WORKSPACE.

This file is collected last on purpose, so that a run stopping at its first
failure has run every other test before it.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from helpers import bench_params, pair

pytestmark = pytest.mark.gpu


def _inputs(h=96, w=128, n_iter=13, seed=9):
    from vfs_b200 import EquidistantCam
    from vfs_b200.vector_field import get_vector_fields, get_grid_zero
    p = pair(w, height=h, t=(0.12, 0.01, 0.0), seed=seed, n_level=3)
    prm = bench_params(h, w, n_level=3, n_warp=3, n_iter=n_iter)
    cam = EquidistantCam(p.intrinsics)
    cam.setup_module()
    tvf, cvf = get_vector_fields(get_grid_zero((h, w)), cam, cam, p.R, p.t, 1)
    return p, prm, tvf, cvf


def _plan_solve(p, prm, tvf, cvf):
    from vfs_b200 import VFS
    vfs = VFS(prm)
    vfs.setup_module()
    vfs.compute_pyramid_sizes()
    vfs.create_mask_pyramid(p.mask)
    vfs.create_vector_field_pyramid(tvf, cvf)
    want = vfs.solve_stereo(p.img_ref, p.img_other).cpu().numpy()
    assert np.isfinite(want).all()
    return want


class _StaticCall:
    """Device copies of one problem's inputs and an output buffer; enqueue()
    issues vfs_solve_stereo_static on torch's current stream and returns
    without synchronising."""

    def __init__(self, p, prm, tvf, cvf):
        dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dt).contiguous()
        self.prm = prm
        self.mask, self.tvf, self.cvf = dev(p.mask, torch.uint8), dev(tvf, torch.float32), dev(cvf, torch.float32)
        self.ref, self.oth = dev(p.img_ref, torch.uint8), dev(p.img_other, torch.uint8)
        self.out = torch.full((prm.height, prm.width, 2), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()  # inputs in place before any other stream uses them

    def enqueue(self):
        from vfs_b200 import _lib
        cp = _lib.VfsParams.from_param_bag(self.prm)
        rc = _lib.lib().vfs_solve_stereo_static(ctypes.byref(cp), self.mask.data_ptr(), self.prm.width,
                                                self.tvf.data_ptr(), self.cvf.data_ptr(), self.ref.data_ptr(),
                                                self.oth.data_ptr(), self.out.data_ptr(), _lib.stream())
        _lib.check(rc, "vfs_solve_stereo_static")
        return self.out


def _same_bits(want, got, what):
    same = want.view(np.uint32) == got.view(np.uint32)
    assert same.all(), f"{what}: {np.count_nonzero(~same)} of {same.size} values differ from the plan path"


def test_static_solve_matches_plan_solve(gpu):
    p, prm, tvf, cvf = _inputs()
    want = _plan_solve(p, prm, tvf, cvf)
    call = _StaticCall(p, prm, tvf, cvf)
    for i in range(2):  # two calls in a row share the scratch
        got = call.enqueue().cpu().numpy()
        _same_bits(want, got, f"call {i}")


def test_static_solve_back_to_back_across_parameter_changes(gpu):
    # A at 96x128 with 13 iterations, B at 80x112 with 7, then A again: each
    # call after the first changes the parameters and so rebuilds the plan
    # over the scratch while the previous call's kernels may still run
    probs = {"A": _inputs(96, 128, n_iter=13, seed=9), "B": _inputs(80, 112, n_iter=7, seed=4)}
    want = {k: _plan_solve(*v) for k, v in probs.items()}
    calls = [("A", _StaticCall(*probs["A"])), ("B", _StaticCall(*probs["B"])), ("A", _StaticCall(*probs["A"]))]
    side = torch.cuda.Stream()  # non-blocking: not ordered with the legacy default stream
    with torch.cuda.stream(side):
        outs = [c.enqueue() for _, c in calls]  # no host synchronisation between the calls
    side.synchronize()
    for i, ((k, _), out) in enumerate(zip(calls, outs)):
        _same_bits(want[k], out.cpu().numpy(), f"call {i} ({k})")


def test_static_solve_rejects_sizes_beyond_the_scratch(gpu):
    from vfs_b200 import _lib
    big = bench_params(2048, 2048, n_level=5, n_warp=1, n_iter=1)
    need = ctypes.c_size_t(0)
    cp = _lib.VfsParams.from_param_bag(big)
    _lib.call("vfs_plan_workspace_size", ctypes.byref(cp), ctypes.byref(need))
    assert need.value > _lib.lib().vfs_static_scratch_bytes()
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    rc = _lib.lib().vfs_solve_stereo_static(ctypes.byref(cp), dummy.data_ptr(), 2048, dummy.data_ptr(),
                                            dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                            dummy.data_ptr(), _lib.stream())
    assert rc == _lib.VFS_ERR_WORKSPACE
    assert "static scratch" in _lib.lib().vfs_last_error().decode()
