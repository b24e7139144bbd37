"""The allocation-free whole solve (vfs_solve_stereo_static) against the plan path.

vfs_solve_stereo_static exists for callers that cannot call cudaMalloc: it
takes its workspace from a scratch array compiled into the library instead of
from the caller.  Here it is called through the C ABI twice in a row and each
result must be bit-identical to the workspace-based plan path
(vfs_plan_solve through VFS.solve_stereo) on the same inputs; a size whose
workspace exceeds the scratch must be rejected with VFS_ERR_WORKSPACE.

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


def _inputs(gpu):
    from vfs_b200 import EquidistantCam
    from vfs_b200.vector_field import get_vector_fields, get_grid_zero
    h, w = 96, 128
    p = pair(w, height=h, t=(0.12, 0.01, 0.0), seed=9, n_level=3)
    prm = bench_params(h, w, n_level=3, n_warp=3, n_iter=13)
    cam = EquidistantCam(p.intrinsics)
    cam.setup_module()
    tvf, cvf = get_vector_fields(get_grid_zero((h, w)), cam, cam, p.R, p.t, 1)
    return p, prm, tvf, cvf


def _static_solve(prm, p, tvf, cvf):
    from vfs_b200 import _lib
    dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a)).to("cuda", dt).contiguous()
    mask, t_d, c_d = dev(p.mask, torch.uint8), dev(tvf, torch.float32), dev(cvf, torch.float32)
    ref, oth = dev(p.img_ref, torch.uint8), dev(p.img_other, torch.uint8)
    out = torch.full((prm.height, prm.width, 2), float("nan"), dtype=torch.float32, device="cuda")
    cp = _lib.VfsParams.from_param_bag(prm)
    rc = _lib.lib().vfs_solve_stereo_static(ctypes.byref(cp), mask.data_ptr(), prm.width, t_d.data_ptr(),
                                            c_d.data_ptr(), ref.data_ptr(), oth.data_ptr(), out.data_ptr(),
                                            _lib.stream())
    _lib.check(rc, "vfs_solve_stereo_static")
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_static_solve_matches_plan_solve(gpu):
    from vfs_b200 import VFS
    p, prm, tvf, cvf = _inputs(gpu)
    vfs = VFS(prm)
    vfs.setup_module()
    vfs.compute_pyramid_sizes()
    vfs.create_mask_pyramid(p.mask)
    vfs.create_vector_field_pyramid(tvf, cvf)
    want = vfs.solve_stereo(p.img_ref, p.img_other).cpu().numpy()
    assert np.isfinite(want).all()
    for call in range(2):  # two calls in a row share the scratch
        got = _static_solve(prm, p, tvf, cvf)
        same = want.view(np.uint32) == got.view(np.uint32)
        assert same.all(), f"call {call}: {np.count_nonzero(~same)} of {same.size} values differ from the plan path"


def test_static_solve_rejects_sizes_beyond_the_scratch(gpu):
    from vfs_b200 import _lib
    p, prm, tvf, cvf = _inputs(gpu)
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
