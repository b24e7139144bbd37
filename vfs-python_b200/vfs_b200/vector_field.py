"""Drop-in for the reference's vector-field generator (Python/vector_field.py:28-65).

``get_vector_fields`` returns (tvf, cvf) as NumPy arrays, as the reference
does.  For the standard grids (``get_grid_zero``/``get_grid_one``) and the
unit-length normaliser the whole chain runs as one kernel; any other grid or
normaliser takes the reference's step-by-step chain on torch tensors.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import call, stream


def default_normalizer(x: torch.Tensor) -> torch.Tensor:
    """The normaliser of Python/main_equidistant.py:60 on torch tensors."""
    return x / torch.linalg.norm(x, dim=2)[:, :, None]


def get_grid_zero(sz) -> torch.Tensor:
    """Python/vector_field.py:58-62: (H, W, 2) float32 pixel coordinates."""
    uv = np.empty((*sz, 2), dtype=np.int32)
    uv[:, :, 0] = np.arange(0, sz[1])[np.newaxis, :]
    uv[:, :, 1] = np.arange(0, sz[0])[:, np.newaxis]
    g = torch.as_tensor(uv.astype(np.float32)).cuda()
    g._vfs_grid_offset = 0.0
    return g


def get_grid_one(sz) -> torch.Tensor:
    """Python/vector_field.py:64-65."""
    g = get_grid_zero(sz) + 1
    g._vfs_grid_offset = 1.0
    return g


def get_vector_fields(grid, camera_ref, camera_other, R, t, t_scale, normalizer=None):
    if isinstance(t_scale, (float, int)):
        t_scale = (t_scale, t_scale)
    t = np.asarray(t, dtype=np.float64).reshape(3)
    R = np.asarray(R, dtype=np.float64).reshape(3, 3)
    off = getattr(grid, "_vfs_grid_offset", None)
    if off is not None and (normalizer is None or normalizer is default_normalizer):
        camera_ref.setup_module()
        h, w = grid.shape[:2]
        tvf = torch.empty((h, w, 2), dtype=torch.float32, device="cuda")
        cvf = torch.empty((h, w, 2), dtype=torch.float32, device="cuda")
        Rd = (ctypes.c_double * 9)(*R.reshape(-1).tolist())
        td = (ctypes.c_double * 3)(*t.tolist())
        sd = (ctypes.c_double * 2)(float(t_scale[0]), float(t_scale[1]))
        call("vfs_vector_fields", tvf.data_ptr(), cvf.data_ptr(), *camera_ref._k(), *camera_other._k(), Rd, td, sd,
             float(off), h, w, stream())
        return tvf.cpu().numpy(), cvf.cpu().numpy()
    # the reference's chain, Python/vector_field.py:31-56
    normalizer = normalizer or default_normalizer
    grid = grid.to(device="cuda", dtype=torch.float32).contiguous()
    XYZ = camera_ref.get_XYZs(grid)
    XYZ = normalizer(XYZ).contiguous()
    st = torch.tensor((t_scale[0] * t)[np.newaxis, np.newaxis, :], dtype=torch.float32, device="cuda")
    tvf_forward = camera_ref.get_UVs((XYZ + st).contiguous())
    st = torch.tensor((t_scale[1] * t)[np.newaxis, np.newaxis, :], dtype=torch.float32, device="cuda")
    tvf_backward = camera_ref.get_UVs((XYZ - st).contiguous())
    tvf = (tvf_forward - tvf_backward) / 2
    tvf /= torch.linalg.norm(tvf, dim=2)[:, :, None]
    Rt = torch.tensor(R.T, dtype=torch.float32, device="cuda")
    RXYZ = (XYZ.reshape(-1, 3) @ Rt).reshape(XYZ.shape).contiguous()
    cvf = camera_other.get_UVs(RXYZ) - grid
    return tvf.cpu().numpy(), cvf.cpu().numpy()
