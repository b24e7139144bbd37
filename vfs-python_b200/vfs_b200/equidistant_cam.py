"""Drop-in for the reference's ``EquidistantCam`` (Python/equidistant_cam.py:34-206).

Equidistant fisheye model r = f * theta (Python/equidistant_cam.cuh:32-59).
The intrinsics are rounded to float32 as the reference's constant upload
does (Python/equidistant_cam.py:44-46, 67-70) and passed to each kernel by
value.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import call, stream


class EquidistantCam:
    def __init__(self, p):
        self.f = p[0]
        self.u0 = p[1]
        self.v0 = p[2]
        self.gpu_module = None
        self.rays = None
        self.mask = None
        self.sz = None

    def get_intrincs_array(self):
        return np.array([self.f, self.u0, self.v0], dtype=np.float32)

    def _k(self):
        f, u0, v0 = (float(v) for v in self.get_intrincs_array())
        return f, u0, v0

    def compile_module(self):
        self.gpu_module = _lib.lib()

    def setup_module(self):
        if self.gpu_module is None:
            self.compile_module()

    def get_rays(self, sz=None):
        """getRays, Python/equidistant_cam.py:72-92."""
        self.setup_module()
        if sz is None:
            sz = self.sz
        rays = torch.empty((sz[0], sz[1], 3), dtype=torch.float32, device="cuda")
        call("vfs_cam_get_rays", rays.data_ptr(), *self._k(), rays.shape[0], rays.shape[1], stream())
        self.rays = rays
        return rays

    def get_UVs(self, xyz):
        """getUVFromXYZ, Python/equidistant_cam.py:94-114."""
        self.setup_module()
        assert xyz.is_contiguous()
        assert xyz.dtype == torch.float32
        uv = torch.empty((*xyz.shape[:2], 2), dtype=torch.float32, device="cuda")
        call("vfs_cam_get_uvs", uv.data_ptr(), xyz.data_ptr(), *self._k(), uv.shape[0], uv.shape[1], stream())
        return uv

    def get_XYZs(self, uv):
        """getXYZFromUV, Python/equidistant_cam.py:116-136."""
        self.setup_module()
        uv = uv.contiguous()
        assert uv.dtype == torch.float32
        xyz = torch.empty((*uv.shape[:2], 3), dtype=torch.float32, device="cuda")
        call("vfs_cam_get_xyzs", xyz.data_ptr(), uv.data_ptr(), *self._k(), xyz.shape[0], xyz.shape[1], stream())
        return xyz

    def get_thetas(self):
        """getThetas, Python/equidistant_cam.py:138-159."""
        if self.rays is None:
            self.get_rays()
        thetas = torch.empty_like(self.rays)
        call("vfs_cam_get_thetas", thetas.data_ptr(), self.rays.data_ptr(), thetas.shape[0], thetas.shape[1],
             stream())
        return thetas

    def create_default_mask(self, sz=None):
        """Python/equidistant_cam.py:161-170."""
        if sz is None:
            sz = self.sz
        self.mask = torch.full((sz[0], sz[1]), 1, dtype=torch.uint8, device="cuda")

    def set_mask(self, mask):
        """Python/equidistant_cam.py:172-178 (the mask is read directly; no texture is needed)."""
        if isinstance(mask, torch.Tensor):
            self.mask = mask.to(device="cuda", dtype=torch.uint8).contiguous()
        else:
            self.mask = torch.as_tensor(np.ascontiguousarray(mask, dtype=np.uint8)).cuda()

    def get_xyz_from_distance(self, D):
        """getXYZFromDistance, Python/equidistant_cam.py:180-206."""
        self.setup_module()
        if not isinstance(D, torch.Tensor):
            D = torch.as_tensor(np.ascontiguousarray(D, dtype=np.float32))
        D = D.to(device="cuda", dtype=torch.float32).contiguous()
        if self.rays is None:
            self.get_rays(D.shape[:2])
        if self.mask is None:
            self.create_default_mask(D.shape[:2])
        assert tuple(D.shape) == tuple(self.rays.shape[:2])
        xyz = torch.empty_like(self.rays)
        call("vfs_cam_xyz_from_distance", xyz.data_ptr(), self.rays.data_ptr(), D.data_ptr(), self.mask.data_ptr(),
             self.mask.shape[1], xyz.shape[0], xyz.shape[1], stream())
        return xyz
