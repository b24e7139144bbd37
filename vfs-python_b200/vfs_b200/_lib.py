"""ctypes binding of libvfs_b200.so (C ABI in include/vfs_b200.h).

The library is built in place by ``vfs-python_b200/build.py``.  There is no
fallback: if the library is missing or CUDA is unavailable every entry point
raises.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvfs_b200.so")

VFS_OK = 0
VFS_ERR_ARG = 1
VFS_ERR_ALIGN = 2
VFS_ERR_WORKSPACE = 3
VFS_ERR_CUDA = 4
VFS_ERR_STATE = 5

TEX_U8, TEX_F32, TEX_F32X2 = 0, 2, 3


class VfsParams(ctypes.Structure):
    """Mirror of ``VfsParams`` in include/vfs_b200.h."""
    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int),
        ("beta", ctypes.c_double), ("gamma", ctypes.c_double), ("alpha0", ctypes.c_double),
        ("alpha1", ctypes.c_double), ("timeStepLambda", ctypes.c_double), ("Lambda", ctypes.c_double),
        ("fScale", ctypes.c_double), ("limitRange", ctypes.c_double),
        ("nLevel", ctypes.c_int), ("nWarpIters", ctypes.c_int), ("nSolverIters", ctypes.c_int),
    ]

    @classmethod
    def from_param_bag(cls, p) -> "VfsParams":
        return cls(int(p.width), int(p.height), float(p.beta), float(p.gamma), float(p.alpha0), float(p.alpha1),
                   float(p.timeStepLambda), float(p.Lambda), float(p.fScale), float(p.limitRange), int(p.nLevel),
                   int(p.nWarpIters), int(p.nSolverIters))


class VfsSolveStats(ctypes.Structure):
    """Mirror of ``VfsSolveStats`` in include/vfs_b200.h."""
    _fields_ = [("kernels_per_solve", ctypes.c_longlong), ("tgv_ms", ctypes.c_double),
                ("tgv_alg_bytes", ctypes.c_double), ("tgv_launches", ctypes.c_longlong),
                ("tgv_intervals", ctypes.c_int), ("tgv_ms_level", ctypes.c_double * 16),
                ("recompute_ms", ctypes.c_double)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_D = ctypes.c_double
_SZ = ctypes.c_size_t
_U64 = ctypes.c_uint64
_PRM = ctypes.POINTER(VfsParams)

# name -> argtypes
_SIGS = {
    "vfs_version": [],
    "vfs_last_error": [],
    "vfs_texture_create": [_P, _I, _I, _SZ, _I, _I, ctypes.POINTER(_U64)],
    "vfs_texture_destroy": [_U64],
    "vfs_cast_and_scale": [_P, _P, _I, _I, _P],
    "vfs_downsample_image": [_P, _U64, _I, _I, _P],
    "vfs_downsample_vector_field": [_P, _U64, _I, _I, _P],
    "vfs_downsample_mask": [_P, _U64, _I, _I, _P],
    "vfs_warping_image": [_P, _P, _U64, _I, _I, _P],
    "vfs_gaussian": [_P, _U64, _P, _SZ, _I, _I, _P],
    "vfs_compute_tensor_eta": [_P, _P, _U64, _P, _SZ, _PRM, _I, _I, _P],
    "vfs_find_warping_vector": [_P, _P, _U64, _I, _I, _P],
    "vfs_compute_derivatives": [_P, _U64, _U64, _U64, _I, _I, _P],
    "vfs_update_dual_variables": [_P, _P, _P, _F, _P, _P, _P, _P, _SZ, _PRM, _I, _I, _P],
    "vfs_l1_thresholding": [_P, _F, _P, _P, _P, _P, _P, _P, _SZ, _PRM, _I, _I, _P],
    "vfs_update_primal_variables": [_P, _P, _F, _F, _P, _P, _P, _P, _P, _P, _P, _P, _SZ, _PRM, _I, _I, _P],
    "vfs_median_filter": [_P, _P, _P, _SZ, _I, _I, _P],
    "vfs_compute_optical_flow_with_clamp": [_P, _P, _P, _P, _P, _SZ, _PRM, _I, _I, _P],
    "vfs_upsampling_vector_field1": [_P, _U64, _PRM, _I, _I, _P],
    "vfs_upsampling_vector_field": [_P, _U64, _PRM, _I, _I, _P],
    "vfs_triangulate_rays": [_P, _P, _P, _P, _P, _SZ, _I, _I, _P],
    "vfs_triangulate_rays_lsq": [_P, _P, _P, _P, _P, _SZ, _I, _I, _P],
    "vfs_cam_get_rays": [_P, _F, _F, _F, _I, _I, _P],
    "vfs_cam_get_uvs": [_P, _P, _F, _F, _F, _I, _I, _P],
    "vfs_cam_get_xyzs": [_P, _P, _F, _F, _F, _I, _I, _P],
    "vfs_cam_get_thetas": [_P, _P, _I, _I, _P],
    "vfs_cam_xyz_from_distance": [_P, _P, _P, _P, _SZ, _I, _I, _P],
    "vfs_vector_fields": [_P, _P, _F, _F, _F, _F, _F, _F, _P, _P, _P, _F, _I, _I, _P],
    "vfs_plan_workspace_size": [_PRM, ctypes.POINTER(_SZ)],
    "vfs_plan_create": [_PRM, _P, _SZ, ctypes.POINTER(_P)],
    "vfs_plan_destroy": [_P],
    "vfs_plan_sizes": [_P, _P],
    "vfs_plan_set_mask": [_P, _P, _SZ, _P],
    "vfs_plan_set_vector_fields": [_P, _P, _P, _P],
    "vfs_plan_solve": [_P, _P, _P, _P, _P],
    "vfs_plan_triangulate": [_P, _F, _F, _F, _P, _P, _P],
    "vfs_plan_triangulate_lsq": [_P, _F, _F, _F, _P, _P, _P],
    "vfs_plan_set_tgv_variant": [_P, _I],
    "vfs_plan_set_graph": [_P, _I],
    "vfs_tgv_variants": [_P, _I, _P],
    "vfs_static_scratch_bytes": [],
    "vfs_batch_workspace_size": [_PRM, _I, _P, _P, ctypes.POINTER(_SZ)],
    "vfs_batch_create": [_PRM, _I, _P, _P, _P, _SZ, ctypes.POINTER(_P)],
    "vfs_batch_destroy": [_P],
    "vfs_batch_set_pair": [_P, _I, _P, _SZ, _P, _P, _P],
    "vfs_batch_solve": [_P, _P, _P, _P, _P],
    "vfs_batch_triangulate": [_P, _I, _F, _F, _F, _P, _P, _P],
    "vfs_batch_triangulate_lsq": [_P, _I, _F, _F, _F, _P, _P, _P],
    "vfs_batch_set_level_variant": [_P, _I, _I],
    "vfs_batch_set_graph": [_P, _I],
    "vfs_batch_set_group_bytes": [_P, _SZ],
    "vfs_batch_set_timing": [_P, _I],
    "vfs_batch_stats": [_P, ctypes.POINTER(VfsSolveStats)],
    "vfs_solve_stereo_static": [_PRM, _P, _SZ, _P, _P, _P, _P, _P, _P],
    "vfs_plan_set_timing": [_P, _I],
    "vfs_plan_set_cluster": [_P, _I],
    "vfs_plan_set_level_variant": [_P, _I, _I],
    "vfs_plan_level_cluster": [_P, _I],
    "vfs_plan_stats": [_P, ctypes.POINTER(VfsSolveStats)],
    "vfs_step_schedule": [_I, _D, _P],
    "vfs_grad_workspace_size": [_PRM, _I, ctypes.POINTER(_SZ)],
    "vfs_grad_create": [_PRM, _I, _F, _F, _F, _D, _P, _SZ, ctypes.POINTER(_P)],
    "vfs_grad_destroy": [_P],
    "vfs_grad_plan": [_P],
    "vfs_grad_forward": [_P, _P, _P, _P, _P, _P, _P],
    "vfs_grad_backward": [_P, _P, _P, _P, _P, _P],
    "vfs_grad_set_options": [_P, _I, _I],
    "vfs_grad_set_level_form": [_P, _I, _I],
    "vfs_grad_set_triangulation": [_P, _I],
    "vfs_grad_set_timing": [_P, _I],
    "vfs_grad_stats": [_P, ctypes.POINTER(VfsSolveStats)],
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python vfs-python_b200/build.py` "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = (ctypes.c_char_p if name == "vfs_last_error" else
                          ctypes.c_size_t if name == "vfs_static_scratch_bytes" else
                          ctypes.c_void_p if name == "vfs_grad_plan" else ctypes.c_int)
        _lib = L
    return _lib


class VfsError(RuntimeError):
    pass


def check(rc: int, what: str) -> None:
    if rc == VFS_OK:
        return
    msg = lib().vfs_last_error().decode(errors="replace")
    if rc == VFS_ERR_ARG:
        raise ValueError(f"{what}: {msg}")
    if rc == VFS_ERR_STATE:
        raise AssertionError(f"{what}: {msg}")
    raise VfsError(f"{what} failed ({rc}): {msg}")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def stream() -> int:
    """Handle of torch's current CUDA stream (every call is ordered on it)."""
    return torch.cuda.current_stream().cuda_stream


def require_cuda(t: torch.Tensor, what: str) -> None:
    if not t.is_cuda:
        raise ValueError(f"{what} must be a CUDA tensor")
    if not t.is_contiguous():
        raise AssertionError(f"{what} must be C-contiguous")
