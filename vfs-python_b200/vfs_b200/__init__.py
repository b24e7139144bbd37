"""B200-native variational fisheye stereo (drop-in for eshibusawa/VFS-Python).

    from vfs_b200 import VFS, vfs_params, EquidistantCam, get_vector_fields

The modules mirror the reference's (``vfs``, ``vfs_params``,
``equidistant_cam``, ``vector_field``, ``texture``); the compute runs in
``libvfs_b200.so`` (C ABI: include/vfs_b200.h).
"""
from .vfs_params import vfs_params
from .vfs import VFS
from .equidistant_cam import EquidistantCam
from .vector_field import get_vector_fields, get_grid_zero, get_grid_one, default_normalizer
from .texture import create_texture_object
from .grad import DepthSolver

__all__ = ["VFS", "vfs_params", "EquidistantCam", "get_vector_fields", "get_grid_zero", "get_grid_one",
           "default_normalizer", "create_texture_object", "DepthSolver"]
