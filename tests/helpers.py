"""Shared test inputs: parameter bags and synthetic pairs."""
from __future__ import annotations

import os
import subprocess

import numpy as np

from vfs_b200.synthetic import make_pair
from vfs_b200.vfs_params import vfs_params


def bench_params(h, w, n_level=4, n_warp=10, n_iter=50):
    """The stereo workloads' solver settings (scale 0.5, lambda 50)."""
    p = vfs_params()
    p.width, p.height = w, h
    p.nLevel, p.fScale = n_level, 2.0
    p.nWarpIters, p.nSolverIters = n_warp, n_iter
    p.Lambda, p.alpha0, p.alpha1, p.beta, p.gamma = 50.0, 17.0, 1.2, 9.0, 0.85
    return p


def default_params(h, w, n_level=6, n_warp=3, n_iter=20):
    """The reference's vfs_params defaults (fScale 1.2, Lambda 5), fewer loops."""
    p = vfs_params()
    p.width, p.height = w, h
    p.nLevel, p.nWarpIters, p.nSolverIters = n_level, n_warp, n_iter
    return p


def pair(size, t=(0.1, 0.0, 0.0), seed=0, n_level=4, height=None):
    return make_pair(size, t, seed=seed, n_level=n_level, height=height)


def bits(a) -> np.ndarray:
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def reference_dir() -> str:
    """The reference checkout's Python directory (VFS_REFERENCE, else the
    default oracle/refgpu/Makefile holds); "" when make cannot say."""
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "refgpu")
    try:
        r = subprocess.run(["make", "-s", "-C", here, "print-ref"], capture_output=True, text=True, timeout=30)
    except (OSError, subprocess.SubprocessError):
        return ""
    return r.stdout.strip() if r.returncode == 0 else ""
