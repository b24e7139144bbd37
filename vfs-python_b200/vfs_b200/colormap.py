"""Depth colour maps, as the reference's ``depth_to_colormap``
(Python/colormap.py:286-292): inverse depth between near and far mapped onto
a 256-entry jet table, BGR u8, black where depth <= 0.

The table is MATLAB's ``jet(256)`` generated from its published construction
(piecewise-linear ramps of width n = 64) and rounded to 4 decimals, which is
the reference's printed table; it is stored BGR as the reference flips it.
The reference's ``astype(np.int)`` fails under NumPy >= 1.24; plain ``int``
is used here.  Visual output only: host NumPy, no GPU work.
"""
from __future__ import annotations

import math

import numpy as np


def jet(m: int = 256) -> np.ndarray:
    """(m, 3) RGB jet colour map in [0, 1]."""
    n = math.ceil(m / 4)
    u = np.concatenate([np.arange(1, n + 1) / n, np.ones(n - 1), np.arange(n, 0, -1) / n])
    g = math.ceil(n / 2) - (1 if m % 4 == 1 else 0) + np.arange(1, u.size + 1)  # 1-based rows
    r, b = g + n, g - n
    J = np.zeros((m, 3))
    for ch, idx in ((0, r), (1, g), (2, b)):
        ok = (idx >= 1) & (idx <= m)
        J[idx[ok] - 1, ch] = u[ok]
    return J


colormap_rgb = np.round(jet(256), 4)
colormap = np.fliplr(colormap_rgb)  # BGR, as the reference stores it


def depth_to_colormap(depth, min_z, max_z):
    """(H, W) depth (NumPy or torch) -> (H, W, 3) u8 BGR image."""
    if hasattr(depth, "detach"):
        depth = depth.detach().cpu().numpy()
    depth = np.asarray(depth)
    mask = depth > 0
    delta = 1 / min_z - 1 / max_z
    with np.errstate(divide="ignore", invalid="ignore"):
        x = np.maximum(0, np.minimum(1 / (depth + 1e-6) - 1 / max_z, delta) / delta)
    index = np.round(np.nan_to_num(x, nan=0.0) * 255).astype(int)
    img = (colormap[index] * 255).astype(np.uint8)
    img[~mask] = (0, 0, 0)
    return img
