"""Seeded synthetic fisheye stereo pairs (the reference ships no benchmark data).

A scene is a range field over the reference camera's pixels (a tilted plane
plus eight Gaussian bumps, clipped to [1, 10] m) textured with 4-octave value
noise in [0, 255] that is evaluated analytically at continuous coordinates.
The second view sees every reference point ``X`` at ``R (X + t)``, the
convention of the reference's vector-field generator and triangulation
(Python/vector_field.py:36-54, Python/vfs.cu:728-734): the calibration field
``project(R X) - grid`` undoes R, and the translation field and triangulation
work on ``X + t``.  R defaults to the identity.  For each pixel of the second
image the reference pixel that lands there (after undoing R) is found by
fixed-point iteration on the flow, so the second image needs no resampling.

The mask is the reference driver's circle (Python/main_equidistant.py:52-53)
with margin ``max(10, 2**(nLevel-1))`` pixels.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def equidistant_intrinsics(width: int, height: int):
    """180 degree field of view: f = (W/2)/(pi/2), principal point at the centre."""
    return ((width / 2.0) / (math.pi / 2.0), width / 2.0, height / 2.0)


def _project(X, f, cx, cy):
    R = np.hypot(X[..., 0], X[..., 1])
    th = np.arctan2(R, X[..., 2])
    ph = np.arctan2(X[..., 1], X[..., 0])
    return np.stack([f * th * np.cos(ph) + cx, f * th * np.sin(ph) + cy], -1)


def _unproject(uv, f, cx, cy):
    x = uv[..., 0] - cx
    y = uv[..., 1] - cy
    th = np.hypot(x, y) / f
    ph = np.arctan2(y, x)
    return np.stack([np.cos(ph) * np.sin(th), np.sin(ph) * np.sin(th), np.cos(th)], -1)


class _ValueNoise:
    def __init__(self, rng, width, height, octaves=4):
        self.cells = [width / 16.0 / (2 ** o) for o in range(octaves)]
        self.amps = [0.5 ** o for o in range(octaves)]
        self.pad = 2.0 * max(width, height)
        self.lat = []
        for c in self.cells:
            n = int(math.ceil((max(width, height) + 2 * self.pad) / c)) + 3
            self.lat.append(rng.uniform(0.0, 1.0, (n, n)))

    def __call__(self, x, y):
        acc = np.zeros(np.shape(x))
        for c, a, L in zip(self.cells, self.amps, self.lat):
            gx = (np.asarray(x) + self.pad) / c
            gy = (np.asarray(y) + self.pad) / c
            gx = np.clip(gx, 0, L.shape[1] - 2.000001)
            gy = np.clip(gy, 0, L.shape[0] - 2.000001)
            ix = np.floor(gx).astype(np.int64)
            iy = np.floor(gy).astype(np.int64)
            fx = gx - ix
            fy = gy - iy
            sx = fx * fx * (3 - 2 * fx)
            sy = fy * fy * (3 - 2 * fy)
            v = ((1 - sx) * (1 - sy) * L[iy, ix] + sx * (1 - sy) * L[iy, ix + 1]
                 + (1 - sx) * sy * L[iy + 1, ix] + sx * sy * L[iy + 1, ix + 1])
            acc += a * v
        return 255.0 * acc / sum(self.amps)


class _Range:
    def __init__(self, rng, width, height):
        self.w, self.h = width, height
        self.d0 = rng.uniform(3.0, 6.0)
        self.gx = rng.uniform(-2.0, 2.0)
        self.gy = rng.uniform(-2.0, 2.0)
        self.bumps = []
        for _ in range(8):
            self.bumps.append((rng.uniform(0, width), rng.uniform(0, height),
                               rng.uniform(width / 20.0, width / 8.0),
                               rng.choice([-1.0, 1.0]) * rng.uniform(0.5, 2.0)))

    def __call__(self, x, y):
        d = self.d0 + self.gx * (x - self.w / 2) / self.w + self.gy * (y - self.h / 2) / self.h
        for bx, by, s, a in self.bumps:
            d = d + a * np.exp(-((x - bx) ** 2 + (y - by) ** 2) / (2 * s * s))
        return np.clip(d, 1.0, 10.0)


@dataclass
class StereoPair:
    img_ref: np.ndarray          # (H, W) uint8
    img_other: np.ndarray        # (H, W) uint8
    mask: np.ndarray             # (H, W) uint8, 255 = valid
    intrinsics: tuple            # (f, u0, v0)
    R: np.ndarray                # (3, 3)
    t: np.ndarray                # (3, 1)
    depth: np.ndarray            # (H, W) float32 z-depth of the reference view
    seed: int = 0
    meta: dict = field(default_factory=dict)


def circle_mask(height: int, width: int, margin: int) -> np.ndarray:
    """Filled circle centred at (W//2, H//2) with radius W//2 - margin, as
    ``cv2.circle(mask, (W//2, H//2), W//2 - margin, 255, -1)``."""
    import cv2
    mask = np.zeros((height, width), np.uint8)
    cv2.circle(mask, (width // 2, height // 2), width // 2 - margin, 255, -1)
    return mask


def rotation_xyz(rx: float, ry: float, rz: float) -> np.ndarray:
    """Rotation matrix Rz(rz) @ Ry(ry) @ Rx(rx), angles in radians."""
    cx, sx, cy, sy, cz, sz = np.cos(rx), np.sin(rx), np.cos(ry), np.sin(ry), np.cos(rz), np.sin(rz)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def vector_fields(pair: StereoPair, t_scale=1.0):
    """The pair's translation and calibration fields (tvf, cvf), (H, W, 2)
    float32, from float64 camera math: what get_vector_fields(get_grid_zero,
    cam, cam, R, t, t_scale) computes (Python/vector_field.py:28-56), so that
    solvers fed from different implementations can be given identical
    fields.  tvf = normalize((project(X + s0 t) - project(X - s1 t)) / 2) and
    cvf = project(R X) - grid, X the unit ray of each pixel."""
    s0, s1 = (t_scale, t_scale) if np.isscalar(t_scale) else t_scale
    H, W = pair.img_ref.shape
    f, cx, cy = pair.intrinsics
    t = np.asarray(pair.t, np.float64).reshape(3)
    yy, xx = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    grid = np.stack([xx, yy], -1)
    X = _unproject(grid, f, cx, cy)
    X = X / np.linalg.norm(X, axis=-1, keepdims=True)
    d = (_project(X + s0 * t, f, cx, cy) - _project(X - s1 * t, f, cx, cy)) / 2
    with np.errstate(invalid="ignore", divide="ignore"):
        tvf = d / np.linalg.norm(d, axis=-1, keepdims=True)
    cvf = _project(X @ np.asarray(pair.R, np.float64).T, f, cx, cy) - grid
    return tvf.astype(np.float32), cvf.astype(np.float32)


def uneven_workload(n_pairs: int = 32, seed: int = 0, sides=(480, 640, 800, 1024), t_range=(0.05, 0.2)):
    """(side, t, seed) of each pair of the batched uneven workload: square
    sides drawn uniformly from ``sides``, translation direction uniform on the
    unit sphere with magnitude uniform in ``t_range`` metres, pair i seeded
    with i."""
    rng = np.random.default_rng(seed)
    sz = rng.choice(list(sides), size=n_pairs)
    out = []
    for i in range(n_pairs):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        out.append((int(sz[i]), tuple(d * rng.uniform(*t_range)), i))
    return out


def make_pair(size: int, t, seed: int = 0, n_level: int = 4, height: int | None = None, R=None) -> StereoPair:
    """One seeded pair at ``size`` x ``size`` (or ``height`` x ``size``);
    ``R`` (3x3) rotates the second view, X_other = R (X + t)."""
    W = int(size)
    H = int(height if height is not None else size)
    t = np.asarray(t, np.float64).reshape(3)
    R = np.eye(3) if R is None else np.asarray(R, np.float64).reshape(3, 3)
    rng = np.random.default_rng(seed)
    f, cx, cy = equidistant_intrinsics(W, H)
    noise = _ValueNoise(rng, W, H)
    rng_field = _Range(rng, W, H)

    yy, xx = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    img_ref = noise(xx, yy)

    def flow(px, py):
        ray = _unproject(np.stack([px, py], -1), f, cx, cy)
        X = rng_field(px, py)[..., None] * ray + t
        uv = _project(X, f, cx, cy)
        return uv[..., 0] - px, uv[..., 1] - py

    # target of the fixed point: the second view's pixel with R undone
    if np.array_equal(R, np.eye(3)):
        gx, gy = xx, yy
    else:
        d = _unproject(np.stack([xx, yy], -1), f, cx, cy) @ R  # rows R^T d
        g = _project(d, f, cx, cy)
        gx, gy = g[..., 0], g[..., 1]
    p1x, p1y = gx.copy(), gy.copy()
    for _ in range(30):
        fx, fy = flow(p1x, p1y)
        p1x = 0.5 * p1x + 0.5 * (gx - fx)
        p1y = 0.5 * p1y + 0.5 * (gy - fy)
    img_other = noise(p1x, p1y)

    ray = _unproject(np.stack([xx, yy], -1), f, cx, cy)
    depth = (rng_field(xx, yy) * ray[..., 2]).astype(np.float32)
    margin = max(10, 2 ** (n_level - 1))
    mask = circle_mask(H, W, margin)
    q = lambda a: np.clip(np.round(a), 0, 255).astype(np.uint8)
    return StereoPair(q(img_ref), q(img_other), mask, (f, cx, cy), R, t.reshape(3, 1), depth, seed,
                      {"margin": margin})
