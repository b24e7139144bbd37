"""Test infrastructure: a float64 NumPy restatement of the reference solver.

This is the FP64 oracle for the B200 stereo path and the timed CPU baseline.
It restates, array-at-a-time, every kernel of the reference's ``Python/vfs.cu``
and ``Python/template_cam.cu`` / ``Python/equidistant_cam.cuh`` and the host
orchestration of ``Python/vfs.py`` / ``Python/vector_field.py``; each function
cites the lines it follows.  The product never imports it.

Texture sampling.  The reference samples nearly every input through CUDA
texture objects (normalised coordinates, mirror addressing, linear filtering;
``Python/vfs.py:96-98``).  Two models are offered:

``mode="exact"``
    coordinates in float64, exact bilinear weights;
``mode="tex8"``
    coordinates computed in float32 exactly as the kernel computes them,
    1-D weights rounded half-up to 8 fractional bits and the corner product
    ``a*b`` rounded the same way (the other three corner weights keep the
    marginals).  Measured on a B200: the 1-D model reproduces the hardware to
    <= 1 ulp on every sample (98.4 % bit-exact); the 2-D corner-weight rule
    matches 98 % of random samples exactly, the rest within about 1/256 of a
    local intensity step.  The texture unit's own 2-D arithmetic is not fully
    known, so FP64-vs-reference comparisons carry a tolerance.

Point-sampled masks use the texel rule measured on a B200: the normalised
coordinate is truncated to 21 fractional bits before it is scaled by the
texture width (``_point_index``); this reproduces the reference's mask pyramid
(``downSamplingMask``) exactly at every size probed.

Out-of-buffer reads.  The reference's dual/threshold/primal kernels read flat
neighbours ``index +- 1`` / ``index +- width``; past either end of the buffer
they read whatever memory is there.  Here (and in the product, and in the
guarded reference harness) those reads return 0.
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32
F64 = np.float64


# ---------------------------------------------------------------- sampling
def _q8(v):
    return np.floor(v * 256.0 + 0.5) / 256.0


def _mirror_index(i, n):
    i = np.mod(i, 2 * n)
    return np.where(i >= n, 2 * n - 1 - i, i)


def tex_linear(T, x, y, mode="exact"):
    """Linear-filtered, mirror-addressed, normalised-coordinate fetch.

    Follows the texture semantics the reference sets up in
    ``Python/vfs.py:96-98`` (``create_texture_object`` in
    ``Python/texture.py:27-55``).  ``T`` is (H, W) or (H, W, C).
    """
    H, W = T.shape[:2]
    x = np.asarray(x, F64)
    y = np.asarray(y, F64)
    u = x * W - 0.5
    v = y * H - 0.5
    i0 = np.floor(u)
    j0 = np.floor(v)
    a = u - i0
    b = v - j0
    i0 = i0.astype(np.int64)
    j0 = j0.astype(np.int64)
    if mode == "tex8":
        a = _q8(a)
        b = _q8(b)
        w11 = _q8(a * b)
        w01 = a - w11
        w10 = b - w11
        w00 = 1.0 - a - b + w11
    else:
        w00 = (1 - a) * (1 - b)
        w01 = a * (1 - b)
        w10 = (1 - a) * b
        w11 = a * b
    I0, I1 = _mirror_index(i0, W), _mirror_index(i0 + 1, W)
    J0, J1 = _mirror_index(j0, H), _mirror_index(j0 + 1, H)
    Td = np.asarray(T, F64)
    if Td.ndim == 3:
        w00, w01, w10, w11 = (w[..., None] for w in (w00, w01, w10, w11))
    return w00 * Td[J0, I0] + w01 * Td[J0, I1] + w10 * Td[J1, I0] + w11 * Td[J1, I1]


def _point_index(xn, n):
    """Texel picked by point sampling at normalised float32 coordinate ``xn``."""
    xt = np.floor(np.asarray(xn, F64) * 2.0 ** 21) / 2.0 ** 21
    return _mirror_index(np.floor(xt * n).astype(np.int64), n)


def mask_neighbours(M):
    """Mask at a pixel and at its E/W/S/N neighbours, as the kernels read it.

    ``NearestNeighbor<uchar>::get`` (``Python/vfs.cu:54-59``) at integer
    ``X+-1``/``Y+-1`` with mirror addressing returns the edge texel for
    ``X=-1`` and ``X=W`` (``Python/vfs.cu:359, 371, 448-467, 537-553``).
    """
    H, W = M.shape
    Mb = np.asarray(M) != 0
    xs = np.arange(W)
    ys = np.arange(H)
    mE = Mb[:, np.minimum(xs + 1, W - 1)]
    mW = Mb[:, np.maximum(xs - 1, 0)]
    mS = Mb[np.minimum(ys + 1, H - 1), :]
    mN = Mb[np.maximum(ys - 1, 0), :]
    return Mb, mE, mW, mS, mN


def flat_get(a, off):
    """``a.flat[i + off]`` per pixel (per channel), 0 outside the buffer."""
    H, W = a.shape[:2]
    n = H * W
    af = a.reshape(n, -1)
    out = np.zeros_like(af)
    idx = np.arange(n) + off
    ok = (idx >= 0) & (idx < n)
    out[ok] = af[idx[ok]]
    return out.reshape(a.shape)


def _grid(H, W, dtype):
    Y, X = np.meshgrid(np.arange(H, dtype=dtype), np.arange(W, dtype=dtype), indexing="ij")
    return X, Y


def _ft(mode):
    return F32 if mode == "tex8" else F64


# ---------------------------------------------------------------- vfs.cu kernels
def cast_and_scale(img_u8):
    """``castAndScale``, Python/vfs.cu:145-156: u8 / 256."""
    return np.asarray(img_u8, F64) / 256.0


def down_sampling(T, Hc, Wc, mode="exact"):
    """``downSamplingImage`` / ``downSamplingVectorField`` via ``Bilinear``,
    Python/vfs.cu:35-49, 171-184."""
    ft = _ft(mode)
    X, Y = _grid(Hc, Wc, ft)
    dx = ft(1.0) / ft(Wc)
    dy = ft(1.0) / ft(Hc)
    x = (X + ft(0.5)) * dx
    y = (Y + ft(0.5)) * dy
    dx = dx * ft(0.25)
    dy = dy * ft(0.25)
    s = (tex_linear(T, x - dx, y, mode) + tex_linear(T, x + dx, y, mode)
         + tex_linear(T, x, y - dy, mode) + tex_linear(T, x, y + dy, mode))
    return 0.25 * s


def down_sampling_mask(M, Hc, Wc):
    """``downSamplingMask``: point sample at ``(X+0.5)/Wc``, Python/vfs.cu:54-59, 176-179."""
    Hf, Wf = M.shape
    xs = (np.arange(Wc, dtype=F32) + F32(0.5)) / F32(Wc)
    ys = (np.arange(Hc, dtype=F32) + F32(0.5)) / F32(Hc)
    ix = _point_index(xs, Wf)
    iy = _point_index(ys, Hf)
    return np.asarray(M)[iy[:, None], ix[None, :]].astype(np.uint8)


def warping_image(T, warp, mode="exact"):
    """``warpingImage``, Python/vfs.cu:61-66, 186-202: I((X+wx+0.5)/W, (Y+wy+0.5)/H)."""
    H, W = warp.shape[:2]
    ft = _ft(mode)
    X, Y = _grid(H, W, ft)
    w = np.asarray(warp, ft)
    x = (X + w[..., 0] + ft(0.5)) / ft(W)
    y = (Y + w[..., 1] + ft(0.5)) / ft(H)
    return tex_linear(T, x, y, mode)


find_warping_vector = warping_image
"""``findWarpingVector``, Python/vfs.cu:283-302 (same sampling on the vector field)."""


def gaussian_masked(T, M, mode="exact"):
    """``gaussianMasked``, Python/vfs.cu:81-102, 204-226 (3x3 binomial, masked -> 0)."""
    H, W = T.shape
    ft = _ft(mode)
    X, Y = _grid(H, W, ft)
    dx = ft(1.0) / ft(W)
    dy = ft(1.0) / ft(H)
    x = (X + ft(0.5)) * dx
    y = (Y + ft(0.5)) * dy
    t = lambda a, b: tex_linear(T, a, b, mode)
    v0 = t(x, y)
    v1 = t(x - dx, y - dy) + t(x - dx, y + dy) + t(x + dx, y - dy) + t(x + dx, y + dy)
    v2 = t(x - dx, y) + t(x + dx, y) + t(x, y - dy) + t(x, y + dy)
    out = 0.25 * v0 + 0.0625 * v1 + 0.125 * v2
    return np.where(np.asarray(M) != 0, out, 0.0)


def compute_tensor_eta(T, M, p, mode="exact"):
    """``computeTensorEtaMasked`` + ``computeEta``, Python/vfs.cu:106-118, 228-281.

    Returns (abc, eta), each (H, W, 3).
    """
    H, W = T.shape
    ft = _ft(mode)
    X, Y = _grid(H, W, ft)
    dx = ft(1.0) / ft(W)
    dy = ft(1.0) / ft(H)
    x = (X + ft(0.5)) * dx
    y = (Y + ft(0.5)) * dy
    t = lambda a, b: tex_linear(T, a, b, mode)
    g0 = t(x + dx, y + dy) - t(x, y + dy)
    g1 = t(x + dx, y + dy) - t(x + dx, y)
    ng = np.hypot(g0, g1)
    with np.errstate(divide="ignore", invalid="ignore"):
        n0 = g0 / ng
        n1 = g1 / ng
    small = ng < 1e-8
    n0 = np.where(small, 1.0, n0)
    n1 = np.where(small, 0.0, n1)
    t0, t1 = n1, -n0
    wgt = np.maximum(np.exp(-p.beta * ng ** p.gamma), 1e-8)
    a = wgt * n0 * n0 + t0 * t0
    b = wgt * n1 * n1 + t1 * t1
    c = wgt * n0 * n1 + t0 * t1
    a11 = p.alpha1 * p.alpha1
    a004 = 4 * p.alpha0 * p.alpha0
    e0 = a11 * (a * a + b * b + 2 * c * c) + a11 * ((a + c) ** 2 + (b + c) ** 2)
    e1 = a11 * (b * b + c * c) + a004
    e2 = a11 * (a * a + c * c) + a004
    m = (np.asarray(M) != 0)[..., None]
    abc = np.where(m, np.stack([a, b, c], -1), 0.0)
    eta = np.where(m, np.stack([e0, e1, e2], -1), 0.0)
    return abc, eta


def compute_derivatives(ref, other, tvf, mode="exact"):
    """``computeDerivatives``, Python/vfs.cu:120-142, 304-324 -> (H, W, 2) = (Iu, Iz)."""
    H, W = ref.shape
    ft = _ft(mode)
    X, Y = _grid(H, W, ft)
    x = (X + ft(0.5)) / ft(W)
    y = (Y + ft(0.5)) / ft(H)
    vec = tex_linear(tvf, x, y, mode)
    vx = vec[..., 0].astype(ft)
    vy = vec[..., 1].astype(ft)
    norm = np.hypot(vx, vy).astype(ft)
    dx = (vx / norm / ft(W)).astype(ft)
    dy = (vy / norm / ft(H)).astype(ft)
    tr = lambda a, b: tex_linear(ref, a, b, mode)
    to = lambda a, b: tex_linear(other, a, b, mode)
    two = ft(2)
    v0 = tr(x - two * dx, y - two * dy) - tr(x - dx, y - dy) * 8 + tr(x + dx, y + dy) * 8 - tr(x + two * dx, y + two * dy)
    v1 = to(x - two * dx, y - two * dy) - to(x - dx, y - dy) * 8 + to(x + dx, y + dy) * 8 - to(x + two * dx, y + two * dy)
    v2 = tr(x, y)
    v3 = to(x, y)
    return np.stack([(v0 + v1) / 24.0, v3 - v2], -1)


def update_dual_variables(p_, q_, sigma, u, v, abc, M, prm):
    """``updateDualVariables``, Python/vfs.cu:326-419.  Returns (p, tp, q)."""
    Mb, mE, mW, mS, mN = mask_neighbours(M)
    uE, uW, uS, uN = flat_get(u, 1), flat_get(u, -1), flat_get(u, u.shape[1]), flat_get(u, -u.shape[1])
    vE, vW, vS, vN = flat_get(v, 1), flat_get(v, -1), flat_get(v, v.shape[1]), flat_get(v, -v.shape[1])
    vx, vy = v[..., 0], v[..., 1]
    gux = np.where(mE, uE - u - vx, u - uW - vx)
    gvx = np.where(mE, vE[..., 0] - vx, vx - vW[..., 0])
    gvw = np.where(mE, vE[..., 1] - vy, vy - vW[..., 1])
    guy = np.where(mS, uS - u - vy, u - uN - vy)
    gvy = np.where(mS, vS[..., 1] - vy, vy - vN[..., 1])
    gvz = np.where(mS, vS[..., 0] - vx, vx - vN[..., 0])
    a, b, c = abc[..., 0], abc[..., 1], abc[..., 2]
    tux = a * gux + c * guy
    tuy = c * gux + b * guy
    scale = prm.alpha1 * sigma / 3.0
    px = p_[..., 0] + scale * tux
    py = p_[..., 1] + scale * tuy
    nrm = np.maximum(np.hypot(px, py), 1.0)
    px, py = px / nrm, py / nrm
    tpx = a * px + c * py
    tpy = c * px + b * py
    scale = prm.alpha0 * sigma / 2.0
    Q = q_ + scale * np.stack([gvx, gvy, gvz, gvw], -1)
    nrm = np.maximum(np.sqrt(np.sum(Q * Q, -1)), 1.0)
    Q = Q / nrm[..., None]
    m2 = Mb[..., None]
    return (np.where(m2, np.stack([px, py], -1), 0.0), np.where(m2, np.stack([tpx, tpy], -1), 0.0),
            np.where(m2, Q, 0.0))


def l1_thresholding(tau, tp, u, u_, deriv, eta, M, prm):
    """``l1Thresholding``, Python/vfs.cu:421-505."""
    Mb, mE, mW, mS, mN = mask_neighbours(M)
    W = u.shape[1]
    tpW = flat_get(tp, -1)
    tpN = flat_get(tp, -W)
    gx = np.where(mE & mW, tp[..., 0] - tpW[..., 0], np.where(~mE, -tpW[..., 0], tp[..., 0]))
    gy = np.where(mS & mN, tp[..., 1] - tpN[..., 1], np.where(~mS, -tpN[..., 1], tp[..., 1]))
    Iu, Iz = deriv[..., 0], deriv[..., 1]
    eps = 1e-7
    with np.errstate(divide="ignore", invalid="ignore"):
        te = np.where(np.abs(eta[..., 0]) < eps, tau, tau / eta[..., 0])
        ut = u_ + te * (gx + gy)
        rho = Iu * (ut - u) + Iz
        bound = prm.Lambda * te * Iu * Iu
        mid = np.where(np.abs(Iu) < eps, ut - u, (ut - u) - rho / Iu)
        du = np.where((rho <= bound) & (rho >= -bound), mid,
                      np.where(rho < -bound, (ut - u) + prm.Lambda * te * Iu,
                               np.where(rho > bound, (ut - u) - prm.Lambda * te * Iu, 0.0)))
    return np.where(Mb, u + du, 0.0)


def update_primal_variables(tau, mu, p, q, u, u_, v_, abc, eta, M, prm):
    """``updatePrimalVariables``, Python/vfs.cu:507-581.  Returns (u_bar, v_bar)."""
    Mb, mE, mW, mS, mN = mask_neighbours(M)
    W = u.shape[1]
    qW = flat_get(q, -1)
    qN = flat_get(q, -W)
    gqx = np.where(mE, q[..., 0], 0.0) - np.where(mW, qW[..., 0], 0.0)
    gqw = np.where(mE, q[..., 3], 0.0) - np.where(mW, qW[..., 3], 0.0)
    gqy = np.where(mS, q[..., 1], 0.0) - np.where(mN, qN[..., 1], 0.0)
    gqz = np.where(mS, q[..., 2], 0.0) - np.where(mN, qN[..., 2], 0.0)
    a, b, c = abc[..., 0], abc[..., 1], abc[..., 2]
    tux = a * p[..., 0] + c * p[..., 1]
    tuy = c * p[..., 0] + b * p[..., 1]
    eps = 1e-7
    with np.errstate(divide="ignore", invalid="ignore"):
        t1 = np.where(np.abs(eta[..., 1]) < eps, tau, tau / eta[..., 1])
        t2 = np.where(np.abs(eta[..., 2]) < eps, tau, tau / eta[..., 2])
    Vx = t1 * (prm.alpha1 * tux + prm.alpha0 * (gqx + gqz)) + v_[..., 0]
    Vy = t2 * (prm.alpha1 * tuy + prm.alpha0 * (gqw + gqy)) + v_[..., 1]
    uo = mu * (u - u_) + u
    vo = np.stack([mu * (Vx - v_[..., 0]) + Vx, mu * (Vy - v_[..., 1]) + Vy], -1)
    return np.where(Mb, uo, 0.0), np.where(Mb[..., None], vo, 0.0)


def median_filter(u, M):
    """``medianFilter`` (5x5, clamp-to-edge), Python/vfs.cu:583-639."""
    H, W = u.shape
    ys = np.arange(H)
    xs = np.arange(W)
    taps = []
    for j in range(5):
        yy = np.clip(ys + j - 2, 0, H - 1)
        for i in range(5):
            xx = np.clip(xs + i - 2, 0, W - 1)
            taps.append(u[yy[:, None], xx[None, :]])
    med = np.sort(np.stack(taps, 0), axis=0)[12]
    return np.where(np.asarray(M) != 0, med, u)


def compute_optical_flow_with_clamp(warp, u_before, u_med, tvec, M, prm):
    """``computeOpticalFlowWithClamp``, Python/vfs.cu:641-676 (in place on warp, u_before)."""
    m = np.asarray(M) != 0
    delta = np.minimum(u_med - u_before, prm.limitRange)
    u_before[m] = u_before[m] + delta[m]
    warp[m, 0] = delta[m] * tvec[m, 0] + warp[m, 0]
    warp[m, 1] = delta[m] * tvec[m, 1] + warp[m, 1]
    return warp, u_before


def upsampling(coarse, Hf, Wf, scale, mode="exact"):
    """``upSamplingVectorField(1)`` via ``NearestNeighborScaled``, Python/vfs.cu:69-79, 678-705."""
    ft = _ft(mode)
    X, Y = _grid(Hf, Wf, ft)
    x = (X + ft(0.5)) / ft(Wf)
    y = (Y + ft(0.5)) / ft(Hf)
    return scale * tex_linear(coarse, x, y, mode)


def triangulate_rays(rays, rays_o, t, M):
    """``triangulateRays``, Python/vfs.cu:707-745 (x components only)."""
    xr = rays[..., 0] / rays[..., 2]
    yr = rays[..., 1] / rays[..., 2]
    xo = rays_o[..., 0] / rays_o[..., 2]
    with np.errstate(divide="ignore", invalid="ignore"):
        Z = (t[0] - t[2] * xo) / (xo - xr)
    out = np.stack([Z * xr, Z * yr, Z], -1)
    m = np.asarray(M) != 0
    out[~m] = (0.0, 0.0, -1.0)
    return out


def triangulate_rays_lsq(rays, rays_o, t, M):
    """Least-squares option beside ``triangulateRays`` (Python/vfs.cu:707-745),
    with no reference counterpart: the point on the reference ray closest to
    the other camera's ray ``-t + s * rays_o`` (the reference's convention,
    the other camera sees X at X + t), using all three components of t."""
    r = np.asarray(rays, F64)
    o = np.asarray(rays_o, F64)
    tt = np.asarray(t, F64).reshape(3)
    n = np.cross(r, o)
    m = np.cross(np.broadcast_to(-tt, o.shape), o)
    with np.errstate(divide="ignore", invalid="ignore"):
        lam = np.sum(m * n, -1) / np.sum(n * n, -1)
    out = lam[..., None] * r
    msk = np.asarray(M) != 0
    out[~msk] = (0.0, 0.0, -1.0)
    return out


# ---------------------------------------------------------------- camera
class EquidistantCam64:
    """``EquidistantCamera`` (Python/equidistant_cam.cuh:32-59) and the
    ``EquidistantCam`` kernels getRays/getUVFromXYZ/getXYZFromUV
    (Python/template_cam.cu:25-86), in float64."""

    def __init__(self, p):
        self.f, self.u0, self.v0 = (float(F32(v)) for v in p[:3])

    def project(self, X):
        R = np.hypot(X[..., 0], X[..., 1])
        theta = np.arctan2(R, X[..., 2])
        phi = np.arctan2(X[..., 1], X[..., 0])
        return np.stack([self.f * theta * np.cos(phi) + self.u0, self.f * theta * np.sin(phi) + self.v0], -1)

    def unproject(self, uv):
        x = uv[..., 0] - self.u0
        y = uv[..., 1] - self.v0
        theta = np.hypot(x, y) / self.f
        phi = np.arctan2(y, x)
        st = np.sin(theta)
        return np.stack([np.cos(phi) * st, np.sin(phi) * st, np.cos(theta)], -1)

    get_UVs = project
    get_XYZs = unproject

    def get_rays(self, sz):
        return self.unproject(get_grid_zero(sz))


def get_grid_zero(sz):
    """Python/vector_field.py:58-62."""
    Y, X = np.meshgrid(np.arange(sz[0], dtype=F64), np.arange(sz[1], dtype=F64), indexing="ij")
    return np.stack([X, Y], -1)


def get_vector_fields(grid, cam_ref, cam_other, R, t, t_scale):
    """Python/vector_field.py:28-56 with the normalizer of Python/main_equidistant.py:60."""
    if isinstance(t_scale, (float, int)):
        t_scale = (t_scale, t_scale)
    t = np.asarray(t, F64).reshape(3)
    XYZ = cam_ref.unproject(np.asarray(grid, F64))
    XYZ = XYZ / np.linalg.norm(XYZ, axis=2)[..., None]
    fwd = cam_ref.project(XYZ + t_scale[0] * t)
    bwd = cam_ref.project(XYZ - t_scale[1] * t)
    tvf = (fwd - bwd) / 2
    tvf = tvf / np.linalg.norm(tvf, axis=2)[..., None]
    RXYZ = XYZ @ np.asarray(R, F64).T
    cvf = cam_other.project(RXYZ) - grid
    return tvf, cvf


# ---------------------------------------------------------------- orchestration
def step_schedule(n_iters, time_step_lambda):
    """(sigma, tau, mu) per TGV iteration, with the reference's NumPy scalar
    arithmetic (Python/vfs.py:494-515).  Under NumPy >= 2 the scalars become
    float32 after the first iteration; the values returned are those float32
    numbers, as the kernels receive them (``cp.float32(...)``)."""
    out = []
    tau = 1.
    sigma = 1. / tau
    for _ in range(n_iters):
        if sigma < 1000:
            mu = 1 / np.sqrt(1 + 0.7 * tau * time_step_lambda).astype(np.float32)
        else:
            mu = 1
        out.append((float(np.float32(sigma)), float(np.float32(tau)), float(np.float32(mu))))
        sigma = sigma / mu
        tau = tau * mu
    return out


class VFS64:
    """``VFS`` (Python/vfs.py:33-559) in float64 NumPy."""

    def __init__(self, param, mode="exact"):
        self.param = param
        self.mode = mode

    def compute_pyramid_sizes(self):
        """Python/vfs.py:84-91."""
        sizes = []
        h, w = self.param.height, self.param.width
        for _ in range(self.param.nLevel):
            sizes.append((h, w))
            h = int(h / self.param.fScale)
            w = int(w / self.param.fScale)
        self.sizes = sizes

    def create_mask_pyramid(self, mask):
        """Python/vfs.py:159-187."""
        masks = [np.asarray(mask, np.uint8)]
        for sz in self.sizes[1:]:
            masks.append(down_sampling_mask(masks[-1], *sz))
        self.masks = masks

    def create_vector_field_pyramid(self, translation, calibration):
        """Python/vfs.py:189-218."""
        self.calibration = np.asarray(calibration, F64)
        tr = [np.asarray(translation, F64)]
        for sz in self.sizes[1:]:
            tr.append(down_sampling(tr[-1], *sz, mode=self.mode))
        self.translations = tr

    def create_image_pyramid(self, img_ref, img_other):
        """Python/vfs.py:93-157."""
        ref0 = cast_and_scale(img_ref)
        other0 = cast_and_scale(img_other)
        other0 = warping_image(other0, self.calibration, self.mode)
        refs, others = [ref0], [other0]
        for sz in self.sizes[1:]:
            refs.append(down_sampling(refs[-1], *sz, mode=self.mode))
            others.append(down_sampling(others[-1], *sz, mode=self.mode))
        self.refs, self.others = refs, others

    def solve_stereo(self, img_ref, img_other, levels=None, n_warps=None, n_iters=None):
        """Python/vfs.py:460-533.  ``levels``/``n_warps``/``n_iters`` bound the
        work (a prefix of the coarse-to-fine loops) for timing samples."""
        prm = self.param
        self.create_image_pyramid(img_ref, img_other)
        n_warps = prm.nWarpIters if n_warps is None else n_warps
        n_iters = prm.nSolverIters if n_iters is None else n_iters
        sched = step_schedule(n_iters, prm.timeStepLambda)
        L = len(self.sizes)
        for k in range(L, 0, -1):
            if levels is not None and (L - k) >= levels:
                break
            s = self.sizes[k - 1]
            M = self.masks[k - 1]
            if k == L:
                warp = np.zeros((*s, 2))
                u = np.zeros(s)
                u_ = np.zeros(s)
            smoothed = gaussian_masked(self.refs[k - 1], M, self.mode)
            abc, eta = compute_tensor_eta(smoothed, M, prm, self.mode)
            for _ in range(n_warps):
                tvec = find_warping_vector(self.translations[k - 1], warp, self.mode)
                warped = warping_image(self.others[k - 1], warp, self.mode)
                deriv = compute_derivatives(self.refs[k - 1], warped, self.translations[k - 1], self.mode)
                p = np.zeros((*s, 2))
                q = np.zeros((*s, 4))
                v_ = np.zeros((*s, 2))
                u_before = u.copy()
                for sigma, tau, mu in sched:
                    p, tp, q = update_dual_variables(p, q, sigma, u_, v_, abc, M, prm)
                    u = l1_thresholding(tau, tp, u, u_, deriv, eta, M, prm)
                    u_, v_ = update_primal_variables(tau, mu, p, q, u, u_, v_, abc, eta, M, prm)
                u_med = median_filter(u, M)
                warp, u_before = compute_optical_flow_with_clamp(warp, u_before, u_med, tvec, M, prm)
                u = u_before
            if k > 1:
                ss = self.sizes[k - 2]
                u_ = upsampling(u, *ss, prm.fScale, self.mode)
                u = u_.copy()
                warp = upsampling(warp, *ss, prm.fScale, self.mode)
        warp = warp.copy()
        if warp.shape[:2] == self.masks[0].shape:
            warp[self.masks[0] == 0, :] = 0
        self.warpUV = warp
        return warp

    def triangulate_flow(self, camera, translation, method="reference"):
        """Python/vfs.py:535-559 (``method="lsq"``: ``triangulate_rays_lsq``)."""
        sz = self.warpUV.shape[:2]
        rays = camera.get_rays(sz)
        rays_o = camera.unproject(get_grid_zero(sz) + self.warpUV)
        tri = triangulate_rays_lsq if method == "lsq" else triangulate_rays
        return tri(rays, rays_o, np.asarray(translation, F64).reshape(3), self.masks[0])
