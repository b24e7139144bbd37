"""Test infrastructure: float64 reverse mode of the whole stereo solve.

The forward is oracle/np64/vfs64.py's coarse-to-fine solve (the reference's
``VFS.solve_stereo`` + ``triangulate_flow``, Python/vfs.py:460-559, with the
vector fields of Python/vector_field.py:28-56), taken as a function of

* the two images in the solver's own scale (``castAndScale`` output,
  Python/vfs.cu:145-156: u8 / 256),
* the translation ``t`` (which moves the epipolar field and the triangulation),
* theta = (Lambda, alpha0, alpha1, beta, gamma),

to the depth map ``xyz[..., 2]``.  ``solve`` runs it and keeps a tape;
``backward`` returns the vector-Jacobian product for a depth cotangent.

Rules at the non-smooth points (the CUDA adjoint follows the same ones):

* texture fetches: the derivative of exact bilinear interpolation at the
  fetch coordinate (the hardware's 8-bit weight rounding is passed straight
  through), right-sided at texel centres;
* median: the cotangent goes to the pixel whose tap the sort selected;
* ``min(., limitRange)``: to the first argument unless the limit is taken;
* shrink and projections: the active branch (oracle/np64/adjoint64.py).

The CPU tests check this against float64 central differences.
"""
from __future__ import annotations

import copy
import math

import numpy as np

from . import vfs64 as V
from .adjoint64 import iteration_forward, iteration_reverse

F64 = np.float64
THETA = ("Lambda", "alpha0", "alpha1", "beta", "gamma")


# ---------------------------------------------------------------- fetches
def sample_vjp(T, x, y, g):
    """Adjoint of ``tex_linear(T, x, y)`` (exact weights, mirror addressing).

    Returns (gT, gx, gy): the cotangent scattered onto the texels and the
    derivative with respect to the normalised coordinates (summed over
    channels).
    """
    H, W = T.shape[:2]
    Td = np.asarray(T, F64)
    two_d = Td.ndim == 2
    if two_d:
        Td = Td[..., None]
        g = np.asarray(g, F64)[..., None]
    u = np.asarray(x, F64) * W - 0.5
    v = np.asarray(y, F64) * H - 0.5
    i0 = np.floor(u)
    j0 = np.floor(v)
    a = (u - i0)[..., None]
    b = (v - j0)[..., None]
    i0 = i0.astype(np.int64)
    j0 = j0.astype(np.int64)
    I0, I1 = V._mirror_index(i0, W), V._mirror_index(i0 + 1, W)
    J0, J1 = V._mirror_index(j0, H), V._mirror_index(j0 + 1, H)
    gT = np.zeros_like(Td)
    np.add.at(gT, (J0, I0), (1 - a) * (1 - b) * g)
    np.add.at(gT, (J0, I1), a * (1 - b) * g)
    np.add.at(gT, (J1, I0), (1 - a) * b * g)
    np.add.at(gT, (J1, I1), a * b * g)
    t00, t01, t10, t11 = Td[J0, I0], Td[J0, I1], Td[J1, I0], Td[J1, I1]
    du = (1 - b) * (t01 - t00) + b * (t11 - t10)
    dv = (1 - a) * (t10 - t00) + a * (t11 - t01)
    gx = np.sum(g * du, -1) * W
    gy = np.sum(g * dv, -1) * H
    return (gT[..., 0] if two_d else gT), gx, gy


def _centre_coords(H, W):
    X, Y = V._grid(H, W, F64)
    return (X + 0.5) / W, (Y + 0.5) / H


def down_sampling_vjp(shape_f, g):
    """Adjoint of ``down_sampling`` (Python/vfs.cu:35-49, 171-184)."""
    Hc, Wc = g.shape[:2]
    T = np.zeros(shape_f)
    x, y = _centre_coords(Hc, Wc)
    dx, dy = 0.25 / Wc, 0.25 / Hc
    out = np.zeros(shape_f)
    for xs, ys in ((x - dx, y), (x + dx, y), (x, y - dy), (x, y + dy)):
        out += sample_vjp(T, xs, ys, 0.25 * g)[0]
    return out


def upsampling_vjp(shape_c, g, scale):
    """Adjoint of ``upsampling`` (Python/vfs.cu:69-79, 678-705)."""
    Hf, Wf = g.shape[:2]
    x, y = _centre_coords(Hf, Wf)
    return sample_vjp(np.zeros(shape_c), x, y, scale * g)[0]


def warping_image_vjp(T, warp, g):
    """Adjoint of ``warping_image`` / ``find_warping_vector`` (Python/vfs.cu:61-66,
    186-202, 283-302): (gT, g_warp)."""
    H, W = warp.shape[:2]
    X, Y = V._grid(H, W, F64)
    x = (X + warp[..., 0] + 0.5) / W
    y = (Y + warp[..., 1] + 0.5) / H
    gT, gx, gy = sample_vjp(T, x, y, g)
    return gT, np.stack([gx / W, gy / H], -1)


def gaussian_masked_vjp(shape, M, g):
    """Adjoint of ``gaussian_masked`` (Python/vfs.cu:81-102, 204-226)."""
    H, W = shape
    x, y = _centre_coords(H, W)
    dx, dy = 1.0 / W, 1.0 / H
    g = np.where(np.asarray(M) != 0, g, 0.0)
    Z = np.zeros(shape)
    out = sample_vjp(Z, x, y, 0.25 * g)[0]
    for sx, sy in ((-dx, -dy), (-dx, dy), (dx, -dy), (dx, dy)):
        out += sample_vjp(Z, x + sx, y + sy, 0.0625 * g)[0]
    for sx, sy in ((-dx, 0), (dx, 0), (0, -dy), (0, dy)):
        out += sample_vjp(Z, x + sx, y + sy, 0.125 * g)[0]
    return out


# ---------------------------------------------------------------- per-level pieces
def tensor_eta_vjp(T, M, prm, g_abc, g_eta):
    """Adjoint of ``compute_tensor_eta`` (Python/vfs.cu:106-118, 228-281).

    Returns (gT, {alpha0, alpha1, beta, gamma})."""
    H, W = T.shape
    x, y = _centre_coords(H, W)
    dx, dy = 1.0 / W, 1.0 / H
    t = lambda a, b: V.tex_linear(T, a, b)
    g0 = t(x + dx, y + dy) - t(x, y + dy)
    g1 = t(x + dx, y + dy) - t(x + dx, y)
    ng = np.hypot(g0, g1)
    small = ng < 1e-8
    with np.errstate(divide="ignore", invalid="ignore"):
        n0 = np.where(small, 1.0, g0 / ng)
        n1 = np.where(small, 0.0, g1 / ng)
        ngg = np.where(ng > 0, ng ** prm.gamma, 0.0)
        lng = np.where(ng > 0, np.log(np.where(ng > 0, ng, 1.0)), 0.0)
    e = np.exp(-prm.beta * ngg)
    live = e > 1e-8
    w = np.where(live, e, 1e-8)
    a = w * n0 * n0 + n1 * n1
    b = w * n1 * n1 + n0 * n0
    c = w * n0 * n1 - n0 * n1
    a11 = prm.alpha1 * prm.alpha1
    m = np.asarray(M) != 0
    ga = np.where(m, g_abc[..., 0], 0.0)
    gb = np.where(m, g_abc[..., 1], 0.0)
    gc = np.where(m, g_abc[..., 2], 0.0)
    ge0 = np.where(m, g_eta[..., 0], 0.0)
    ge1 = np.where(m, g_eta[..., 1], 0.0)
    ge2 = np.where(m, g_eta[..., 2], 0.0)
    # eta
    ga = ga + a11 * (ge0 * (2 * a + 2 * (a + c)) + ge2 * 2 * a)
    gb = gb + a11 * (ge0 * (2 * b + 2 * (b + c)) + ge1 * 2 * b)
    gc = gc + a11 * (ge0 * (4 * c + 2 * (a + c) + 2 * (b + c)) + ge1 * 2 * c + ge2 * 2 * c)
    g_a11 = (ge0 * (a * a + b * b + 2 * c * c + (a + c) ** 2 + (b + c) ** 2)
             + ge1 * (b * b + c * c) + ge2 * (a * a + c * c))
    g_alpha1 = np.sum(g_a11) * 2 * prm.alpha1
    g_alpha0 = np.sum(ge1 + ge2) * 8 * prm.alpha0
    # abc
    gw = ga * n0 * n0 + gb * n1 * n1 + gc * n0 * n1
    gn0 = ga * 2 * w * n0 + gb * 2 * n0 + gc * (w - 1) * n1
    gn1 = ga * 2 * n1 + gb * 2 * w * n1 + gc * (w - 1) * n0
    gE = np.where(live, gw * e, 0.0)              # d/d(-beta ng^gamma)
    g_beta = -np.sum(gE * ngg)
    g_gamma = -np.sum(gE * prm.beta * ngg * lng)
    with np.errstate(divide="ignore", invalid="ignore"):
        g_ng = np.where(small, 0.0, -gE * prm.beta * prm.gamma * ngg / np.where(small, 1.0, ng))
        dot = gn0 * n0 + gn1 * n1
        gg0 = np.where(small, 0.0, (gn0 - n0 * dot) / np.where(small, 1.0, ng)) + g_ng * n0
        gg1 = np.where(small, 0.0, (gn1 - n1 * dot) / np.where(small, 1.0, ng)) + g_ng * n1
    Z = np.zeros_like(T, dtype=F64)
    gT = sample_vjp(Z, x + dx, y + dy, gg0 + gg1)[0]
    gT += sample_vjp(Z, x, y + dy, -gg0)[0]
    gT += sample_vjp(Z, x + dx, y, -gg1)[0]
    return gT, {"alpha0": g_alpha0, "alpha1": g_alpha1, "beta": g_beta, "gamma": g_gamma}


def derivatives_vjp(ref, other, tvf, g):
    """Adjoint of ``compute_derivatives`` (Python/vfs.cu:120-142, 304-324).

    Returns (g_ref, g_other, g_tvf)."""
    H, W = ref.shape
    x, y = _centre_coords(H, W)
    vec = V.tex_linear(tvf, x, y)
    vx, vy = vec[..., 0], vec[..., 1]
    n = np.hypot(vx, vy)
    dx = vx / n / W
    dy = vy / n / H
    g_iu = g[..., 0] / 24.0
    g_iz = g[..., 1]
    g_ref = np.zeros_like(ref, dtype=F64)
    g_oth = np.zeros_like(other, dtype=F64)
    g_dx = np.zeros((H, W))
    g_dy = np.zeros((H, W))
    for k, ck in ((-2, 1.0), (-1, -8.0), (1, 8.0), (2, -1.0)):
        for T, gT in ((ref, g_ref), (other, g_oth)):
            t_, gx, gy = sample_vjp(T, x + k * dx, y + k * dy, ck * g_iu)
            gT += t_
            g_dx += k * gx
            g_dy += k * gy
    g_ref += sample_vjp(np.zeros_like(g_ref), x, y, -g_iz)[0]
    g_oth += sample_vjp(np.zeros_like(g_oth), x, y, g_iz)[0]
    n3 = n ** 3
    g_vx = (g_dx / W) * vy * vy / n3 + (g_dy / H) * (-vx * vy / n3)
    g_vy = (g_dx / W) * (-vx * vy / n3) + (g_dy / H) * vx * vx / n3
    g_tvf = sample_vjp(np.zeros(tvf.shape), x, y, np.stack([g_vx, g_vy], -1))[0]
    return g_ref, g_oth, g_tvf


def median_source(u, M):
    """Flat index of the pixel whose tap ``median_filter`` returns (Python/vfs.cu:583-639)."""
    H, W = u.shape
    ys = np.arange(H)
    xs = np.arange(W)
    vals, src = [], []
    for j in range(5):
        yy = np.clip(ys + j - 2, 0, H - 1)
        for i in range(5):
            xx = np.clip(xs + i - 2, 0, W - 1)
            vals.append(u[yy[:, None], xx[None, :]])
            src.append(yy[:, None] * W + xx[None, :])
    vals = np.stack(vals, 0)
    src = np.stack(src, 0)
    order = np.argsort(vals, axis=0, kind="stable")[12]
    return np.take_along_axis(src, order[None], 0)[0]


# ---------------------------------------------------------------- camera pieces
def _project_jac(cam, P):
    """d project / d P for the equidistant camera (Python/equidistant_cam.cuh:32-45): (..., 2, 3)."""
    X, Y, Z = P[..., 0], P[..., 1], P[..., 2]
    R = np.hypot(X, Y)
    th = np.arctan2(R, Z)
    with np.errstate(divide="ignore", invalid="ignore"):
        k = np.where(R > 0, cam.f * th / np.where(R > 0, R, 1.0), cam.f / Z)
        s2 = (R / Z) ** 2
        series = cam.f / Z ** 3 * (-2.0 / 3.0 + 0.8 * s2 - 6.0 / 7.0 * s2 * s2)
        direct = cam.f * (Z * R / (R * R + Z * Z) - th) / np.where(R > 0, R, 1.0) ** 3
        D = np.where((Z > 0) & (R < 1e-3 * np.abs(Z)), series, direct)
    dkdZ = -cam.f / (R * R + Z * Z)
    J = np.empty(P.shape[:-1] + (2, 3))
    J[..., 0, 0] = k + X * D * X
    J[..., 0, 1] = X * D * Y
    J[..., 0, 2] = X * dkdZ
    J[..., 1, 0] = Y * D * X
    J[..., 1, 1] = k + Y * D * Y
    J[..., 1, 2] = Y * dkdZ
    return J


def vector_fields_vjp(cam, t, t_scale, shape, g_tvf):
    """d L / d t through ``get_vector_fields``'s tvf (Python/vector_field.py:28-50)."""
    t = np.asarray(t, F64).reshape(3)
    P = cam.unproject(V.get_grid_zero(shape))
    P = P / np.linalg.norm(P, axis=2)[..., None]
    Pf, Pb = P + t_scale * t, P - t_scale * t
    tv = (cam.project(Pf) - cam.project(Pb)) / 2
    n = np.linalg.norm(tv, axis=2)[..., None]
    d = tv / n
    g_tv = (g_tvf - d * np.sum(g_tvf * d, -1)[..., None]) / n
    Jf, Jb = _project_jac(cam, Pf), _project_jac(cam, Pb)
    g = np.einsum("hwi,hwij->j", g_tv / 2, Jf) * t_scale + np.einsum("hwi,hwij->j", -g_tv / 2, Jb) * (-t_scale)
    return g


def _xo_and_grad(cam, uv):
    """x/z of the unprojected ray and its derivative w.r.t. (u, v)."""
    x = uv[..., 0] - cam.u0
    y = uv[..., 1] - cam.v0
    rho = np.hypot(x, y)
    th = rho / cam.f
    with np.errstate(divide="ignore", invalid="ignore"):
        G = np.where(rho > 0, np.tan(th) / np.where(rho > 0, rho, 1.0), 1.0 / cam.f)
        Gp_over_rho = np.where(th < 1e-3, (2.0 / 3.0 + 8.0 / 15.0 * th * th) / cam.f ** 3,
                               (rho / (cam.f * np.cos(th) ** 2) - np.tan(th)) / np.where(rho > 0, rho, 1.0) ** 3)
    ro = cam.unproject(uv)
    xo = ro[..., 0] / ro[..., 2]
    return xo, G + x * x * Gp_over_rho, x * y * Gp_over_rho


def triangulate_vjp(cam, warp, t, M, g_depth):
    """Adjoint of the depth map of ``triangulate_flow`` (Python/vfs.py:535-559,
    Python/vfs.cu:707-745): (g_warp, g_t)."""
    t = np.asarray(t, F64).reshape(3)
    H, W = warp.shape[:2]
    grid = V.get_grid_zero((H, W))
    rr = cam.unproject(grid)
    xr = rr[..., 0] / rr[..., 2]
    xo, dxo_du, dxo_dv = _xo_and_grad(cam, grid + warp)
    m = (np.asarray(M) != 0) & (g_depth != 0)
    g = np.where(m, g_depth, 0.0)
    D = xo - xr
    with np.errstate(divide="ignore", invalid="ignore"):
        gZ_xo = np.where(m, g * (t[2] * xr - t[0]) / (D * D), 0.0)
        g_t = np.array([np.sum(np.where(m, g / D, 0.0)), 0.0, np.sum(np.where(m, -g * xo / D, 0.0))])
    return np.stack([gZ_xo * dxo_du, gZ_xo * dxo_dv], -1), g_t


def _unproject_and_jac(cam, uv):
    """Unit ray of ``EquidistantCamera::unproject`` (Python/equidistant_cam.cuh:46-59)
    at uv and its Jacobian d ray / d (u, v), shape (..., 3, 2).  With
    x, y relative to the principal point, rho = |(x, y)|, theta = rho / f and
    S = sin(theta) / rho: ray = (S x, S y, cos theta)."""
    x = uv[..., 0] - cam.u0
    y = uv[..., 1] - cam.v0
    rho = np.hypot(x, y)
    th = rho / cam.f
    small = th < 1e-3
    with np.errstate(divide="ignore", invalid="ignore"):
        rs = np.where(small, 1.0, rho)
        S = np.where(small, (1 - th * th / 6 + th ** 4 / 120) / cam.f, np.sin(th) / rs)
        Sp = np.where(small, (-1.0 / 3 + th * th / 30) / cam.f ** 3,  # (dS/drho) / rho
                      (rho * np.cos(th) / cam.f - np.sin(th)) / rs ** 3)
    ray = np.stack([S * x, S * y, np.cos(th)], -1)
    J = np.empty(uv.shape[:-1] + (3, 2))
    J[..., 0, 0] = S + x * x * Sp
    J[..., 0, 1] = J[..., 1, 0] = x * y * Sp
    J[..., 1, 1] = S + y * y * Sp
    J[..., 2, 0] = -S * x / cam.f
    J[..., 2, 1] = -S * y / cam.f
    return ray, J


def triangulate_lsq_vjp(cam, warp, t, M, g_depth):
    """Adjoint of the depth map of ``triangulate_flow(method="lsq")``
    (vfs64.triangulate_rays_lsq; no reference counterpart): (g_warp, g_t).
    depth = lambda r_z with lambda = (m . n) / (n . n), n = r x o,
    m = (-t) x o, o = unproject(grid + warp)."""
    t = np.asarray(t, F64).reshape(3)
    H, W = warp.shape[:2]
    grid = V.get_grid_zero((H, W))
    rr = cam.unproject(grid)
    ro, J = _unproject_and_jac(cam, grid + warp)
    msk = (np.asarray(M) != 0) & (g_depth != 0)
    n = np.cross(rr, ro)
    m = np.cross(np.broadcast_to(-t, ro.shape), ro)
    nn = np.sum(n * n, -1)
    with np.errstate(divide="ignore", invalid="ignore"):
        lam = np.sum(m * n, -1) / nn
        g_lam = np.where(msk, g_depth * rr[..., 2], 0.0)
        gm = (g_lam / nn)[..., None] * n
        gn = (g_lam / nn)[..., None] * (m - 2 * lam[..., None] * n)
    gm = np.where(msk[..., None], gm, 0.0)
    gn = np.where(msk[..., None], gn, 0.0)
    # m = (-t) x o: d/d(-t) = o x gm, d/do = gm x (-t); n = r x o: d/do = gn x r
    g_t = -np.sum(np.cross(ro, gm), axis=(0, 1))
    g_o = np.cross(gm, np.broadcast_to(-t, ro.shape)) + np.cross(gn, rr)
    g_warp = np.einsum("...i,...ij->...j", g_o, J)
    return np.where(msk[..., None], g_warp, 0.0), g_t


# ---------------------------------------------------------------- whole solve
class Problem:
    """What stays fixed while the solve is differentiated: parameters (loop
    counts, fScale, limitRange, timeStepLambda), camera, mask, ``t_scale``,
    and the triangulation rule ("reference": Python/vfs.cu:728-734; "lsq":
    least squares along the reference ray)."""

    def __init__(self, prm, cam, mask, t_scale=1.0, triangulation="reference"):
        self.prm = prm
        self.cam = cam
        self.mask = np.asarray(mask, np.uint8)
        self.t_scale = float(t_scale)
        if triangulation not in ("reference", "lsq"):
            raise ValueError(triangulation)
        self.triangulation = triangulation


def _params(prob, theta):
    prm = copy.copy(prob.prm)
    for k, v in zip(THETA, theta):
        setattr(prm, k, float(v))
    return prm


def solve(prob, I0, I1, t, theta, mode="exact", tape=False):
    """Depth map of the coarse-to-fine solve (Python/vfs.py:460-559) for float
    images ``I0``/``I1`` (u8 / 256).  With ``tape`` returns (depth, tape)."""
    prm = _params(prob, theta)
    H, W = I0.shape
    cam = prob.cam
    t = np.asarray(t, F64).reshape(3)
    tvf, cvf = V.get_vector_fields(V.get_grid_zero((H, W)), cam, cam, np.eye(3), t, prob.t_scale)
    vfs = V.VFS64(prm, mode)
    vfs.compute_pyramid_sizes()
    vfs.create_mask_pyramid(prob.mask)
    sizes, masks = vfs.sizes, vfs.masks
    tvfs = [tvf]
    refs = [np.asarray(I0, F64)]
    others = [V.warping_image(np.asarray(I1, F64), cvf, mode)]
    for sz in sizes[1:]:
        tvfs.append(V.down_sampling(tvfs[-1], *sz, mode=mode))
        refs.append(V.down_sampling(refs[-1], *sz, mode=mode))
        others.append(V.down_sampling(others[-1], *sz, mode=mode))
    sched = V.step_schedule(prm.nSolverIters, prm.timeStepLambda)
    L = len(sizes)
    levels = {}
    for k in range(L, 0, -1):
        s, M = sizes[k - 1], masks[k - 1]
        m = np.asarray(M) != 0
        if k == L:
            warp = np.zeros((*s, 2))
            u = np.zeros(s)
            u_ = np.zeros(s)
        smoothed = V.gaussian_masked(refs[k - 1], M, mode)
        abc, eta = V.compute_tensor_eta(smoothed, M, prm, mode)
        wrecs = []
        for _ in range(prm.nWarpIters):
            rec = {"warp_in": warp.copy(), "u_in": u.copy()}
            tvec = V.find_warping_vector(tvfs[k - 1], warp, mode)
            warped = V.warping_image(others[k - 1], warp, mode)
            deriv = V.compute_derivatives(refs[k - 1], warped, tvfs[k - 1], mode)
            cst = {"abc": abc, "eta": eta, "deriv": deriv}
            st = {"u": u.copy(), "ub": u_.copy(), "v": np.zeros((*s, 2)), "p": np.zeros((*s, 2)),
                  "q": np.zeros((*s, 4))}
            its = []
            for sigma, tau, mu in sched:
                out, inter = iteration_forward(st, cst, prm, sigma, tau, mu, M)
                if tape:
                    its.append((st, inter, sigma, tau, mu))
                st = out
            u_T, u_ = st["u"], st["ub"]
            med = V.median_filter(u_T, M)
            raw = med - u
            delta = np.minimum(raw, prm.limitRange)
            u = np.where(m, u + delta, u)
            warp = np.where(m[..., None], warp + delta[..., None] * tvec, warp)
            if tape:
                rec.update(tvec=tvec, warped=warped, cst=cst, its=its, delta=delta,
                           active=raw < prm.limitRange, med_src=median_source(u_T, M))
                wrecs.append(rec)
        levels[k] = {"smoothed": smoothed, "warps": wrecs}
        if k > 1:
            ss = sizes[k - 2]
            u_ = V.upsampling(u, *ss, prm.fScale, mode)
            u = u_.copy()
            warp = V.upsampling(warp, *ss, prm.fScale, mode)
    warp = np.where((masks[0] != 0)[..., None], warp, 0.0)
    tri = V.triangulate_rays_lsq if prob.triangulation == "lsq" else V.triangulate_rays
    depth = tri(cam.get_rays((H, W)), cam.unproject(V.get_grid_zero((H, W)) + warp), t, masks[0])[..., 2]
    if not tape:
        return depth
    return depth, {"prm": prm, "t": t, "cvf": cvf, "I1": np.asarray(I1, F64), "sizes": sizes, "masks": masks,
                   "tvfs": tvfs, "refs": refs, "others": others, "levels": levels, "warp": warp}


def backward(prob, tp, g_depth):
    """Vector-Jacobian product of ``solve`` for the depth cotangent ``g_depth``.

    Returns {"I0", "I1", "t", "theta"}."""
    prm, sizes, masks = tp["prm"], tp["sizes"], tp["masks"]
    cam = prob.cam
    L = len(sizes)
    tri_vjp = triangulate_lsq_vjp if prob.triangulation == "lsq" else triangulate_vjp
    g_warp, g_t = tri_vjp(cam, tp["warp"], tp["t"], masks[0], g_depth)
    g_warp = np.where((masks[0] != 0)[..., None], g_warp, 0.0)
    g_u = np.zeros(sizes[0])
    g_ub = np.zeros(sizes[0])
    g_th = dict.fromkeys(THETA, 0.0)
    g_refs = [np.zeros(s) for s in sizes]
    g_others = [np.zeros(s) for s in sizes]
    g_tvfs = [np.zeros((*s, 2)) for s in sizes]
    for k in range(1, L + 1):
        M = masks[k - 1]
        m = np.asarray(M) != 0
        lv = tp["levels"][k]
        g_abc = np.zeros((*sizes[k - 1], 3))
        g_eta = np.zeros((*sizes[k - 1], 3))
        for rec in reversed(lv["warps"]):
            tvec, delta = rec["tvec"], rec["delta"]
            g_delta = np.where(m, g_u + np.sum(g_warp * tvec, -1), 0.0)
            g_tvec = np.where(m[..., None], delta[..., None] * g_warp, 0.0)
            g_med = np.where(rec["active"], g_delta, 0.0)
            g_u_in = g_u - g_med
            g_uT = np.zeros(sizes[k - 1])
            np.add.at(g_uT.reshape(-1), rec["med_src"][m], g_med[m])
            g_st = {"u": g_uT, "ub": g_ub, "v": np.zeros((*sizes[k - 1], 2)),
                    "p": np.zeros((*sizes[k - 1], 2)), "q": np.zeros((*sizes[k - 1], 4))}
            g_deriv = np.zeros((*sizes[k - 1], 2))
            for st, inter, sigma, tau, mu in reversed(rec["its"]):
                r = iteration_reverse(st, rec["cst"], prm, sigma, tau, mu, M, inter, g_st)
                g_st = {n: r[n] for n in ("u", "ub", "v", "p", "q")}
                g_abc += r["abc"]
                g_eta += r["eta"]
                g_deriv += r["deriv"]
                for n in ("Lambda", "alpha0", "alpha1"):
                    g_th[n] += r[n]
            g_u_in = g_u_in + g_st["u"]
            g_ub = g_st["ub"]
            gr, gw, gtv = derivatives_vjp(tp["refs"][k - 1], rec["warped"], tp["tvfs"][k - 1], g_deriv)
            g_refs[k - 1] += gr
            g_tvfs[k - 1] += gtv
            gT, gwarp_w = warping_image_vjp(tp["others"][k - 1], rec["warp_in"], gw)
            g_others[k - 1] += gT
            gT, gwarp_t = warping_image_vjp(tp["tvfs"][k - 1], rec["warp_in"], g_tvec)
            g_tvfs[k - 1] += gT
            g_warp = g_warp + gwarp_w + gwarp_t
            g_u = g_u_in
        gS, gth = tensor_eta_vjp(lv["smoothed"], M, prm, g_abc, g_eta)
        for n, v in gth.items():
            g_th[n] += v
        g_refs[k - 1] += gaussian_masked_vjp(sizes[k - 1], M, gS)
        if k < L:
            sc = sizes[k]
            g_u = upsampling_vjp(sc, g_u + g_ub, prm.fScale)
            g_ub = np.zeros(sc)
            g_warp = upsampling_vjp((*sc, 2), g_warp, prm.fScale)
    for l in range(L - 1, 0, -1):
        g_refs[l - 1] += down_sampling_vjp(sizes[l - 1], g_refs[l])
        g_others[l - 1] += down_sampling_vjp(sizes[l - 1], g_others[l])
        g_tvfs[l - 1] += down_sampling_vjp((*sizes[l - 1], 2), g_tvfs[l])
    g_I1 = warping_image_vjp(tp["I1"], tp["cvf"], g_others[0])[0]
    g_t = g_t + vector_fields_vjp(cam, tp["t"], prob.t_scale, sizes[0], g_tvfs[0])
    return {"I0": g_refs[0], "I1": g_I1, "t": g_t, "theta": np.array([g_th[n] for n in THETA])}
