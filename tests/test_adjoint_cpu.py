"""CPU: the float64 reverse mode of a TGV iteration against finite differences."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import bench_params


def _problem(seed, h=6, w=7, all_ones=False):
    rng = np.random.default_rng(seed)
    M = np.full((h, w), 255, np.uint8) if all_ones else (rng.uniform(0, 1, (h, w)) > 0.25).astype(np.uint8) * 255
    st = {"u": rng.normal(0, 1, (h, w)), "ub": rng.normal(0, 1, (h, w)), "v": rng.normal(0, 0.3, (h, w, 2)),
          "p": rng.normal(0, 0.4, (h, w, 2)), "q": rng.normal(0, 0.2, (h, w, 4))}
    a = rng.uniform(0.2, 1.0, (h, w))
    cst = {"abc": np.stack([a, rng.uniform(0.2, 1.0, (h, w)), rng.normal(0, 0.2, (h, w))], -1),
           "eta": np.stack([rng.uniform(1, 5, (h, w)), rng.uniform(1100, 1300, (h, w)),
                            rng.uniform(1100, 1300, (h, w))], -1),
           "deriv": np.stack([rng.normal(0, 0.3, (h, w)), rng.normal(0, 0.05, (h, w))], -1)}
    prm = bench_params(h, w)
    prm.Lambda = 5.0
    return st, cst, prm, M, rng


def _loss(out, wts):
    return sum(np.sum(out[k] * wts[k]) for k in wts)


@pytest.mark.parametrize("seed,all_ones", [(0, False), (1, False), (2, True), (3, False)])
def test_iteration_vjp_matches_finite_differences(seed, all_ones):
    from oracle.np64 import adjoint64 as A
    from oracle.np64 import vfs64 as V
    st, cst, prm, M, rng = _problem(seed, all_ones=all_ones)
    sigma, tau, mu = 2.5, 0.4, 0.9
    out, inter = A.iteration_forward(st, cst, prm, sigma, tau, mu, M)
    # the forward is the oracle's
    p2, tp2, q2 = V.update_dual_variables(st["p"], st["q"], sigma, st["ub"], st["v"], cst["abc"], M, prm)
    u2 = V.l1_thresholding(tau, tp2, st["u"], st["ub"], cst["deriv"], cst["eta"], M, prm)
    ub2, vb2 = V.update_primal_variables(tau, mu, p2, q2, u2, st["ub"], st["v"], cst["abc"], cst["eta"], M, prm)
    for k, ref in (("p", p2), ("q", q2), ("u", u2), ("ub", ub2), ("v", vb2)):
        assert np.allclose(out[k], ref, rtol=1e-12, atol=1e-12), k
    wts = {k: rng.normal(0, 1, out[k].shape) for k in out}
    g = A.iteration_reverse(st, cst, prm, sigma, tau, mu, M, inter, wts)
    h = 1e-6

    def L_of(st_, cst_, prm_):
        o, _ = A.iteration_forward(st_, cst_, prm_, sigma, tau, mu, M)
        return _loss(o, wts)

    for group, src in (("state", st), ("const", cst)):
        for k in src:
            d = rng.normal(0, 1, src[k].shape)
            plus = {kk: vv.copy() for kk, vv in src.items()}
            minus = {kk: vv.copy() for kk, vv in src.items()}
            plus[k] = plus[k] + h * d
            minus[k] = minus[k] - h * d
            if group == "state":
                fd = (L_of(plus, cst, prm) - L_of(minus, cst, prm)) / (2 * h)
            else:
                fd = (L_of(st, plus, prm) - L_of(st, minus, prm)) / (2 * h)
            an = np.sum(g[k] * d)
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (k, fd, an)
    for name in ("Lambda", "alpha0", "alpha1"):
        import copy
        pp, pm = copy.copy(prm), copy.copy(prm)
        setattr(pp, name, getattr(prm, name) + h)
        setattr(pm, name, getattr(prm, name) - h)
        fd = (L_of(st, cst, pp) - L_of(st, cst, pm)) / (2 * h)
        assert abs(fd - g[name]) <= 1e-6 * max(1.0, abs(fd)), (name, fd, g[name])


def _fd_check(f, x, vjp, rng, h=1e-6, rtol=1e-6):
    y = f(x)
    w = rng.normal(0, 1, np.shape(y))
    d = rng.normal(0, 1, np.shape(x))
    fd = (np.sum(w * f(x + h * d)) - np.sum(w * f(x - h * d))) / (2 * h)
    an = np.sum(vjp(x, w) * d)
    assert abs(fd - an) <= rtol * max(1.0, abs(fd)), (fd, an)


def test_stage_vjps_match_finite_differences():
    import copy
    from oracle.np64 import grad64 as G
    from oracle.np64 import vfs64 as V
    rng = np.random.default_rng(1)
    H, W = 13, 17
    T = rng.uniform(0, 1, (H, W))
    T2 = rng.uniform(0, 1, (H, W, 2))
    M = (rng.uniform(0, 1, (H, W)) > 0.2).astype(np.uint8) * 255
    warp = rng.normal(0, 2, (H, W, 2))
    _fd_check(lambda a: V.down_sampling(a, 6, 8), T, lambda a, w: G.down_sampling_vjp(a.shape, w), rng)
    _fd_check(lambda a: V.down_sampling(a, 6, 8), T2, lambda a, w: G.down_sampling_vjp(a.shape, w), rng)
    _fd_check(lambda a: V.upsampling(a, 26, 34, 2.0), T, lambda a, w: G.upsampling_vjp(a.shape, w, 2.0), rng)
    _fd_check(lambda a: V.warping_image(a, warp), T, lambda a, w: G.warping_image_vjp(a, warp, w)[0], rng)
    _fd_check(lambda a: V.warping_image(T2, a), warp, lambda a, w: G.warping_image_vjp(T2, a, w)[1], rng, rtol=1e-5)
    _fd_check(lambda a: V.gaussian_masked(a, M), T, lambda a, w: G.gaussian_masked_vjp(a.shape, M, w), rng)
    prm = bench_params(H, W)
    both = lambda a, p=prm: np.concatenate(V.compute_tensor_eta(a, M, p), -1)
    _fd_check(both, T, lambda a, w: G.tensor_eta_vjp(a, M, prm, w[..., :3], w[..., 3:])[0], rng, rtol=1e-5)
    for name in ("alpha0", "alpha1", "beta", "gamma"):
        def f(v, name=name):
            p = copy.copy(prm)
            setattr(p, name, float(v))
            return both(T, p)
        _fd_check(f, np.float64(getattr(prm, name)),
                  lambda a, w, name=name: G.tensor_eta_vjp(T, M, prm, w[..., :3], w[..., 3:])[1][name], rng, rtol=1e-4)
    tvf = rng.normal(0, 1, (H, W, 2))
    ref, oth = rng.uniform(0, 1, (H, W)), rng.uniform(0, 1, (H, W))
    _fd_check(lambda a: V.compute_derivatives(a, oth, tvf), ref, lambda a, w: G.derivatives_vjp(a, oth, tvf, w)[0], rng)
    _fd_check(lambda a: V.compute_derivatives(ref, a, tvf), oth, lambda a, w: G.derivatives_vjp(ref, a, tvf, w)[1], rng)
    _fd_check(lambda a: V.compute_derivatives(ref, oth, a), tvf, lambda a, w: G.derivatives_vjp(ref, oth, a, w)[2], rng)
    from vfs_b200.synthetic import equidistant_intrinsics
    cam = V.EquidistantCam64(equidistant_intrinsics(48, 48))
    t = np.array([0.12, 0.03, 0.05])
    _fd_check(lambda a: V.get_vector_fields(V.get_grid_zero((48, 48)), cam, cam, np.eye(3), a, 1.0)[0], t,
              lambda a, w: G.vector_fields_vjp(cam, a, 1.0, (48, 48), w), rng, rtol=1e-5)
    Mm = np.zeros((48, 48), np.uint8)
    Mm[8:40, 8:40] = 255
    wp = rng.normal(2, 1, (48, 48, 2))

    def tri(a, tt=t):
        z = V.triangulate_rays(cam.get_rays((48, 48)), cam.unproject(V.get_grid_zero((48, 48)) + a), tt, Mm)[..., 2]
        return np.where(Mm != 0, z, 0)
    _fd_check(tri, wp, lambda a, w: G.triangulate_vjp(cam, a, t, Mm, w)[0], rng, rtol=1e-5)
    _fd_check(lambda a: tri(wp, a), t, lambda a, w: G.triangulate_vjp(cam, wp, a, Mm, w)[1], rng)

    def tri_lsq(a, tt=t):
        z = V.triangulate_rays_lsq(cam.get_rays((48, 48)), cam.unproject(V.get_grid_zero((48, 48)) + a), tt,
                                   Mm)[..., 2]
        return np.where(Mm != 0, z, 0)
    _fd_check(tri_lsq, wp, lambda a, w: G.triangulate_lsq_vjp(cam, a, t, Mm, w)[0], rng, rtol=1e-5)
    _fd_check(lambda a: tri_lsq(wp, a), t, lambda a, w: G.triangulate_lsq_vjp(cam, wp, a, Mm, w)[1], rng)
    # the unprojection Jacobian, including the series branch at the principal point
    uv = np.concatenate([rng.uniform(0, 48, (40, 2)), cam.u0 + rng.normal(0, 1e-3, (8, 2)),
                         np.array([[cam.u0, cam.v0]])])
    ray, Jac = G._unproject_and_jac(cam, uv)
    assert np.allclose(ray, cam.unproject(uv), rtol=0, atol=1e-15)
    for j in range(2):
        e = np.eye(2)[j] * 1e-6
        fd = (cam.unproject(uv + e) - cam.unproject(uv - e)) / 2e-6
        assert np.allclose(Jac[..., j], fd, rtol=0, atol=1e-8)


@pytest.mark.parametrize("triangulation", ["reference", "lsq"])
def test_solve_vjp_matches_finite_differences(triangulation):
    """Whole coarse-to-fine solve, depth cotangent -> images, t, theta.

    The unrolled solve is piecewise smooth: median selection, the limitRange
    clamp, the shrink cases and the unit-ball projections switch inside a
    1e-4 stencil on this problem, so the float64 differences are taken at
    h = 1e-8 along image directions, 1e-7 along t and 1e-5 along theta, where
    they have converged (along t.y, h = 1e-6 is still 6e-5..1e-4 off for both
    triangulation rules, 1e-7 agrees to 3e-7; along theta the least-squares
    depths carry more rounding noise, 3e-4 at h = 1e-6 against 4e-5 at 1e-5).
    """
    from oracle.np64 import grad64 as G
    from oracle.np64 import vfs64 as V
    from helpers import pair
    P = pair(48, t=(0.12, 0.01, 0.0), n_level=2)
    prm = bench_params(48, 48, n_level=2, n_warp=2, n_iter=6)
    prob = G.Problem(prm, V.EquidistantCam64(P.intrinsics), P.mask, triangulation=triangulation)
    nz = np.random.default_rng(9)     # continuous images: no exact ties in the median windows
    I0 = P.img_ref / 256.0 + nz.uniform(0, 1 / 256, (48, 48))
    I1 = P.img_other / 256.0 + nz.uniform(0, 1 / 256, (48, 48))
    t = P.t.reshape(3)
    theta = np.array([prm.Lambda, prm.alpha0, prm.alpha1, prm.beta, prm.gamma])
    d0, tape = G.solve(prob, I0, I1, t, theta, tape=True)
    good = (P.mask != 0) & np.isfinite(d0) & (np.abs(d0) < 50)
    rng = np.random.default_rng(0)
    wts = np.where(good, rng.normal(0, 1, good.shape), 0)
    g = G.backward(prob, tape, wts)
    L = lambda *a: np.sum(np.where(good, wts * G.solve(prob, *a), 0))
    base = [I0, I1, t, theta]
    checks = [(0, rng.normal(0, 1, I0.shape), g["I0"]), (1, rng.normal(0, 1, I1.shape), g["I1"])]
    checks += [(2, np.eye(3)[j], g["t"]) for j in range(3)]
    checks += [(3, np.eye(5)[j], g["theta"]) for j in range(5)]
    for i, d, gi in checks:
        h = {0: 1e-8, 1: 1e-8, 2: 1e-7, 3: 1e-5}[i]
        ap, am = list(base), list(base)
        ap[i] = base[i] + h * d
        am[i] = base[i] - h * d
        fd = (L(*ap) - L(*am)) / (2 * h)
        an = np.sum(gi * d)
        assert abs(fd - an) <= 1e-4 * max(1.0, abs(fd)), (i, fd, an)
