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
