"""Test infrastructure: float64 reverse mode of the TGV solver iterations.

The forward is oracle/np64/vfs64.py's (the reference's updateDualVariables ->
l1Thresholding -> updatePrimalVariables, Python/vfs.cu:326-581); here each
iteration's vector-Jacobian product is written out by hand, taking the active
branch at the non-smooth points (the unit-ball projections, the three-case
L1 shrink).  It is checked against float64 finite differences in the CPU
tests and serves as the specification the CUDA adjoint is tested against.

State of an iteration: u, ub (u_), v (v_, 2), p (2), q (4).  Per-warp
constants: abc (3), eta (3), deriv (Iu, Iz), the mask.  Parameters:
Lambda, alpha0, alpha1.
"""
from __future__ import annotations

import numpy as np

from .vfs64 import flat_get, mask_neighbours

EPS = 1e-7


def _scatter(g, off, val):
    """g.flat[i + off] += val[i] for in-buffer targets (the transpose of flat_get)."""
    H, W = g.shape[:2]
    n = H * W
    gf = g.reshape(n, -1)
    vf = val.reshape(n, -1)
    idx = np.arange(n) + off
    ok = (idx >= 0) & (idx < n)
    np.add.at(gf, idx[ok], vf[ok])


def iteration_forward(st, cst, prm, sigma, tau, mu, M):
    """One iteration with every intermediate the reverse needs."""
    u, ub, v, p, q = st["u"], st["ub"], st["v"], st["p"], st["q"]
    abc, eta, deriv = cst["abc"], cst["eta"], cst["deriv"]
    Mb, mE, mW, mS, mN = mask_neighbours(M)
    W = u.shape[1]
    a, b, c = abc[..., 0], abc[..., 1], abc[..., 2]
    vx, vy = v[..., 0], v[..., 1]
    uE, uW, uS, uN = flat_get(ub, 1), flat_get(ub, -1), flat_get(ub, W), flat_get(ub, -W)
    vE, vW, vS, vN = flat_get(v, 1), flat_get(v, -1), flat_get(v, W), flat_get(v, -W)
    gUx = np.where(mE, uE - ub - vx, ub - uW - vx)
    gVx = np.where(mE, vE[..., 0] - vx, vx - vW[..., 0])
    gVw = np.where(mE, vE[..., 1] - vy, vy - vW[..., 1])
    gUy = np.where(mS, uS - ub - vy, ub - uN - vy)
    gVy = np.where(mS, vS[..., 1] - vy, vy - vN[..., 1])
    gVz = np.where(mS, vS[..., 0] - vx, vx - vN[..., 0])
    tux = a * gUx + c * gUy
    tuy = c * gUx + b * gUy
    sP = prm.alpha1 * sigma / 3.0
    sQ = prm.alpha0 * sigma / 2.0
    P = np.stack([p[..., 0] + sP * tux, p[..., 1] + sP * tuy], -1)
    nP = np.maximum(np.hypot(P[..., 0], P[..., 1]), 1.0)
    pn = P / nP[..., None]
    gV = np.stack([gVx, gVy, gVz, gVw], -1)
    Q = q + sQ * gV
    nQ = np.maximum(np.sqrt((Q * Q).sum(-1)), 1.0)
    qn = Q / nQ[..., None]
    m2 = Mb[..., None]
    pn = np.where(m2, pn, 0.0)
    qn = np.where(m2, qn, 0.0)
    tp = np.where(m2, np.stack([a * pn[..., 0] + c * pn[..., 1], c * pn[..., 0] + b * pn[..., 1]], -1), 0.0)
    # threshold
    tpW = flat_get(tp, -1)
    tpN = flat_get(tp, -W)
    gTx = np.where(mE & mW, tp[..., 0] - tpW[..., 0], np.where(~mE, -tpW[..., 0], tp[..., 0]))
    gTy = np.where(mS & mN, tp[..., 1] - tpN[..., 1], np.where(~mS, -tpN[..., 1], tp[..., 1]))
    Iu, Iz = deriv[..., 0], deriv[..., 1]
    small_ex = np.abs(eta[..., 0]) < EPS
    with np.errstate(divide="ignore", invalid="ignore"):
        te = np.where(small_ex, tau, tau / eta[..., 0])
    ut = ub + te * (gTx + gTy)
    rho = Iu * (ut - u) + Iz
    B = prm.Lambda * te * Iu * Iu
    mid = (rho <= B) & (rho >= -B)
    lo = rho < -B
    hi = rho > B
    small_iu = np.abs(Iu) < EPS
    with np.errstate(divide="ignore", invalid="ignore"):
        un = np.where(mid, np.where(small_iu, ut, ut - rho / Iu),
                      np.where(lo, ut + prm.Lambda * te * Iu, np.where(hi, ut - prm.Lambda * te * Iu, u)))
    un = np.where(Mb, un, 0.0)
    # primal
    qW = flat_get(qn, -1)
    qN = flat_get(qn, -W)
    gQx = np.where(mE, qn[..., 0], 0.0) - np.where(mW, qW[..., 0], 0.0)
    gQw = np.where(mE, qn[..., 3], 0.0) - np.where(mW, qW[..., 3], 0.0)
    gQy = np.where(mS, qn[..., 1], 0.0) - np.where(mN, qN[..., 1], 0.0)
    gQz = np.where(mS, qn[..., 2], 0.0) - np.where(mN, qN[..., 2], 0.0)
    small_ey = np.abs(eta[..., 1]) < EPS
    small_ez = np.abs(eta[..., 2]) < EPS
    with np.errstate(divide="ignore", invalid="ignore"):
        t1 = np.where(small_ey, tau, tau / eta[..., 1])
        t2 = np.where(small_ez, tau, tau / eta[..., 2])
    tu2x, tu2y = tp[..., 0], tp[..., 1]
    Vx = vx + t1 * (prm.alpha1 * tu2x + prm.alpha0 * (gQx + gQz))
    Vy = vy + t2 * (prm.alpha1 * tu2y + prm.alpha0 * (gQw + gQy))
    ubn = np.where(Mb, un + mu * (un - ub), 0.0)
    vbn = np.where(m2, np.stack([Vx + mu * (Vx - vx), Vy + mu * (Vy - vy)], -1), 0.0)
    out = {"u": un, "ub": ubn, "v": vbn, "p": pn, "q": qn}
    inter = dict(mE=mE, mW=mW, mS=mS, mN=mN, Mb=Mb, gUx=gUx, gUy=gUy, gV=gV, tux=tux, tuy=tuy, sP=sP, sQ=sQ,
                 P=P, nP=nP, pn=pn, Q=Q, nQ=nQ, qn=qn, tp=tp, gTx=gTx, gTy=gTy, te=te, small_ex=small_ex, ut=ut,
                 rho=rho, mid=mid, lo=lo, hi=hi, small_iu=small_iu, gQx=gQx, gQy=gQy, gQz=gQz, gQw=gQw, t1=t1,
                 t2=t2, small_ey=small_ey, small_ez=small_ez, Vx=Vx, Vy=Vy)
    return out, inter


def iteration_reverse(st, cst, prm, sigma, tau, mu, M, inter, g_out):
    """Vector-Jacobian product of one iteration.  g_out holds the adjoints of
    the outputs (u, ub, v, p, q); returns the adjoints of the inputs and of
    the constants and parameters (dict)."""
    u, ub, v = st["u"], st["ub"], st["v"]
    abc, eta, deriv = cst["abc"], cst["eta"], cst["deriv"]
    a, b, c = abc[..., 0], abc[..., 1], abc[..., 2]
    Iu, Iz = deriv[..., 0], deriv[..., 1]
    I = inter
    W = u.shape[1]
    Mb = I["Mb"]
    gu_in = np.zeros_like(u)
    gub_in = np.zeros_like(ub)
    gv_in = np.zeros_like(v)
    gp_in = np.zeros_like(st["p"])
    gq_in = np.zeros_like(st["q"])
    g_abc = np.zeros_like(abc)
    g_eta = np.zeros_like(eta)
    g_deriv = np.zeros_like(deriv)
    g = {"Lambda": 0.0, "alpha0": 0.0, "alpha1": 0.0}

    # ---- primal reverse
    gubn = np.where(Mb, g_out["ub"], 0.0)
    gvbn = np.where(Mb[..., None], g_out["v"], 0.0)
    gun = np.where(Mb, g_out["u"], 0.0) + (1 + mu) * gubn
    gub_in += -mu * gubn
    gVx = (1 + mu) * gvbn[..., 0]
    gVy = (1 + mu) * gvbn[..., 1]
    gv_in[..., 0] += gVx - mu * gvbn[..., 0]
    gv_in[..., 1] += gVy - mu * gvbn[..., 1]
    inner_x = prm.alpha1 * I["tp"][..., 0] + prm.alpha0 * (I["gQx"] + I["gQz"])
    inner_y = prm.alpha1 * I["tp"][..., 1] + prm.alpha0 * (I["gQw"] + I["gQy"])
    gt1 = inner_x * gVx
    gt2 = inner_y * gVy
    g_tp = np.zeros_like(I["tp"])
    g_tp[..., 0] += I["t1"] * prm.alpha1 * gVx
    g_tp[..., 1] += I["t2"] * prm.alpha1 * gVy
    g["alpha1"] += np.sum(I["t1"] * I["tp"][..., 0] * gVx + I["t2"] * I["tp"][..., 1] * gVy)
    g["alpha0"] += np.sum(I["t1"] * (I["gQx"] + I["gQz"]) * gVx + I["t2"] * (I["gQw"] + I["gQy"]) * gVy)
    ggQx = I["t1"] * prm.alpha0 * gVx
    ggQz = ggQx
    ggQw = I["t2"] * prm.alpha0 * gVy
    ggQy = ggQw
    with np.errstate(divide="ignore", invalid="ignore"):
        g_eta[..., 1] += np.where(I["small_ey"], 0.0, -I["t1"] / eta[..., 1] * gt1)
        g_eta[..., 2] += np.where(I["small_ez"], 0.0, -I["t2"] / eta[..., 2] * gt2)
    g_qn = np.zeros_like(I["qn"])
    g_qn[..., 0] += np.where(I["mE"], ggQx, 0.0)
    g_qn[..., 3] += np.where(I["mE"], ggQw, 0.0)
    g_qn[..., 1] += np.where(I["mS"], ggQy, 0.0)
    g_qn[..., 2] += np.where(I["mS"], ggQz, 0.0)
    sW = np.zeros_like(I["qn"])
    sW[..., 0] = np.where(I["mW"], -ggQx, 0.0)
    sW[..., 3] = np.where(I["mW"], -ggQw, 0.0)
    _scatter(g_qn, -1, sW)
    sN = np.zeros_like(I["qn"])
    sN[..., 1] = np.where(I["mN"], -ggQy, 0.0)
    sN[..., 2] = np.where(I["mN"], -ggQz, 0.0)
    _scatter(g_qn, -W, sN)

    # ---- threshold reverse
    mid, lo, hi = I["mid"], I["lo"], I["hi"]
    small_iu = I["small_iu"]
    te = I["te"]
    gut = np.zeros_like(u)
    gte = np.zeros_like(u)
    # middle band, |Iu| >= eps: un = u - Iz / Iu (the expression's value)
    m_mid = Mb & mid & ~small_iu
    with np.errstate(divide="ignore", invalid="ignore"):
        gu_in += np.where(m_mid, gun, 0.0)
        g_deriv[..., 1] += np.where(m_mid, -gun / Iu, 0.0)
        g_deriv[..., 0] += np.where(m_mid, gun * Iz / (Iu * Iu), 0.0)
    m_mid0 = Mb & mid & small_iu
    gut += np.where(m_mid0, gun, 0.0)
    m_lo = Mb & ~mid & lo
    m_hi = Mb & ~mid & ~lo & hi
    m_none = Mb & ~mid & ~lo & ~hi  # NaN comparisons: un = u
    gu_in += np.where(m_none, gun, 0.0)
    sgn = np.where(m_lo, 1.0, np.where(m_hi, -1.0, 0.0))
    m_lh = m_lo | m_hi
    gut += np.where(m_lh, gun, 0.0)
    g["Lambda"] += np.sum(np.where(m_lh, sgn * te * Iu * gun, 0.0))
    gte += np.where(m_lh, sgn * prm.Lambda * Iu * gun, 0.0)
    g_deriv[..., 0] += np.where(m_lh, sgn * prm.Lambda * te * gun, 0.0)
    # ut = ub + te * (gTx + gTy)
    gub_in += gut
    gte += (I["gTx"] + I["gTy"]) * gut
    ggT = te * gut
    with np.errstate(divide="ignore", invalid="ignore"):
        g_eta[..., 0] += np.where(I["small_ex"], 0.0, -te / eta[..., 0] * gte)
    mE, mW, mS, mN = I["mE"], I["mW"], I["mS"], I["mN"]
    g_tp[..., 0] += np.where(mE & mW, ggT, np.where(~mE, 0.0, ggT))
    sx = np.where(mE & mW, -ggT, np.where(~mE, -ggT, 0.0))
    g_tp[..., 1] += np.where(mS & mN, ggT, np.where(~mS, 0.0, ggT))
    sy = np.where(mS & mN, -ggT, np.where(~mS, -ggT, 0.0))
    s = np.zeros_like(I["tp"])
    s[..., 0] = sx
    _scatter(g_tp, -1, s)
    s = np.zeros_like(I["tp"])
    s[..., 1] = sy
    _scatter(g_tp, -W, s)

    # ---- dual reverse
    m2 = Mb[..., None]
    g_tp = np.where(m2, g_tp, 0.0)
    g_qn = np.where(m2, g_qn, 0.0)
    pn = I["pn"]
    g_pn = np.where(m2, g_out["p"], 0.0)
    g_pn[..., 0] += a * g_tp[..., 0] + c * g_tp[..., 1]
    g_pn[..., 1] += c * g_tp[..., 0] + b * g_tp[..., 1]
    g_abc[..., 0] += pn[..., 0] * g_tp[..., 0]
    g_abc[..., 1] += pn[..., 1] * g_tp[..., 1]
    g_abc[..., 2] += pn[..., 1] * g_tp[..., 0] + pn[..., 0] * g_tp[..., 1]
    g_qn = g_qn + np.where(m2, g_out["q"], 0.0)

    def proj_rev(X, nX, xn, gxn):
        inside = nX <= 1.0
        dot = np.sum(xn * gxn, -1, keepdims=True)
        return np.where(inside[..., None], gxn, (gxn - xn * dot) / nX[..., None])

    gP = proj_rev(I["P"], I["nP"], pn, g_pn)
    gQ = proj_rev(I["Q"], I["nQ"], I["qn"], g_qn)
    gp_in += gP
    gq_in += gQ
    ggV = I["sQ"] * gQ
    g["alpha0"] += np.sum(sigma / 2.0 * np.sum(I["gV"] * gQ, -1))
    gtux = I["sP"] * gP[..., 0]
    gtuy = I["sP"] * gP[..., 1]
    g["alpha1"] += np.sum(sigma / 3.0 * (I["tux"] * gP[..., 0] + I["tuy"] * gP[..., 1]))
    ggUx = a * gtux + c * gtuy
    ggUy = c * gtux + b * gtuy
    g_abc[..., 0] += I["gUx"] * gtux
    g_abc[..., 1] += I["gUy"] * gtuy
    g_abc[..., 2] += I["gUy"] * gtux + I["gUx"] * gtuy
    # gU, gV from ub and v at the pixel and its neighbours
    ggVx, ggVy, ggVz, ggVw = ggV[..., 0], ggV[..., 1], ggV[..., 2], ggV[..., 3]
    gvx = -ggUx  # gUx has -vx
    gvy = -ggUy
    # E/W branch
    gub_in += np.where(mE, -ggUx, ggUx)
    _scatter(gub_in, 1, np.where(mE, ggUx, 0.0))
    _scatter(gub_in, -1, np.where(mE, 0.0, -ggUx))
    gvx += np.where(mE, -ggVx, ggVx)
    gvy += np.where(mE, -ggVw, ggVw)
    sE = np.stack([np.where(mE, ggVx, 0.0), np.where(mE, ggVw, 0.0)], -1)
    sW2 = np.stack([np.where(mE, 0.0, -ggVx), np.where(mE, 0.0, -ggVw)], -1)
    _scatter(gv_in, 1, sE)
    _scatter(gv_in, -1, sW2)
    # S/N branch
    gub_in += np.where(mS, -ggUy, ggUy)
    _scatter(gub_in, W, np.where(mS, ggUy, 0.0))
    _scatter(gub_in, -W, np.where(mS, 0.0, -ggUy))
    gvy += np.where(mS, -ggVy, ggVy)
    gvx += np.where(mS, -ggVz, ggVz)
    sS = np.stack([np.where(mS, ggVz, 0.0), np.where(mS, ggVy, 0.0)], -1)
    sN2 = np.stack([np.where(mS, 0.0, -ggVz), np.where(mS, 0.0, -ggVy)], -1)
    _scatter(gv_in, W, sS)
    _scatter(gv_in, -W, sN2)
    gv_in[..., 0] += np.where(Mb, gvx, 0.0)
    gv_in[..., 1] += np.where(Mb, gvy, 0.0)
    return {"u": gu_in, "ub": gub_in, "v": gv_in, "p": gp_in, "q": gq_in, "abc": g_abc, "eta": g_eta,
            "deriv": g_deriv, **g}
