"""GPU: the reverse mode of the solve (vfs_grad_*, DepthSolver) against the
float64 reverse mode of oracle/np64/grad64.py on the same inputs."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import bench_params, pair

pytestmark = pytest.mark.gpu


def _problem(size=64, n_level=2, n_warp=3, n_iter=10, seed=0, t=(0.12, 0.01, 0.0)):
    P = pair(size, t=t, n_level=n_level, seed=seed)
    prm = bench_params(size, size, n_level=n_level, n_warp=n_warp, n_iter=n_iter)
    nz = np.random.default_rng(9)  # continuous images: no exact ties in the median windows
    I0 = (P.img_ref + nz.uniform(0, 1, P.img_ref.shape)).astype(np.float32)
    I1 = (P.img_other + nz.uniform(0, 1, P.img_other.shape)).astype(np.float32)
    return P, prm, I0, I1


def _solver(P, prm, ckpt=4, triangulation="reference"):
    from vfs_b200 import DepthSolver, EquidistantCam
    return DepthSolver(prm, EquidistantCam(P.intrinsics), P.mask, t_scale=1.0, ckpt_every=ckpt,
                       triangulation=triangulation)


def _theta(prm):
    return np.array([prm.Lambda, prm.alpha0, prm.alpha1, prm.beta, prm.gamma])


@pytest.mark.parametrize("triangulation", ["reference", "lsq"])
def test_grad_forward_is_the_plain_solve(triangulation):
    """The recording forward gives the drop-in solve's depth bit for bit."""
    from vfs_b200 import VFS, EquidistantCam
    from vfs_b200.vector_field import get_vector_fields, get_grid_zero
    P = pair(96, t=(0.12, 0.01, 0.0), n_level=3)
    prm = bench_params(96, 96, n_level=3, n_warp=3, n_iter=20)
    cam = EquidistantCam(P.intrinsics)
    tvf, cvf = get_vector_fields(get_grid_zero(P.img_ref.shape), cam, cam, np.eye(3), P.t, 1)
    v = VFS(prm)
    v.setup_module()
    v.compute_pyramid_sizes()
    v.create_mask_pyramid(P.mask)
    v.create_vector_field_pyramid(tvf, cvf)
    v.solve_stereo(P.img_ref, P.img_other)
    want = v.triangulate_flow(cam, P.t, method=triangulation)[..., 2].cpu().numpy()
    s = _solver(P, prm, ckpt=7, triangulation=triangulation)
    got = s.forward_pass(torch.as_tensor(P.img_ref).float().cuda(), torch.as_tensor(P.img_other).float().cuda(),
                         torch.tensor(P.t.reshape(3)), torch.tensor(_theta(prm))).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def _gpu_grads(s, I0, I1, t, theta, wts):
    d = s.forward_pass(torch.as_tensor(I0).cuda(), torch.as_tensor(I1).cuda(), torch.tensor(t), torch.tensor(theta))
    g_ref, g_other, g_t, g_th = s.backward_pass(torch.as_tensor(wts, dtype=torch.float32).cuda())
    torch.cuda.synchronize()
    return d.cpu().numpy(), g_ref.cpu().numpy(), g_other.cpu().numpy(), g_t.cpu().numpy(), g_th.cpu().numpy()


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


REL_TOL = 1e-3  # relative agreement asked of the gradients


@pytest.mark.parametrize("triangulation,t,size,levels,warps,iters,tol", [
    ("reference", (0.12, 0.01, 0.0), 64, 2, 3, 10, REL_TOL),
    ("lsq", (0.06, 0.1, 0.02), 64, 2, 3, 10, REL_TOL),
    # 256x256 through 3 levels x 3 warps x 20 iterations: measured 5.5e-3 (images), <= 8.2e-3 (theta)
    ("reference", (0.12, 0.01, 0.0), 256, 3, 3, 20, 1e-2),
])
def test_grad_matches_float64_reverse_mode(triangulation, t, size, levels, warps, iters, tol):
    """Same inputs, same cotangent: CUDA float32 gradients against the float64
    reverse mode run along the texture-quantised forward ("tex8"), for both
    triangulation rules (the least-squares one on a mostly vertical baseline)
    and for a 256x256 pair.

    The float64 forward reproduces the GPU's texture weights for 98 % of the
    samples, so the two trajectories differ slightly (median depth 4e-6
    relative at 256x256), and the unrolled solve's derivative is large (image
    gradients up to 1e6-1e8 at 256x256): the agreement of the gradients falls
    with the size of the solve.  Measured on a B200 (images / worst theta):
    64x64 2x3x10 1.3e-4 / 2.5e-4; 256x256 3x3x20 5.5e-3 / 8.2e-3; 3x3x10
    8.9e-3 / 3.1e-2; 3x5x50 0.12 / 1.4; 3x5x20 7.6 / 7.7 (gradients 1.7e8)."""
    from oracle.np64 import grad64 as G
    from oracle.np64 import vfs64 as V
    P, prm, I0, I1 = _problem(size=size, n_level=levels, n_warp=warps, n_iter=iters, t=t)
    t = P.t.reshape(3).astype(np.float64)
    theta = _theta(prm)
    s = _solver(P, prm, ckpt=4, triangulation=triangulation)
    d, g_ref, g_other, g_t, g_th = _gpu_grads(s, I0, I1, t, theta, np.zeros(I0.shape))
    good = (P.mask != 0) & np.isfinite(d) & (np.abs(d) < 30)
    prob = G.Problem(prm, V.EquidistantCam64(P.intrinsics), P.mask, triangulation=triangulation)
    d64, tape = G.solve(prob, I0 / 256.0, I1 / 256.0, t, theta, mode="tex8", tape=True)
    good &= np.isfinite(d64) & (np.abs(d64) < 30)  # plausible depth on both sides
    if triangulation == "lsq":
        # this baseline puts the epipole inside the image; beside it the rays
        # are nearly parallel (|r x o| ~ 2e-5), the depth gradient reaches 1e7
        # and float32 ray rounding alone moves it by 1 %: leave parallax below
        # 1 mrad out of the loss (40 of 1403 pixels here)
        grid = V.get_grid_zero(P.mask.shape)
        par = np.linalg.norm(np.cross(prob.cam.unproject(grid), prob.cam.unproject(grid + tape["warp"])), axis=-1)
        good &= par > 1e-3
    wts = np.where(good, np.random.default_rng(0).normal(0, 1, good.shape), 0.0)
    d, g_ref, g_other, g_t, g_th = _gpu_grads(s, I0, I1, t, theta, wts)
    g = G.backward(prob, tape, wts)
    for name, v in (("CUDA image", g_ref), ("CUDA other", g_other), ("CUDA t", g_t), ("CUDA theta", g_th),
                    ("float64 image", g["I0"]), ("float64 other", g["I1"]), ("float64 theta", g["theta"])):
        assert np.isfinite(v).all(), f"{name} gradient not finite at {np.count_nonzero(~np.isfinite(v))} entries"
    assert _rel(g_ref, g["I0"] / 256.0) < tol
    assert _rel(g_other, g["I1"] / 256.0) < tol
    for k in range(3):
        assert abs(g_t[k] - g["t"][k]) <= tol * np.abs(g["t"]).max(), (k, g_t, g["t"])
    for k in range(5):
        assert abs(g_th[k] - g["theta"][k]) <= tol * abs(g["theta"][k]), (k, g_th, g["theta"])


def test_grad_matches_float64_central_differences():
    """CUDA gradients of one scalar (alpha1) and of one pixel of each image
    against float64 central differences of the float64 forward.  One level
    and one warp: every texture fetch then samples at coordinates that do not
    depend on the inputs (the flow is zero while the derivatives are formed),
    so the texture-quantised forward is piecewise smooth in every input and
    its differences converge: at h = 1e-8 (images, u8 / 256 units) and 1e-5
    (alpha1), where the median, clamp, shrink and projection switches of the
    unrolled solve are not crossed."""
    from oracle.np64 import grad64 as G
    from oracle.np64 import vfs64 as V
    P, prm, I0, I1 = _problem(size=64, n_level=1, n_warp=1, n_iter=30)
    t = P.t.reshape(3).astype(np.float64)
    theta = _theta(prm)
    s = _solver(P, prm, ckpt=5)
    d = _gpu_grads(s, I0, I1, t, theta, np.zeros(I0.shape))[0]
    good = (P.mask != 0) & np.isfinite(d) & (np.abs(d) < 30)
    wts = np.where(good, np.random.default_rng(3).normal(0, 1, good.shape), 0.0)
    _, g_ref, g_other, _, g_th = _gpu_grads(s, I0, I1, t, theta, wts)
    prob = G.Problem(prm, V.EquidistantCam64(P.intrinsics), P.mask)
    A0, A1 = I0 / 256.0, I1 / 256.0
    L = lambda a0, a1, th: float(np.sum(np.where(good, wts * G.solve(prob, a0, a1, t, th, mode="tex8"), 0.0)))
    h = 1e-5
    e = np.eye(5)[2]
    fd = (L(A0, A1, theta + h * e) - L(A0, A1, theta - h * e)) / (2 * h)
    assert abs(g_th[2] - fd) <= REL_TOL * abs(fd), ("alpha1", g_th[2], fd)
    h = 1e-8
    for name, g, pick in (("I0", g_ref, 0), ("I1", g_other, 1)):
        y, x = np.unravel_index(np.argmax(np.abs(g)), g.shape)
        dA = np.zeros_like(A0)
        dA[y, x] = h
        args_p = [A0 + dA, A1, theta] if pick == 0 else [A0, A1 + dA, theta]
        args_m = [A0 - dA, A1, theta] if pick == 0 else [A0, A1 - dA, theta]
        fd = (L(*args_p) - L(*args_m)) / (2 * h) / 256.0  # per u8 unit, as the CUDA gradient
        assert abs(g[y, x] - fd) <= REL_TOL * abs(fd), (name, (y, x), g[y, x], fd)


def test_grad_independent_of_checkpoint_spacing():
    P, prm, I0, I1 = _problem(n_iter=9)
    t = P.t.reshape(3).astype(np.float64)
    theta = _theta(prm)
    s = _solver(P, prm)
    d = _gpu_grads(s, I0, I1, t, theta, np.zeros(I0.shape))[0]
    s.release()
    good = (P.mask != 0) & np.isfinite(d) & (np.abs(d) < 30)
    wts = np.where(good, np.random.default_rng(1).normal(0, 1, good.shape), 0.0) * 1e-3
    outs = []
    for ck in (1, 2, 4, 9, 100):
        s = _solver(P, prm, ckpt=ck)
        outs.append(_gpu_grads(s, I0, I1, t, theta, wts))
        s.release()
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0])
        for a, b in zip(o[1:], outs[0][1:]):
            assert _rel(a, b) < 1e-4


def test_autograd_function():
    P, prm, I0, I1 = _problem(n_warp=2, n_iter=6)
    s = _solver(P, prm, ckpt=3)
    a = torch.as_tensor(I0).cuda().requires_grad_()
    b = torch.as_tensor(I1).cuda().requires_grad_()
    t = torch.tensor(P.t.reshape(3), dtype=torch.float64, requires_grad=True)
    th = torch.tensor(_theta(prm), requires_grad=True)
    depth = s(a, b, t, th)
    m = torch.as_tensor(P.mask != 0).cuda() & torch.isfinite(depth) & (depth.abs() < 30)
    gt = torch.as_tensor(P.depth).cuda()
    loss = (depth - gt).abs()[m].mean()
    depth2 = s(a, b, t, th)  # a second forward: the first one's backward records its tape again
    loss.backward()
    assert torch.isfinite(a.grad).all() and torch.isfinite(b.grad).all()
    assert torch.isfinite(t.grad).all() and torch.isfinite(th.grad).all()
    g_depth = torch.zeros_like(depth)
    g_depth[m] = torch.sign((depth - gt)[m]) / m.sum()
    s.forward_pass(a.detach(), b.detach(), t.detach(), th.detach())
    g_ref, g_other, g_t, g_th = s.backward_pass(g_depth)
    assert _rel(a.grad.cpu().numpy(), g_ref.cpu().numpy()) < 1e-5
    assert _rel(th.grad.numpy(), g_th.cpu().numpy()) < 1e-5
    assert torch.equal(depth2, depth)


def test_backward_kernel_forms_agree():
    """Tiled and three-kernel reverse steps, recording and one-iteration
    recomputation: the same gradients (float atomics reorder sums only)."""
    P, prm, I0, I1 = _problem(n_iter=9)
    t = P.t.reshape(3).astype(np.float64)
    theta = _theta(prm)
    s = _solver(P, prm, ckpt=5)
    d = _gpu_grads(s, I0, I1, t, theta, np.zeros(I0.shape))[0]
    good = (P.mask != 0) & np.isfinite(d) & (np.abs(d) < 30)
    wts = np.where(good, np.random.default_rng(2).normal(0, 1, good.shape), 0.0) * 1e-3
    outs = []
    forms = [(0, -1), (1, -1), (0, 0), (1, 0), (1, 124), (1, 216), (1, 220), (1, 221), (1, 222), (1, 224), (2, 0), (3, 0),
             (4, 0), (5, 0)]
    forms += [(b, 0) for b in (11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 22, 23, 24, 25)]
    for fused, tv in forms:
        s.set_options(fused, tv)
        outs.append(_gpu_grads(s, I0, I1, t, theta, wts))
    s1 = _solver(P, prm, ckpt=1)  # every state recorded, no recomputation
    for fused in (1, 11, 14, 16):
        s1.set_options(fused, 0)
        outs.append(_gpu_grads(s1, I0, I1, t, theta, wts))
    s1.set_level_forms([16, 15])  # per-level forms
    outs.append(_gpu_grads(s1, I0, I1, t, theta, wts))
    for o in outs[1:]:
        for a, b in zip(o[1:], outs[0][1:]):
            assert _rel(a, b) < 1e-5


def test_checkpointing_sized_to_memory():
    """ckpt_every="auto" picks the densest spacing whose workspace fits the
    budget and gives the gradients of that spacing chosen by hand."""
    from vfs_b200 import DepthSolver, EquidistantCam, grad
    P, prm, I0, I1 = _problem(n_iter=9)
    t = P.t.reshape(3).astype(np.float64)
    theta = _theta(prm)
    budget = grad.workspace_bytes(prm, 5)
    auto = DepthSolver(prm, EquidistantCam(P.intrinsics), P.mask, ckpt_every="auto", memory_budget=budget)
    assert auto.ckpt_every == grad.checkpoint_interval(prm, budget) and auto.workspace_bytes <= budget
    d = _gpu_grads(auto, I0, I1, t, theta, np.zeros(I0.shape))[0]
    good = (P.mask != 0) & np.isfinite(d) & (np.abs(d) < 30)
    wts = np.where(good, np.random.default_rng(3).normal(0, 1, good.shape), 0.0) * 1e-3
    got = _gpu_grads(auto, I0, I1, t, theta, wts)
    want = _gpu_grads(_solver(P, prm, ckpt=auto.ckpt_every), I0, I1, t, theta, wts)
    for a, b in zip(got[1:], want[1:]):
        assert _rel(a, b) < 1e-5


@pytest.mark.parametrize("size,seed,n_iter,noisy", [(512, 6, 30, False), (256, 0, 50, True)])
def test_grad_finite_next_to_nan_flow(size, seed, n_iter, noisy):
    """On these pairs the forward flow is NaN at a few pixels (41 at 512x512,
    10 at 256x256) beside the epipole of t = (0.1, 0, 0), as with the
    reference's own kernels (the epipolar direction is undefined there).
    With the depth loss restricted to plausible depths the gradients stay
    finite: transposed fetches give non-finite coordinates zero weight, and
    the reverse kernels drop non-finite cotangent contributions (a NaN state
    would otherwise carry NaN to every cotangent through the stencil; at
    256x256 with 250 iterations per level it did)."""
    from vfs_b200 import DepthSolver, EquidistantCam
    P = pair(size, t=(0.1, 0.0, 0.0), seed=seed, n_level=3)
    prm = bench_params(size, size, n_level=3, n_warp=5, n_iter=n_iter)
    s = DepthSolver(prm, EquidistantCam(P.intrinsics), P.mask, ckpt_every=10)
    I0, I1 = P.img_ref.astype(np.float32), P.img_other.astype(np.float32)
    if noisy:  # the images of the 256x256 gradient comparison (sub-u8 noise)
        nz = np.random.default_rng(9)
        I0 = (P.img_ref + nz.uniform(0, 1, P.img_ref.shape)).astype(np.float32)
        I1 = (P.img_other + nz.uniform(0, 1, P.img_other.shape)).astype(np.float32)
    a = torch.as_tensor(I0).cuda()
    b = torch.as_tensor(I1).cuda()
    t = torch.tensor(P.t.reshape(3), dtype=torch.float64)
    d = s.forward_pass(a, b, t, torch.tensor(_theta(prm)))
    assert int(torch.isnan(d).sum()) > 0  # the case this test is about
    gt = torch.as_tensor(P.depth).cuda()
    m = torch.as_tensor(P.mask != 0).cuda() & torch.isfinite(d) & (d > 0) & (d < 50)
    g = torch.where(m, torch.sign(d - gt), torch.zeros_like(d)) / m.sum()
    for r in s.backward_pass(g):
        assert torch.isfinite(r).all()
