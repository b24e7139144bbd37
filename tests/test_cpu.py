"""CPU tests: the C ABI's host side, the step schedule, and the float64 oracle
pinned against golden outputs of the reference's own kernels.

No GPU is used.  tests/golden/ref_small.npz was produced on a B200 by
tests/golden/make_golden.py from the reference's CUDA kernels (built from its
sources) with the reference's host call order.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from helpers import bench_params, default_params, pair
from vfs_b200.synthetic import make_pair

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "vfs_b200.h")
GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_small.npz")


@pytest.fixture(scope="module")
def lib():
    from vfs_b200 import _lib
    return _lib


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLDEN))


# ---------------------------------------------------------------- C ABI, host side
def test_library_exports_every_header_symbol(lib):
    declared = re.findall(r"VFS_API\s+(?:int|size_t|const char\*|VfsPlan\*)\s+(vfs_\w+)", open(HEADER).read())
    assert len(declared) >= 40
    out = subprocess.run(["nm", "-D", "--defined-only", lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert sorted(set(declared) - exported) == []
    assert sorted(exported - set(declared)) == []
    L = lib.lib()
    for name in declared:
        assert hasattr(L, name)


def test_step_schedule_matches_reference_numpy_rules(lib):
    from oracle.np64.vfs64 import step_schedule
    for n, tsl in [(100, 1.0), (50, 1.0), (7, 0.3), (3000, 3.0)]:
        out = np.zeros(3 * n, np.float32)
        lib.call("vfs_step_schedule", n, tsl, out.ctypes.data)
        want = np.array(step_schedule(n, tsl), np.float32).reshape(-1)
        assert np.array_equal(out.view(np.uint32), want.view(np.uint32))


def _prm(lib, **kw):
    p = bench_params(64, 80, n_level=3)
    for k, v in kw.items():
        setattr(p, k, v)
    return lib.VfsParams.from_param_bag(p)


def test_workspace_size_and_parameter_validation(lib):
    n = ctypes.c_size_t(0)
    lib.call("vfs_plan_workspace_size", ctypes.byref(_prm(lib)), ctypes.byref(n))
    small = n.value
    lib.call("vfs_plan_workspace_size", ctypes.byref(_prm(lib, width=800, height=800)), ctypes.byref(n))
    assert n.value > 50 * small
    for bad in (dict(width=0), dict(nLevel=0), dict(fScale=1.0), dict(nSolverIters=-1), dict(Lambda=float("nan")),
                dict(nLevel=12)):  # 64 / 2**11 == 0: a level of size zero
        with pytest.raises(ValueError):
            lib.call("vfs_plan_workspace_size", ctypes.byref(_prm(lib, **bad)), ctypes.byref(n))


def test_plan_create_rejects_missing_workspace(lib):
    plan = ctypes.c_void_p(0)
    rc = lib.lib().vfs_plan_create(ctypes.byref(_prm(lib)), None, 0, ctypes.byref(plan))
    assert rc == lib.VFS_ERR_WORKSPACE
    assert "workspace of" in lib.lib().vfs_last_error().decode()


def test_static_solve_rejects_oversize_before_touching_cuda(lib):
    p = lib.VfsParams.from_param_bag(bench_params(2048, 2048, n_level=5, n_warp=1, n_iter=1))
    dummy = ctypes.c_void_p(16)
    rc = lib.lib().vfs_solve_stereo_static(ctypes.byref(p), dummy, 2048, dummy, dummy, dummy, dummy, dummy, None)
    assert rc == lib.VFS_ERR_WORKSPACE


def test_null_arguments_are_rejected(lib):
    rc = lib.lib().vfs_cast_and_scale(None, None, 4, 4, None)
    assert rc == lib.VFS_ERR_ARG
    # texture bases must be 512-byte aligned and pitches multiples of 32 bytes
    # covering a row; both are checked before any CUDA call
    tex = ctypes.c_uint64()
    rc = lib.lib().vfs_texture_create(ctypes.c_void_p(0x1100), 4, 4, 64, 2, 1, ctypes.byref(tex))
    assert rc == lib.VFS_ERR_ALIGN
    rc = lib.lib().vfs_texture_create(ctypes.c_void_p(0x1000), 4, 8, 20, 2, 1, ctypes.byref(tex))
    assert rc == lib.VFS_ERR_ALIGN
    rc = lib.lib().vfs_texture_create(ctypes.c_void_p(0x1000), 4, 8, 32, 7, 1, ctypes.byref(tex))
    assert rc == lib.VFS_ERR_ARG


def test_synthetic_pairs_are_deterministic():
    a = pair(64, seed=3)
    b = pair(64, seed=3)
    c = pair(64, seed=4)
    assert np.array_equal(a.img_ref, b.img_ref) and np.array_equal(a.img_other, b.img_other)
    assert not np.array_equal(a.img_ref, c.img_ref)
    assert a.img_ref.dtype == np.uint8 and a.mask.max() == 255


def test_least_squares_triangulation_arguments_are_checked_on_the_host(lib):
    """The least-squares entry points and options validate their arguments
    before any CUDA call."""
    L = lib.lib()
    t = (ctypes.c_float * 3)(0.1, 0.0, 0.0)
    d = ctypes.c_void_p(16)
    assert L.vfs_triangulate_rays_lsq(None, d, d, t, d, 8, 4, 4, None) == lib.VFS_ERR_ARG
    assert L.vfs_triangulate_rays_lsq(d, d, d, None, d, 8, 4, 4, None) == lib.VFS_ERR_ARG
    assert L.vfs_plan_triangulate_lsq(None, 1.0, 0.0, 0.0, t, d, None) == lib.VFS_ERR_ARG
    assert L.vfs_batch_triangulate_lsq(None, 0, 1.0, 0.0, 0.0, t, d, None) == lib.VFS_ERR_ARG
    assert L.vfs_grad_set_triangulation(None, 1) == lib.VFS_ERR_ARG
    from vfs_b200 import DepthSolver
    with pytest.raises(ValueError):
        DepthSolver(bench_params(16, 16, n_level=1), (10.0, 8.0, 8.0), np.zeros((16, 16), np.uint8),
                    triangulation="midpoint")
    from vfs_b200.vfs import VFS
    with pytest.raises(ValueError):
        VFS.triangulate_flow(object(), None, (0.1, 0, 0), method="midpoint")
    from vfs_b200.batch import VFSBatch
    with pytest.raises(ValueError):
        VFSBatch.triangulate(object(), 0, None, (0.1, 0, 0), method="midpoint")


def test_synthetic_rotation_is_undone_by_the_calibration_field():
    """A rotated second view, warped by the reference's calibration field
    (cvf = project(R X) - grid, Python/vector_field.py:50-54, applied as in
    Python/vfs.py:150-153), matches the unrotated second view of the same scene."""
    from oracle.np64 import vfs64 as V
    from vfs_b200.synthetic import rotation_xyz
    n = 96
    R = rotation_xyz(0.03, -0.04, 0.02)
    a = pair(n, t=(0.1, 0.02, 0.0), seed=3)
    b = make_pair(n, (0.1, 0.02, 0.0), seed=3, R=R)
    assert np.array_equal(a.img_ref, b.img_ref) and np.array_equal(b.R, R)
    cam = V.EquidistantCam64(b.intrinsics)
    tvf_a, cvf_a = V.get_vector_fields(V.get_grid_zero((n, n)), cam, cam, a.R, a.t, 1)
    tvf_b, cvf_b = V.get_vector_fields(V.get_grid_zero((n, n)), cam, cam, b.R, b.t, 1)
    assert np.abs(cvf_a).max() < 1e-9 and np.abs(cvf_b).max() > 1.0
    assert np.array_equal(tvf_a, tvf_b)  # the translation field ignores R
    calib = V.warping_image(b.img_other.astype(np.float64), cvf_b)
    inner = a.mask != 0
    diff = np.abs(calib - a.img_other)[inner]
    unrelated = np.abs(b.img_other.astype(np.float64) - a.img_other)[inner]
    assert diff.mean() < 4.0 and unrelated.mean() > 4 * diff.mean(), (diff.mean(), unrelated.mean())


def test_lsq_triangulation_recovers_points_for_any_baseline():
    """The least-squares option recovers exact points for every baseline
    direction; the reference's x-only formula (Python/vfs.cu:728-734) is exact
    only while t.x dominates and fails for a vertical baseline."""
    from oracle.np64 import vfs64 as V
    rng = np.random.default_rng(0)
    n = 2000
    d = rng.normal(size=(n, 3))
    d[:, 2] = np.abs(d[:, 2]) + 0.2
    X = d / np.linalg.norm(d, axis=1, keepdims=True) * rng.uniform(1, 10, (n, 1))
    M = np.ones(n, np.uint8)
    unit = lambda v: v / np.linalg.norm(v, axis=-1, keepdims=True)
    for t in [(0.1, 0.0, 0.0), (0.12, 0.01, 0.0), (0.0, 0.1, 0.0), (0.03, -0.05, 0.08)]:
        t = np.asarray(t)
        r, o = unit(X), unit(X + t)
        got = V.triangulate_rays_lsq(r, o, t, M)
        assert np.allclose(got, X, rtol=1e-9, atol=0), t
        ref = V.triangulate_rays(r, o, t, M)
        if t[0] != 0:
            assert np.allclose(ref, X, rtol=1e-6, atol=0), t
        else:
            assert not np.allclose(ref, X, rtol=1e-2, atol=0, equal_nan=False)
    # masked pixels take the reference's (0, 0, -1)
    M[:3] = 0
    out = V.triangulate_rays_lsq(unit(X), unit(X + 0.1), np.full(3, 0.1), M)
    assert np.array_equal(out[:3], np.tile([0.0, 0.0, -1.0], (3, 1)))


# ---------------------------------------------------------------- oracle vs golden
def _within(a, b, atol, frac=1.0, what=""):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, what
    ok = np.abs(a - b) <= atol
    assert ok.mean() >= frac, f"{what}: {100 * (1 - ok.mean()):.3f}% beyond {atol}, max {np.abs(a - b).max()}"


def test_oracle_mask_pyramid_exact(gold):
    from oracle.np64 import vfs64 as V
    m = gold["mask_0"]
    for k in (1, 2):
        h, w = gold[f"mask_{k}"].shape
        got = V.down_sampling_mask(gold[f"mask_{k - 1}"], h, w)
        assert np.array_equal(got, gold[f"mask_{k}"]), f"mask level {k}"
    assert np.array_equal(m, gold["mask"])


def test_oracle_pyramids(gold):
    from oracle.np64 import vfs64 as V
    for k in (1, 2):
        h, w = gold[f"ref_{k}"].shape
        _within(V.down_sampling(gold[f"ref_{k - 1}"], h, w, "tex8"), gold[f"ref_{k}"], 2e-3, what=f"ref {k}")
        _within(V.down_sampling(gold[f"other_{k - 1}"], h, w, "tex8"), gold[f"other_{k}"], 2e-3, what=f"other {k}")
        _within(V.down_sampling(gold[f"tvf_{k - 1}"], h, w, "tex8"), gold[f"tvf_{k}"], 2e-3, what=f"tvf {k}")
    _within(V.cast_and_scale(gold["img_ref"]), gold["ref_0"], 0, what="castAndScale")
    _within(V.warping_image(V.cast_and_scale(gold["img_other"]), gold["cvf"], "tex8"), gold["other_0"], 2e-3,
            what="calibration warp")


@pytest.mark.parametrize("k", [0, 1])
def test_oracle_step_kernels(gold, k):
    from oracle.np64 import vfs64 as V
    prm = bench_params(*gold[f"ref_{k}"].shape, n_level=3)
    M = gold[f"mask_{k}"]
    g = lambda n: gold[f"L{k}_out_{n}"]
    i = lambda n: gold[f"L{k}_in_{n}"].astype(np.float64)
    _within(V.gaussian_masked(gold[f"ref_{k}"], M, "tex8"), g("smooth"), 1e-6, what="gaussian")
    abc, eta = V.compute_tensor_eta(g("smooth"), M, prm, "tex8")
    _within(abc, g("abc"), 2e-5, what="tensor")
    _within(eta, g("eta"), 2e-5 * np.abs(g("eta")).max(), what="eta")
    _within(V.find_warping_vector(gold[f"tvf_{k}"], i("warp"), "tex8"), g("tvec"), 2e-3, what="findWarpingVector")
    _within(V.warping_image(gold[f"other_{k}"], i("warp"), "tex8"), g("warped"), 3e-3, what="warpingImage")
    d = V.compute_derivatives(gold[f"ref_{k}"], g("warped"), gold[f"tvf_{k}"], "tex8")
    _within(d, g("deriv"), 3e-3, frac=0.999, what="computeDerivatives")
    sigma, tau, mu = (float(v) for v in gold[f"L{k}_sched"])
    # the solver steps have no texture reads: float64 vs float32 on identical inputs
    p, tp, q = V.update_dual_variables(i("p"), i("q"), sigma, i("ub"), i("vb"), g("abc"), M, prm)
    _within(p, g("p"), 1e-5, what="dual p")
    _within(tp, g("tp"), 1e-5, what="dual tp")
    _within(q, g("q"), 1e-5, what="dual q")
    u = V.l1_thresholding(tau, g("tp"), i("u"), i("ub"), g("deriv"), g("eta"), M, prm)
    _within(u, g("u"), 1e-4, frac=0.999, what="threshold")
    ub, vb = V.update_primal_variables(tau, mu, g("p"), g("q"), g("u"), i("ub"), i("vb"), g("abc"), g("eta"), M, prm)
    _within(ub, g("ub"), 1e-4, what="primal u_")
    _within(vb, g("vb"), 1e-4, what="primal v_")
    med = V.median_filter(g("u").astype(np.float64), M)
    assert np.array_equal(med.astype(np.float32), g("median"))
    warp = i("warp").copy()
    ubf = i("ub").copy()
    V.compute_optical_flow_with_clamp(warp, ubf, g("median").astype(np.float64), g("tvec").astype(np.float64), M,
                                      prm)
    _within(warp, g("clamp_warp"), 1e-5, what="clamp warp")
    _within(ubf, g("clamp_u"), 1e-5, what="clamp u")
    if k > 0:
        fh, fw = gold[f"ref_{k - 1}"].shape
        _within(V.upsampling(g("clamp_u"), fh, fw, 2.0, "tex8"), g("up1"), 1e-5, what="upsample1")
        _within(V.upsampling(g("clamp_warp"), fh, fw, 2.0, "tex8"), g("up2"), 1e-5, what="upsample2")


def test_oracle_camera(gold):
    from oracle.np64 import vfs64 as V
    cam = V.EquidistantCam64(gold["intrinsics"])
    h, w = gold["mask"].shape
    _within(cam.get_rays((h, w)), gold["cam_rays"], 2e-6, what="rays")
    xyz = cam.unproject(gold["cam_uv_in"].astype(np.float64))
    _within(xyz, gold["cam_xyz"], 2e-6, what="getXYZFromUV")
    _within(cam.project(gold["cam_xyz"].astype(np.float64)), gold["cam_uv"], 2e-4, what="getUVFromXYZ")


def test_oracle_end_to_end_default_params(gold):
    """The whole reference-default solve (Lambda 5, fScale 1.2) in float64 stays
    close to the reference kernels' float32 result."""
    from oracle.np64 import vfs64 as V
    h, w = gold["mask"].shape
    prm = default_params(h, w, n_level=4, n_warp=2, n_iter=9)
    v = V.VFS64(prm, "tex8")
    v.compute_pyramid_sizes()
    v.create_mask_pyramid(gold["mask"])
    v.create_vector_field_pyramid(gold["tvf"], gold["cvf"])
    warp = v.solve_stereo(gold["img_ref"], gold["img_other"])
    m = gold["mask"] > 0
    d = np.abs(warp - gold["e2e_default_warp"])[m]
    assert np.median(d) < 1e-3 and np.percentile(d, 99) < 0.05, (np.median(d), np.percentile(d, 99))


def test_grad_workspace_size_and_validation(lib):
    """Reverse-mode plan sizing (no GPU needed): recording every state costs
    about ckpt_every times the checkpointed tape; bad arguments are rejected
    before any CUDA call."""
    n1, n10 = ctypes.c_size_t(0), ctypes.c_size_t(0)
    prm = _prm(lib)
    lib.call("vfs_grad_workspace_size", ctypes.byref(prm), 1, ctypes.byref(n1))
    lib.call("vfs_grad_workspace_size", ctypes.byref(prm), 10, ctypes.byref(n10))
    plan = ctypes.c_size_t(0)
    lib.call("vfs_plan_workspace_size", ctypes.byref(prm), ctypes.byref(plan))
    assert n1.value > 4 * n10.value > 4 * plan.value
    with pytest.raises(ValueError):
        lib.call("vfs_grad_workspace_size", ctypes.byref(prm), 0, ctypes.byref(n1))
    with pytest.raises(ValueError):
        lib.call("vfs_grad_workspace_size", ctypes.byref(_prm(lib, nLevel=0)), 10, ctypes.byref(n1))
    gp = ctypes.c_void_p(0)
    rc = lib.lib().vfs_grad_create(ctypes.byref(prm), 10, 100.0, 32.0, 32.0, 1.0, None, 0, ctypes.byref(gp))
    assert rc == lib.VFS_ERR_WORKSPACE
    rc = lib.lib().vfs_grad_create(ctypes.byref(prm), 10, 0.0, 32.0, 32.0, 1.0, None, 0, ctypes.byref(gp))
    assert rc == lib.VFS_ERR_ARG  # focal length must be positive
    assert lib.lib().vfs_grad_set_options(None, 11, 0) == lib.VFS_ERR_ARG
    assert lib.lib().vfs_grad_backward(None, None, None, None, None, None) == lib.VFS_ERR_ARG


def test_bench_algorithmic_bytes_and_profile_files():
    """bench.py's roofline basis: 113 B per pixel-iteration, 60 per pixel-warp,
    41 per pixel-level, summed over the pyramid (1.989e10 B per 512x512 map with
    4 levels x 10 warps x 50 iterations; 9.688e10 B per 800x800 map with
    5 x 10 x 100), and the ncu summaries it scales traffic from are present."""
    import json
    import bench
    p = bench.params()
    assert bench.alg_bytes_per_map(p) == 96878952500
    p.width = p.height = 512
    p.nLevel, p.nSolverIters = 4, 50
    assert abs(bench.alg_bytes_per_map(p) - 1.989e10) < 1e7
    for name in list(bench.TRAFFIC_FILES.values()) + list(bench.REV_TRAFFIC_FILES.values()):
        d = json.load(open(os.path.join(ROOT, "profiles", name)))
        assert 0 < d["dram_bytes_per_alg_byte"] < 1
        assert abs(d["dram_bytes_per_alg_byte"] - (d["dram_read_bytes"] + d["dram_write_bytes"]) / d["alg_bytes"]) < 1e-3
    # the dominant kernel's launches: K iterations each (no GPU needed to ask)
    assert bench.variant_iters(232) == 2 and bench.variant_iters(221) == 3 and bench.variant_iters(134) == 4


def test_checkpoint_spacing_sized_to_memory():
    """DepthSolver(ckpt_every="auto"): the densest checkpoint spacing whose
    reverse-mode workspace fits the budget (800x800, 5 levels x 10 warps x 100
    iterations: every state recorded needs 34.6 GB, every 10 iterations 4.1 GB;
    the workspace is least near 50, since the backward buffers one interval)."""
    from vfs_b200 import grad
    from vfs_b200.vfs_params import vfs_params
    p = vfs_params(np.zeros((800, 800), np.uint8))
    p.nLevel, p.nWarpIters, p.nSolverIters, p.fScale = 5, 10, 100, 2.0
    w = {k: grad.workspace_bytes(p, k) for k in grad.CKPT_CANDIDATES}
    assert abs(w[1] - 34.589e9) < 1e7 and abs(w[10] - 4.121e9) < 1e7
    assert grad.checkpoint_interval(p, 180e9) == 1
    assert grad.checkpoint_interval(p, w[2]) == 2
    assert grad.checkpoint_interval(p, w[10]) == 10
    assert grad.checkpoint_interval(p, min(w.values())) == min(w, key=w.get)
    with pytest.raises(MemoryError):
        grad.checkpoint_interval(p, min(w.values()) - 1)


def test_bench_variant_iters_of_non_variant():
    """The cluster-resident kernel's id is not a tile variant: 0 iterations."""
    import bench
    assert bench.variant_iters(1000) == 0
