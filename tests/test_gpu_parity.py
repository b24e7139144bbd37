"""GPU parity: the B200 kernels against the reference's own kernels.

The reference side runs the reference's CUDA kernels (built from its sources
into oracle/_ref by oracle/refgpu/Makefile) with the reference's host call
order (oracle/refgpu/refpath.py).  Both sides get identical inputs; every
comparison is bit-exact (float32 bit patterns), since the B200 kernels
perform the same float32 operations and sample through the same texture
hardware.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import bench_params, default_params, pair, bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_mod(gpu):
    from oracle.refgpu import refpath
    return refpath


def _np(t):
    return t.detach().cpu().numpy()


def assert_bits_equal(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} vs {b.shape}"
    same = bits(a) == bits(b)
    if not same.all():
        idx = np.argwhere(~same)[:5]
        raise AssertionError(f"{what}: {np.count_nonzero(~same)} of {same.size} differ; first at {idx.tolist()}: "
                             f"{a[tuple(idx[0])]} vs {b[tuple(idx[0])]}")


def _fields(p):
    from oracle.np64 import vfs64 as V
    cam = V.EquidistantCam64(p.intrinsics)
    tvf, cvf = V.get_vector_fields(V.get_grid_zero(p.img_ref.shape), cam, cam, p.R, p.t, 1)
    return tvf.astype(np.float32), cvf.astype(np.float32)


def _both(ref_mod, prm, p, mask=None, lib_name=None):
    from vfs_b200.vfs import VFS
    tvf, cvf = _fields(p)
    mask = p.mask if mask is None else mask
    r = ref_mod.RefVFS(prm, lib_name)
    o = VFS(prm)
    for v in (r, o):
        v.setup_module()
        v.compute_pyramid_sizes()
        v.create_mask_pyramid(mask)
        v.create_vector_field_pyramid(tvf, cvf)
    return r, o


@pytest.mark.parametrize("size", [(80, 96), (61, 53)])
def test_pyramids_bit_exact(ref_mod, size):
    h, w = size
    p = pair(w, height=h, seed=3, n_level=3)
    prm = bench_params(h, w, n_level=3)
    r, o = _both(ref_mod, prm, p)
    r.create_image_pyramid(p.img_ref, p.img_other)
    o.create_image_pyramid(p.img_ref, p.img_other)
    torch.cuda.synchronize()
    for k in range(prm.nLevel):
        assert_bits_equal(_np(r.masks[k]), _np(o.masks[k]), f"mask level {k}")
        assert_bits_equal(_np(r.translations[k]), _np(o.translations[k]), f"tvf level {k}")
        assert_bits_equal(_np(r.refs[k]), _np(o.refs[k]), f"ref level {k}")
        assert_bits_equal(_np(r.others[k]), _np(o.others[k]), f"other level {k}")


def test_default_params_pyramids_bit_exact(ref_mod):
    """fScale 1.2: box taps straddle texels, the mask texel choice depends on rounding."""
    p = pair(100, height=90, seed=5, n_level=6)
    prm = default_params(90, 100, n_level=6)
    r, o = _both(ref_mod, prm, p, lib_name="default")
    r.create_image_pyramid(p.img_ref, p.img_other)
    o.create_image_pyramid(p.img_ref, p.img_other)
    torch.cuda.synchronize()
    for k in range(prm.nLevel):
        assert_bits_equal(_np(r.masks[k]), _np(o.masks[k]), f"mask level {k}")
        assert_bits_equal(_np(r.translations[k]), _np(o.translations[k]), f"tvf level {k}")
        assert_bits_equal(_np(r.refs[k]), _np(o.refs[k]), f"ref level {k}")
        assert_bits_equal(_np(r.others[k]), _np(o.others[k]), f"other level {k}")


def _rand_state(rng, h, w):
    f = lambda *s, sc=1.0: (rng.standard_normal(s) * sc).astype(np.float32)
    return dict(p=f(h, w, 2, sc=0.3), q=f(h, w, 4, sc=0.3), u=f(h, w, sc=2.0), ub=f(h, w, sc=2.0),
                vb=f(h, w, 2, sc=0.2), warp=f(h, w, 2, sc=1.5))


@pytest.mark.parametrize("all_ones_mask", [False, True])
def test_step_kernels_bit_exact(ref_mod, all_ones_mask):
    """Every per-step kernel on the same random inputs (the all-ones mask makes
    the border pixels read their flat, row-wrapping neighbours)."""
    h, w = 72, 88
    p = pair(w, height=h, seed=7, n_level=3)
    prm = bench_params(h, w, n_level=3)
    mask = np.full((h, w), 255, np.uint8) if all_ones_mask else p.mask
    r, o = _both(ref_mod, prm, p, mask=mask)
    r.create_image_pyramid(p.img_ref, p.img_other)
    o.create_image_pyramid(p.img_ref, p.img_other)
    rng = np.random.default_rng(11)
    for k in (0, 1):
        s = r.sizes[k]
        st = _rand_state(rng, *s)
        R = {n: ref_mod.to_device(v) for n, v in st.items()}
        O = {n: torch.as_tensor(v).cuda() for n, v in st.items()}
        rm, om = r.masks_to[k], o.masks_to[k]
        # gaussian + tensor
        rs = r.gaussian(r.refs_to[k], rm, s)
        os_ = o.gaussian(o.refs_to[k], om, s)
        assert_bits_equal(_np(rs), _np(os_), f"gaussian L{k}")
        rabc, reta = r.compute_tensor_eta(rs, rm)
        oabc, oeta = o.compute_tensor_eta(os_, om)
        assert_bits_equal(_np(rabc), _np(oabc), f"tensor L{k}")
        assert_bits_equal(_np(reta), _np(oeta), f"eta L{k}")
        # warp-dependent gathers
        rt = r.find_warping_vector(R["warp"], r.translations_to[k])
        ot = o.find_warping_vector(O["warp"], o.translations_to[k])
        assert_bits_equal(_np(rt), _np(ot), f"findWarpingVector L{k}")
        rw = r.warping_image(r.others_to[k], R["warp"])
        ow = o.warping_image(o.others_to[k], O["warp"])
        assert_bits_equal(_np(rw), _np(ow), f"warpingImage L{k}")
        rd = r.compute_derivatives(rw, r.refs_to[k], r.translations_to[k])
        od = o.compute_derivatives(ow, o.refs_to[k], o.translations_to[k])
        assert_bits_equal(_np(rd), _np(od), f"computeDerivatives L{k}")
        # one TGV iteration, then a second from its outputs
        for it, (sigma, tau, mu) in enumerate([(1.0, 1.0, 0.76696503), (1.3038405, 0.76696503, 0.8205865)]):
            rp, rtp, rq = r.update_dual_variables(R["p"], R["q"], sigma, R["ub"], R["vb"], rabc, rm)
            op, otp, oq = o.update_dual_variables(O["p"], O["q"], sigma, O["ub"], O["vb"], oabc, om)
            assert_bits_equal(_np(rp), _np(op), f"dual p L{k} it{it}")
            assert_bits_equal(_np(rtp), _np(otp), f"dual tp L{k} it{it}")
            assert_bits_equal(_np(rq), _np(oq), f"dual q L{k} it{it}")
            ru = r.l1_thresholding(tau, rtp, R["u"], R["ub"], rd, reta, rm)
            ou = o.l1_thresholding(tau, otp, O["u"], O["ub"], od, oeta, om)
            assert_bits_equal(_np(ru), _np(ou), f"threshold L{k} it{it}")
            rub, rvb = r.update_primal_variables(tau, mu, rp, rq, ru, R["ub"], R["vb"], rabc, reta, rm)
            oub, ovb = o.update_primal_variables(tau, mu, op, oq, ou, O["ub"], O["vb"], oabc, oeta, om)
            assert_bits_equal(_np(rub), _np(oub), f"primal u_ L{k} it{it}")
            assert_bits_equal(_np(rvb), _np(ovb), f"primal v_ L{k} it{it}")
            R.update(p=rp, q=rq, u=ru, ub=rub, vb=rvb)
            O.update(p=op, q=oq, u=ou, ub=oub, vb=ovb)
        # median, clamp, upsampling
        rmed = r.median_filter(R["u"], rm)
        omed = o.median_filter(O["u"], om)
        assert_bits_equal(_np(rmed), _np(omed), f"median L{k}")
        rwp, rubf = r.compute_optical_flow_with_clamp(R["warp"], R["ub"], rmed, rt, rm)
        owp, oubf = o.compute_optical_flow_with_clamp(O["warp"], O["ub"], omed, ot, om)
        torch.cuda.synchronize()
        assert_bits_equal(_np(rwp), _np(owp), f"clamp warp L{k}")
        assert_bits_equal(_np(rubf), _np(oubf), f"clamp u L{k}")
        if k > 0:
            fs = r.sizes[k - 1]
            assert_bits_equal(_np(r.upsampling_vector_field1(rubf, fs)), _np(o.upsampling_vector_field1(oubf, fs)),
                              f"upsample1 L{k}")
            assert_bits_equal(_np(r.upsampling_vector_field(rwp, fs)), _np(o.upsampling_vector_field(owp, fs)),
                              f"upsample2 L{k}")


def _solve_pair(ref_mod, prm, p, lib_name=None, mask=None, variants=((4, False),)):
    """Reference solve vs the fused solve under each (TGV variant, cluster) config."""
    from vfs_b200.equidistant_cam import EquidistantCam
    r, o = _both(ref_mod, prm, p, lib_name=lib_name, mask=mask)
    rw = _np(r.solve_stereo(p.img_ref, p.img_other))
    rcam = ref_mod.RefEquidistantCam(p.intrinsics, lib_name or ref_mod.param_set_for(prm))
    rcam.setup_module()
    rxyz = _np(r.triangulate_flow(rcam, p.t))
    cam = EquidistantCam(p.intrinsics)
    cam.setup_module()
    outs = {}
    for v, cluster in variants:
        o.tgv_iters_per_launch = v
        o.use_cluster = cluster
        o.release()
        try:
            ow = _np(o.solve_stereo(p.img_ref, p.img_other))
        except Exception as e:
            raise AssertionError(f"TGV variant {v} (cluster {cluster}): {e}") from e
        oxyz = _np(o.triangulate_flow(cam, p.t))
        outs[(v, cluster)] = (ow, oxyz)
    return (rw, rxyz), outs, o, cam


@pytest.mark.parametrize("n_iter", [13, 20])
def test_solve_bit_exact_bench_params(ref_mod, n_iter):
    h, w = 96, 128
    p = pair(w, height=h, t=(0.12, 0.01, 0.0), seed=1, n_level=3)
    prm = bench_params(h, w, n_level=3, n_warp=3, n_iter=n_iter)
    from vfs_b200 import _lib
    import ctypes
    n = _lib.lib().vfs_tgv_variants(None, 0, None)
    ids = (ctypes.c_int * n)()
    assert _lib.lib().vfs_tgv_variants(ids, n, None) == n
    configs = [(ids[i], False) for i in range(n)] + [(134, True)]
    (rw, rxyz), outs, o, cam = _solve_pair(ref_mod, prm, p, variants=configs)
    for v, (ow, oxyz) in outs.items():
        assert_bits_equal(rw, ow, f"warpUV (iterations per launch {v})")
        assert_bits_equal(rxyz, oxyz, f"xyz (iterations per launch {v})")
    # the step-by-step path agrees too
    sw = _np(o.solve_stereo_steps(p.img_ref, p.img_other))
    assert_bits_equal(rw, sw, "warpUV (per-step path)")
    sxyz = _np(o.triangulate_flow(cam, p.t))
    assert_bits_equal(rxyz, sxyz, "xyz (per-step path)")


def test_solve_bit_exact_default_params(ref_mod):
    h, w = 90, 100
    p = pair(w, height=h, seed=2, n_level=6)
    prm = default_params(h, w, n_level=6, n_warp=2, n_iter=9)
    (rw, rxyz), outs, _, _ = _solve_pair(ref_mod, prm, p, lib_name="default",
                                         variants=((4, False), (134, False), (134, True)))
    for v, (ow, oxyz) in outs.items():
        assert_bits_equal(rw, ow, f"warpUV {v}")
        assert_bits_equal(rxyz, oxyz, f"xyz {v}")


def test_solve_bit_exact_all_ones_mask(ref_mod):
    """No mask: border pixels take the reference's flat (row-wrapping) reads."""
    h, w = 64, 80
    p = pair(w, height=h, seed=4, n_level=3)
    prm = bench_params(h, w, n_level=3, n_warp=2, n_iter=10)
    ones = np.full((h, w), 255, np.uint8)
    (rw, rxyz), outs, _, _ = _solve_pair(ref_mod, prm, p, mask=ones, variants=((1, False), (4, False), (134, True)))
    for v, (ow, oxyz) in outs.items():
        assert_bits_equal(rw, ow, f"warpUV (iterations per launch {v})")
        assert_bits_equal(rxyz, oxyz, f"xyz (iterations per launch {v})")


def test_camera_and_vector_fields(ref_mod):
    from vfs_b200.equidistant_cam import EquidistantCam
    from vfs_b200.vector_field import get_vector_fields, get_grid_zero, get_grid_one
    h, w = 70, 90
    intr = (w / 2 / (np.pi / 2), w / 2, h / 2)
    rc = ref_mod.RefEquidistantCam(intr)
    rc.setup_module()
    oc = EquidistantCam(intr)
    oc.setup_module()
    assert_bits_equal(_np(rc.get_rays((h, w))), _np(oc.get_rays((h, w))), "getRays")
    assert_bits_equal(_np(rc.get_thetas()), _np(oc.get_thetas()), "getThetas")
    rng = np.random.default_rng(0)
    uv = (rng.uniform(0, 1, (h, w, 2)) * [w, h]).astype(np.float32)
    rxyz = rc.get_XYZs(ref_mod.to_device(uv))
    oxyz = oc.get_XYZs(torch.as_tensor(uv).cuda())
    assert_bits_equal(_np(rxyz), _np(oxyz), "getXYZFromUV")
    assert_bits_equal(_np(rc.get_UVs(rxyz)), _np(oc.get_UVs(oxyz)), "getUVFromXYZ")
    D = rng.uniform(1, 10, (h, w)).astype(np.float32)
    m = (rng.uniform(0, 1, (h, w)) > 0.3).astype(np.uint8)
    rc.set_mask(m)
    oc.set_mask(m)
    assert_bits_equal(_np(rc.get_xyz_from_distance(ref_mod.to_device(D))),
                      _np(oc.get_xyz_from_distance(torch.as_tensor(D).cuda())), "getXYZFromDistance")
    # vector fields: the fused kernel vs the reference's chain (5e-4 px is the
    # reference test's bound, Python/test_vector_field.py:40)
    R = np.eye(3)
    th = 0.05
    R2 = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    for Rm, t, ts, gridf, rgridf in [(R, [[0.1], [0.0], [0.0]], 1, get_grid_zero, ref_mod.get_grid_zero),
                                     (R2, [[0.05], [0.1], [0.02]], (1, 0.01), get_grid_one, ref_mod.get_grid_one)]:
        rt, rcv = ref_mod.get_vector_fields(rgridf((h, w)), rc, rc, Rm, np.asarray(t), ts)
        ot, ocv = get_vector_fields(gridf((h, w)), oc, oc, Rm, np.asarray(t), ts)
        assert np.nanmax(np.abs(rt - ot)) < 5e-4
        assert np.nanmax(np.abs(rcv - ocv)) < 5e-4


def test_autotuned_levels_bit_exact(ref_mod):
    """The autotuner's per-level kernel choice (tiles, iterations per launch,
    cluster kernel) changes speed only: the solve stays bit-identical."""
    from vfs_b200.autotune import variants, CLUSTER
    h, w = 96, 128
    p = pair(w, height=h, t=(0.12, 0.01, 0.0), seed=6, n_level=3)
    prm = bench_params(h, w, n_level=3, n_warp=2, n_iter=11)
    r, o = _both(ref_mod, prm, p)
    rw = _np(r.solve_stereo(p.img_ref, p.img_other))
    choice = o.autotune(p.img_ref, p.img_other, repeats=1)
    assert len(choice) == prm.nLevel
    assert all(c in variants() or c == CLUSTER for c in choice)
    o.configure(use_graph=True)
    assert_bits_equal(rw, _np(o.solve_stereo(p.img_ref, p.img_other)), f"warpUV with {choice}")
    # every single choice applied to all levels agrees as well
    for c in (162, 192, CLUSTER):
        o.set_level_variants([c] * prm.nLevel)
        assert_bits_equal(rw, _np(o.solve_stereo(p.img_ref, p.img_other)), f"warpUV with {c} everywhere")


def test_solve_bit_exact_rotated_pair(ref_mod):
    """A second view rotated by R (X_other = R (X + t)): the calibration warp by
    cvf (Python/vfs.py:150-153) is no longer a near-identity, and the solve
    still matches the reference's kernels bit for bit."""
    from vfs_b200.synthetic import make_pair, rotation_xyz
    h, w = 96, 128
    p = make_pair(w, (0.1, 0.03, 0.01), seed=8, n_level=3, height=h, R=rotation_xyz(0.02, -0.03, 0.015))
    prm = bench_params(h, w, n_level=3, n_warp=3, n_iter=13)
    (rw, rxyz), outs, o, cam = _solve_pair(ref_mod, prm, p, variants=((4, False), (134, False)))
    _, cvf = _fields(p)
    assert np.abs(cvf).max() > 1.0
    for v, (ow, oxyz) in outs.items():
        assert_bits_equal(rw, ow, f"warpUV {v}")
        assert_bits_equal(rxyz, oxyz, f"xyz {v}")


def test_lsq_triangulation_against_float64(ref_mod):
    """triangulate_flow(method="lsq") (fused plan kernel and the ray-by-ray
    entry point) against the float64 oracle's least-squares triangulation of
    the same flow.  Where the parallax angle exceeds 1 mrad the float32 result
    is within 1e-3 relative of float64; the two GPU paths agree bit for bit."""
    from oracle.np64 import vfs64 as V
    h, w = 96, 128
    t = (0.05, 0.1, 0.02)  # mostly vertical: the reference formula is ill-conditioned here
    p = pair(w, height=h, t=t, seed=5, n_level=3)
    prm = bench_params(h, w, n_level=3, n_warp=3, n_iter=13)
    _, o = _both(ref_mod, prm, p)
    from vfs_b200.equidistant_cam import EquidistantCam
    cam = EquidistantCam(p.intrinsics)
    cam.setup_module()
    flow = _np(o.solve_stereo(p.img_ref, p.img_other))
    fused = _np(o.triangulate_flow(cam, p.t, method="lsq"))
    steps = _np(o.solve_stereo_steps(p.img_ref, p.img_other))
    assert_bits_equal(flow, steps, "flow (plan vs per-step path)")
    raywise = _np(o.triangulate_flow(cam, p.t, method="lsq"))
    assert_bits_equal(fused, raywise, "lsq xyz (fused vs ray-by-ray)")
    cam64 = V.EquidistantCam64(p.intrinsics)
    rays = cam64.get_rays((h, w))
    rays_o = cam64.unproject(V.get_grid_zero((h, w)) + flow.astype(np.float64))
    want = V.triangulate_rays_lsq(rays, rays_o, np.asarray(t, np.float64), p.mask)
    m = p.mask != 0
    assert np.array_equal(fused[~m], np.tile(np.float32([0, 0, -1]), (np.count_nonzero(~m), 1)))
    parallax = np.linalg.norm(np.cross(rays, rays_o), axis=-1)
    sel = m & (parallax > 1e-3) & np.isfinite(want).all(-1)
    assert sel.sum() > 0.5 * m.sum()
    rel = np.abs(fused[sel, 2] - want[sel, 2]) / np.abs(want[sel, 2])
    assert rel.max() < 1e-3, (rel.max(), np.median(rel))
    assert np.median(rel) < 1e-5


@pytest.mark.parametrize("h,w,n_level,n_warp,n_iter,mask_kind", [
    (17, 23, 2, 2, 5, "circle"),    # smaller than every tile
    (61, 53, 3, 2, 7, "circle"),    # odd, ragged sizes
    (48, 40, 1, 1, 1, "circle"),    # one level, one warp, one iteration
    (64, 64, 3, 2, 6, "zero"),      # every pixel masked: every tile skips its iterations
])
def test_solve_bit_exact_edge_cases(ref_mod, h, w, n_level, n_warp, n_iter, mask_kind):
    p = pair(w, height=h, seed=11, n_level=max(n_level, 2))
    prm = bench_params(h, w, n_level=n_level, n_warp=n_warp, n_iter=n_iter)
    mask = np.zeros((h, w), np.uint8) if mask_kind == "zero" else p.mask
    variants = ((4, False), (134, False), (220, False), (222, False), (224, False), (134, True))
    (rw, rxyz), outs, _, _ = _solve_pair(ref_mod, prm, p, mask=mask, variants=variants)
    if mask_kind == "zero":
        assert not rw.any()
    for v, (ow, oxyz) in outs.items():
        assert_bits_equal(rw, ow, f"warpUV {v}")
        assert_bits_equal(rxyz, oxyz, f"xyz {v}")
