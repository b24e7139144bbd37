"""GPU: the B200 kernels reproduce the committed reference-kernel fixtures bit for bit.

tests/golden/ref_small.npz holds outputs of the reference's own CUDA kernels
(tests/golden/make_golden.py); this check needs neither the reference nor its
build at test time.
"""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from helpers import bench_params, default_params

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_small.npz")


def _eq(a, b, what):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape, what
    va = a.view(np.uint32) if a.dtype == np.float32 else a
    vb = b.view(np.uint32) if b.dtype == np.float32 else b
    bad = np.count_nonzero(va != vb)
    assert bad == 0, f"{what}: {bad} of {a.size} differ"


@pytest.fixture(scope="module")
def gold(gpu):
    return dict(np.load(GOLDEN))


def _vfs(prm, g):
    from vfs_b200 import VFS
    v = VFS(prm)
    v.setup_module()
    v.compute_pyramid_sizes()
    v.create_mask_pyramid(g["mask"])
    v.create_vector_field_pyramid(g["tvf"], g["cvf"])
    return v


def test_golden_pyramids_and_steps(gold):
    g = gold
    h, w = g["mask"].shape
    prm = bench_params(h, w, n_level=3, n_warp=3, n_iter=13)
    v = _vfs(prm, g)
    v.create_image_pyramid(g["img_ref"], g["img_other"])
    torch.cuda.synchronize()
    for k in range(3):
        _eq(v.masks[k].cpu().numpy(), g[f"mask_{k}"], f"mask {k}")
        _eq(v.translations[k].cpu().numpy(), g[f"tvf_{k}"], f"tvf {k}")
        _eq(v.refs[k].cpu().numpy(), g[f"ref_{k}"], f"ref {k}")
        _eq(v.others[k].cpu().numpy(), g[f"other_{k}"], f"other {k}")
    for k in (0, 1):
        s = v.sizes[k]
        T = lambda n: torch.as_tensor(g[f"L{k}_in_{n}"]).cuda().contiguous()
        gout = lambda n: g[f"L{k}_out_{n}"]
        m = v.masks_to[k]
        sm = v.gaussian(v.refs_to[k], m, s)
        abc, eta = v.compute_tensor_eta(sm, m)
        tv = v.find_warping_vector(T("warp"), v.translations_to[k])
        wi = v.warping_image(v.others_to[k], T("warp"))
        de = v.compute_derivatives(wi, v.refs_to[k], v.translations_to[k])
        sigma, tau, mu = (float(x) for x in g[f"L{k}_sched"])
        p, tp, q = v.update_dual_variables(T("p"), T("q"), sigma, T("ub"), T("vb"), abc, m)
        u = v.l1_thresholding(tau, tp, T("u"), T("ub"), de, eta, m)
        ub, vb = v.update_primal_variables(tau, mu, p, q, u, T("ub"), T("vb"), abc, eta, m)
        med = v.median_filter(u, m)
        wp, ubf = v.compute_optical_flow_with_clamp(T("warp"), T("ub"), med, tv, m)
        got = dict(smooth=sm, abc=abc, eta=eta, tvec=tv, warped=wi, deriv=de, p=p, tp=tp, q=q, u=u, ub=ub, vb=vb,
                   median=med, clamp_warp=wp, clamp_u=ubf)
        if k > 0:
            fs = v.sizes[k - 1]
            got["up1"] = v.upsampling_vector_field1(ubf, fs)
            got["up2"] = v.upsampling_vector_field(wp, fs)
        torch.cuda.synchronize()
        for n, t in got.items():
            _eq(t.cpu().numpy(), gout(n), f"level {k} {n}")


@pytest.mark.parametrize("which", ["bench", "default"])
def test_golden_end_to_end(gold, which):
    from vfs_b200 import EquidistantCam
    g = gold
    h, w = g["mask"].shape
    prm = bench_params(h, w, n_level=3, n_warp=3, n_iter=13) if which == "bench" else \
        default_params(h, w, n_level=4, n_warp=2, n_iter=9)
    v = _vfs(prm, g)
    cam = EquidistantCam(tuple(g["intrinsics"]))
    cam.setup_module()
    for graph in (False, True):
        v.configure(use_graph=graph)
        warp = v.solve_stereo(g["img_ref"], g["img_other"]).cpu().numpy()
        xyz = v.triangulate_flow(cam, g["t"]).cpu().numpy()
        _eq(warp, g[f"e2e_{which}_warp"], f"{which} flow (graph {graph})")
        _eq(xyz, g[f"e2e_{which}_xyz"], f"{which} xyz (graph {graph})")
    _eq(cam.get_rays((h, w)).cpu().numpy(), g["cam_rays"], "rays")
    xyz = cam.get_XYZs(torch.as_tensor(g["cam_uv_in"]).cuda())
    _eq(xyz.cpu().numpy(), g["cam_xyz"], "getXYZFromUV")
    _eq(cam.get_UVs(xyz).cpu().numpy(), g["cam_uv"], "getUVFromXYZ")
