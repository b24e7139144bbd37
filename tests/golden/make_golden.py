"""Generates tests/golden/ref_small.npz from the reference's own CUDA kernels.

Run on a GPU machine after `make -C oracle/refgpu` (which builds the
reference's kernels from its sources into oracle/_ref):

    python tests/golden/make_golden.py [out.npz]

Inputs are a seeded synthetic fisheye pair at 48x64 and seeded random solver
states; every output is produced by the reference kernels through the
reference's host call order (oracle/refgpu/refpath.py).  The fixtures pin the
float64 oracle (CPU tests) and the B200 kernels (GPU tests) without needing
the reference at test time.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "vfs-python_b200"), os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

from helpers import bench_params, default_params, pair  # noqa: E402
from oracle.np64 import vfs64 as V  # noqa: E402
from oracle.refgpu import refpath  # noqa: E402

H, W = 48, 64


def np_(t):
    return t.detach().cpu().numpy()


def main(out_path):
    torch.manual_seed(0)
    g = {}
    p = pair(W, height=H, t=(0.1, 0.0, 0.0), seed=0, n_level=3)
    cam64 = V.EquidistantCam64(p.intrinsics)
    tvf, cvf = V.get_vector_fields(V.get_grid_zero((H, W)), cam64, cam64, p.R, p.t, 1)
    tvf, cvf = tvf.astype(np.float32), cvf.astype(np.float32)
    g.update(img_ref=p.img_ref, img_other=p.img_other, mask=p.mask, tvf=tvf, cvf=cvf,
             intrinsics=np.array(p.intrinsics, np.float64), t=p.t.reshape(3))

    # ---- pyramids and per-kernel outputs (bench parameters, 3 levels)
    prm = bench_params(H, W, n_level=3, n_warp=3, n_iter=13)
    r = refpath.RefVFS(prm, "bench")
    r.compute_pyramid_sizes()
    r.create_mask_pyramid(p.mask)
    r.create_vector_field_pyramid(tvf, cvf)
    r.create_image_pyramid(p.img_ref, p.img_other)
    for k in range(prm.nLevel):
        g[f"mask_{k}"] = np_(r.masks[k])
        g[f"tvf_{k}"] = np_(r.translations[k])
        g[f"ref_{k}"] = np_(r.refs[k])
        g[f"other_{k}"] = np_(r.others[k])
    rng = np.random.default_rng(1)
    for k in (0, 1):
        s = r.sizes[k]
        f = lambda *sh, sc=1.0: (rng.standard_normal(sh) * sc).astype(np.float32)
        st = dict(p=f(*s, 2, sc=0.3), q=f(*s, 4, sc=0.3), u=f(*s, sc=2.0), ub=f(*s, sc=2.0), vb=f(*s, 2, sc=0.2),
                  warp=f(*s, 2, sc=1.5))
        for n_, v in st.items():
            g[f"L{k}_in_{n_}"] = v
        R = {n_: refpath.to_device(v) for n_, v in st.items()}
        rm = r.masks_to[k]
        sm = r.gaussian(r.refs_to[k], rm, s)
        abc, eta = r.compute_tensor_eta(sm, rm)
        tv = r.find_warping_vector(R["warp"], r.translations_to[k])
        wi = r.warping_image(r.others_to[k], R["warp"])
        de = r.compute_derivatives(wi, r.refs_to[k], r.translations_to[k])
        sigma, tau, mu = V.step_schedule(2, 1.0)[1]
        pp, tp, qq = r.update_dual_variables(R["p"], R["q"], sigma, R["ub"], R["vb"], abc, rm)
        uu = r.l1_thresholding(tau, tp, R["u"], R["ub"], de, eta, rm)
        ub2, vb2 = r.update_primal_variables(tau, mu, pp, qq, uu, R["ub"], R["vb"], abc, eta, rm)
        med = r.median_filter(uu, rm)
        wp, ubf = r.compute_optical_flow_with_clamp(R["warp"], R["ub"], med, tv, rm)
        out = dict(smooth=sm, abc=abc, eta=eta, tvec=tv, warped=wi, deriv=de, p=pp, tp=tp, q=qq, u=uu, ub=ub2,
                   vb=vb2, median=med, clamp_warp=wp, clamp_u=ubf)
        if k > 0:
            fs = r.sizes[k - 1]
            out["up1"] = r.upsampling_vector_field1(ubf, fs)
            out["up2"] = r.upsampling_vector_field(wp, fs)
        for n_, v in out.items():
            g[f"L{k}_out_{n_}"] = np_(v)
        g[f"L{k}_sched"] = np.array([sigma, tau, mu], np.float32)

    # ---- end to end: bench parameters and the reference defaults
    cam = refpath.RefEquidistantCam(p.intrinsics, "bench")
    cam.setup_module()
    g["e2e_bench_warp"] = np_(r.solve_stereo(p.img_ref, p.img_other))
    g["e2e_bench_xyz"] = np_(r.triangulate_flow(cam, p.t))
    prm_d = default_params(H, W, n_level=4, n_warp=2, n_iter=9)
    rd = refpath.RefVFS(prm_d, "default")
    rd.compute_pyramid_sizes()
    rd.create_mask_pyramid(p.mask)
    rd.create_vector_field_pyramid(tvf, cvf)
    g["e2e_default_warp"] = np_(rd.solve_stereo(p.img_ref, p.img_other))
    g["e2e_default_xyz"] = np_(rd.triangulate_flow(cam, p.t))

    # ---- camera kernels
    g["cam_rays"] = np_(cam.get_rays((H, W)))
    uv = (rng.uniform(0, 1, (H, W, 2)) * [W, H]).astype(np.float32)
    g["cam_uv_in"] = uv
    xyz = cam.get_XYZs(refpath.to_device(uv))
    g["cam_xyz"] = np_(xyz)
    g["cam_uv"] = np_(cam.get_UVs(xyz))
    np.savez_compressed(out_path, **g)
    print(f"wrote {out_path}: {len(g)} arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_small.npz"))
