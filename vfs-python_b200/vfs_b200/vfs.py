"""Drop-in for the reference's ``VFS`` class (Python/vfs.py:33-559).

Same constructor, methods, call order and results; device arrays are torch
CUDA tensors instead of CuPy arrays, and every launch is asynchronous on
torch's current stream (the reference synchronises the device after each).

``solve_stereo`` runs the fused B200 path: one plan (libvfs_b200's
``vfs_plan_*``) holds all pyramids and solver state in one workspace, and the
TGV iterations run in the temporally blocked kernel.  The per-kernel methods
(``warping_image`` ... ``upsampling_vector_field``) mirror the reference's
launch wrappers one to one and are the parity hooks; ``solve_stereo_steps``
chains them in the reference's order.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .texture import Texture
from ._lib import call, ptr, stream


def _dev(a, dtype) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        t = a.to(device="cuda", dtype=dtype)
    else:
        t = torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)
    return t.contiguous()


class VFS:
    def __init__(self, param):
        self.param = param
        self.gpu_module = None
        self._plan = None
        self._plan_key = None
        self._workspace = None
        self._plan_mask = False
        self._plan_fields = False
        self.tgv_iters_per_launch = 134
        self.use_graph = False
        self.timing = False
        self.use_cluster = False

    # ---- Python/vfs.py:38-74
    def setup_module(self):
        if self.gpu_module is None:
            self.gpu_module = _lib.lib()

    def compile_module(self):
        self.setup_module()

    @staticmethod
    def compute_optical_flow(u, vec):
        """Python/vfs.py:76-82."""
        assert len(u.shape) == 2
        assert len(vec.shape) == 3
        assert u.shape == vec.shape[:2]
        assert vec.shape[2] == 2
        return u[:, :, None] * vec

    def _prm(self) -> _lib.VfsParams:
        return _lib.VfsParams.from_param_bag(self.param)

    # ---- Python/vfs.py:84-91
    def compute_pyramid_sizes(self):
        sizes = []
        h, w = self.param.height, self.param.width
        for _ in range(self.param.nLevel):
            sizes.append((h, w))
            h = int(h / self.param.fScale)
            w = int(w / self.param.fScale)
        self.sizes = sizes

    # ---- the fused plan ----------------------------------------------------
    def _key(self):
        p = self.param
        return (p.width, p.height, p.beta, p.gamma, p.alpha0, p.alpha1, p.timeStepLambda, p.Lambda, p.fScale,
                p.limitRange, p.nLevel, p.nWarpIters, p.nSolverIters)

    def _ensure_plan(self):
        self.setup_module()
        key = self._key()
        if self._plan is not None and self._plan_key == key:
            return self._plan
        self.release()
        prm = self._prm()
        nbytes = ctypes.c_size_t(0)
        call("vfs_plan_workspace_size", ctypes.byref(prm), ctypes.byref(nbytes))
        self._workspace = torch.empty(nbytes.value + 256, dtype=torch.uint8, device="cuda")
        plan = ctypes.c_void_p(0)
        call("vfs_plan_create", ctypes.byref(prm), self._workspace.data_ptr(), self._workspace.numel(),
             ctypes.byref(plan))
        call("vfs_plan_set_tgv_variant", plan, int(self.tgv_iters_per_launch))
        call("vfs_plan_set_graph", plan, 1 if self.use_graph else 0)
        call("vfs_plan_set_timing", plan, 1 if self.timing else 0)
        call("vfs_plan_set_cluster", plan, 1 if self.use_cluster else 0)
        for l, v in enumerate(getattr(self, "level_variants", [])[:self.param.nLevel]):
            call("vfs_plan_set_level_variant", plan, l, int(v))
        self._plan, self._plan_key = plan, key
        self._plan_mask = self._plan_fields = False
        return plan

    def configure(self, iters_per_launch=None, use_graph=None, timing=None, cluster=None):
        """Fused-path options: TGV iterations per launch (1, 2, 4), CUDA-graph
        replay of the whole solve, and TGV event timing (see ``solve_stats``)."""
        if iters_per_launch is not None:
            self.tgv_iters_per_launch = int(iters_per_launch)
        if use_graph is not None:
            self.use_graph = bool(use_graph)
        if timing is not None:
            self.timing = bool(timing)
        if cluster is not None:
            self.use_cluster = bool(cluster)
        if self._plan is not None:
            call("vfs_plan_set_tgv_variant", self._plan, int(self.tgv_iters_per_launch))
            call("vfs_plan_set_graph", self._plan, 1 if self.use_graph else 0)
            call("vfs_plan_set_timing", self._plan, 1 if self.timing else 0)
            call("vfs_plan_set_cluster", self._plan, 1 if self.use_cluster else 0)

    def set_level_variants(self, choice):
        """Per-level TGV kernel ids, finest level first (0: the default kernel,
        1000: the cluster-resident kernel)."""
        self.level_variants = list(choice)
        if self._plan is not None:
            for l, v in enumerate(self.level_variants):
                call("vfs_plan_set_level_variant", self._plan, l, int(v))

    def autotune(self, img_ref, img_other, **kw):
        """Times every TGV kernel on this plan's levels and keeps the fastest
        per level (results are bit-identical whichever kernel runs)."""
        from .autotune import autotune
        return autotune(self, _dev(img_ref, torch.uint8), _dev(img_other, torch.uint8), **kw)

    def solve_stats(self) -> dict:
        """Statistics of the last fused solve (synchronises the current stream)."""
        torch.cuda.current_stream().synchronize()
        st = _lib.VfsSolveStats()
        call("vfs_plan_stats", self._plan, ctypes.byref(st))
        out = {k: getattr(st, k) for k, _ in st._fields_}
        out["tgv_ms_level"] = list(st.tgv_ms_level)[:self.param.nLevel]
        return out

    def release(self):
        """Frees the plan (and its workspace)."""
        if self._plan is not None:
            torch.cuda.current_stream().synchronize()
            _lib.lib().vfs_plan_destroy(self._plan)
            self._plan = None
            self._workspace = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def _sync_plan_inputs(self):
        plan = self._ensure_plan()
        if not self._plan_mask:
            assert hasattr(self, "masks"), "create_mask_pyramid must be called before solve_stereo"
            call("vfs_plan_set_mask", plan, self.masks[0].data_ptr(), self.masks[0].shape[1], stream())
            self._plan_mask = True
        if not self._plan_fields:
            assert hasattr(self, "calibration"), "create_vector_field_pyramid must be called before solve_stereo"
            call("vfs_plan_set_vector_fields", plan, self.translations[0].data_ptr(), self.calibration.data_ptr(),
                 stream())
            self._plan_fields = True
        return plan

    # ---- pyramids, Python/vfs.py:93-218 -------------------------------------
    def _ct(self, t, linear=True):
        return Texture(t, linear)

    def create_image_pyramid_(self, img_f32):
        self.setup_module()
        pyr = [img_f32]
        pyr_to = []
        for sz in self.sizes[1:]:
            d = torch.empty(sz, dtype=torch.float32, device="cuda")
            to = self._ct(pyr[-1])
            call("vfs_downsample_image", d.data_ptr(), to.handle, d.shape[0], d.shape[1], stream())
            pyr.append(d)
            pyr_to.append(to)
        pyr_to.append(self._ct(pyr[-1]))
        return pyr, pyr_to

    def create_image_pyramid(self, img_ref, img_other):
        self.setup_module()
        assert tuple(img_ref.shape) == tuple(img_other.shape)
        img_ref_gpu = _dev(img_ref, torch.uint8)
        img_other_gpu = _dev(img_other, torch.uint8)
        ref0 = torch.empty(img_ref_gpu.shape, dtype=torch.float32, device="cuda")
        other0 = torch.empty(img_other_gpu.shape, dtype=torch.float32, device="cuda")
        for s, d in zip((img_ref_gpu, img_other_gpu), (ref0, other0)):
            call("vfs_cast_and_scale", d.data_ptr(), s.data_ptr(), s.shape[0], s.shape[1], stream())
        refs, refs_to = self.create_image_pyramid_(ref0)
        to = self._ct(other0)
        other0_warp = self.warping_image(to, self.calibration)
        others, others_to = self.create_image_pyramid_(other0_warp)
        self.refs, self.others = refs, others
        self.refs_to, self.others_to = refs_to, others_to

    def create_mask_pyramid(self, mask):
        self.setup_module()
        masks = [_dev(mask, torch.uint8)]
        masks_to = []
        for sz in self.sizes[1:]:
            d = torch.empty(sz, dtype=torch.uint8, device="cuda")
            to = self._ct(masks[-1], linear=False)
            call("vfs_downsample_mask", d.data_ptr(), to.handle, d.shape[0], d.shape[1], stream())
            masks.append(d)
            masks_to.append(to)
        masks_to.append(self._ct(masks[-1], linear=False))
        self.masks = masks
        self.masks_to = masks_to
        self._plan_mask = False

    def create_vector_field_pyramid(self, translation, calibration):
        self.setup_module()
        self.calibration = _dev(calibration, torch.float32)
        translations = [_dev(translation, torch.float32)]
        translations_to = []
        for sz in self.sizes[1:]:
            d = torch.empty((*sz, 2), dtype=torch.float32, device="cuda")
            to = self._ct(translations[-1])
            call("vfs_downsample_vector_field", d.data_ptr(), to.handle, d.shape[0], d.shape[1], stream())
            translations.append(d)
            translations_to.append(to)
        translations_to.append(self._ct(translations[-1]))
        self.translations = translations
        self.translations_to = translations_to
        self._plan_fields = False

    # ---- per-kernel wrappers, Python/vfs.py:220-458 --------------------------
    @staticmethod
    def _mask(to_mask):
        return to_mask.data_ptr, to_mask.pitch

    def warping_image(self, to, warp):
        warp = _dev(warp, torch.float32)
        d = torch.empty(warp.shape[:2], dtype=torch.float32, device="cuda")
        call("vfs_warping_image", d.data_ptr(), warp.data_ptr(), to.handle, d.shape[0], d.shape[1], stream())
        return d

    def gaussian(self, to, to_mask, sz):
        d = torch.empty(tuple(sz), dtype=torch.float32, device="cuda")
        m, mp = self._mask(to_mask)
        call("vfs_gaussian", d.data_ptr(), to.handle, m, mp, d.shape[0], d.shape[1], stream())
        return d

    def compute_tensor_eta(self, img, to_mask):
        to = self._ct(img)
        d_tensor = torch.empty((*img.shape, 3), dtype=torch.float32, device="cuda")
        d_eta = torch.empty((*img.shape, 3), dtype=torch.float32, device="cuda")
        m, mp = self._mask(to_mask)
        prm = self._prm()
        call("vfs_compute_tensor_eta", d_tensor.data_ptr(), d_eta.data_ptr(), to.handle, m, mp, ctypes.byref(prm),
             d_tensor.shape[0], d_tensor.shape[1], stream())
        return d_tensor, d_eta

    def find_warping_vector(self, warpUV, to_translation):
        assert warpUV.is_contiguous()
        d = torch.empty_like(warpUV)
        call("vfs_find_warping_vector", d.data_ptr(), warpUV.data_ptr(), to_translation.handle, d.shape[0],
             d.shape[1], stream())
        return d

    def compute_derivatives(self, wapred_other, to_ref, to_translation):
        d = torch.empty((*wapred_other.shape, 2), dtype=torch.float32, device="cuda")
        to = self._ct(wapred_other)
        call("vfs_compute_derivatives", d.data_ptr(), to_ref.handle, to.handle, to_translation.handle, d.shape[0],
             d.shape[1], stream())
        return d

    def update_dual_variables(self, p, q, sigma, u, v, tensor_abc, to_mask):
        for t in (p, q, u, v, tensor_abc):
            assert t.is_contiguous()
        assert tuple(u.shape) == tuple(v.shape[:2])
        tp = torch.empty_like(p)
        m, mp = self._mask(to_mask)
        prm = self._prm()
        call("vfs_update_dual_variables", p.data_ptr(), tp.data_ptr(), q.data_ptr(), float(np.float32(sigma)),
             u.data_ptr(), v.data_ptr(), tensor_abc.data_ptr(), m, mp, ctypes.byref(prm), p.shape[0], p.shape[1],
             stream())
        return p, tp, q

    def l1_thresholding(self, tau, tp, u, u_, derivatives, eta, to_mask):
        for t in (tp, u, u_, derivatives, eta):
            assert t.is_contiguous()
        assert u.shape == u_.shape
        us = torch.empty_like(u)
        m, mp = self._mask(to_mask)
        prm = self._prm()
        call("vfs_l1_thresholding", us.data_ptr(), float(np.float32(tau)), tp.data_ptr(), u.data_ptr(),
             u_.data_ptr(), derivatives.data_ptr(), eta.data_ptr(), m, mp, ctypes.byref(prm), us.shape[0],
             us.shape[1], stream())
        return us

    def update_primal_variables(self, tau, mu, p, q, u, u_, v_, tensor_abc, eta, to_mask):
        for t in (p, q, u, u_, v_, tensor_abc, eta):
            assert t.is_contiguous()
        assert tuple(u_.shape) == tuple(v_.shape[:2])
        us = torch.empty_like(u_)
        vs = torch.empty_like(v_)
        m, mp = self._mask(to_mask)
        prm = self._prm()
        call("vfs_update_primal_variables", us.data_ptr(), vs.data_ptr(), float(np.float32(tau)),
             float(np.float32(mu)), p.data_ptr(), q.data_ptr(), u.data_ptr(), u_.data_ptr(), v_.data_ptr(),
             tensor_abc.data_ptr(), eta.data_ptr(), m, mp, ctypes.byref(prm), us.shape[0], us.shape[1], stream())
        return us, vs

    def median_filter(self, u, to_mask):
        assert u.is_contiguous()
        d = torch.empty_like(u)
        m, mp = self._mask(to_mask)
        call("vfs_median_filter", d.data_ptr(), u.data_ptr(), m, mp, d.shape[0], d.shape[1], stream())
        return d

    def compute_optical_flow_with_clamp(self, warpUV_, u_, u, translation_vector, to_mask):
        for t in (warpUV_, u_, u):
            assert t.is_contiguous()
        m, mp = self._mask(to_mask)
        prm = self._prm()
        call("vfs_compute_optical_flow_with_clamp", warpUV_.data_ptr(), u_.data_ptr(), u.data_ptr(),
             translation_vector.data_ptr(), m, mp, ctypes.byref(prm), warpUV_.shape[0], warpUV_.shape[1], stream())
        return warpUV_, u_

    def upsampling_vector_field1(self, u, shape):
        d = torch.empty(tuple(shape), dtype=torch.float32, device="cuda")
        to = self._ct(u)
        prm = self._prm()
        call("vfs_upsampling_vector_field1", d.data_ptr(), to.handle, ctypes.byref(prm), d.shape[0], d.shape[1],
             stream())
        return d

    def upsampling_vector_field(self, warp, shape):
        d = torch.empty((*shape, 2), dtype=torch.float32, device="cuda")
        to = self._ct(warp)
        prm = self._prm()
        call("vfs_upsampling_vector_field", d.data_ptr(), to.handle, ctypes.byref(prm), d.shape[0], d.shape[1],
             stream())
        return d

    # ---- Python/vfs.py:460-533 -----------------------------------------------
    def solve_stereo(self, img_ref, img_other):
        """Fused solve; returns warpUV (H, W, 2) float32 on the device."""
        plan = self._sync_plan_inputs()
        ref = _dev(img_ref, torch.uint8)
        oth = _dev(img_other, torch.uint8)
        assert tuple(ref.shape) == tuple(oth.shape) == (self.param.height, self.param.width)
        out = torch.empty((self.param.height, self.param.width, 2), dtype=torch.float32, device="cuda")
        call("vfs_plan_solve", plan, ref.data_ptr(), oth.data_ptr(), out.data_ptr(), stream())
        self.warpUV = out
        self._fused_flow = out
        return out

    def solve_stereo_steps(self, img_ref, img_other):
        """The reference's solve loop (Python/vfs.py:460-533) over the
        per-kernel entry points, one launch per reference kernel."""
        self.create_image_pyramid(img_ref, img_other)
        sched = _step_schedule(self.param.nSolverIters, self.param.timeStepLambda)
        for s, k in zip(self.sizes[::-1], range(len(self.sizes), 0, -1)):
            s2, s4 = (*s, 2), (*s, 4)
            if s == self.sizes[-1]:
                warpUV_ref = torch.zeros(s2, dtype=torch.float32, device="cuda")
                u = torch.zeros(s, dtype=torch.float32, device="cuda")
                u_ = torch.zeros(s, dtype=torch.float32, device="cuda")
            ref_smoothed = self.gaussian(self.refs_to[k - 1], self.masks_to[k - 1], s)
            abc, eta = self.compute_tensor_eta(ref_smoothed, self.masks_to[k - 1])
            for _kw in range(self.param.nWarpIters):
                tvec = self.find_warping_vector(warpUV_ref, self.translations_to[k - 1])
                other_warped = self.warping_image(self.others_to[k - 1], warpUV_ref)
                derivatives = self.compute_derivatives(other_warped, self.refs_to[k - 1],
                                                       self.translations_to[k - 1])
                p = torch.zeros(s2, dtype=torch.float32, device="cuda")
                q = torch.zeros(s4, dtype=torch.float32, device="cuda")
                v_ = torch.zeros(s2, dtype=torch.float32, device="cuda")
                u_before_solver = u.clone()
                for sigma, tau, mu in sched:
                    p, tp, q = self.update_dual_variables(p, q, sigma, u_, v_, abc, self.masks_to[k - 1])
                    u = self.l1_thresholding(tau, tp, u, u_, derivatives, eta, self.masks_to[k - 1])
                    u_, v_ = self.update_primal_variables(tau, mu, p, q, u, u_, v_, abc, eta, self.masks_to[k - 1])
                u_filtered = self.median_filter(u, self.masks_to[k - 1])
                warpUV_ref, u = self.compute_optical_flow_with_clamp(warpUV_ref, u_before_solver, u_filtered, tvec,
                                                                     self.masks_to[k - 1])
            if k > 1:
                ss = self.sizes[k - 2]
                u_ = self.upsampling_vector_field1(u, ss)
                u = u_.clone()
                warpUV_ref = self.upsampling_vector_field(warpUV_ref, ss)
        warpUV_ref[self.masks[0] == 0, :] = 0
        self.warpUV = warpUV_ref
        return warpUV_ref

    # ---- Python/vfs.py:535-559
    def triangulate_flow(self, camera, translation, method="reference"):
        """Rays of the grid and of grid + flow, triangulated with the
        translation.  ``method="reference"`` is the reference's formula
        (x components, t.x and t.z only); ``method="lsq"`` is the
        least-squares point on the reference ray closest to the other ray,
        which uses all of t (for baselines mostly along y or z)."""
        if method not in ("reference", "lsq"):
            raise ValueError(f"triangulation method {method!r}: use 'reference' or 'lsq'")
        sfx = "_lsq" if method == "lsq" else ""
        t = np.asarray(translation, dtype=np.float32).reshape(-1)
        assert t.size == 3
        h, w = self.warpUV.shape[:2]
        out = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
        tt = (ctypes.c_float * 3)(*t.tolist())
        if self._plan is not None and getattr(self, "_fused_flow", None) is self.warpUV:
            # getRays + getXYZFromUV + triangulateRays in one kernel on the
            # plan's copy of the flow
            call("vfs_plan_triangulate" + sfx, self._plan, float(np.float32(camera.f)), float(np.float32(camera.u0)),
                 float(np.float32(camera.v0)), tt, out.data_ptr(), stream())
            return out
        # rays of the grid and of grid + flow, then triangulateRays
        rays = camera.get_rays((h, w))
        from .vector_field import get_grid_zero
        rays_other = camera.get_XYZs(get_grid_zero((h, w)) + self.warpUV)
        m = self.masks_to[0]
        call("vfs_triangulate_rays" + sfx, out.data_ptr(), rays.data_ptr(), rays_other.data_ptr(), tt, m.data_ptr,
             m.pitch, h, w, stream())
        return out


def _step_schedule(n, time_step_lambda):
    out = np.zeros(3 * max(n, 1), dtype=np.float32)
    call("vfs_step_schedule", int(n), float(time_step_lambda), out.ctypes.data)
    return [tuple(float(v) for v in out[3 * i:3 * i + 3]) for i in range(n)]
