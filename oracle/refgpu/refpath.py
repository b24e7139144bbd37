"""Test infrastructure: the reference's GPU path, driven without CuPy.

The kernels that run here are the reference's own (``Python/vfs.cu``,
``Python/equidistant_cam.cuh``, ``Python/template_cam.cu``), compiled from the
reference checkout by ``oracle/refgpu/Makefile`` into
``oracle/_ref/libvfsref_<params>.so``.  This module restates the reference's
host-side orchestration (``Python/vfs.py``, ``Python/equidistant_cam.py``,
``Python/vector_field.py``, ``Python/texture.py``) on torch CUDA tensors with
the same call order, the same per-call texture objects (cudaArray copies) and a
device-wide synchronisation after every launch, exactly as the reference does.

Allocation has two modes.  The default (parity checking) differs from
running the reference under CuPy, deliberately:

* every array is allocated with zero-filled guard bands around it, so the
  reference kernels' out-of-bounds border reads (flat ``index-width`` at row 0,
  ``index+width`` at the last row) read zeros instead of whatever the CuPy
  memory pool had placed next to the array;
* outputs that the reference allocates with ``cp.empty`` are zero-filled.

``set_plain_allocation(True)`` (timing) allocates as CuPy does instead:
``cp.empty`` becomes ``torch.empty`` (no fill kernel, no guard bands) and
``cp.zeros`` becomes ``torch.zeros``, both from torch's caching allocator as
CuPy's arrays come from its memory pool.  Every reference kernel writes each
in-bounds element of its output, so the two modes give the same results
wherever the mask keeps the border pixels out (the out-of-bounds reads need an
unmasked pixel in the first or last row or column of some level).

It is used by the GPU parity tests, the golden-fixture generator and the
``--impl reference`` arm of ``bench.py``; the product never imports it.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF_DIR = os.path.join(os.path.dirname(_HERE), "_ref")

# cudaTextureAddressMode / cudaTextureFilterMode / cudaTextureReadMode values
ADDR_WRAP, ADDR_CLAMP, ADDR_MIRROR, ADDR_BORDER = 0, 1, 2, 3
FILTER_POINT, FILTER_LINEAR = 0, 1
READ_ELEMENT = 0

# Parameter sets baked into the reference builds (oracle/refgpu/Makefile).
PARAM_SETS = {
    "bench": dict(fScale=2.0, beta=9.0, gamma=0.85, alpha0=17.0, alpha1=1.2, Lambda=50.0, limitRange=0.1),
    "default": dict(fScale=1.2, beta=9.0, gamma=0.85, alpha0=17.0, alpha1=1.2, Lambda=5.0, limitRange=0.1),
}

_LIBS: dict = {}


def param_set_for(param) -> str:
    """Name of the reference build whose baked constants equal ``param``'s."""
    for name, vals in PARAM_SETS.items():
        if all(float(getattr(param, k)) == float(v) for k, v in vals.items()):
            return name
    raise ValueError("no reference build for these parameters; add a variant to oracle/refgpu/Makefile")


def load(name: str = "bench") -> ctypes.CDLL:
    if name not in _LIBS:
        path = os.path.join(_REF_DIR, f"libvfsref_{name}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle/refgpu` where the reference checkout exists")
        _LIBS[name] = ctypes.CDLL(path)
    return _LIBS[name]


def _p(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _chk(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"reference {what} failed with CUDA error {rc}")


_DT_BYTES = {torch.uint8: 1, torch.int16: 2, torch.float32: 4, torch.int32: 4}


_PLAIN = False


def set_plain_allocation(enable: bool) -> None:
    """Allocate as CuPy does (see the module docstring) instead of with
    zero-filled guard bands."""
    global _PLAIN
    _PLAIN = bool(enable)


def zeros(shape, dtype=torch.float32) -> torch.Tensor:
    """``cp.zeros``: zero-filled (with zero guard bands unless plain)."""
    return torch.zeros(shape, dtype=dtype, device="cuda") if _PLAIN else alloc(shape, dtype)


def alloc(shape, dtype=torch.float32, guard_elems: int | None = None) -> torch.Tensor:
    """``cp.empty``: a zero-filled CUDA tensor with zero guard bands before
    and after it, or, with plain allocation, an uninitialised one."""
    if _PLAIN:
        return torch.empty(shape, dtype=dtype, device="cuda")
    n = int(np.prod(shape))
    if guard_elems is None:
        row = int(np.prod(shape[1:])) if len(shape) > 1 else n
        guard_elems = row + 64
    # keep the view 256-byte aligned, as cudaMalloc would
    esz = _DT_BYTES[dtype]
    g = ((guard_elems * esz + 255) // 256) * 256 // esz
    buf = torch.zeros(g + n + g, dtype=dtype, device="cuda")
    return buf[g:g + n].view(*shape)


def to_device(arr, dtype=torch.float32) -> torch.Tensor:
    a = torch.as_tensor(np.ascontiguousarray(arr))
    out = alloc(tuple(a.shape), dtype)
    out.copy_(a.to(dtype))
    return out


class RefTexture:
    """A texture object over a cudaArray copy, as Python/texture.py:27-55."""

    def __init__(self, lib, img: torch.Tensor, address_mode=ADDR_BORDER, filter_mode=FILTER_POINT,
                 read_mode=READ_ELEMENT, normalized=0):
        assert img.is_contiguous()
        if img.dtype == torch.uint8:
            kind = 0
        elif img.dtype == torch.int16:
            kind = 1
        elif img.dtype == torch.float32 and img.dim() == 2:
            kind = 2
        else:
            assert img.dtype == torch.float32 and img.dim() == 3 and img.shape[2] == 2
            kind = 3
        self._lib = lib
        self.tex = ctypes.c_ulonglong(0)
        self.arr = ctypes.c_void_p(0)
        _chk(lib.ref_tex_create(_p(img), img.shape[0], img.shape[1], kind, address_mode, filter_mode,
                                read_mode, normalized, ctypes.byref(self.tex), ctypes.byref(self.arr)),
             "texture create")

    @property
    def handle(self) -> ctypes.c_ulonglong:
        return self.tex

    def __del__(self):
        try:
            self._lib.ref_tex_destroy(self.tex, self.arr)
        except Exception:
            pass


def _sync(lib):
    _chk(lib.ref_sync(), "device synchronize")


class RefEquidistantCam:
    """Python/equidistant_cam.py:34-206 on the reference kernels."""

    def __init__(self, p, lib_name: str = "bench"):
        self.f, self.u0, self.v0 = p[0], p[1], p[2]
        self.lib = load(lib_name)
        self.rays = None
        self.mask = None
        self.to_mask = None

    def setup_module(self):
        # Python/equidistant_cam.py:67-70 -> util_cuda.upload_constant
        p = np.array([self.f, self.u0, self.v0], dtype=np.float32)
        _chk(self.lib.ref_cam_set_intrinsics(ctypes.c_float(p[0]), ctypes.c_float(p[1]), ctypes.c_float(p[2])),
             "constant upload")

    def get_rays(self, sz):
        rays = alloc((sz[0], sz[1], 3))
        _chk(self.lib.ref_getRays(_p(rays), sz[0], sz[1]), "getRays")
        _sync(self.lib)
        self.rays = rays
        return rays

    def get_UVs(self, xyz):
        assert xyz.is_contiguous() and xyz.dtype == torch.float32
        uv = alloc((xyz.shape[0], xyz.shape[1], 2))
        _chk(self.lib.ref_getUVFromXYZ(_p(uv), _p(xyz), uv.shape[0], uv.shape[1]), "getUVFromXYZ")
        _sync(self.lib)
        return uv

    def get_XYZs(self, uv):
        assert uv.is_contiguous() and uv.dtype == torch.float32
        xyz = alloc((uv.shape[0], uv.shape[1], 3))
        _chk(self.lib.ref_getXYZFromUV(_p(xyz), _p(uv), xyz.shape[0], xyz.shape[1]), "getXYZFromUV")
        _sync(self.lib)
        return xyz

    def get_thetas(self):
        thetas = alloc(tuple(self.rays.shape))
        _chk(self.lib.ref_getThetas(_p(thetas), _p(self.rays), thetas.shape[0], thetas.shape[1]), "getThetas")
        _sync(self.lib)
        return thetas

    def set_mask(self, mask):
        m = to_device(mask, torch.uint8)
        self.mask = m
        self.to_mask = RefTexture(self.lib, m, ADDR_BORDER, FILTER_POINT, READ_ELEMENT, 0)

    def get_xyz_from_distance(self, D):
        if self.rays is None:
            self.get_rays(D.shape[:2])
        if self.mask is None:
            self.set_mask(np.ones(D.shape[:2], np.uint8))
        xyz = alloc(tuple(self.rays.shape))
        _chk(self.lib.ref_getXYZFromDistance(_p(xyz), _p(self.rays), _p(D), self.to_mask.handle,
                                             xyz.shape[0], xyz.shape[1]), "getXYZFromDistance")
        _sync(self.lib)
        return xyz


def get_grid_zero(sz) -> torch.Tensor:
    """Python/vector_field.py:58-62."""
    uv = np.empty((*sz, 2), dtype=np.int32)
    uv[:, :, 0] = np.arange(0, sz[1])[np.newaxis, :]
    uv[:, :, 1] = np.arange(0, sz[0])[:, np.newaxis]
    return to_device(uv.astype(np.float32))


def get_grid_one(sz) -> torch.Tensor:
    """Python/vector_field.py:64-65."""
    g = get_grid_zero(sz)
    out = alloc(tuple(g.shape))
    out.copy_(g + 1)
    return out


def normalizer_default(x: torch.Tensor) -> torch.Tensor:
    """The normalizer lambda of Python/main_equidistant.py:60."""
    out = alloc(tuple(x.shape))
    out.copy_(x / torch.linalg.norm(x, dim=2)[:, :, None])
    return out


def get_vector_fields(grid, camera_ref, camera_other, R, t, t_scale, normalizer=normalizer_default):
    """Python/vector_field.py:28-56 (returns NumPy arrays, as the reference does)."""
    if isinstance(t_scale, (float, int)):
        t_scale = (t_scale, t_scale)
    t = np.asarray(t, dtype=np.float64).reshape(3, 1)
    XYZ = camera_ref.get_XYZs(grid)
    XYZ = normalizer(XYZ)
    st = torch.tensor((t_scale[0] * t)[np.newaxis, np.newaxis, :, 0], dtype=torch.float32, device="cuda")
    a = alloc(tuple(XYZ.shape)); a.copy_(XYZ + st)
    tvf_forward = camera_ref.get_UVs(a)
    st = torch.tensor((t_scale[1] * t)[np.newaxis, np.newaxis, :, 0], dtype=torch.float32, device="cuda")
    b = alloc(tuple(XYZ.shape)); b.copy_(XYZ - st)
    tvf_backward = camera_ref.get_UVs(b)
    tvf = (tvf_forward - tvf_backward) / 2
    norm = torch.linalg.norm(tvf, dim=2)
    tvf /= norm[:, :, None]
    XYZ_ = XYZ.reshape(-1, 3)
    Rt = torch.tensor(np.asarray(R).T, dtype=torch.float32, device="cuda")
    # cp.dot of float32 operands: a float32 GEMM.  torch's matmul may use TF32
    # unless disabled; the reference's cuBLAS call does not.
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        RXYZ = torch.matmul(XYZ_, Rt).reshape(XYZ.shape)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    c = alloc(tuple(RXYZ.shape)); c.copy_(RXYZ)
    uv_other = camera_other.get_UVs(c)
    cvf = uv_other - grid
    return tvf.cpu().numpy(), cvf.cpu().numpy()


class RefVFS:
    """Python/vfs.py:33-559 on the reference kernels."""

    def __init__(self, param, lib_name: str | None = None):
        self.param = param
        self.lib = load(lib_name or param_set_for(param))

    def setup_module(self):
        pass

    # ---- Python/vfs.py:84-91
    def compute_pyramid_sizes(self):
        sizes = []
        h, w = self.param.height, self.param.width
        for _ in range(self.param.nLevel):
            sizes.append((h, w))
            h = int(h / self.param.fScale)
            w = int(w / self.param.fScale)
        self.sizes = sizes

    def _launch(self, name, *args):
        _chk(getattr(self.lib, name)(*args), name)
        _sync(self.lib)

    def _ct(self, t, filt=FILTER_LINEAR):
        return RefTexture(self.lib, t, ADDR_MIRROR, filt, READ_ELEMENT, 1)

    # ---- Python/vfs.py:93-119
    def create_image_pyramid_(self, img_f32):
        pyr = [img_f32]
        pyr_to = []
        for sz in self.sizes[1:]:
            d = alloc(sz)
            to = self._ct(pyr[-1])
            self._launch("ref_downSamplingImage", _p(d), to.handle, d.shape[0], d.shape[1])
            pyr.append(d)
            pyr_to.append(to)
        pyr_to.append(self._ct(pyr[-1]))
        return pyr, pyr_to

    # ---- Python/vfs.py:121-157
    def create_image_pyramid(self, img_ref, img_other):
        assert img_ref.shape == img_other.shape
        img_ref_gpu = to_device(img_ref, torch.uint8)
        img_other_gpu = to_device(img_other, torch.uint8)
        ref0 = alloc(tuple(img_ref_gpu.shape))
        other0 = alloc(tuple(img_other_gpu.shape))
        for s, d in zip((img_ref_gpu, img_other_gpu), (ref0, other0)):
            self._launch("ref_castAndScale", _p(d), _p(s), s.shape[0], s.shape[1])
        refs, refs_to = self.create_image_pyramid_(ref0)
        to = self._ct(other0)
        other0_warp = self.warping_image(to, self.calibration)
        others, others_to = self.create_image_pyramid_(other0_warp)
        self.refs, self.others = refs, others
        self.refs_to, self.others_to = refs_to, others_to

    # ---- Python/vfs.py:159-187
    def create_mask_pyramid(self, mask):
        masks = [to_device(mask, torch.uint8)]
        masks_to = []
        for sz in self.sizes[1:]:
            d = alloc(sz, torch.uint8)
            to = self._ct(masks[-1], FILTER_POINT)
            self._launch("ref_downSamplingMask", _p(d), to.handle, d.shape[0], d.shape[1])
            masks.append(d)
            masks_to.append(to)
        masks_to.append(self._ct(masks[-1], FILTER_POINT))
        self.masks = masks
        self.masks_to = masks_to

    # ---- Python/vfs.py:189-218
    def create_vector_field_pyramid(self, translation, calibration):
        self.calibration = to_device(np.asarray(calibration, dtype=np.float32))
        translations = [to_device(np.asarray(translation, dtype=np.float32))]
        translations_to = []
        for sz in self.sizes[1:]:
            d = alloc((*sz, 2))
            to = self._ct(translations[-1])
            self._launch("ref_downSamplingVectorField", _p(d), to.handle, d.shape[0], d.shape[1])
            translations.append(d)
            translations_to.append(to)
        translations_to.append(self._ct(translations[-1]))
        self.translations = translations
        self.translations_to = translations_to

    # ---- per-kernel wrappers, Python/vfs.py:220-458
    def warping_image(self, to, warp):
        d = alloc(tuple(warp.shape[:2]))
        self._launch("ref_warpingImage", _p(d), _p(warp), to.handle, d.shape[0], d.shape[1])
        return d

    def gaussian(self, to, to_mask, sz):
        d = alloc(tuple(sz))
        self._launch("ref_gaussianMasked", _p(d), to.handle, to_mask.handle, d.shape[0], d.shape[1])
        return d

    def compute_tensor_eta(self, img, to_mask):
        to = self._ct(img)
        d_tensor = alloc((*img.shape, 3))
        d_eta = alloc((*img.shape, 3))
        self._launch("ref_computeTensorEtaMasked", _p(d_tensor), _p(d_eta), to.handle, to_mask.handle,
                     d_tensor.shape[0], d_tensor.shape[1])
        return d_tensor, d_eta

    def find_warping_vector(self, warpUV, to_translation):
        d = alloc(tuple(warpUV.shape))
        self._launch("ref_findWarpingVector", _p(d), _p(warpUV), to_translation.handle, d.shape[0], d.shape[1])
        return d

    def compute_derivatives(self, warped_other, to_ref, to_translation):
        d = alloc((*warped_other.shape, 2))
        to = self._ct(warped_other)
        self._launch("ref_computeDerivatives", _p(d), to_ref.handle, to.handle, to_translation.handle,
                     d.shape[0], d.shape[1])
        return d

    def update_dual_variables(self, p, q, sigma, u, v, tensor_abc, to_mask):
        tp = alloc(tuple(p.shape))
        self._launch("ref_updateDualVariables", _p(p), _p(tp), _p(q), ctypes.c_float(sigma), _p(u), _p(v),
                     _p(tensor_abc), to_mask.handle, p.shape[0], p.shape[1])
        return p, tp, q

    def l1_thresholding(self, tau, tp, u, u_, derivatives, eta, to_mask):
        us = alloc(tuple(u.shape))
        self._launch("ref_l1Thresholding", _p(us), ctypes.c_float(tau), _p(tp), _p(u), _p(u_), _p(derivatives),
                     _p(eta), to_mask.handle, us.shape[0], us.shape[1])
        return us

    def update_primal_variables(self, tau, mu, p, q, u, u_, v_, tensor_abc, eta, to_mask):
        us = alloc(tuple(u_.shape))
        vs = alloc(tuple(v_.shape))
        self._launch("ref_updatePrimalVariables", _p(us), _p(vs), ctypes.c_float(tau), ctypes.c_float(mu),
                     _p(p), _p(q), _p(u), _p(u_), _p(v_), _p(tensor_abc), _p(eta), to_mask.handle,
                     us.shape[0], us.shape[1])
        return us, vs

    def median_filter(self, u, to_mask):
        d = alloc(tuple(u.shape))
        self._launch("ref_medianFilter", _p(d), _p(u), to_mask.handle, d.shape[0], d.shape[1])
        return d

    def compute_optical_flow_with_clamp(self, warpUV_, u_, u, translation_vector, to_mask):
        self._launch("ref_computeOpticalFlowWithClamp", _p(warpUV_), _p(u_), _p(u), _p(translation_vector),
                     to_mask.handle, warpUV_.shape[0], warpUV_.shape[1])
        return warpUV_, u_

    def upsampling_vector_field1(self, u, shape):
        d = alloc(tuple(shape))
        to = self._ct(u)
        self._launch("ref_upSamplingVectorField1", _p(d), to.handle, d.shape[0], d.shape[1])
        return d

    def upsampling_vector_field(self, warp, shape):
        d = alloc((*shape, 2))
        to = self._ct(warp)
        self._launch("ref_upSamplingVectorField", _p(d), to.handle, d.shape[0], d.shape[1])
        return d

    # ---- Python/vfs.py:460-533
    def solve_stereo(self, img_ref, img_other):
        self.create_image_pyramid(img_ref, img_other)
        for s, k in zip(self.sizes[::-1], range(len(self.sizes), 0, -1)):
            s2 = (*s, 2)
            s4 = (*s, 4)
            if s == self.sizes[-1]:
                warpUV_ref = zeros(s2)
                u = zeros(s)
                u_ = zeros(s)
            ref_smoothed = self.gaussian(self.refs_to[k - 1], self.masks_to[k - 1], s)
            abc, eta = self.compute_tensor_eta(ref_smoothed, self.masks_to[k - 1])
            for _kw in range(self.param.nWarpIters):
                translation_vector_ref = self.find_warping_vector(warpUV_ref, self.translations_to[k - 1])
                other_warped = self.warping_image(self.others_to[k - 1], warpUV_ref)
                derivatives = self.compute_derivatives(other_warped, self.refs_to[k - 1],
                                                       self.translations_to[k - 1])
                p = zeros(s2)
                q = zeros(s4)
                v_ = zeros(s2)
                tau = 1.
                sigma = 1. / tau
                u_before_solver = alloc(s)
                u_before_solver.copy_(u)
                for _ks in range(self.param.nSolverIters):
                    if sigma < 1000:
                        mu = 1 / np.sqrt(1 + 0.7 * tau * self.param.timeStepLambda).astype(np.float32)
                    else:
                        mu = 1
                    p, tp, q = self.update_dual_variables(p, q, sigma, u_, v_, abc, self.masks_to[k - 1])
                    u = self.l1_thresholding(tau, tp, u, u_, derivatives, eta, self.masks_to[k - 1])
                    u_, v_ = self.update_primal_variables(tau, mu, p, q, u, u_, v_, abc, eta, self.masks_to[k - 1])
                    sigma = sigma / mu
                    tau = tau * mu
                u_filtered = self.median_filter(u, self.masks_to[k - 1])
                warpUV_ref, u = self.compute_optical_flow_with_clamp(warpUV_ref, u_before_solver, u_filtered,
                                                                     translation_vector_ref, self.masks_to[k - 1])
            if k > 1:
                ss = self.sizes[k - 2]
                u_ = self.upsampling_vector_field1(u, ss)
                u = alloc(tuple(ss))
                u.copy_(u_)
                warpUV_ref = self.upsampling_vector_field(warpUV_ref, ss)
        warpUV_ref[self.masks[0] == 0, :] = 0
        self.warpUV = warpUV_ref
        return warpUV_ref

    # ---- Python/vfs.py:535-559
    def triangulate_flow(self, camera, translation):
        rays = camera.get_rays(tuple(self.warpUV.shape[:2]))
        uv = get_grid_zero(tuple(self.warpUV.shape[:2]))
        a = alloc(tuple(uv.shape)); a.copy_(uv + self.warpUV)
        rays_other = camera.get_XYZs(a)
        translation_ = to_device(np.asarray(translation, dtype=np.float32).reshape(-1))
        d = alloc(tuple(rays.shape))
        self._launch("ref_triangulateRays", _p(d), _p(rays), _p(rays_other), _p(translation_),
                     self.masks_to[0].handle, d.shape[0], d.shape[1])
        return d
