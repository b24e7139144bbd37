"""Texture objects for the per-step API, in place of the reference's
``create_texture_object`` (Python/texture.py:27-55).

The reference copies each array into a cudaArray and binds a bindless texture
to it.  Here the copy goes into a pitch-linear buffer (512-byte aligned base,
128-byte row pitch) and the texture is bound to that buffer; on B200 the two
return bit-identical samples.  Supported, as the solver uses them: u8, f32 and
2-channel f32 arrays, mirror addressing with normalised coordinates, linear or
point filtering (Python/vfs.py:96-98, 169-171).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

# cudaTextureAddressMode / cudaTextureFilterMode / cudaTextureReadMode values
cudaAddressModeWrap, cudaAddressModeClamp, cudaAddressModeMirror, cudaAddressModeBorder = 0, 1, 2, 3
cudaFilterModePoint, cudaFilterModeLinear = 0, 1
cudaReadModeElementType = 0

_PITCH = 128
_BASE = 512


def pitched_copy(img: torch.Tensor):
    """(buffer, view, pitch_bytes): ``view`` is a (h, pitch/elem, ...) view of a
    512-byte-aligned buffer whose first ``w`` columns hold ``img``."""
    h, w = img.shape[:2]
    ch = 1 if img.dim() == 2 else img.shape[2]
    esz = img.element_size() * ch
    pitch = (w * esz + _PITCH - 1) // _PITCH * _PITCH
    raw = torch.empty(h * pitch + _BASE, dtype=torch.uint8, device=img.device)
    off = (-raw.data_ptr()) % _BASE
    body = raw[off:off + h * pitch]
    per_row = pitch // img.element_size()
    view = body.view(img.dtype).view(h, per_row)
    if ch > 1:
        view = view.view(h, per_row // ch, ch)
    view[:, :w].copy_(img)
    return raw, view, pitch


class Texture:
    """A bindless texture over a pitched copy of ``img`` (kept alive here)."""

    def __init__(self, img: torch.Tensor, linear: bool):
        if not img.is_cuda:
            raise ValueError("texture source must be a CUDA tensor")
        if img.dtype == torch.uint8 and img.dim() == 2:
            kind = _lib.TEX_U8
        elif img.dtype == torch.float32 and img.dim() == 2:
            kind = _lib.TEX_F32
        elif img.dtype == torch.float32 and img.dim() == 3 and img.shape[2] == 2:
            kind = _lib.TEX_F32X2
        else:
            raise ValueError(f"unsupported texture source {img.dtype} {tuple(img.shape)}")
        self.shape = tuple(img.shape)
        self._raw, self.view, self.pitch = pitched_copy(img.contiguous())
        self.handle = ctypes.c_uint64(0)
        self._live = False
        _lib.call("vfs_texture_create", self.view.data_ptr(), self.shape[0], self.shape[1], self.pitch, kind,
                  1 if linear else 0, ctypes.byref(self.handle))
        self._live = True

    @property
    def data_ptr(self) -> int:
        return self.view.data_ptr()

    def __del__(self):
        if getattr(self, "_live", False):
            try:
                # kernels that sample this texture may still be queued
                torch.cuda.current_stream().synchronize()
                _lib.lib().vfs_texture_destroy(self.handle)
            except Exception:
                pass


def create_texture_object(img_gpu, addressMode=cudaAddressModeBorder, filterMode=cudaFilterModePoint,
                          readMode=cudaReadModeElementType, normalizedCoords=0):
    """Drop-in for Python/texture.py:27-55 for the modes the solver uses."""
    if addressMode != cudaAddressModeMirror or not normalizedCoords or readMode != cudaReadModeElementType:
        raise NotImplementedError("only mirror-addressed, normalised, element-type textures are supported")
    return Texture(img_gpu, linear=(filterMode == cudaFilterModeLinear))
