"""Batched solve of many stereo pairs of uneven resolution (no counterpart in
the reference, which solves one pair per ``VFS.solve_stereo`` call).

    b = VFSBatch(param, sizes=[(h0, w0), (h1, w1), ...])
    for i, (mask, tvf, cvf) in enumerate(per_pair): b.set_pair(i, mask, tvf, cvf)
    warps = b.solve(img_refs, img_others)          # list of (H_i, W_i, 2) tensors
    xyz = b.triangulate(i, camera_i, t_i)

All pairs share ``param``'s solver settings (``param.width/height`` are
ignored).  Per pair the result is bit-identical to ``VFS.solve_stereo``; the
pairs advance level by level together and each TGV pass is one kernel launch
over the tiles of every pair (or, with ``configure(group_bytes=...)``, of each
group of pairs whose solver state fits that budget), captured with the rest of
the batch as one CUDA graph.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import call, stream
from .vfs import _dev


class VFSBatch:
    def __init__(self, param, sizes, use_graph: bool = True):
        self.param = param
        self.sizes = [(int(h), int(w)) for h, w in sizes]
        n = len(self.sizes)
        self._prm = _lib.VfsParams.from_param_bag(param)
        hs = (ctypes.c_int * n)(*[h for h, _ in self.sizes])
        ws = (ctypes.c_int * n)(*[w for _, w in self.sizes])
        nbytes = ctypes.c_size_t(0)
        call("vfs_batch_workspace_size", ctypes.byref(self._prm), n, hs, ws, ctypes.byref(nbytes))
        self._workspace = torch.empty(nbytes.value + 512, dtype=torch.uint8, device="cuda")
        self._batch = ctypes.c_void_p(0)
        call("vfs_batch_create", ctypes.byref(self._prm), n, hs, ws, self._workspace.data_ptr(),
             self._workspace.numel(), ctypes.byref(self._batch))
        call("vfs_batch_set_graph", self._batch, 1 if use_graph else 0)
        self._keep = [None] * n

    def __len__(self):
        return len(self.sizes)

    def set_pair(self, i, mask, tvf, cvf):
        """Mask (H, W) u8 and vector fields (H, W, 2) of pair i (as
        create_mask_pyramid + create_vector_field_pyramid)."""
        m = _dev(mask, torch.uint8)
        t = _dev(tvf, torch.float32)
        c = _dev(cvf, torch.float32)
        assert tuple(m.shape) == self.sizes[i] and tuple(t.shape) == (*self.sizes[i], 2)
        call("vfs_batch_set_pair", self._batch, int(i), m.data_ptr(), m.shape[1], t.data_ptr(), c.data_ptr(),
             stream())
        self._keep[i] = (m, t, c)

    def set_level_variants(self, choice):
        for l, v in enumerate(choice):
            call("vfs_batch_set_level_variant", self._batch, l, int(v))

    def configure(self, use_graph=None, timing=None, group_bytes=None):
        """group_bytes: working-set budget of a launch group (vfs_batch_set_group_bytes;
        0: all pairs of a level in one launch per pass)."""
        if use_graph is not None:
            call("vfs_batch_set_graph", self._batch, 1 if use_graph else 0)
        if group_bytes is not None:
            call("vfs_batch_set_group_bytes", self._batch, int(group_bytes))
        if timing is not None:
            call("vfs_batch_set_timing", self._batch, 1 if timing else 0)

    def solve(self, img_refs, img_others):
        n = len(self.sizes)
        refs = [_dev(a, torch.uint8) for a in img_refs]
        oths = [_dev(a, torch.uint8) for a in img_others]
        outs = [torch.empty((*self.sizes[i], 2), dtype=torch.float32, device="cuda") for i in range(n)]
        P = ctypes.c_void_p * n
        call("vfs_batch_solve", self._batch, P(*[r.data_ptr() for r in refs]), P(*[o.data_ptr() for o in oths]),
             P(*[o.data_ptr() for o in outs]), stream())
        self._inputs = (refs, oths)
        return outs

    def triangulate(self, i, camera, translation, method="reference"):
        """Depth points of pair i (VFS.triangulate_flow's two methods)."""
        if method not in ("reference", "lsq"):
            raise ValueError(f"triangulation method {method!r}: use 'reference' or 'lsq'")
        t = np.asarray(translation, dtype=np.float32).reshape(-1)
        out = torch.empty((*self.sizes[i], 3), dtype=torch.float32, device="cuda")
        f, u0, v0 = camera._k()
        call("vfs_batch_triangulate" + ("_lsq" if method == "lsq" else ""), self._batch, int(i), f, u0, v0, (ctypes.c_float * 3)(*t.tolist()),
             out.data_ptr(), stream())
        return out

    def stats(self) -> dict:
        torch.cuda.current_stream().synchronize()
        st = _lib.VfsSolveStats()
        call("vfs_batch_stats", self._batch, ctypes.byref(st))
        out = {k: getattr(st, k) for k, _ in st._fields_}
        out["tgv_ms_level"] = list(st.tgv_ms_level)[:self.param.nLevel]
        return out

    def autotune(self, img_refs, img_others, candidates=None, repeats: int = 1):
        """Per-level choice of the batched TGV kernel (1xx variants)."""
        from .autotune import variants
        cands = candidates or [v for v in variants() if v >= 100]
        nlev = self.param.nLevel
        self.configure(use_graph=True, timing=True)
        best = [(float("inf"), 134)] * nlev
        for c in cands:
            self.set_level_variants([c] * nlev)
            times = None
            for _ in range(repeats + 1):
                self.solve(img_refs, img_others)
                lv = self.stats()["tgv_ms_level"]
                times = lv if times is None else [min(a, b) for a, b in zip(times, lv)]
            best = [min(b, (t, c)) for b, t in zip(best, times)]
        choice = [c for _, c in best]
        self.set_level_variants(choice)
        self.configure(timing=False)
        return choice

    def release(self):
        if getattr(self, "_batch", None):
            torch.cuda.current_stream().synchronize()
            _lib.lib().vfs_batch_destroy(self._batch)
            self._batch = None
            self._workspace = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
