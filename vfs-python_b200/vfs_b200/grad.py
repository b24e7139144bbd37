"""Differentiable depth from the stereo solve (no counterpart in the reference,
which is forward only).

``DepthSolver`` fixes what is not differentiated (the parameter bag's loop
counts, fScale, limitRange and timeStepLambda, the camera, the mask,
``t_scale``) and maps

    (img_ref, img_other, t, theta) -> depth = triangulate_flow(solve_stereo(...), t)[..., 2]

with theta = (Lambda, alpha0, alpha1, beta, gamma).  The translation also
moves the epipolar field, ``get_vector_fields(grid, cam, cam, I, t, t_scale)``.
Images are float32 CUDA tensors in the u8 range (u8 images converted with
``.float()`` give the plain solve's result bit for bit).  The backward pass is
the hand-written reverse mode of libvfs_b200 (``vfs_grad_*``): the forward
records the flow, u and u_ at each warp's start and the solver state every
``ckpt_every`` iterations; the backward recomputes each interval and runs the
adjoint kernels.  ``ckpt_every=1`` records every state and recomputes nothing
(fastest; 3.6 GB at 512x512 with 3x5x50, 35 GB at 800x800 with 5x10x100);
``ckpt_every=10`` needs about a tenth of that.  ``autotune`` picks the kernel
of each level for both passes.

    solver = DepthSolver(param, camera, mask)
    depth = solver(img_ref, img_other, t, theta)       # autograd-aware
    # DepthSolver(..., triangulation="lsq") uses all three components of t
    loss = (depth - gt).abs()[mask != 0].mean(); loss.backward()
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr, stream

THETA = ("Lambda", "alpha0", "alpha1", "beta", "gamma")

# checkpoint spacings tried by checkpoint_interval, densest first
CKPT_CANDIDATES = (1, 2, 5, 10, 20, 25, 50, 100)


def workspace_bytes(param, ckpt_every: int) -> int:
    """Device workspace of a DepthSolver with this parameter bag and spacing."""
    need = ctypes.c_size_t(0)
    call("vfs_grad_workspace_size", ctypes.byref(_lib.VfsParams.from_param_bag(param)), int(ckpt_every),
         ctypes.byref(need))
    return int(need.value)


def checkpoint_interval(param, budget_bytes: int, candidates=CKPT_CANDIDATES) -> int:
    """The densest checkpoint spacing whose workspace fits ``budget_bytes``
    (denser spacings recompute less in the backward: 1 records every state and
    recomputes nothing).  The workspace is not monotonic in the spacing: sparse
    checkpoints save the recorded states, but the backward then buffers every
    state of one interval.  Raises MemoryError if no candidate fits."""
    need = {int(k): workspace_bytes(param, k) for k in candidates}
    for k in sorted(need):
        if need[k] <= budget_bytes:
            return k
    k_min = min(need, key=need.get)
    raise MemoryError(f"no checkpoint spacing in {tuple(sorted(need))} fits {int(budget_bytes)} bytes "
                      f"(the least, every {k_min} iterations, needs {need[k_min]})")


class DepthSolver:
    def __init__(self, param, camera, mask, t_scale: float = 1.0, ckpt_every=10, level_variants=None,
                 triangulation: str = "reference", memory_budget: int | None = None):
        """``triangulation``: "reference" (the reference's x-only formula) or
        "lsq" (least squares along the reference ray, all of t; the choice for
        baselines with large y or z components).  ``ckpt_every="auto"`` sizes
        the checkpointing to the memory: the densest spacing whose workspace
        fits ``memory_budget`` bytes (default: 90 % of the device memory free
        now; give each of several solvers its share)."""
        if triangulation not in ("reference", "lsq"):
            raise ValueError(f"triangulation {triangulation!r}: use 'reference' or 'lsq'")
        self.param = param
        self.prm = _lib.VfsParams.from_param_bag(param)
        if ckpt_every == "auto":
            budget = memory_budget if memory_budget is not None else int(0.9 * torch.cuda.mem_get_info()[0])
            ckpt_every = checkpoint_interval(param, budget)
        self.ckpt_every = int(ckpt_every)
        self.workspace_bytes = workspace_bytes(param, self.ckpt_every)
        self._ws = torch.empty(self.workspace_bytes + 1024, dtype=torch.uint8, device="cuda")
        gp = ctypes.c_void_p(0)
        f, u0, v0 = camera._k() if hasattr(camera, "_k") else (float(x) for x in camera)
        call("vfs_grad_create", ctypes.byref(self.prm), self.ckpt_every, f, u0, v0, float(t_scale),
             self._ws.data_ptr(), self._ws.numel(), ctypes.byref(gp))
        self._gp = gp
        self.shape = (int(param.height), int(param.width))
        m = mask if isinstance(mask, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(mask))
        self._mask = m.to(device="cuda", dtype=torch.uint8).contiguous()
        if tuple(self._mask.shape) != self.shape:
            raise AssertionError(f"mask shape {tuple(self._mask.shape)} != {self.shape}")
        self._plan = _lib.lib().vfs_grad_plan(self._gp)
        self.triangulation = triangulation
        call("vfs_grad_set_triangulation", self._gp, int(triangulation == "lsq"))
        call("vfs_plan_set_mask", self._plan, self._mask.data_ptr(), self.shape[1], stream())
        for lvl, var in enumerate(level_variants or []):
            if var:
                call("vfs_plan_set_level_variant", self._plan, lvl, int(var))
        self._scal = torch.zeros(8, dtype=torch.float64, device="cuda")
        self._generation = 0
        self._recorded = None

    def set_options(self, fused_reverse: int = 11, trace_variant: int = 0) -> None:
        """Backward kernel forms (see vfs_grad_set_options in vfs_b200.h): the
        reverse-step kernel (11..20, 22..25 two to four iterations per launch, 1..5 one
        tiled kernel per iteration, 0 three gather kernels) and the TGV variant
        recomputing checkpoint intervals (0 automatic, -1 one iteration per launch)."""
        call("vfs_grad_set_options", self._gp, int(fused_reverse), int(trace_variant))

    def set_level_forms(self, forms) -> None:
        """Reverse-step kernel form per level (finest first; 0 = the plan's)."""
        for lvl, f in enumerate(forms):
            call("vfs_grad_set_level_form", self._gp, lvl, int(f))
        self.level_forms = list(forms)

    def autotune(self, img_ref, img_other, t, theta=None, g_depth=None,
                 forms=(11, 20, 22, 23, 24, 25, 13, 18, 17, 19, 12, 15, 16, 14), fwd_variants=(134, 124, 212, 216, 207, 220, 221, 222, 224, 232),
                 repeats: int = 2):
        """Choose, per level, the recording forward's TGV kernel and then the
        reverse-step form, by timing whole passes (levels are independent, so
        one sweep per level suffices).  Returns the reverse forms, finest
        level first; the forward choice is kept in ``level_variants``."""
        theta = self.theta_of() if theta is None else theta
        n_level = int(self.param.nLevel)
        # the recording forward's TGV kernel per level, among the variants that
        # have a recording form
        fwd_chosen = []
        for lvl in range(n_level):
            best = None
            for var in fwd_variants:
                call("vfs_plan_set_level_variant", self._plan, lvl, int(var))
                self.forward_pass(img_ref, img_other, t, theta)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(repeats):
                    self.forward_pass(img_ref, img_other, t, theta)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / repeats
                if best is None or ms < best[0]:
                    best = (ms, int(var))
            fwd_chosen.append(best[1])
            call("vfs_plan_set_level_variant", self._plan, lvl, best[1])
        self.level_variants = fwd_chosen
        depth = self.forward_pass(img_ref, img_other, t, theta)
        if g_depth is None:  # unit cotangent where the depth is finite and not near-singular
            g_depth = torch.where(torch.isfinite(depth) & (depth.abs() < 1e3) & (self._mask != 0),
                                  torch.ones_like(depth), torch.zeros_like(depth))
        chosen = [int(forms[0])] * n_level
        self.set_level_forms(chosen)

        def timed():
            self.backward_pass(g_depth)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(repeats):
                self.backward_pass(g_depth)
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / repeats

        for lvl in range(n_level):
            best = None
            for f in forms:
                call("vfs_grad_set_level_form", self._gp, lvl, int(f))
                ms = timed()
                if best is None or ms < best[0]:
                    best = (ms, int(f))
            chosen[lvl] = best[1]
            call("vfs_grad_set_level_form", self._gp, lvl, chosen[lvl])
        self.level_forms = chosen
        return chosen

    def set_timing(self, enable: bool) -> None:
        call("vfs_grad_set_timing", self._gp, int(bool(enable)))

    def backward_stats(self) -> dict:
        """Timing of the last backward's reverse TGV launches (set_timing(True) first)."""
        torch.cuda.current_stream().synchronize()
        st = _lib.VfsSolveStats()
        call("vfs_grad_stats", self._gp, ctypes.byref(st))
        return {"tgv_ms": st.tgv_ms, "tgv_alg_bytes": st.tgv_alg_bytes, "tgv_launches": st.tgv_launches,
                "tgv_ms_level": list(st.tgv_ms_level)[: int(self.param.nLevel)], "recompute_ms": st.recompute_ms}

    def theta_of(self, param=None) -> torch.Tensor:
        p = param or self.param
        return torch.tensor([float(getattr(p, k)) for k in THETA], dtype=torch.float64)

    def __call__(self, img_ref, img_other, t, theta=None):
        if theta is None:
            theta = self.theta_of()
        return _DepthFunction.apply(self, img_ref, img_other, torch.as_tensor(t, dtype=torch.float64),
                                    torch.as_tensor(theta, dtype=torch.float64))

    # ---- the two passes (also usable without autograd)
    def _check(self, img, what):
        _lib.require_cuda(img, what)
        if img.dtype != torch.float32 or tuple(img.shape) != self.shape:
            raise AssertionError(f"{what} must be float32 {self.shape}")

    def forward_pass(self, img_ref, img_other, t, theta) -> torch.Tensor:
        self._check(img_ref, "img_ref")
        self._check(img_other, "img_other")
        tv = [float(x) for x in torch.as_tensor(t, dtype=torch.float64).reshape(3).tolist()]
        th = [float(x) for x in torch.as_tensor(theta, dtype=torch.float64).reshape(5).tolist()]
        depth = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        call("vfs_grad_forward", self._gp, img_ref.data_ptr(), img_other.data_ptr(), (ctypes.c_double * 3)(*tv),
             (ctypes.c_double * 5)(*th), depth.data_ptr(), stream())
        self._generation += 1
        return depth

    def backward_pass(self, g_depth: torch.Tensor):
        g_depth = g_depth.to(device="cuda", dtype=torch.float32).contiguous()
        g_ref = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        g_other = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        call("vfs_grad_backward", self._gp, g_depth.data_ptr(), g_ref.data_ptr(), g_other.data_ptr(),
             self._scal.data_ptr(), stream())
        return g_ref, g_other, self._scal[:3].clone(), self._scal[3:].clone()

    def release(self) -> None:
        if self._gp:
            torch.cuda.current_stream().synchronize()
            _lib.lib().vfs_grad_destroy(self._gp)
            self._gp = None
            self._ws = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class _DepthFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, solver, img_ref, img_other, t, theta):
        depth = solver.forward_pass(img_ref.detach(), img_other.detach(), t.detach(), theta.detach())
        ctx.solver = solver
        ctx.generation = solver._generation
        ctx.save_for_backward(img_ref, img_other, t, theta)
        return depth

    @staticmethod
    def backward(ctx, g_depth):
        solver = ctx.solver
        img_ref, img_other, t, theta = ctx.saved_tensors
        if solver._generation != ctx.generation:
            # another forward ran on this solver since: record this one's tape again
            solver.forward_pass(img_ref.detach(), img_other.detach(), t.detach(), theta.detach())
            ctx.generation = solver._generation
        g_ref, g_other, g_t, g_theta = solver.backward_pass(g_depth)
        return (None, g_ref if ctx.needs_input_grad[1] else None, g_other if ctx.needs_input_grad[2] else None,
                g_t.to(t.device) if ctx.needs_input_grad[3] else None,
                g_theta.to(theta.device) if ctx.needs_input_grad[4] else None)
