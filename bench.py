"""Benchmark: depth maps/s of the variational fisheye stereo solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one step = one depth map): an 800x800 equidistant fisheye pair
(f = 400/(pi/2), principal point at the centre, t = (0.12, 0.01, 0) m, no
rotation), 5-level pyramid at scale 0.5, 10 warps per level, 100 TGV
iterations, lambda 50, alpha0 17, alpha1 1.2, beta 9, gamma 0.85, float32;
solve_stereo followed by triangulate_flow.  The pair is synthetic (seeded
range field + value-noise texture, see vfs_b200/synthetic.py): the reference
publishes no benchmark data.  Both arms get the same images, mask and
epipolar/calibration fields (float64 camera math, vfs_b200.synthetic.vector_fields).

``value``: device time of K steps with inputs resident in HBM (CUDA events on
the solve's stream; L2 is flushed by writing 256 MiB between steps, outside
the timed events).  ``e2e``: the same through the public Python API from
pinned host images, with the host->device copy of both images and the
device->host copy of the depth map inside the timed region.  ``batched``: the
32-pair uneven workload in one batched graph (pairs sharded over ranks by
cost); ``batched800``: eight pairs of the headline configuration per GPU in
one batched graph (the fused-batched form of ``value``, which solves one pair
at a time).  ``parity_vs_reference``: after the timed region, the same pair solved
by the reference's own kernels (oracle/_ref), compared bit for bit.

With N > 1 GPUs (``--gpus N`` starts the N ranks through torch.distributed.run
when it is not already running under it) each rank solves its own pair (weak
scaling, no collective on the data path); times are the max over ranks (NCCL).
``--dry-run`` runs the rank plumbing on CPU with gloo and no GPU work.

``--impl reference``: the reference's own CUDA kernels (built from its sources
into oracle/_ref) under the reference's host loop, which launches one kernel
per step and synchronises the device after each, on the same pair; rank 0
only.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "vfs-python_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "depth maps/s at 800² fused-batched vs plain on one B200 @≤1e-4 err; fwd+bwd/s"
UNIT = "depth maps/s"
SIZE = 800
T = (0.12, 0.01, 0.0)
N_LEVEL, N_WARP, N_ITER = 5, 10, 100
ALG_BYTES_ITER, ALG_BYTES_WARP, ALG_BYTES_LEVEL = 113, 60, 41


def params():
    from vfs_b200.vfs_params import vfs_params
    p = vfs_params()
    p.width = p.height = SIZE
    p.nLevel, p.fScale, p.nWarpIters, p.nSolverIters = N_LEVEL, 2.0, N_WARP, N_ITER
    p.Lambda, p.alpha0, p.alpha1, p.beta, p.gamma = 50.0, 17.0, 1.2, 9.0, 0.85
    p.timeStepLambda, p.limitRange = 1.0, 0.1
    return p


def level_pixels(p):
    out, h, w = [], p.height, p.width
    for _ in range(p.nLevel):
        out.append(h * w)
        h, w = int(h / p.fScale), int(w / p.fScale)
    return out


def alg_bytes_per_map(p):
    return sum(n * (p.nWarpIters * (p.nSolverIters * ALG_BYTES_ITER + ALG_BYTES_WARP) + ALG_BYTES_LEVEL)
               for n in level_pixels(p))


def variant_iters(variant):
    """Iterations per launch of a compiled TGV kernel variant (0 for an id
    that is not one, such as the cluster-resident kernel's)."""
    from vfs_b200 import _lib
    lib = _lib.lib()
    n = lib.vfs_tgv_variants(None, 0, None)
    ids, its = (ctypes.c_int * n)(), (ctypes.c_int * n)()
    lib.vfs_tgv_variants(ids, n, its)
    return dict(zip(ids, its)).get(variant, 0)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to start: wait for its first row (taken
            # before the timed region, so dropped) so that the 200 ms samples
            # cover the whole timed region
            t0 = time.time()
            while not self.rows and time.time() - t0 < 10 and self.proc.poll() is None:
                time.sleep(0.02)
            self.rows.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for n, v in zip(names, r[4:8]):
                    if v.lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def launch_ranks(args) -> int:
    """--gpus N outside torch.distributed.run: start N ranks through it (one
    process per GPU, rendezvous on 127.0.0.1) with the same arguments; rank 0
    prints the line.  Returns the launcher's exit status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def dist_init(dry_run=False):
    n = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not dry_run:
        torch.cuda.set_device(local)
    if n > 1:
        import datetime
        if dry_run:
            torch.distributed.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        else:
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                                 device_id=torch.device("cuda", local))
    return n, rank, local


def max_over_ranks(x: float, n: int) -> float:
    """Max over ranks (NCCL on GPUs, gloo in a dry run): time-like figures."""
    from vfs_b200.distributed import max_over_ranks as _max
    return float(x) if n == 1 else _max(x)


def barrier(n, dry_run=False):
    if n > 1:
        torch.distributed.barrier()
    if not dry_run:
        torch.cuda.synchronize()


def cpu_model() -> str:
    """lscpu's model name of this host (or /proc/cpuinfo's)."""
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in out.splitlines():
            if line.startswith("Model name:"):
                return line.split(":", 1)[1].strip()
    except (OSError, subprocess.SubprocessError):
        pass
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def make_inputs(seed):
    from vfs_b200.synthetic import make_pair
    return make_pair(SIZE, T, seed=seed, n_level=N_LEVEL)


def setup_b200(pair, p):
    """The drop-in VFS set up for one pair, with the pair's float64 fields
    (the same arrays the reference arm and the parity check get)."""
    from vfs_b200 import VFS, EquidistantCam
    from vfs_b200.synthetic import vector_fields
    cam = EquidistantCam(pair.intrinsics)
    cam.setup_module()
    tvf, cvf = vector_fields(pair)
    vfs = VFS(p)
    vfs.setup_module()
    vfs.compute_pyramid_sizes()
    vfs.create_mask_pyramid(pair.mask)
    vfs.create_vector_field_pyramid(tvf, cvf)
    return vfs, cam


def cpu_baseline_sample(pair, p, budget_s=20.0):
    """float64 NumPy oracle on the host, one core: the finest level's
    per-level and per-warp work plus a few TGV iterations, extrapolated to a
    full depth map by pixel-iteration counts."""
    from oracle.np64 import vfs64 as V
    cam = V.EquidistantCam64(pair.intrinsics)
    tvf, cvf = V.get_vector_fields(V.get_grid_zero(pair.img_ref.shape), cam, cam, pair.R, pair.t, 1)
    v = V.VFS64(p)
    v.compute_pyramid_sizes()
    v.create_mask_pyramid(pair.mask)
    v.create_vector_field_pyramid(tvf, cvf)
    v.create_image_pyramid(pair.img_ref, pair.img_other)
    M = v.masks[0]
    s = v.sizes[0]
    t0 = time.perf_counter()
    sm = V.gaussian_masked(v.refs[0], M)
    abc, eta = V.compute_tensor_eta(sm, M, p)
    t_level = time.perf_counter() - t0
    warp = np.zeros((*s, 2))
    u = np.zeros(s)
    u_ = np.zeros(s)
    t0 = time.perf_counter()
    tvec = V.find_warping_vector(v.translations[0], warp)
    warped = V.warping_image(v.others[0], warp)
    deriv = V.compute_derivatives(v.refs[0], warped, v.translations[0])
    t_warp = time.perf_counter() - t0
    p_ = np.zeros((*s, 2))
    q = np.zeros((*s, 4))
    vb = np.zeros((*s, 2))
    ub4 = u.copy()
    sched = V.step_schedule(p.nSolverIters, p.timeStepLambda)
    n_it = 0
    t0 = time.perf_counter()
    for sigma, tau, mu in sched:
        p_, tp, q = V.update_dual_variables(p_, q, sigma, u_, vb, abc, M, p)
        u = V.l1_thresholding(tau, tp, u, u_, deriv, eta, M, p)
        u_, vb = V.update_primal_variables(tau, mu, p_, q, u, u_, vb, abc, eta, M, p)
        n_it += 1
        if time.perf_counter() - t0 > budget_s or n_it >= 20:
            break
    t_iter = (time.perf_counter() - t0) / n_it
    t1 = time.perf_counter()
    med = V.median_filter(u, M)
    V.compute_optical_flow_with_clamp(warp, ub4, med, tvec, M, p)
    t_warp += time.perf_counter() - t1
    n0 = s[0] * s[1]
    per_px = lambda t: t / n0
    t_map = sum(n * (p.nWarpIters * (p.nSolverIters * per_px(t_iter) + per_px(t_warp)) + per_px(t_level))
                for n in level_pixels(p))
    return {"value": 1.0 / t_map, "unit": UNIT, "cores": 1, "kind": "port", "cpu_model": cpu_model(),
            "host_cpus": os.cpu_count(),
            "sample": f"float64 NumPy oracle (one thread) at 800x800: the finest level's per-level and per-warp "
                      f"work once and {n_it} TGV iterations ({t_iter:.2f} s each), extrapolated by pixel-iterations "
                      f"to 5 levels x 10 warps x 100 iterations ({t_map:.0f} s per map)"}


def parity_vs_reference(pair, p, flow, xyz):
    """Checker, outside every timed region: the same pair (images, mask,
    fields, parameters) solved by the reference's own kernels (oracle/_ref,
    built from the reference's sources) under the reference's host loop,
    compared with this run's flow and xyz.  Depth error over mask != 0 where
    the reference depth is finite and in (0, 100] m."""
    from oracle.refgpu import refpath
    from vfs_b200.synthetic import vector_fields
    tvf, cvf = vector_fields(pair)
    r = refpath.RefVFS(p, "bench")
    r.compute_pyramid_sizes()
    r.create_mask_pyramid(pair.mask)
    r.create_vector_field_pyramid(tvf, cvf)
    cam = refpath.RefEquidistantCam(pair.intrinsics, "bench")
    cam.setup_module()
    rflow = r.solve_stereo(pair.img_ref, pair.img_other).cpu().numpy()
    rxyz = r.triangulate_flow(cam, pair.t).cpu().numpy()
    flow, xyz = np.ascontiguousarray(flow), np.ascontiguousarray(xyz)
    zr, zo = rxyz[..., 2].astype(np.float64), xyz[..., 2].astype(np.float64)
    sel = (pair.mask != 0) & np.isfinite(zr) & (zr > 0) & (zr <= 100)
    both = np.isfinite(rflow) & np.isfinite(flow)
    return {"checker": "reference kernels (oracle/_ref) on the same pair, fields and parameters",
            "flow_values_differing": int(np.count_nonzero(rflow.view(np.uint32) != flow.view(np.uint32))),
            "xyz_values_differing": int(np.count_nonzero(rxyz.view(np.uint32) != xyz.view(np.uint32))),
            "flow_values": int(flow.size),
            "max_abs_flow_diff_px": float(np.abs(rflow[both] - flow[both]).max()) if both.any() else None,
            "median_rel_depth_err": float(np.median(np.abs(zo[sel] - zr[sel]) / zr[sel])) if sel.any() else None,
            "depth_pixels_compared": int(sel.sum())}


# ncu captures of the finest level's kernel, by TGV variant
TRAFFIC_FILES = {232: "k_tgv_reg_26x26_800x800_ncu.json", 221: "k_tgv_reg_36x36_800x800_ncu.json",
                 134: "k_tgv_reg_800x800_ncu.json"}


def load_traffic(name="k_tgv_reg_800x800_ncu.json"):
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def run_b200(args, n, rank, local):
    p = params()
    pair = make_inputs(seed=rank)
    vfs, cam = setup_b200(pair, p)
    vfs.configure(iters_per_launch=args.iters_per_launch, use_graph=not args.no_graph, timing=True)
    ref_d = torch.as_tensor(pair.img_ref).cuda()
    oth_d = torch.as_tensor(pair.img_other).cuda()
    if args.level_variants:
        level_choice = [int(v) for v in args.level_variants.split(",")]
        vfs.set_level_variants(level_choice)
    else:
        level_choice = vfs.autotune(ref_d, oth_d) if not args.no_autotune else None
    tune_top = None
    if level_choice and not args.level_variants:
        from vfs_b200.autotune import last_table
        tab = (last_table(vfs) or {}).get("table", {})
        tune_top = [sorted(((round(ms[l], 3), int(v)) for v, ms in tab.items()))[:4] for l in range(N_LEVEL)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        vfs.solve_stereo(ref_d, oth_d)
        return vfs.triangulate_flow(cam, pair.t)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kernels = vfs.solve_stats()["kernels_per_solve"] + 1

    # ---- device-resident throughput
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    tgv_ms = tgv_ms_fine = tgv_bytes = 0.0
    tgv_launches = 0
    barrier(n)
    torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed steps (ncu --nvtx-include timed/)
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
            st = vfs.solve_stats()  # synchronises
            tgv_ms += st["tgv_ms"]
            tgv_ms_fine += st["tgv_ms_level"][0]
            tgv_bytes += st["tgv_alg_bytes"]
            tgv_launches += st["tgv_launches"]
    torch.cuda.nvtx.range_pop()
    barrier(n)
    elapsed = sum(a.elapsed_time(b) for a, b in ev) / 1e3
    t_max = max_over_ranks(elapsed, n)
    value = n * args.steps / t_max

    # ---- end to end through the public API from pinned host memory
    h_ref = torch.as_tensor(pair.img_ref).pin_memory()
    h_oth = torch.as_tensor(pair.img_other).pin_memory()
    h_depth = torch.empty((SIZE, SIZE), dtype=torch.float32).pin_memory()

    def e2e_step():
        d_ref = h_ref.to("cuda", non_blocking=True)
        d_oth = h_oth.to("cuda", non_blocking=True)
        vfs.solve_stereo(d_ref, d_oth)
        xyz = vfs.triangulate_flow(cam, pair.t)
        h_depth.copy_(xyz[:, :, 2], non_blocking=True)

    xyz_np = step().cpu().numpy()  # one more solve, for the parity check
    flow_np = vfs.warpUV.cpu().numpy()
    vfs.configure(timing=False)
    for _ in range(args.warmup):
        e2e_step()
    barrier(n)
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        ev2[i][0].record(stream)
        e2e_step()
        ev2[i][1].record(stream)
        ev2[i][1].synchronize()
    barrier(n)
    e2e_t = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev2) / 1e3, n)
    e2e_value = n * args.steps / e2e_t
    depth = h_depth.numpy()
    m = (pair.mask > 0) & (pair.depth > 0)

    peak, peak_kind = measured_peak()
    # the dominant kernel: the finest level's TGV kernel (one variant, one
    # shape); its launches per solve are nWarpIters x ceil(nSolverIters / K)
    # and each processes K iterations of every pixel of the level
    fine = level_choice[0] if level_choice else args.iters_per_launch
    k_fine = variant_iters(fine) or N_ITER  # the cluster-resident kernel: one launch per warp
    fine_launches = N_WARP * -(-N_ITER // k_fine)
    fine_bytes_per_launch = SIZE * SIZE * ALG_BYTES_ITER * (N_ITER * N_WARP) / fine_launches
    fine_launch_us = 1e3 * tgv_ms_fine / (fine_launches * args.steps) if tgv_ms_fine > 0 else None
    achieved = fine_bytes_per_launch / (fine_launch_us / 1e6) / 1e9 if fine_launch_us else None
    all_achieved = tgv_bytes / (tgv_ms / 1e3) / 1e9 if tgv_ms > 0 else None
    traffic = None
    tr = load_traffic(TRAFFIC_FILES[fine]) if fine in TRAFFIC_FILES else None
    if tr:
        traffic = tr["dram_bytes_per_alg_byte"] * fine_bytes_per_launch
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": n, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded range field + value-noise texture, 800x800 fisheye pair per rank)",
        "config": {"workload": "800x800 equidistant fisheye pair, 5 levels x 10 warps x 100 TGV iterations, "
                               "solve_stereo + triangulate_flow",
                   "size": SIZE, "levels": N_LEVEL, "warps": N_WARP, "iterations": N_ITER, "lambda": 50.0,
                   "t": list(T), "tgv_kernel_default": args.iters_per_launch,
                   "tgv_kernel_per_level": level_choice, "cuda_graph": not args.no_graph,
                   "autotune_fastest_per_level_ms_variant": tune_top,
                   "l2": "flushed between steps (256 MiB write outside the timed events)",
                   "parallelism": f"dp{n} (independent pairs)"},
        "roofline": {"bound": "hbm",
                     "kernel": f"k_tgv_reg variant {fine} (fused TGV, {k_fine} iterations per launch) on the "
                               f"{SIZE}x{SIZE} level",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                     "traffic": traffic,
                     "alg_bytes_per_launch": fine_bytes_per_launch, "avg_launch_us": fine_launch_us,
                     "launches_per_step": fine_launches,
                     "share_of_step": (tgv_ms_fine / 1e3) / elapsed if elapsed else None,
                     "basis": "113 algorithmic bytes per pixel-iteration x the level's pixels x the launch's "
                              "iterations, over the launches' CUDA-event time (events around each warp's TGV "
                              "launches of the level, summed over the timed steps)",
                     "all_tgv_levels": {"achieved": all_achieved,
                                        "frac": (all_achieved / peak) if all_achieved else None,
                                        "alg_bytes_per_launch": tgv_bytes / max(tgv_launches, 1),
                                        "avg_launch_us": 1e3 * tgv_ms / max(tgv_launches, 1),
                                        "share_of_step": (tgv_ms / 1e3) / elapsed if elapsed else None}},
        "alg_bytes_per_map": alg_bytes_per_map(p),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * SIZE * SIZE,
                "d2h_bytes_per_step": 4 * SIZE * SIZE},
        "gpu_launches": int(kernels * args.steps),
        "clocks": clk.summary(),
        "depth_vs_ground_truth": {
            "median_rel_err": float(np.median(np.abs(depth[m] - pair.depth[m]) / pair.depth[m])),
            "note": "against the synthetic scene's true depth, not a parity figure: at Lambda 50 the "
                    "reference's method itself drifts from the true depth"},
    }
    if not args.no_fwd_bwd:
        # the same pair through the differentiable solve (no collective on the
        # data path: every rank measures its own), iterates checkpointed every
        # 10 iterations and recomputed in the backward, and every state recorded
        plain_ms = 1e3 * t_max / args.steps
        fbs = {}
        for ck in (10, 1):
            fb = fwd_bwd_timing(pair, p, ckpt=ck, plain_ms=plain_ms, flush=flush, local=local)
            fb["ms_fwd_bwd"] = max_over_ranks(fb["ms_fwd_bwd"], n)
            fb["ratio_to_forward"] = fb["ms_fwd_bwd"] / plain_ms
            fb["fwd_bwd_per_s"] = n * 1e3 / fb["ms_fwd_bwd"]
            fbs[ck] = fb
        line["fwd_bwd"] = fbs[10]
        line["fwd_bwd_every_state_recorded"] = fbs[1]
    del flush
    if not args.no_batched:
        line["batched"] = run_batched(args, n, rank, local, steps=max(3, min(args.steps, 10)))
        # the same 800x800 configuration fused-batched: 8 pairs per GPU in one batched graph
        line["batched800"] = run_batched800(args, n, rank, local, steps=max(3, min(args.steps, 5)))
    if rank == 0 and not args.no_parity:
        line["parity_vs_reference"] = parity_vs_reference(pair, p, flow_np, xyz_np)
    if n == 1 and rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(pair, p, budget_s=args.cpu_budget)
    return line


def _batched_pair(args):
    """One pair of the batched workload and its fields (process-pool worker)."""
    import os as _os
    import sys as _sys
    _sys.path[:0] = [ROOT, _os.path.join(ROOT, "vfs-python_b200")]
    from vfs_b200.synthetic import make_pair, vector_fields
    size, t, seed = args
    pp = make_pair(size, t, seed=seed, n_level=4)
    return pp, vector_fields(pp)


def run_batched(args, n, rank, local, steps=None):
    """32 pairs of uneven resolution, 4 levels x 10 warps x 50 iterations,
    solved as one batch (one graph, one TGV launch per pass over all pairs)."""
    import multiprocessing as mpc
    from vfs_b200.batch import VFSBatch
    from vfs_b200.distributed import shard, pair_cost
    from vfs_b200.synthetic import uneven_workload
    steps = steps or args.steps
    work = uneven_workload()
    costs = [pair_cost(s, s, 4, 2.0, 10, 50) for s, _, _ in work]
    mine = shard(costs, n, rank)
    with mpc.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        made = pool.map(_batched_pair, [work[i] for i in mine])
    pairs = [m[0] for m in made]
    p = params()
    p.nLevel, p.nWarpIters, p.nSolverIters = 4, 10, 50
    sizes = [pp.img_ref.shape for pp in pairs]
    batch = VFSBatch(p, sizes)
    for i, (pp, (tvf, cvf)) in enumerate(made):
        batch.set_pair(i, pp.mask, tvf, cvf)
    refs = [torch.as_tensor(pp.img_ref).cuda() for pp in pairs]
    oths = [torch.as_tensor(pp.img_other).cuda() for pp in pairs]
    cands = [int(c) for c in args.batch_candidates.split(",")] if args.batch_candidates else None
    choice = batch.autotune(refs, oths, candidates=cands) if not args.no_autotune else None
    batch.configure(use_graph=True, timing=True)
    for _ in range(args.warmup):
        batch.solve(refs, oths)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    barrier(n)
    tot = 0.0
    tgv = 0.0
    with ClockSampler(local) as clk:
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            batch.solve(refs, oths)
            e1.record()
            e1.synchronize()
            tot += e0.elapsed_time(e1) / 1e3
            tgv += batch.stats()["tgv_ms"] / 1e3
    barrier(n)
    t_max = max_over_ranks(tot, n)
    value = len(work) * steps / t_max
    del flush
    batch.release()
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": n, "steps": steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_max / steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (per-pair seeds)",
            "config": {"workload": "batched: 32 pairs, sides from {480, 640, 800, 1024}, random translation "
                                   "directions, 4 levels x 10 warps x 50 TGV iterations, one batched graph",
                       "pairs_this_rank": len(pairs), "tgv_kernel_per_level": choice,
                       "parallelism": f"dp{n} (pairs sharded by cost)",
                       "l2": "flushed between steps (256 MiB write outside the timed events)"},
            "tgv_share_of_step": tgv / tot if tot else None, "clocks": clk.summary()}


def run_batched800(args, n, rank, local, steps=None):
    """The 800x800 drop-in configuration (5 levels x 10 warps x 100
    iterations) for several pairs at once (per-pair seeds): one batched graph
    per step, then each pair's triangulation.  Batching fills the SMs on the
    latency-bound coarse levels, which one pair alone cannot."""
    import multiprocessing as mpc
    from vfs_b200.batch import VFSBatch
    steps = steps or args.steps
    from vfs_b200 import EquidistantCam
    from vfs_b200.synthetic import vector_fields
    seeds = [rank * args.pairs + i for i in range(args.pairs)]
    with mpc.get_context("spawn").Pool(min(args.pairs, os.cpu_count() or 1)) as pool:
        pairs = pool.map(make_inputs, seeds)
    p = params()
    batch = VFSBatch(p, [pp.img_ref.shape for pp in pairs])
    cams = []
    for i, pp in enumerate(pairs):
        cam = EquidistantCam(pp.intrinsics)
        cam.setup_module()
        batch.set_pair(i, pp.mask, *vector_fields(pp))
        cams.append(cam)
    refs = [torch.as_tensor(pp.img_ref).cuda() for pp in pairs]
    oths = [torch.as_tensor(pp.img_other).cuda() for pp in pairs]
    choice = batch.autotune(refs, oths) if not args.no_autotune else None
    batch.configure(use_graph=True, timing=True)

    def step():
        batch.solve(refs, oths)
        return [batch.triangulate(i, cams[i], pairs[i].t) for i in range(len(pairs))]

    for _ in range(args.warmup):
        step()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    barrier(n)
    tot = tgv = 0.0
    tgv_level = None
    with ClockSampler(local) as clk:
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            step()
            e1.record()
            e1.synchronize()
            tot += e0.elapsed_time(e1) / 1e3
            st = batch.stats()
            tgv += st["tgv_ms"] / 1e3
            lv = st.get("tgv_ms_level")
            if lv is not None:
                tgv_level = list(lv) if tgv_level is None else [a + b for a, b in zip(tgv_level, lv)]
    barrier(n)
    t_max = max_over_ranks(tot, n)
    value = n * len(pairs) * steps / t_max
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": n, "steps": steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_max / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (per-pair seeds)",
            "tgv_ms_per_level_per_step": [x / steps for x in tgv_level] if tgv_level else None,
            "config": {"workload": f"batched 800x800: {len(pairs)} pairs per GPU, 5 levels x 10 warps x 100 TGV "
                                   "iterations, one batched graph + triangulate_flow per pair",
                       "pairs_per_gpu": len(pairs), "tgv_kernel_per_level": choice,
                       "parallelism": f"dp{n} (independent pairs)",
                       "l2": "flushed between steps (256 MiB write outside the timed events)"},
            "tgv_share_of_step": tgv / tot if tot else None, "clocks": clk.summary()}


def run_reference(args, n, rank, local):
    """The reference's CUDA kernels (oracle/_ref) under the reference's host
    loop (Python/vfs.py:460-559), allocating as CuPy does (no fill kernels for
    cp.empty arrays), on the same pair, fields and parameters as the B200 arm;
    L2 flushed between steps outside the timed events, as in the B200 arm."""
    from oracle.refgpu import refpath
    from vfs_b200.synthetic import vector_fields
    refpath.set_plain_allocation(True)
    p = params()
    pair = make_inputs(seed=0)
    tvf, cvf = vector_fields(pair)
    r = refpath.RefVFS(p, "bench")
    r.compute_pyramid_sizes()
    r.create_mask_pyramid(pair.mask)
    r.create_vector_field_pyramid(tvf, cvf)
    cam = refpath.RefEquidistantCam(pair.intrinsics, "bench")
    cam.setup_module()

    def step():
        r.solve_stereo(pair.img_ref, pair.img_other)
        return r.triangulate_flow(cam, pair.t)

    for _ in range(args.warmup):
        step()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    el = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            step()
            e1.record()
            e1.synchronize()
            el += e0.elapsed_time(e1) / 1e3
    value = args.steps / el
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "impl": "reference", "data": "synthetic (same pair and fields as the b200 arm, seed 0)",
        "config": {"workload": "800x800 equidistant fisheye pair, 5 levels x 10 warps x 100 TGV iterations, "
                               "solve_stereo + triangulate_flow",
                   "size": SIZE, "levels": N_LEVEL, "warps": N_WARP, "iterations": N_ITER, "lambda": 50.0,
                   "t": list(T), "parallelism": "single GPU",
                   "allocation": "as CuPy: cp.empty -> uninitialised, cp.zeros -> zero-filled (torch's caching "
                                 "allocator in place of CuPy's pool)",
                   "l2": "flushed between steps (256 MiB write outside the timed events)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference", "cpu_model": cpu_model(),
                         "sample": f"{args.steps} full 800x800 solves: the reference's CUDA kernels on the B200, "
                                   "launched and synchronised one at a time by one host thread"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
        "wall_s": time.perf_counter() - t0,
    }


def loss_mask(depth, valid):
    """Pixels the depth loss uses: inside the mask with a plausible depth.  Near
    the epipoles the flow carries almost no disparity and the triangulated
    depth (and its float32 gradient, which grows as 1/disparity^2) explodes."""
    return valid & torch.isfinite(depth) & (depth > 0) & (depth < 50)


def _grad_step_parts(solver, ref_f, oth_f, t, theta, gt, valid):
    """One forward + backward through DepthSolver with an L1 depth loss; returns the cotangents."""
    depth = solver.forward_pass(ref_f, oth_f, t, theta)
    m = loss_mask(depth, valid)
    g = torch.where(m, torch.sign(depth - gt), torch.zeros_like(depth)) / m.sum().clamp(min=1)
    return solver.backward_pass(g)


# ncu captures of the reverse kernel, by reverse form
REV_TRAFFIC_FILES = {23: "k_rev_block_24x21_800x800_ncu.json", 20: "k_rev_block_28x16_800x800_ncu.json",
                     11: "k_rev_block_800x800_ncu.json"}


def reverse_roofline(solver, run_once):
    """Live roofline of the reverse TGV launches: one extra forward + backward
    with event timing around the reverse launches (outside any timed loop);
    traffic from the capture of the finest level's reverse form."""
    forms = getattr(solver, "level_forms", None) or [11]
    tr = load_traffic(REV_TRAFFIC_FILES[forms[0]]) if forms[0] in REV_TRAFFIC_FILES else None
    solver.set_timing(True)
    run_once()
    st = solver.backward_stats()
    solver.set_timing(False)
    peak, kind = measured_peak()
    achieved = st["tgv_alg_bytes"] / (st["tgv_ms"] / 1e3) / 1e9 if st["tgv_ms"] > 0 else None
    return {"bound": "hbm", "kernel": f"k_rev_block (reverse TGV iterations; finest level form {forms[0]})",
            "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "peak_source": kind,
            "alg_bytes_per_pixel_iteration": 241, "alg_bytes_per_launch": st["tgv_alg_bytes"] / max(st["tgv_launches"], 1),
            "avg_launch_us": 1e3 * st["tgv_ms"] / max(st["tgv_launches"], 1), "reverse_tgv_ms": st["tgv_ms"],
            "reverse_tgv_ms_per_level": st["tgv_ms_level"], "recompute_ms": st.get("recompute_ms"),
            "traffic": (tr["dram_bytes_per_alg_byte"] * st["tgv_alg_bytes"] / max(st["tgv_launches"], 1)) if tr else None}


def fwd_bwd_timing(pair, p, steps=3, warmup=1, ckpt=1, plain_ms=None, flush=None, local=0):
    """Forward + hand-written backward of one solve through DepthSolver (L1
    depth loss against the pair's ground truth), per-level reverse forms
    autotuned first.  Device time with inputs resident."""
    from vfs_b200 import DepthSolver, EquidistantCam
    cam = EquidistantCam(pair.intrinsics)
    solver = DepthSolver(p, cam, pair.mask, t_scale=1.0, ckpt_every=ckpt)
    ref_f = torch.as_tensor(pair.img_ref).float().cuda()
    oth_f = torch.as_tensor(pair.img_other).float().cuda()
    t = torch.tensor(np.asarray(pair.t, np.float64).reshape(3))
    theta = solver.theta_of()
    gt = torch.as_tensor(pair.depth).cuda()
    valid = torch.as_tensor(pair.mask != 0).cuda()
    forms = solver.autotune(ref_f, oth_f, t, theta)
    for _ in range(warmup):
        _grad_step_parts(solver, ref_f, oth_f, t, theta, gt, valid)
    torch.cuda.synchronize()
    f_ms = b_ms = 0.0
    with ClockSampler(local) as clk:
        for _ in range(steps):
            if flush is not None:
                flush.zero_()
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record()
            depth = solver.forward_pass(ref_f, oth_f, t, theta)
            e[1].record()
            m = loss_mask(depth, valid)
            g = torch.where(m, torch.sign(depth - gt), torch.zeros_like(depth)) / m.sum().clamp(min=1)
            solver.backward_pass(g)
            e[2].record()
            torch.cuda.synchronize()
            f_ms += e[0].elapsed_time(e[1])
            b_ms += e[1].elapsed_time(e[2])
    out = {"ms_fwd_bwd": (f_ms + b_ms) / steps, "ms_recording_forward": f_ms / steps, "ms_backward": b_ms / steps,
           "clocks": clk.summary(), "ckpt_every": ckpt, "reverse_forms_per_level": forms,
           "recording_forward_variants": getattr(solver, "level_variants", None),
           "workspace_gb": solver.workspace_bytes / 1e9,
           "roofline": reverse_roofline(solver, lambda: _grad_step_parts(solver, ref_f, oth_f, t, theta, gt, valid))}
    if plain_ms:
        out["ratio_to_forward"] = out["ms_fwd_bwd"] / plain_ms
    solver.release()
    return out


GRAD_WORKLOADS = {
    # 8 pairs at 512x512, 3 levels x 5 warps x 50 iterations, t = (0.1, 0, 0)
    "grad": dict(size=512, n_pairs=8, levels=3, warps=5, iters=50, ckpt=10, random_t=False),
    # parameter learning: 16 pairs at 1024x1024, 5 x 10 x 100, translation
    # direction uniform on the sphere with magnitude in [0.05, 0.3] m
    "learn": dict(size=1024, n_pairs=16, levels=5, warps=10, iters=100, ckpt=1, random_t=True),
}


def run_grad(args, n, rank, local):
    """fwd+bwd solves/s of a parameter-learning step: per pair the L1 loss of
    the depth map against ground truth and its gradients w.r.t. both images,
    t and theta; theta gradients summed over pairs and ranks (NCCL), SGD step."""
    from vfs_b200 import DepthSolver, EquidistantCam
    from vfs_b200.synthetic import make_pair
    wl = GRAD_WORKLOADS[args.workload]
    size, n_pairs = wl["size"], wl["n_pairs"]
    ckpt = args.ckpt if args.ckpt else wl["ckpt"]
    p = params()
    p.width = p.height = size
    p.nLevel, p.nWarpIters, p.nSolverIters = wl["levels"], wl["warps"], wl["iters"]
    rng = np.random.default_rng(1000 + rank)
    pairs = []
    for i in range(n_pairs):
        if wl["random_t"]:
            d = rng.standard_normal(3)
            t_i = tuple(d / np.linalg.norm(d) * rng.uniform(0.05, 0.3))
        else:
            t_i = (0.1, 0.0, 0.0)
        pairs.append(make_pair(size, t_i, seed=n_pairs * rank + i, n_level=wl["levels"]))
    cam = EquidistantCam(pairs[0].intrinsics)
    torch.cuda.reset_peak_memory_stats()
    solver = DepthSolver(p, cam, pairs[0].mask, t_scale=1.0, ckpt_every=ckpt)
    dev = [(torch.as_tensor(q.img_ref).float().cuda(), torch.as_tensor(q.img_other).float().cuda(),
            torch.tensor(np.asarray(q.t, np.float64).reshape(3)), torch.as_tensor(q.depth).cuda()) for q in pairs]
    valid = torch.as_tensor(pairs[0].mask != 0).cuda()
    theta = solver.theta_of().clone()
    forms = solver.autotune(dev[0][0], dev[0][1], dev[0][2], theta)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # the plain forward of the same pairs (solve_stereo + triangulate_flow)
    plains = []
    for q in pairs:
        vfs, cam_q = setup_b200(q, p)
        vfs.configure(use_graph=True)
        plains.append((vfs, cam_q, torch.as_tensor(q.img_ref).cuda(), torch.as_tensor(q.img_other).cuda(), q.t))
    def plain_step():
        for vfs, cam_q, a, b, tq in plains:
            vfs.solve_stereo(a, b)
            vfs.triangulate_flow(cam_q, tq)

    def step():
        # one parameter-learning step: gradients of every pair's L1 depth
        # losses, summed over pairs and (NCCL all-reduce) over ranks, then
        # an SGD update of (lambda, alpha0, alpha1, beta, gamma)
        g_theta = torch.zeros(5, dtype=torch.float64, device="cuda")
        for a, b, tq, gt in dev:
            g_theta += _grad_step_parts(solver, a, b, tq, theta, gt, valid)[3]
        if n > 1:
            torch.distributed.all_reduce(g_theta)
        # the unrolled solve's derivative can be huge (at 1024x1024, 5x10x100
        # the theta gradients measured 1e3..1e24): clip to unit norm
        g = g_theta.cpu()
        theta.sub_(args.lr * g / max(1.0, float(g.norm())))

    for _ in range(args.warmup):
        step()
        plain_step()
    barrier(n)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    evp = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record()
            step()
            ev[i][1].record()
            flush.zero_()
            evp[i][0].record()
            plain_step()
            evp[i][1].record()
        torch.cuda.synchronize()
    barrier(n)
    t_grad = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / 1e3, n)
    t_plain = max_over_ranks(sum(a.elapsed_time(b) for a, b in evp) / 1e3, n)
    value = n * n_pairs * args.steps / t_grad
    # end to end through the autograd API: pinned host images in, image and
    # parameter gradients out
    host = [(torch.as_tensor(q.img_ref).float().pin_memory(), torch.as_tensor(q.img_other).float().pin_memory())
            for q in pairs]
    h_out = [(torch.empty((size, size)).pin_memory(), torch.empty((size, size)).pin_memory(),
              torch.empty(8, dtype=torch.float64).pin_memory()) for _ in pairs]

    def e2e_step():
        for (ha, hb), (ga_h, gb_h, gs_h), (_, _, tq, gt) in zip(host, h_out, dev):
            a = ha.to("cuda", non_blocking=True).requires_grad_()
            b = hb.to("cuda", non_blocking=True).requires_grad_()
            tt = tq.clone().requires_grad_()
            th = theta.clone().requires_grad_()
            depth = solver(a, b, tt, th)
            m = loss_mask(depth.detach(), valid)
            loss = (depth - gt).abs()[m].mean()
            loss.backward()
            ga_h.copy_(a.grad, non_blocking=True)
            gb_h.copy_(b.grad, non_blocking=True)
            gs_h[:3].copy_(tt.grad, non_blocking=True)
            gs_h[3:].copy_(th.grad, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    barrier(n)
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        e2e_step()
    e1.record()
    torch.cuda.synchronize()
    barrier(n)
    e2e_t = max_over_ranks(e0.elapsed_time(e1) / 1e3, n)
    a0, b0, t0_, gt0 = dev[0]
    roof = reverse_roofline(solver, lambda: _grad_step_parts(solver, a0, b0, t0_, theta, gt0, valid))
    desc = (f"{n_pairs} pairs at {size}x{size}, {wl['levels']} levels x {wl['warps']} warps x {wl['iters']} TGV "
            f"iterations, " + ("translation direction uniform on the sphere, |t| in [0.05, 0.3] m" if wl["random_t"]
                               else "t = (0.1, 0, 0) m"))
    return {
        "metric": f"fwd+bwd solves/s ({desc}, L1 depth loss)", "value": value, "unit": "solves/s",
        "n_gpus": n, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_grad / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic ({n_pairs} seeded {size}x{size} fisheye pairs per rank)",
        "config": {"workload": desc + "; depth -> L1 loss against ground truth -> gradients w.r.t. both images, t, "
                                      "lambda, alpha0, alpha1, beta, gamma; theta gradients summed over pairs and "
                                      "ranks, clipped to unit norm, SGD step", "ckpt_every": ckpt, "reverse_forms_per_level": forms,
                   "recording_forward_variants": getattr(solver, "level_variants", None), "lr": args.lr,
                   "theta_after": [float(x) for x in theta],
                   "l2": "flushed before each step (256 MiB write outside the timed events)",
                   "parallelism": f"dp{n} (independent pairs)"},
        "forward_solves_per_s": n * n_pairs * args.steps / t_plain,
        "ratio_fwd_bwd_to_forward": t_grad / t_plain,
        "workspace_gb": solver.workspace_bytes / 1e9,
        "peak_memory_gb": torch.cuda.max_memory_allocated() / 1e9,
        "roofline": roof,
        "e2e": {"value": n * n_pairs * args.steps / e2e_t, "unit": "solves/s",
                "h2d_bytes_per_step": n_pairs * 2 * size * size * 4,
                "d2h_bytes_per_step": n_pairs * (2 * size * size * 4 + 64)},
        "clocks": clk.summary(),
    }


def dry_run(args, n, rank):
    """The multi-rank plumbing without GPU work (gloo on CPU): each rank takes
    its cost-balanced shard of the batched workload's pairs, the max of a
    per-rank time, and the sum over ranks of a per-rank theta gradient, through
    the same helpers the GPU runs use."""
    from vfs_b200.distributed import shard, pair_cost
    from vfs_b200.synthetic import uneven_workload
    work = uneven_workload()
    costs = [pair_cost(s, s, 4, 2.0, 10, 50) for s, _, _ in work]
    mine = shard(costs, n, rank)
    t_max = max_over_ranks(1.0 + rank, n)
    g = torch.tensor([rank + 1.0, 2.0 * rank, 0.5, -rank, 3.0], dtype=torch.float64)
    if n > 1:
        torch.distributed.all_reduce(g)
        shards = [None] * n
        torch.distributed.all_gather_object(shards, mine)
    else:
        shards = [mine]
    return {"dry_run": True, "n_gpus": n, "world_size": n, "workload": "batched uneven (32 pairs)",
            "shards": shards, "shard_costs": [sum(costs[i] for i in sh) for sh in shards],
            "max_over_ranks": t_max, "theta_grad_sum": g.tolist()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 40 for single, 10 for batched and grad, 3 for learn; "
                         "10 for --impl reference)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--iters-per-launch", type=int, default=134)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--level-variants", default="",
                    help="single: comma-separated TGV kernel per level, finest first (skips the autotuner)")
    ap.add_argument("--workload", default="single", choices=["single", "batched", "batched800", "grad", "learn"],
                    help="single: the 800x800 pair (default); batched: 32 uneven pairs in one batch; "
                         "batched800: --pairs 800x800 pairs in one batch; "
                         "grad: forward + backward of 8 pairs at 512x512; learn: 16 pairs at 1024x1024")
    ap.add_argument("--pairs", type=int, default=8, help="batched800: pairs per GPU")
    ap.add_argument("--batch-candidates", default="",
                    help="batched: comma-separated TGV variants the batch autotuner may choose from (default: all)")
    ap.add_argument("--ckpt", type=int, default=0,
                    help="grad/learn: TGV iterations between recorded states (0: the workload's default)")
    ap.add_argument("--lr", type=float, default=1e-3,
                    help="grad/learn: SGD step on theta (gradient clipped to unit norm) per bench step")
    ap.add_argument("--no-fwd-bwd", action="store_true", help="single: skip the fwd+bwd measurement")
    ap.add_argument("--profile-grad", action="store_true",
                    help="with --profile-case: one forward + backward at the finest level only, 1 warp, "
                         "8 TGV iterations, every state recorded, reverse form --reverse-form")
    ap.add_argument("--reverse-form", type=int, default=11)
    ap.add_argument("--trace-variant", type=int, default=0,
                    help="with --profile-grad: TGV variant of the recording forward, one with a recording "
                         "form (0: the default, 134)")
    ap.add_argument("--no-batched", action="store_true", help="single: skip the batched uneven workload")
    ap.add_argument("--no-parity", action="store_true",
                    help="single: skip the parity check against the reference kernels")
    ap.add_argument("--dry-run", action="store_true",
                    help="rank plumbing only, on CPU with gloo: shards, max-over-ranks and the theta-gradient "
                         "sum; no GPU work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--profile-case", action="store_true",
                    help="small case for ncu: the 800x800 finest level only, 1 warp, 20 TGV iterations, "
                         "kernel --iters-per-launch everywhere (1000: cluster kernel), no graph; two solves")
    ap.add_argument("--profile-size", type=int, default=SIZE)
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 10 if args.impl == "reference" else {"single": 40, "batched": 10, "batched800": 10, "grad": 10,
                                                            "learn": 3}[args.workload]
    args.warmup = max(args.warmup, 1)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args))
    if args.dry_run:
        n, rank, local = dist_init(dry_run=True)
        line = dry_run(args, n, rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if n > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    if args.profile_case and args.profile_grad:
        torch.cuda.set_device(0)
        from vfs_b200 import DepthSolver, EquidistantCam
        from vfs_b200.synthetic import make_pair
        p = params()
        p.width = p.height = args.profile_size
        p.nLevel, p.nWarpIters, p.nSolverIters = 1, 1, 8
        pair = make_pair(args.profile_size, T, seed=0, n_level=N_LEVEL)
        solver = DepthSolver(p, EquidistantCam(pair.intrinsics), pair.mask, ckpt_every=1,
                             level_variants=[args.trace_variant] if args.trace_variant else None)
        solver.set_options(args.reverse_form, 0)
        gt = torch.as_tensor(pair.depth).cuda()
        valid = torch.as_tensor(pair.mask != 0).cuda()
        for _ in range(2):
            _grad_step_parts(solver, torch.as_tensor(pair.img_ref).float().cuda(),
                             torch.as_tensor(pair.img_other).float().cuda(),
                             torch.tensor(np.asarray(pair.t, np.float64).reshape(3)), solver.theta_of(), gt, valid)
        torch.cuda.synchronize()
        print("profile case done")
        return
    if args.profile_case:
        torch.cuda.set_device(0)
        p = params()
        p.nLevel, p.nWarpIters, p.nSolverIters = 1, 1, 20
        from vfs_b200.synthetic import make_pair
        pair = make_pair(args.profile_size, T, seed=0, n_level=N_LEVEL)
        p.width = p.height = args.profile_size
        vfs, _ = setup_b200(pair, p)
        if args.iters_per_launch == 1000:  # the cluster-resident kernel
            vfs.configure(use_graph=False, timing=False)
            vfs.set_level_variants([1000])
        else:
            vfs.configure(iters_per_launch=args.iters_per_launch, use_graph=False, timing=False)
        ref_d = torch.as_tensor(pair.img_ref).cuda()
        oth_d = torch.as_tensor(pair.img_other).cuda()
        for _ in range(2):
            vfs.solve_stereo(ref_d, oth_d)
        torch.cuda.synchronize()
        print("profile case done")
        return
    n, rank, local = dist_init()
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, n, rank, local)), flush=True)
    elif args.workload in ("batched", "batched800"):
        line = (run_batched if args.workload == "batched" else run_batched800)(args, n, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    elif args.workload in ("grad", "learn"):
        line = run_grad(args, n, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    else:
        line = run_b200(args, n, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    if n > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
