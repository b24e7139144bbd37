// Fused TGV solver iterations: state and constant plane sets, launch entry.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "vfs_kernels.cuh"
#include "vfs_pixel.cuh"

namespace vfs {

// Asynchronous global -> shared copies (cp.async): 4 or 16 bytes, zero-filled
// where !ok (the source is then not read); a commit closes a group, a wait
// blocks until at most NG groups are still in flight.
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async16(float* dst, const float* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(ok ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NG>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NG) : "memory"); }

// Solver state of one warp, structure of arrays, flat row-major planes of
// h*w floats (row stride exactly w, as the reference's flat neighbour reads
// assume).  u: thresholded flow increment; ub, vbx, vby: the over-relaxed
// (bar) primal variables u_ and v_; p (2) and q (4): dual variables.
struct TgvState {
  float *u, *ub, *vbx, *vby, *px, *py, *qx, *qy, *qz, *qw;
};

// Per-warp constants, same flat layout: diffusion tensor (a, b, c), the
// preconditioner eta (x, y, z), the image derivatives (iu, iz) and the mask
// code (self/E/W/S/N bits).
struct TgvConsts {
  const float *a, *b, *c, *ex, *ey, *ez, *iu, *iz;
  const uint8_t* code;
  // the same constants as two 16-byte records per pixel, rec[2 f] =
  // (a, b, c, ex) and rec[2 f + 1] = (ey, ez, iu, iz): the register-owned
  // kernels load them with two vector loads instead of eight scalar ones
  // (required by those kernels; the others read the planes)
  const float4* rec = nullptr;
};

// One image of a batched TGV launch: its two state sets (ping-pong), its
// per-warp constants, its size and where its tiles start in the launch.
struct TgvBatchItem {
  TgvState st[2];
  TgvConsts cst;
  int h, w, tiles_x, tile_base;
};

// Tile shape of a register-owned variant (false for other variants).
bool tgv_tile_shape(int variant, int* tx, int* ty);

// The work list of one batched launch, passed by value as the kernel's
// parameter (so the kernel reads the items' pointers from the constant
// parameter space, as a single-image launch reads its arguments): up to
// kBatchParamItems images whose tiles are bid0 .. bid0 + n_tiles - 1 of the
// items' tile numbering (TgvBatchItem::tile_base).
constexpr int kBatchParamItems = 32;
struct TgvBatchParams {
  int n_items, bid0;
  TgvBatchItem items[kBatchParamItems];
};

// Batched launch of a register-owned variant over n_tiles blocks: the items
// read st[parity] and write st[parity ^ 1].
cudaError_t launch_tgv_batch(int variant, const TgvBatchParams& P, int n_tiles, int parity, const float3* sched,
                             int it0, int niter, const SolverConsts& kc, cudaStream_t s);

// Sets the kernels' shared-memory attributes (call before any graph capture).
cudaError_t tgv_prepare();

// Iterations per launch of each compiled variant (0 if unknown), and the
// list of compiled variant ids (returns the count; writes up to cap ids).
int tgv_variant_list(int* ids, int cap);
int tgv_max_iters_per_launch(int variant);

// Runs `niter` (<= the variant's K) iterations starting at schedule index
// it0, reading `in` and writing `out` (distinct buffer sets).  `sched[i]` is
// (sigma, tau, mu) of iteration i.
cudaError_t launch_tgv_block(int variant, const TgvState& in, const TgvState& out, const TgvConsts& c,
                             const float3* sched, int it0, int niter, const SolverConsts& kc, int h, int w,
                             cudaStream_t s);

// Recording form of a register-owned variant (tgv_has_trace): runs `niter`
// (<= K) iterations from `in` and writes the state after iteration s to
// record s - 1 of the trace: the state set whose planes are those of trace0
// moved by (s - 1) * rec_stride floats.
bool tgv_has_trace(int variant);
cudaError_t launch_tgv_trace(int variant, const TgvState& in, const TgvState& trace0, long rec_stride,
                             const TgvConsts& c, const float3* sched, int it0, int niter, const SolverConsts& kc,
                             int h, int w, cudaStream_t s);

// Cluster-resident solve of a whole level (vfs_tgv_cluster.cu): all `niter`
// iterations, then median filter and clamped flow update, in one launch of a
// `cluster`-CTA cluster.  tgv_cluster_size returns the cluster size to use for
// an h x w level (0 if the level does not fit); tgv_cluster_prepare sets the
// kernel attributes and reports the largest cluster the device co-schedules.
int tgv_cluster_size(int h, int w, int max_cluster);
cudaError_t tgv_cluster_prepare(int* max_cluster);
cudaError_t launch_tgv_cluster(int cluster, const TgvState& st, const TgvConsts& c, const float3* sched, int niter,
                               const SolverConsts& kc, Plane<float2> warp, Plane<float> ubefore,
                               Plane<const float2> tvec, float limit, int h, int w, cudaStream_t s);

}  // namespace vfs
