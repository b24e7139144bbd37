// Temporally blocked TGV-L1 primal-dual iterations (the solver loop of
// Python/vfs.py:498-515: updateDualVariables -> l1Thresholding ->
// updatePrimalVariables, Python/vfs.cu:326-581), fused into one kernel that
// runs `k <= K` iterations per launch on a tile held in shared memory.
//
// Geometry.  One iteration at a pixel reads the previous state up to 2 pixels
// towards W/N and 1 pixel towards E/S (the threshold and primal steps read
// tp and q at the W and N neighbours, which the dual step forms from u_ and
// v_ one pixel further out).  A CTA therefore loads its TX x TY tile plus a
// halo of 2K pixels on the low sides and K on the high sides, iterates in
// shared memory while the valid region shrinks by (2, 1) per iteration, and
// writes back only the tile.  State is ping-ponged between two buffer sets
// across launches, so a CTA never reads what a neighbour wrote in the same
// launch.
//
// Flat addressing.  The reference reads data neighbours at flat offsets
// index+-1 and index+-width (row-major, wrapping across rows at the image's
// left and right edges), while it reads the mask in 2-D with edge clamping.
// The window here maps window pixel (wx, wy) to flat index
// (y0-2K+wy)*W + (x0-2K+wx), so every neighbour in the window is the flat
// neighbour the reference reads, including the row wrap; the mask is carried
// as a per-pixel code (self/E/W/S/N bits, computed in 2-D once per level)
// addressed the same flat way.  Flat positions outside [0, H*W) hold zero
// state and a zero code, which is what the reference's guarded reads see and
// keeps them at zero.
//
// Per-pixel arithmetic is vfs_pixel.cuh's, shared with the one-kernel-per-
// step entry points, so the fused solver is bit-identical to them.
#include <cstdio>
#include <string>

#include "vfs_tgv.cuh"

namespace vfs {
namespace {

// Shared-memory planes (structure of arrays, one float per pixel each).
enum SmemPlane {
  sU, sUB, sVBX, sVBY, sPX, sPY, sQX, sQY, sQZ, sQW, sTPX, sTPY,
  sA, sB, sC, sEX, sEY, sEZ, sIU, sIZ, kNumPlanes
};

template <int K, int TX, int TY>
struct TgvGeom {
  static constexpr int WX = TX + 3 * K;
  static constexpr int WY = TY + 3 * K;
  static constexpr int N = WX * WY;
  static constexpr size_t smem_bytes() { return (size_t)kNumPlanes * N * sizeof(float) + ((N + 15) / 16) * 16; }
};

template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) k_tgv_block(TgvState in, TgvState out, TgvConsts cst,
                                                  const float3* __restrict__ sched, int it0, int niter,
                                                  SolverConsts kc, int h, int w) {
  using G = TgvGeom<K, TX, TY>;
  extern __shared__ float4 smem_raw[];
  float* sm = reinterpret_cast<float*>(smem_raw);
  uint8_t* scode = reinterpret_cast<uint8_t*>(sm + (size_t)kNumPlanes * G::N);
  auto P = [&](int plane) { return sm + (size_t)plane * G::N; };

  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const long n = (long)h * w;
  const long base = (long)(y0 - 2 * K) * w + (x0 - 2 * K);

  // ---- load the window (state, per-warp constants, mask code)
  for (int e = threadIdx.x; e < G::N; e += NT) {
    const int wy = e / G::WX, wx = e - wy * G::WX;
    const long f = base + (long)wy * w + wx;
    const bool ok = f >= 0 && f < n;
    P(sU)[e] = ok ? in.u[f] : 0.f;
    P(sUB)[e] = ok ? in.ub[f] : 0.f;
    P(sVBX)[e] = ok ? in.vbx[f] : 0.f;
    P(sVBY)[e] = ok ? in.vby[f] : 0.f;
    P(sPX)[e] = ok ? in.px[f] : 0.f;
    P(sPY)[e] = ok ? in.py[f] : 0.f;
    P(sQX)[e] = ok ? in.qx[f] : 0.f;
    P(sQY)[e] = ok ? in.qy[f] : 0.f;
    P(sQZ)[e] = ok ? in.qz[f] : 0.f;
    P(sQW)[e] = ok ? in.qw[f] : 0.f;
    P(sA)[e] = ok ? cst.a[f] : 0.f;
    P(sB)[e] = ok ? cst.b[f] : 0.f;
    P(sC)[e] = ok ? cst.c[f] : 0.f;
    P(sEX)[e] = ok ? cst.ex[f] : 0.f;
    P(sEY)[e] = ok ? cst.ey[f] : 0.f;
    P(sEZ)[e] = ok ? cst.ez[f] : 0.f;
    P(sIU)[e] = ok ? cst.iu[f] : 0.f;
    P(sIZ)[e] = ok ? cst.iz[f] : 0.f;
    scode[e] = ok ? cst.code[f] : (uint8_t)0;
  }
  __syncthreads();

  const int k = niter < K ? niter : K;
  for (int s = 1; s <= k; ++s) {
    const float3 ss = sched[it0 + s - 1];  // (sigma, tau, mu)
    const float scaleP = kc.alpha1 * ss.x / kc.etaP;
    const float scaleQ = kc.alpha0 * ss.x / kc.etaQ;
    // dual step on [lo-1, hi) x [lo-1, hi), window coordinates
    {
      const int lo = 2 * K - 2 * (k - s) - 1;
      const int hiX = 2 * K + TX + (k - s), hiY = 2 * K + TY + (k - s);
      const int ex = hiX - lo, ey = hiY - lo;
      for (int e = threadIdx.x; e < ex * ey; e += NT) {
        const int ry = e / ex, rx = e - ry * ex;
        const int i = (lo + ry) * G::WX + (lo + rx);
        const uint8_t code = scode[i];
        if (!(code & kSelf)) {
          P(sPX)[i] = P(sPY)[i] = P(sTPX)[i] = P(sTPY)[i] = 0.f;
          P(sQX)[i] = P(sQY)[i] = P(sQZ)[i] = P(sQW)[i] = 0.f;
          continue;
        }
        float2 p = make_float2(P(sPX)[i], P(sPY)[i]), tp;
        float4 q = make_float4(P(sQX)[i], P(sQY)[i], P(sQZ)[i], P(sQW)[i]);
        const float* ub = P(sUB);
        const float* vx = P(sVBX);
        const float* vy = P(sVBY);
        dual_px(code, ub[i], make_float2(vx[i], vy[i]), ub[i + 1], make_float2(vx[i + 1], vy[i + 1]), ub[i - 1],
                make_float2(vx[i - 1], vy[i - 1]), ub[i + G::WX], make_float2(vx[i + G::WX], vy[i + G::WX]),
                ub[i - G::WX], make_float2(vx[i - G::WX], vy[i - G::WX]),
                make_float3(P(sA)[i], P(sB)[i], P(sC)[i]), scaleP, scaleQ, &p, &tp, &q);
        P(sPX)[i] = p.x;
        P(sPY)[i] = p.y;
        P(sTPX)[i] = tp.x;
        P(sTPY)[i] = tp.y;
        P(sQX)[i] = q.x;
        P(sQY)[i] = q.y;
        P(sQZ)[i] = q.z;
        P(sQW)[i] = q.w;
      }
    }
    __syncthreads();
    // threshold + primal steps on [lo, hi) x [lo, hi)
    {
      const int lo = 2 * K - 2 * (k - s);
      const int hiX = 2 * K + TX + (k - s), hiY = 2 * K + TY + (k - s);
      const int ex = hiX - lo, ey = hiY - lo;
      for (int e = threadIdx.x; e < ex * ey; e += NT) {
        const int ry = e / ex, rx = e - ry * ex;
        const int i = (lo + ry) * G::WX + (lo + rx);
        const uint8_t code = scode[i];
        if (!(code & kSelf)) {
          P(sU)[i] = P(sUB)[i] = P(sVBX)[i] = P(sVBY)[i] = 0.f;
          continue;
        }
        const float u = P(sU)[i], ub = P(sUB)[i];
        const float un = threshold_px(code, ss.y, make_float2(P(sTPX)[i], P(sTPY)[i]),
                                      make_float2(P(sTPX)[i - 1], P(sTPY)[i - 1]),
                                      make_float2(P(sTPX)[i - G::WX], P(sTPY)[i - G::WX]), u, ub,
                                      make_float2(P(sIU)[i], P(sIZ)[i]), P(sEX)[i], kc.lambda);
        float uo;
        float2 vo;
        primal_px(code, ss.y, ss.z, make_float2(P(sPX)[i], P(sPY)[i]),
                  make_float4(P(sQX)[i], P(sQY)[i], P(sQZ)[i], P(sQW)[i]),
                  make_float4(P(sQX)[i - 1], P(sQY)[i - 1], P(sQZ)[i - 1], P(sQW)[i - 1]),
                  make_float4(P(sQX)[i - G::WX], P(sQY)[i - G::WX], P(sQZ)[i - G::WX], P(sQW)[i - G::WX]), un, ub,
                  make_float2(P(sVBX)[i], P(sVBY)[i]), make_float3(P(sA)[i], P(sB)[i], P(sC)[i]),
                  make_float3(P(sEX)[i], P(sEY)[i], P(sEZ)[i]), kc.alpha0, kc.alpha1, &uo, &vo);
        P(sU)[i] = un;
        P(sUB)[i] = uo;
        P(sVBX)[i] = vo.x;
        P(sVBY)[i] = vo.y;
      }
    }
    __syncthreads();
  }

  // ---- write back the tile (real pixels only)
  for (int e = threadIdx.x; e < TX * TY; e += NT) {
    const int ty = e / TX, tx = e - ty * TX;
    const int X = x0 + tx, Y = y0 + ty;
    if (X >= w || Y >= h) continue;
    const int i = (2 * K + ty) * G::WX + (2 * K + tx);
    const long f = (long)Y * w + X;
    out.u[f] = P(sU)[i];
    out.ub[f] = P(sUB)[i];
    out.vbx[f] = P(sVBX)[i];
    out.vby[f] = P(sVBY)[i];
    out.px[f] = P(sPX)[i];
    out.py[f] = P(sPY)[i];
    out.qx[f] = P(sQX)[i];
    out.qy[f] = P(sQY)[i];
    out.qz[f] = P(sQZ)[i];
    out.qw[f] = P(sQW)[i];
  }
}

template <int K, int TX, int TY, int NT>
cudaError_t launch_block(const TgvState& in, const TgvState& out, const TgvConsts& c, const float3* sched, int it0,
                         int niter, const SolverConsts& kc, int h, int w, cudaStream_t s) {
  using G = TgvGeom<K, TX, TY>;
  const size_t smem = G::smem_bytes();
  dim3 grid((w + TX - 1) / TX, (h + TY - 1) / TY);
  k_tgv_block<K, TX, TY, NT><<<grid, NT, smem, s>>>(in, out, c, sched, it0, niter, kc, h, w);
  return cudaGetLastError();
}

}  // namespace
}  // namespace vfs

#include "vfs_tgv_reg.cuh"

namespace vfs {
namespace {

template <int K, int TX, int TY, int NT>
cudaError_t prepare_block() {
  return cudaFuncSetAttribute(k_tgv_block<K, TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)TgvGeom<K, TX, TY>::smem_bytes());
}

template <int K, int TX, int TY, int NT>
cudaError_t prepare_reg() {
  cudaError_t e = cudaFuncSetAttribute(k_tgv_reg<K, TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)RegGeom<K, TX, TY>::smem_bytes());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_tgv_reg_batch<K, TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)RegGeom<K, TX, TY>::smem_bytes());
}

template <int K, int TX, int TY, int NT>
cudaError_t batch_reg(const TgvBatchParams& P, int n_tiles, int parity, const float3* sched, int it0, int niter,
                      const SolverConsts& kc, cudaStream_t s);

template <int K, int TX, int TY, int NT>
cudaError_t batch_block(const TgvBatchParams&, int, int, const float3*, int, int, const SolverConsts&, cudaStream_t) {
  return cudaErrorInvalidValue;  // batched launches use the register-owned kernels
}

// A launch configuration that lets the kernel start as a programmatic
// dependent of the previous launch on the stream (the kernels wait for it
// with griddepcontrol.wait before reading what it wrote).
struct PdlLaunch {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  PdlLaunch(dim3 grid, int threads, size_t smem, cudaStream_t s) {
    cfg.gridDim = grid;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
  }
};

template <int K, int TX, int TY, int NT>
cudaError_t launch_reg(const TgvState& in, const TgvState& out, const TgvConsts& c, const float3* sched, int it0,
                       int niter, const SolverConsts& kc, int h, int w, cudaStream_t s) {
  if (!c.rec) return cudaErrorInvalidValue;
  dim3 grid((w + TX - 1) / TX, (h + TY - 1) / TY);
  PdlLaunch L(grid, NT, RegGeom<K, TX, TY>::smem_bytes(), s);
  cudaError_t e = cudaLaunchKernelEx(&L.cfg, k_tgv_reg<K, TX, TY, NT>, in, out, c, sched, it0, niter, kc, h, w);
  if (e != cudaSuccess) {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_tgv_reg<K, TX, TY, NT>);
    fprintf(stderr, "k_tgv_reg<%d,%d,%d,%d>: %s (smem %zu, max dyn %d, regs %d, max threads %d, local %zu)\n", K, TX,
            TY, NT, cudaGetErrorString(e), RegGeom<K, TX, TY>::smem_bytes(), a.maxDynamicSharedSizeBytes, a.numRegs,
            a.maxThreadsPerBlock, a.localSizeBytes);
  }
  return e;
}

// Batched launches are programmatic dependents of the previous launch too
// (the work list is read before griddepcontrol.wait, the state after it).
template <int K, int TX, int TY, int NT>
cudaError_t batch_reg(const TgvBatchParams& P, int n_tiles, int parity, const float3* sched, int it0, int niter,
                      const SolverConsts& kc, cudaStream_t s) {
  for (int i = 0; i < P.n_items; ++i)
    if (!P.items[i].cst.rec) return cudaErrorInvalidValue;
  PdlLaunch L(dim3(n_tiles), NT, RegGeom<K, TX, TY>::smem_bytes(), s);
  return cudaLaunchKernelEx(&L.cfg, k_tgv_reg_batch<K, TX, TY, NT>, P, parity, sched, it0, niter, kc);
}

// Compiled variants: id -> (implementation, iterations per launch, tile).
// Ids below 100 keep all state in shared memory; ids 1xx are register-owned.
// Ids 22x have tiles sized so that a pyramid level of side S = 12 T covers
// at most 144 tiles, one per SM of the 148: the 1024-thread kernels hold one
// CTA per SM, so 169 tiles of a power-of-two side would need a second wave
// (e.g. 34x34 at 400^2, 17x17 at 200^2, 9x9 at 100^2, 27x27 at 320^2).
// 221 (36x36, 3 iterations, a 45x45 window, two pixels per thread) is the
// largest square tile within 1024 x 2 window pixels: the least halo per tile
// pixel, and 529 tiles fill four waves at 800^2 (the 32x32 tiles' 625 need
// five).  Ids 23x are 512-thread kernels with two pixels per thread compiled
// for two CTAs per SM (64 registers): more halo per tile pixel than 221, but
// each CTA's barrier waits overlap the other CTA's work; 232 (26x26, 2
// iterations) is the fastest at 800^2.  One wave of two CTAs per SM on the
// 400^2, 200^2 and 100^2 levels (24x24 K=2, 12x12 K=4, 8x8 K=6: 289, 289
// and 169 tiles) measured slower there than the one-CTA shapes.
#define VFS_TGV_VARIANTS(X)          \
  X(1, block, 1, 32, 16, 256)        \
  X(2, block, 2, 32, 32, 512)        \
  X(4, block, 4, 32, 32, 512)        \
  X(102, reg, 2, 32, 32, 512)        \
  X(103, reg, 3, 32, 32, 512)        \
  X(104, reg, 4, 32, 32, 512)        \
  X(106, reg, 6, 32, 32, 512)        \
  X(114, reg, 4, 64, 16, 512)        \
  X(124, reg, 4, 32, 16, 256)        \
  X(134, reg, 4, 32, 32, 1024)       \
  X(122, reg, 2, 32, 16, 256)        \
  X(162, reg, 2, 16, 16, 256)        \
  X(164, reg, 4, 16, 16, 256)        \
  X(166, reg, 3, 16, 16, 256)        \
  X(182, reg, 2, 16, 8, 128)         \
  X(184, reg, 4, 16, 8, 128)         \
  X(192, reg, 2, 8, 8, 64)           \
  X(135, reg, 4, 32, 28, 1024)       \
  X(136, reg, 4, 32, 24, 1024)       \
  X(174, reg, 4, 24, 24, 512)        \
  X(173, reg, 3, 24, 24, 512)        \
  X(193, reg, 3, 8, 8, 64)           \
  X(201, reg, 2, 16, 16, 512)        \
  X(202, reg, 3, 16, 16, 640)        \
  X(203, reg, 4, 16, 16, 1024)       \
  X(204, reg, 2, 32, 16, 1024)       \
  X(205, reg, 2, 8, 8, 224)          \
  X(206, reg, 3, 8, 8, 320)          \
  X(207, reg, 4, 8, 8, 416)          \
  X(208, reg, 1, 16, 16, 384)        \
  X(209, reg, 1, 8, 8, 128)          \
  X(210, reg, 2, 24, 24, 1024)       \
  X(211, reg, 3, 22, 22, 1024)       \
  X(212, reg, 4, 20, 20, 1024)       \
  X(213, reg, 6, 8, 8, 704)          \
  X(214, reg, 8, 8, 8, 1024)         \
  X(215, reg, 6, 12, 12, 928)        \
  X(216, reg, 5, 16, 16, 1024)       \
  X(217, reg, 6, 14, 14, 1024)       \
  X(220, reg, 3, 34, 34, 1024)       \
  X(221, reg, 3, 36, 36, 1024)       \
  X(222, reg, 4, 17, 17, 864)        \
  X(223, reg, 5, 17, 17, 1024)       \
  X(224, reg, 6, 9, 9, 736)          \
  X(225, reg, 4, 11, 11, 544)        \
  X(226, reg, 4, 27, 27, 1024)       \
  X(230, reg, 3, 23, 23, 512)        \
  X(231, reg, 4, 20, 20, 512)        \
  X(232, reg, 2, 26, 26, 512)        \
  X(233, reg, 3, 22, 22, 512)        \
  X(234, reg, 2, 28, 24, 512)        \
  X(235, reg, 2, 32, 20, 512)        \
  X(236, reg, 2, 24, 28, 512)

// Register-owned variants also compiled in recording form (every
// iteration's state written out), for the reverse mode's recomputation.
#define VFS_TGV_TRACE_VARIANTS(X) \
  X(124, 4, 32, 16, 256)          \
  X(134, 4, 32, 32, 1024)         \
  X(207, 4, 8, 8, 416)            \
  X(212, 4, 20, 20, 1024)         \
  X(216, 5, 16, 16, 1024)         \
  X(220, 3, 34, 34, 1024)         \
  X(221, 3, 36, 36, 1024)         \
  X(222, 4, 17, 17, 864)          \
  X(224, 6, 9, 9, 736)            \
  X(232, 2, 26, 26, 512)

}  // namespace

cudaError_t tgv_prepare() {
  cudaError_t e = cudaSuccess;
#define VFS_PREP(id, impl, K, TX, TY, NT) \
  if (e == cudaSuccess) e = prepare_##impl<K, TX, TY, NT>();
  VFS_TGV_VARIANTS(VFS_PREP)
#undef VFS_PREP
#define VFS_PREP_T(id, K, TX, TY, NT)                                                                      \
  if (e == cudaSuccess)                                                                                    \
    e = cudaFuncSetAttribute(k_tgv_reg_trace<K, TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             (int)RegGeom<K, TX, TY>::smem_bytes());
  VFS_TGV_TRACE_VARIANTS(VFS_PREP_T)
#undef VFS_PREP_T
  return e;
}

bool tgv_has_trace(int variant) {
  switch (variant) {
#define VFS_HAS_T(id, K, TX, TY, NT) \
  case id: return true;
    VFS_TGV_TRACE_VARIANTS(VFS_HAS_T)
#undef VFS_HAS_T
    default: return false;
  }
}

cudaError_t launch_tgv_trace(int variant, const TgvState& in, const TgvState& trace0, long rec_stride,
                             const TgvConsts& c, const float3* sched, int it0, int niter, const SolverConsts& kc,
                             int h, int w, cudaStream_t s) {
  if (h <= 0 || w <= 0 || niter <= 0) return cudaSuccess;
  if (!kc.dscale || !c.rec) return cudaErrorInvalidValue;  // dual-step scales or constant records missing
  switch (variant) {
#define VFS_LAUNCH_T(id, K, TX, TY, NT)                                                                    \
  case id: {                                                                                               \
    if (niter > K) return cudaErrorInvalidValue;                                                           \
    PdlLaunch L(dim3((w + TX - 1) / TX, (h + TY - 1) / TY), NT, RegGeom<K, TX, TY>::smem_bytes(), s);     \
    return cudaLaunchKernelEx(&L.cfg, k_tgv_reg_trace<K, TX, TY, NT>, in, trace0, rec_stride, c, sched, it0, \
                              niter, kc, h, w);                                                            \
  }
    VFS_TGV_TRACE_VARIANTS(VFS_LAUNCH_T)
#undef VFS_LAUNCH_T
    default: return cudaErrorInvalidValue;
  }
}

int tgv_max_iters_per_launch(int variant) {
  switch (variant) {
#define VFS_ITERS(id, impl, K, TX, TY, NT) \
  case id: return K;
    VFS_TGV_VARIANTS(VFS_ITERS)
#undef VFS_ITERS
    default: return 0;
  }
}

int tgv_variant_list(int* ids, int cap) {
  int n = 0;
#define VFS_LIST(id, impl, K, TX, TY, NT) \
  if (ids && n < cap) ids[n] = id;       \
  ++n;
  VFS_TGV_VARIANTS(VFS_LIST)
#undef VFS_LIST
  return n;
}

bool tgv_tile_shape(int variant, int* tx, int* ty) {
  switch (variant) {
#define VFS_SHAPE(id, impl, K, TX, TY, NT) \
  case id:                                \
    *tx = TX;                             \
    *ty = TY;                             \
    return std::string(#impl) == "reg";
    VFS_TGV_VARIANTS(VFS_SHAPE)
#undef VFS_SHAPE
    default: return false;
  }
}

cudaError_t launch_tgv_batch(int variant, const TgvBatchParams& P, int n_tiles, int parity, const float3* sched,
                             int it0, int niter, const SolverConsts& kc, cudaStream_t s) {
  if (P.n_items <= 0 || n_tiles <= 0 || niter <= 0) return cudaSuccess;
  if (P.n_items > kBatchParamItems) return cudaErrorInvalidValue;
  if (!kc.dscale) return cudaErrorInvalidValue;  // dual-step scales not formed
  switch (variant) {
#define VFS_BATCH_V(id, impl, K, TX, TY, NT) \
  case id: return batch_##impl<K, TX, TY, NT>(P, n_tiles, parity, sched, it0, niter, kc, s);
    VFS_TGV_VARIANTS(VFS_BATCH_V)
#undef VFS_BATCH_V
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_tgv_block(int variant, const TgvState& in, const TgvState& out, const TgvConsts& c,
                             const float3* sched, int it0, int niter, const SolverConsts& kc, int h, int w,
                             cudaStream_t s) {
  if (h <= 0 || w <= 0 || niter <= 0) return cudaSuccess;
  if (!kc.dscale) return cudaErrorInvalidValue;  // dual-step scales not formed
  switch (variant) {
#define VFS_LAUNCH_V(id, impl, K, TX, TY, NT) \
  case id: return launch_##impl<K, TX, TY, NT>(in, out, c, sched, it0, niter, kc, h, w, s);
    VFS_TGV_VARIANTS(VFS_LAUNCH_V)
#undef VFS_LAUNCH_V
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace vfs
