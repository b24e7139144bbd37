// Register-owned variant of the temporally blocked TGV kernel (included by
// vfs_tgv.cu; same geometry, same flat addressing, same per-pixel math).
//
// Each thread owns the window pixels e = threadIdx.x + j*NT for the whole
// launch.  Values only the owner reads stay in its registers: u and p (the
// threshold and primal steps read them at the pixel only) and the per-warp
// constants (tensor, eta, derivatives, mask code).  Values that neighbours
// read go to shared memory: u_ and v_ (read at E/W/S/N by the dual step), tp
// and q (read at W/N by the threshold and primal steps).  That is 9 floats of
// shared memory per window pixel instead of 20, and J independent pixels per
// thread for the scheduler to interleave.
#pragma once

namespace vfs {
namespace {

enum RegPlane { rUB, rVX, rVY, rTX, rTY, rQX, rQY, rQZ, rQW, kRegPlanes };

template <int K, int TX, int TY>
struct RegGeom {
  static constexpr int WX = TX + 3 * K;
  static constexpr int WY = TY + 3 * K;
  static constexpr int N = WX * WY;
  // the planes, then (sigma, tau, mu, scaleP, scaleQ) of each of the
  // launch's iterations
  static constexpr size_t smem_bytes() { return ((size_t)kRegPlanes * N + 5 * K) * sizeof(float); }
};

// One CTA's tile whose origin is (x0, y0).
// With TRACE, the state after iteration s (of this launch) is written to the
// record s - 1 of the trace, whose planes are those of `out` moved by
// (s - 1) * rec_stride floats, instead of the final state to `out`.
template <int K, int TX, int TY, int NT, bool TRACE = false>
__device__ __forceinline__ void tgv_reg_tile(const TgvState& in, const TgvState& out, const TgvConsts& cst,
                                             const float3* __restrict__ sched, int it0, int niter,
                                             const SolverConsts& kc, int h, int w, int x0, int y0,
                                             long rec_stride = 0) {
  using G = RegGeom<K, TX, TY>;
  constexpr int WX = G::WX, N = G::N, J = (N + NT - 1) / NT;
  extern __shared__ float4 smem_raw[];
  float* const sm = reinterpret_cast<float*>(smem_raw);
  float* const sUB = sm + rUB * N;
  float* const sVX = sm + rVX * N;
  float* const sVY = sm + rVY * N;
  float* const sTX = sm + rTX * N;
  float* const sTY = sm + rTY * N;
  float* const sQX = sm + rQX * N;
  float* const sQY = sm + rQY * N;
  float* const sQZ = sm + rQZ * N;
  float* const sQW = sm + rQW * N;
  float* const sSch = sm + kRegPlanes * N;

  const long n = (long)h * w;
  const long base = (long)(y0 - 2 * K) * w + (x0 - 2 * K);

  float ru[J], rpx[J], rpy[J], ra[J], rb[J], rc[J], rex[J], rey[J], rez[J], riu[J], riz[J];
  int rcode[J], rwx[J], rwy[J];

  // When launched as a programmatic dependent of the previous TGV launch this
  // CTA may start before that launch ends: the per-warp constants are read
  // first, the state (which that launch writes) only after griddepcontrol.wait
  // (a no-op for an ordinary launch).
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  const int k = niter < K ? niter : K;
  if (threadIdx.x < 5 * k) {  // this launch's step sizes and dual-step scales
    const int t = threadIdx.x / 5, c = threadIdx.x - 5 * t;
    sSch[threadIdx.x] = c < 3 ? reinterpret_cast<const float*>(sched + it0 + t)[c]
                              : reinterpret_cast<const float*>(kc.dscale + it0 + t)[c - 3];
  }
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int e = threadIdx.x + j * NT;
    const int wy = e / WX, wx = e - wy * WX;
    rwx[j] = wx;
    rwy[j] = e < N ? wy : 1 << 20;  // never inside a region
    const long f = base + (long)wy * w + wx;
    const bool ok = e < N && f >= 0 && f < n;
    ra[j] = ok ? cst.a[f] : 0.f;
    rb[j] = ok ? cst.b[f] : 0.f;
    rc[j] = ok ? cst.c[f] : 0.f;
    rex[j] = ok ? cst.ex[f] : 0.f;
    rey[j] = ok ? cst.ey[f] : 0.f;
    rez[j] = ok ? cst.ez[f] : 0.f;
    riu[j] = ok ? cst.iu[f] : 0.f;
    riz[j] = ok ? cst.iz[f] : 0.f;
    rcode[j] = ok ? cst.code[f] : 0;
  }
  // a tile whose pixels are all masked ends with zero state (masked pixels
  // are written 0 every iteration): write that and skip the iterations
  int live = 0;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int tx = rwx[j] - 2 * K, ty = rwy[j] - 2 * K;
    if (tx >= 0 && tx < TX && ty >= 0 && ty < TY && x0 + tx < w && y0 + ty < h && (rcode[j] & kSelf)) live = 1;
  }
  live = __syncthreads_or(live);
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  if (!live) {
    for (int s = 0; s < (TRACE ? k : 1); ++s) {
      const long ro = (long)s * rec_stride;
#pragma unroll
      for (int j = 0; j < J; ++j) {
        const int tx = rwx[j] - 2 * K, ty = rwy[j] - 2 * K;
        if (tx < 0 || tx >= TX || ty < 0 || ty >= TY) continue;
        const int X = x0 + tx, Y = y0 + ty;
        if (X >= w || Y >= h) continue;
        const long f = (long)Y * w + X + ro;
        out.u[f] = out.ub[f] = out.vbx[f] = out.vby[f] = out.px[f] = out.py[f] = 0.f;
        out.qx[f] = out.qy[f] = out.qz[f] = out.qw[f] = 0.f;
      }
    }
    return;
  }
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int e = threadIdx.x + j * NT;
    const long f = base + (long)rwy[j] * w + rwx[j];
    const bool ok = e < N && f >= 0 && f < n;
    ru[j] = ok ? in.u[f] : 0.f;
    rpx[j] = ok ? in.px[f] : 0.f;
    rpy[j] = ok ? in.py[f] : 0.f;
    if (e < N) {
      sUB[e] = ok ? in.ub[f] : 0.f;
      sVX[e] = ok ? in.vbx[f] : 0.f;
      sVY[e] = ok ? in.vby[f] : 0.f;
      sQX[e] = ok ? in.qx[f] : 0.f;
      sQY[e] = ok ? in.qy[f] : 0.f;
      sQZ[e] = ok ? in.qz[f] : 0.f;
      sQW[e] = ok ? in.qw[f] : 0.f;
    }
  }
  __syncthreads();

  for (int s = 1; s <= k; ++s) {
    const float* const sc = sSch + 5 * (s - 1);
    const float3 ss = make_float3(sc[0], sc[1], sc[2]);  // (sigma, tau, mu)
    const float scaleP = sc[3], scaleQ = sc[4];           // alpha1 sigma / etaP, alpha0 sigma / etaQ
    {  // dual step on [lo, hiX) x [lo, hiY)
      const int lo = 2 * K - 2 * (k - s) - 1;
      const int hiX = 2 * K + TX + (k - s), hiY = 2 * K + TY + (k - s);
#pragma unroll
      for (int j = 0; j < J; ++j) {
        if (rwx[j] < lo || rwx[j] >= hiX || rwy[j] < lo || rwy[j] >= hiY) continue;
        const int i = threadIdx.x + j * NT;
        const uint8_t code = (uint8_t)rcode[j];
        if (!(code & kSelf)) {
          rpx[j] = rpy[j] = 0.f;
          sTX[i] = sTY[i] = 0.f;
          sQX[i] = sQY[i] = sQZ[i] = sQW[i] = 0.f;
          continue;
        }
        float2 p = make_float2(rpx[j], rpy[j]), tp;
        float4 q = make_float4(sQX[i], sQY[i], sQZ[i], sQW[i]);
        dual_px(code, sUB[i], make_float2(sVX[i], sVY[i]), sUB[i + 1], make_float2(sVX[i + 1], sVY[i + 1]),
                sUB[i - 1], make_float2(sVX[i - 1], sVY[i - 1]), sUB[i + WX], make_float2(sVX[i + WX], sVY[i + WX]),
                sUB[i - WX], make_float2(sVX[i - WX], sVY[i - WX]), make_float3(ra[j], rb[j], rc[j]), scaleP,
                scaleQ, &p, &tp, &q);
        rpx[j] = p.x;
        rpy[j] = p.y;
        sTX[i] = tp.x;
        sTY[i] = tp.y;
        sQX[i] = q.x;
        sQY[i] = q.y;
        sQZ[i] = q.z;
        sQW[i] = q.w;
      }
    }
    __syncthreads();
    {  // threshold + primal steps on [lo, hiX) x [lo, hiY)
      const int lo = 2 * K - 2 * (k - s);
      const int hiX = 2 * K + TX + (k - s), hiY = 2 * K + TY + (k - s);
#pragma unroll
      for (int j = 0; j < J; ++j) {
        if (rwx[j] < lo || rwx[j] >= hiX || rwy[j] < lo || rwy[j] >= hiY) continue;
        const int i = threadIdx.x + j * NT;
        const uint8_t code = (uint8_t)rcode[j];
        if (!(code & kSelf)) {
          ru[j] = 0.f;
          sUB[i] = sVX[i] = sVY[i] = 0.f;
          continue;
        }
        const float ub = sUB[i];
        const float un = threshold_px(code, ss.y, make_float2(sTX[i], sTY[i]), make_float2(sTX[i - 1], 0.f),
                                      make_float2(0.f, sTY[i - WX]), ru[j], ub, make_float2(riu[j], riz[j]), rex[j],
                                      kc.lambda);
        float uo;
        float2 vo;
        primal_px(code, ss.y, ss.z, make_float2(rpx[j], rpy[j]), make_float4(sQX[i], sQY[i], sQZ[i], sQW[i]),
                  make_float4(sQX[i - 1], 0.f, 0.f, sQW[i - 1]), make_float4(0.f, sQY[i - WX], sQZ[i - WX], 0.f),
                  un, ub, make_float2(sVX[i], sVY[i]), make_float3(ra[j], rb[j], rc[j]),
                  make_float3(rex[j], rey[j], rez[j]), kc.alpha0, kc.alpha1, &uo, &vo);
        ru[j] = un;
        sUB[i] = uo;
        sVX[i] = vo.x;
        sVY[i] = vo.y;
      }
    }
    if constexpr (TRACE) {  // each thread writes the tile pixels it owns
      const long ro = (long)(s - 1) * rec_stride;
#pragma unroll
      for (int j = 0; j < J; ++j) {
        const int tx = rwx[j] - 2 * K, ty = rwy[j] - 2 * K;
        if (tx < 0 || tx >= TX || ty < 0 || ty >= TY) continue;
        const int X = x0 + tx, Y = y0 + ty;
        if (X >= w || Y >= h) continue;
        const int i = threadIdx.x + j * NT;
        const long f = (long)Y * w + X + ro;
        out.u[f] = ru[j];
        out.ub[f] = sUB[i];
        out.vbx[f] = sVX[i];
        out.vby[f] = sVY[i];
        out.px[f] = rpx[j];
        out.py[f] = rpy[j];
        out.qx[f] = sQX[i];
        out.qy[f] = sQY[i];
        out.qz[f] = sQZ[i];
        out.qw[f] = sQW[i];
      }
    }
    __syncthreads();
  }

  // ---- write back the tile (real pixels only)
  if constexpr (!TRACE) {
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int tx = rwx[j] - 2 * K, ty = rwy[j] - 2 * K;
    if (tx < 0 || tx >= TX || ty < 0 || ty >= TY) continue;
    const int X = x0 + tx, Y = y0 + ty;
    if (X >= w || Y >= h) continue;
    const int i = threadIdx.x + j * NT;
    const long f = (long)Y * w + X;
    out.u[f] = ru[j];
    out.ub[f] = sUB[i];
    out.vbx[f] = sVX[i];
    out.vby[f] = sVY[i];
    out.px[f] = rpx[j];
    out.py[f] = rpy[j];
    out.qx[f] = sQX[i];
    out.qy[f] = sQY[i];
    out.qz[f] = sQZ[i];
    out.qw[f] = sQW[i];
  }
  }
}

template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, (NT <= 256 ? 2 : 1))
    k_tgv_reg(TgvState in, TgvState out, TgvConsts cst, const float3* __restrict__ sched, int it0, int niter,
              SolverConsts kc, int h, int w) {
  tgv_reg_tile<K, TX, TY, NT>(in, out, cst, sched, it0, niter, kc, h, w, blockIdx.x * TX, blockIdx.y * TY);
}

// Recording: every iteration's state to the records 0..niter of the trace
// (record r: the planes of trace0 moved by r * rec_stride floats).
template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, (NT <= 256 ? 2 : 1))
    k_tgv_reg_trace(TgvState in, TgvState trace0, long rec_stride, TgvConsts cst, const float3* __restrict__ sched,
                    int it0, int niter, SolverConsts kc, int h, int w) {
  tgv_reg_tile<K, TX, TY, NT, true>(in, trace0, cst, sched, it0, niter, kc, h, w, blockIdx.x * TX, blockIdx.y * TY,
                                    rec_stride);
}

// Batched: one launch over the tiles of many images (the pairs of a batch at
// the same pyramid level and pass).  items[i].tile_base is the first block of
// item i; block b belongs to the last item whose tile_base <= b.
template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, (NT <= 256 ? 2 : 1))
    k_tgv_reg_batch(const TgvBatchItem* __restrict__ items, int n_items, int parity,
                    const float3* __restrict__ sched, int it0, int niter, SolverConsts kc) {
  int lo = 0, hi = n_items - 1;
  const int bid = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].tile_base <= bid) lo = mid;
    else hi = mid - 1;
  }
  const TgvBatchItem& it = items[lo];
  const int t = bid - it.tile_base;
  const int ty = t / it.tiles_x, tx = t - ty * it.tiles_x;
  tgv_reg_tile<K, TX, TY, NT>(it.st[parity], it.st[parity ^ 1], it.cst, sched, it0, niter, kc, it.h, it.w, tx * TX,
                              ty * TY);
}

}  // namespace
}  // namespace vfs
