// Register-owned variant of the temporally blocked TGV kernel (included by
// vfs_tgv.cu; same geometry, same flat addressing, same per-pixel math).
//
// Each thread owns the window pixels e = threadIdx.x + j*NT for the whole
// launch.  Values only the owner reads stay in its registers: u and p (the
// threshold and primal steps read them at the pixel only) and the per-warp
// constants (tensor, eta, derivatives, mask code).  Values that neighbours
// read go to shared memory: u_ and v_ (read at E/W/S/N by the dual step), tp
// and q (read at W/N by the threshold and primal steps).  Kernels whose
// threads own one window pixel store them as records, (u_, v_x, v_y, -) and q
// as float4 and tp as float2, so that one 16- or 8-byte shared-memory access
// moves what a neighbour contributes (~4 % faster on the coarse levels);
// kernels whose threads own two or more keep nine float planes, which need
// fewer registers.  That is 9-10 floats of shared memory per window pixel
// instead of 20, and J independent pixels per thread for the scheduler to
// interleave.
#pragma once

namespace vfs {
namespace {

// the flag added to the codes of a warp whose pixels all have kAllSides
constexpr uint8_t kWarpFull = 32;

// CTAs per SM the register-owned kernels are compiled for: two for blocks of
// up to 256 threads, and for 512-thread blocks whose threads own two window
// pixels (64 registers each, so that two CTAs share an SM and one's barrier
// waits overlap the other's work); one otherwise.
template <int K, int TX, int TY, int NT>
constexpr int reg_min_blocks() {
  return NT <= 256 ? 2 : (NT == 512 && (TX + 3 * K) * (TY + 3 * K) > NT && (TX + 3 * K) * (TY + 3 * K) <= 2 * NT ? 2 : 1);
}

template <int K, int TX, int TY>
struct RegGeom {
  static constexpr int WX = TX + 3 * K;
  static constexpr int WY = TY + 3 * K;
  static constexpr int N = WX * WY;
  // the state (RegSmem: 40 bytes per window pixel packed, 36 as planes),
  // then (sigma, tau, mu, scaleP, scaleQ) of each of the launch's iterations
  static constexpr size_t smem_bytes() { return (size_t)N * (16 + 16 + 8) + 5 * K * sizeof(float); }
};

// The shared-memory state of a tile, in one of two layouts with the same
// values: PACKED keeps (u_, v_x, v_y, -) and q as float4 records and tp as a
// float2, so a neighbour's contribution is one 16- or 8-byte access (fewer
// shared-memory instructions); otherwise nine float planes, which need fewer
// registers (the kernels whose threads own two or more window pixels would
// spill with the records).  Both fit in RegGeom::smem_bytes().
template <bool PACKED, int N>
struct RegSmem {
  float4* base;
  __device__ __forceinline__ float* pl(int p) const { return reinterpret_cast<float*>(base) + p * N; }
  __device__ __forceinline__ float4 uv(int i) const {
    if constexpr (PACKED) return base[i];
    else return make_float4(pl(0)[i], pl(1)[i], pl(2)[i], 0.f);
  }
  __device__ __forceinline__ void set_uv(int i, float4 v) const {
    if constexpr (PACKED) base[i] = v;
    else pl(0)[i] = v.x, pl(1)[i] = v.y, pl(2)[i] = v.z;
  }
  // addresses of component c of pixel i's (u_, v_x, v_y) and q values
  __device__ __forceinline__ float* uv_at(int i, int c) const {
    if constexpr (PACKED) return reinterpret_cast<float*>(base + i) + c;
    else return pl(c) + i;
  }
  __device__ __forceinline__ float* q_at(int i, int c) const {
    if constexpr (PACKED) return reinterpret_cast<float*>(base + N + i) + c;
    else return pl(3 + c) + i;
  }
  __device__ __forceinline__ float4 q(int i) const {
    if constexpr (PACKED) return base[N + i];
    else return make_float4(pl(3)[i], pl(4)[i], pl(5)[i], pl(6)[i]);
  }
  __device__ __forceinline__ void set_q(int i, float4 v) const {
    if constexpr (PACKED) base[N + i] = v;
    else pl(3)[i] = v.x, pl(4)[i] = v.y, pl(5)[i] = v.z, pl(6)[i] = v.w;
  }
  __device__ __forceinline__ float2 tp(int i) const {
    if constexpr (PACKED) return reinterpret_cast<const float2*>(base + 2 * N)[i];
    else return make_float2(pl(7)[i], pl(8)[i]);
  }
  __device__ __forceinline__ void set_tp(int i, float2 v) const {
    if constexpr (PACKED) reinterpret_cast<float2*>(base + 2 * N)[i] = v;
    else pl(7)[i] = v.x, pl(8)[i] = v.y;
  }
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
  // the fast path for fully unmasked warps; the small tiles of the coarse
  // levels (mostly halo and mask edge) measured faster without it
  constexpr bool kFast = TX * TY >= 256;
  extern __shared__ float4 smem_raw[];
  const RegSmem<J == 1, N> S{smem_raw};
  float* const sSch = reinterpret_cast<float*>(smem_raw) + 10 * N;  // after 40 N bytes

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
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 r0 = ok ? cst.rec[2 * f] : z, r1 = ok ? cst.rec[2 * f + 1] : z;
    ra[j] = r0.x, rb[j] = r0.y, rc[j] = r0.z, rex[j] = r0.w;
    rey[j] = r1.x, rez[j] = r1.y, riu[j] = r1.z, riz[j] = r1.w;
    rcode[j] = ok ? cst.code[f] : 0;
    // warps whose pixels are all unmasked with all four neighbours unmasked
    // (most of the image) take a path compiled for that code
    if constexpr (kFast)
      if (__all_sync(0xffffffffu, rcode[j] == kAllSides)) rcode[j] |= kWarpFull;
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
    if (e >= N) continue;
    if constexpr (J > 1) {
      // planes: the shared-memory state straight from global memory with
      // cp.async (zero-filled outside the image), no register staging
      // (800^2 and 400^2 levels 2-3 % faster)
      const long g = ok ? f : 0;
      cp_async4(S.uv_at(e, 0), in.ub + g, ok);
      cp_async4(S.uv_at(e, 1), in.vbx + g, ok);
      cp_async4(S.uv_at(e, 2), in.vby + g, ok);
      cp_async4(S.q_at(e, 0), in.qx + g, ok);
      cp_async4(S.q_at(e, 1), in.qy + g, ok);
      cp_async4(S.q_at(e, 2), in.qz + g, ok);
      cp_async4(S.q_at(e, 3), in.qw + g, ok);
    } else {
      // records: one 16-byte store each (faster here than seven 4-byte copies)
      S.set_uv(e, ok ? make_float4(in.ub[f], in.vbx[f], in.vby[f], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f));
      S.set_q(e, ok ? make_float4(in.qx[f], in.qy[f], in.qz[f], in.qw[f]) : make_float4(0.f, 0.f, 0.f, 0.f));
    }
  }
  if constexpr (J > 1) {
    cp_async_commit();
    cp_async_wait<0>();
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
        // the unmasked step; with the code the literal kAllSides (full) the
        // compiler drops the code tests and the W/N loads, which only
        // pixels without an E/S neighbour read
        auto step = [&](uint8_t cd, bool full) {
          float2 p = make_float2(rpx[j], rpy[j]), tp;
          float4 q = S.q(i);
          const float4 c = S.uv(i), cE = S.uv(i + 1), cS = S.uv(i + WX);
          // (with the fast path compiled in, the other kernels skip them
          // by the code's bits too: fewer registers there)
          const float4 cW = (full || (kFast && (cd & kE))) ? c : S.uv(i - 1);
          const float4 cN = (full || (kFast && (cd & kS))) ? c : S.uv(i - WX);
          dual_px(cd, c.x, make_float2(c.y, c.z), cE.x, make_float2(cE.y, cE.z), cW.x, make_float2(cW.y, cW.z), cS.x,
                  make_float2(cS.y, cS.z), cN.x, make_float2(cN.y, cN.z), make_float3(ra[j], rb[j], rc[j]), scaleP,
                  scaleQ, &p, &tp, &q);
          rpx[j] = p.x;
          rpy[j] = p.y;
          S.set_tp(i, tp);
          S.set_q(i, q);
        };
        auto masked = [&] {
          rpx[j] = rpy[j] = 0.f;
          S.set_tp(i, make_float2(0.f, 0.f));
          S.set_q(i, make_float4(0.f, 0.f, 0.f, 0.f));
        };
        if (kFast && (code & kWarpFull)) step(kAllSides, true);
        else if (!(code & kSelf)) masked();
        else step(code, false);
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
        auto step = [&](uint8_t cd) {
          const float4 c = S.uv(i);
          const float ub = c.x;
          const float un = threshold_px(cd, ss.y, S.tp(i), make_float2(S.tp(i - 1).x, 0.f),
                                        make_float2(0.f, S.tp(i - WX).y), ru[j], ub, make_float2(riu[j], riz[j]),
                                        rex[j], kc.lambda);
          float uo;
          float2 vo;
          const float4 qW = S.q(i - 1), qN = S.q(i - WX);
          primal_px(cd, ss.y, ss.z, make_float2(rpx[j], rpy[j]), S.q(i), make_float4(qW.x, 0.f, 0.f, qW.w),
                    make_float4(0.f, qN.y, qN.z, 0.f), un, ub, make_float2(c.y, c.z), make_float3(ra[j], rb[j], rc[j]),
                    make_float3(rex[j], rey[j], rez[j]), kc.alpha0, kc.alpha1, &uo, &vo);
          ru[j] = un;
          S.set_uv(i, make_float4(uo, vo.x, vo.y, 0.f));
        };
        auto masked = [&] {
          ru[j] = 0.f;
          S.set_uv(i, make_float4(0.f, 0.f, 0.f, 0.f));
        };
        if (kFast && (code & kWarpFull)) step(kAllSides);
        else if (!(code & kSelf)) masked();
        else step(code);
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
        const float4 uv = S.uv(i), q = S.q(i);
        out.u[f] = ru[j];
        out.ub[f] = uv.x;
        out.vbx[f] = uv.y;
        out.vby[f] = uv.z;
        out.px[f] = rpx[j];
        out.py[f] = rpy[j];
        out.qx[f] = q.x;
        out.qy[f] = q.y;
        out.qz[f] = q.z;
        out.qw[f] = q.w;
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
    const float4 uv = S.uv(i), q = S.q(i);
    out.u[f] = ru[j];
    out.ub[f] = uv.x;
    out.vbx[f] = uv.y;
    out.vby[f] = uv.z;
    out.px[f] = rpx[j];
    out.py[f] = rpy[j];
    out.qx[f] = q.x;
    out.qy[f] = q.y;
    out.qz[f] = q.z;
    out.qw[f] = q.w;
  }
  }
}

template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, reg_min_blocks<K, TX, TY, NT>())
    k_tgv_reg(TgvState in, TgvState out, TgvConsts cst, const float3* __restrict__ sched, int it0, int niter,
              SolverConsts kc, int h, int w) {
  tgv_reg_tile<K, TX, TY, NT>(in, out, cst, sched, it0, niter, kc, h, w, blockIdx.x * TX, blockIdx.y * TY);
}

// Recording: every iteration's state to the records 0..niter of the trace
// (record r: the planes of trace0 moved by r * rec_stride floats).
template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, reg_min_blocks<K, TX, TY, NT>())
    k_tgv_reg_trace(TgvState in, TgvState trace0, long rec_stride, TgvConsts cst, const float3* __restrict__ sched,
                    int it0, int niter, SolverConsts kc, int h, int w) {
  tgv_reg_tile<K, TX, TY, NT, true>(in, trace0, cst, sched, it0, niter, kc, h, w, blockIdx.x * TX, blockIdx.y * TY,
                                    rec_stride);
}

// Batched: one launch over the tiles of many images (the pairs of a batch at
// the same pyramid level and pass).  P.items[i].tile_base is the first block
// of item i in the items' numbering, of which the launch covers blocks
// P.bid0 .. P.bid0 + grid - 1; block b belongs to the last item whose
// tile_base <= b.
template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, reg_min_blocks<K, TX, TY, NT>())
    k_tgv_reg_batch(const __grid_constant__ TgvBatchParams P, int parity, const float3* __restrict__ sched, int it0,
                    int niter, SolverConsts kc) {
  int lo = 0, hi = P.n_items - 1;
  const int bid = P.bid0 + (int)blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (P.items[mid].tile_base <= bid) lo = mid;
    else hi = mid - 1;
  }
  const TgvBatchItem& it = P.items[lo];
  const int t = bid - it.tile_base;
  const int ty = t / it.tiles_x, tx = t - ty * it.tiles_x;
  tgv_reg_tile<K, TX, TY, NT>(it.st[parity], it.st[parity ^ 1], it.cst, sched, it0, niter, kc, it.h, it.w, tx * TX,
                              ty * TY);
}

}  // namespace
}  // namespace vfs
