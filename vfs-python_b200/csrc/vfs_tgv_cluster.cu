// Cluster-resident TGV solve for pyramid levels that fit in one thread-block
// cluster's shared memory: all solver iterations of a warp, then the median
// filter and the clamped flow update (Python/vfs.py:498-521), in one launch.
//
// Why: a level of up to ~200x200 pixels is a handful of tiles, so the
// temporally blocked kernel runs it on a few SMs, launch after launch, at the
// latency of one CTA.  Here a cluster of up to 16 CTAs (one per SM) splits the
// level into bands of whole rows; every CTA keeps its band's shared state in
// shared memory and its pixel-local state in registers for the whole solve,
// and reads the neighbour rows of adjacent bands directly from their shared
// memory (distributed shared memory).  Each iteration is two phases (dual
// step; threshold + primal steps) separated by hardware cluster barriers.
//
// Addressing is the reference's flat row-major one (index+-1 wraps across
// rows, index+-width crosses rows), so a band's neighbours are the last
// element(s) of the band above and the first of the band below; flat indices
// outside the image read 0.  Per-pixel arithmetic is vfs_pixel.cuh's, so the
// results are bit-identical to the per-step kernels and to the reference.
#include <cooperative_groups.h>

#include <cstdio>

#include "vfs_kernels.cuh"
#include "vfs_tgv.cuh"

namespace cg = cooperative_groups;

namespace vfs {
namespace {

constexpr int kCNT = 512;                 // threads per CTA
constexpr int kCJ = 6;                    // pixels per thread
constexpr int kCMaxPx = kCNT * kCJ;       // pixels per CTA band
enum ClusterPlane { cUB, cVX, cVY, cTX, cTY, cQX, cQY, cQZ, cQW, cU, kClusterPlanes };
constexpr size_t kClusterSmem = (size_t)kClusterPlanes * kCMaxPx * sizeof(float);

struct Band {
  long f0, f1;   // flat range owned by this CTA
  long stride;   // pixels per band (rows_per_cta * w)
  long n;        // h * w
  int rank;
};

// Shared-memory value of flat pixel g of plane `pl`: local, from the CTA that
// owns g, or 0 outside the image.
__device__ __forceinline__ float sget(const cg::cluster_group& cl, float* sm, int pl, const Band& b, long g) {
  if (g >= b.f0 && g < b.f1) return sm[pl * kCMaxPx + (int)(g - b.f0)];
  if (g < 0 || g >= b.n) return 0.f;
  const int owner = (int)(g / b.stride);
  float* remote = cl.map_shared_rank(sm, owner);
  return remote[pl * kCMaxPx + (int)(g - (long)owner * b.stride)];
}

// Cluster-wide barrier; a cluster of one CTA needs only the CTA barrier,
// which is much cheaper than the cluster barrier's arrive/wait round trip.
__device__ __forceinline__ void csync(const cg::cluster_group& cl, bool single) {
  if (single) __syncthreads();
  else cl.sync();
}

__global__ void __launch_bounds__(kCNT, 1)
    k_tgv_cluster(TgvState st, TgvConsts cst, const float3* __restrict__ sched, int niter, SolverConsts kc,
                  Plane<float2> warp, Plane<float> ubefore, Plane<const float2> tvec, float limit, int h, int w,
                  int rows_per_cta) {
  cg::cluster_group cl = cg::this_cluster();
  const bool single = cl.num_blocks() == 1;
  extern __shared__ float4 smem_raw[];
  float* const sm = reinterpret_cast<float*>(smem_raw);
  Band b;
  b.rank = (int)cl.block_rank();
  b.n = (long)h * w;
  b.stride = (long)rows_per_cta * w;
  b.f0 = min((long)b.rank * b.stride, b.n);
  b.f1 = min(b.f0 + b.stride, b.n);
  const int npx = (int)(b.f1 - b.f0);
  float* const sUB = sm + cUB * kCMaxPx;
  float* const sVX = sm + cVX * kCMaxPx;
  float* const sVY = sm + cVY * kCMaxPx;
  float* const sTX = sm + cTX * kCMaxPx;
  float* const sTY = sm + cTY * kCMaxPx;
  float* const sQX = sm + cQX * kCMaxPx;
  float* const sQY = sm + cQY * kCMaxPx;
  float* const sQZ = sm + cQZ * kCMaxPx;
  float* const sQW = sm + cQW * kCMaxPx;
  float* const sU = sm + cU * kCMaxPx;

  float ru[kCJ], rpx[kCJ], rpy[kCJ], ra[kCJ], rb[kCJ], rc[kCJ], rex[kCJ], rey[kCJ], rez[kCJ], riu[kCJ], riz[kCJ];
  int rcode[kCJ];
#pragma unroll
  for (int j = 0; j < kCJ; ++j) {
    const int e = threadIdx.x + j * kCNT;
    const bool ok = e < npx;
    const long f = b.f0 + e;
    ru[j] = ok ? st.u[f] : 0.f;
    rpx[j] = ok ? st.px[f] : 0.f;
    rpy[j] = ok ? st.py[f] : 0.f;
    ra[j] = ok ? cst.a[f] : 0.f;
    rb[j] = ok ? cst.b[f] : 0.f;
    rc[j] = ok ? cst.c[f] : 0.f;
    rex[j] = ok ? cst.ex[f] : 0.f;
    rey[j] = ok ? cst.ey[f] : 0.f;
    rez[j] = ok ? cst.ez[f] : 0.f;
    riu[j] = ok ? cst.iu[f] : 0.f;
    riz[j] = ok ? cst.iz[f] : 0.f;
    rcode[j] = ok ? cst.code[f] : 0;
    if (ok) {
      sUB[e] = st.ub[f];
      sVX[e] = st.vbx[f];
      sVY[e] = st.vby[f];
      sQX[e] = st.qx[f];
      sQY[e] = st.qy[f];
      sQZ[e] = st.qz[f];
      sQW[e] = st.qw[f];
    }
  }
  csync(cl, single);

  for (int it = 0; it < niter; ++it) {
    const float3 ss = sched[it];  // (sigma, tau, mu)
    const float scaleP = kc.alpha1 * ss.x / kc.etaP;
    const float scaleQ = kc.alpha0 * ss.x / kc.etaQ;
#pragma unroll
    for (int j = 0; j < kCJ; ++j) {  // dual step
      const int e = threadIdx.x + j * kCNT;
      if (e >= npx) continue;
      const uint8_t code = (uint8_t)rcode[j];
      if (!(code & kSelf)) {
        rpx[j] = rpy[j] = 0.f;
        sTX[e] = sTY[e] = 0.f;
        sQX[e] = sQY[e] = sQZ[e] = sQW[e] = 0.f;
        continue;
      }
      const long g = b.f0 + e;
      float2 p = make_float2(rpx[j], rpy[j]), tp;
      float4 q = make_float4(sQX[e], sQY[e], sQZ[e], sQW[e]);
      dual_px(code, sUB[e], make_float2(sVX[e], sVY[e]), sget(cl, sm, cUB, b, g + 1),
              make_float2(sget(cl, sm, cVX, b, g + 1), sget(cl, sm, cVY, b, g + 1)), sget(cl, sm, cUB, b, g - 1),
              make_float2(sget(cl, sm, cVX, b, g - 1), sget(cl, sm, cVY, b, g - 1)), sget(cl, sm, cUB, b, g + w),
              make_float2(sget(cl, sm, cVX, b, g + w), sget(cl, sm, cVY, b, g + w)), sget(cl, sm, cUB, b, g - w),
              make_float2(sget(cl, sm, cVX, b, g - w), sget(cl, sm, cVY, b, g - w)),
              make_float3(ra[j], rb[j], rc[j]), scaleP, scaleQ, &p, &tp, &q);
      rpx[j] = p.x;
      rpy[j] = p.y;
      sTX[e] = tp.x;
      sTY[e] = tp.y;
      sQX[e] = q.x;
      sQY[e] = q.y;
      sQZ[e] = q.z;
      sQW[e] = q.w;
    }
    csync(cl, single);
#pragma unroll
    for (int j = 0; j < kCJ; ++j) {  // threshold + primal steps
      const int e = threadIdx.x + j * kCNT;
      if (e >= npx) continue;
      const uint8_t code = (uint8_t)rcode[j];
      if (!(code & kSelf)) {
        ru[j] = 0.f;
        sUB[e] = sVX[e] = sVY[e] = 0.f;
        continue;
      }
      const long g = b.f0 + e;
      const float ub = sUB[e];
      const float un = threshold_px(code, ss.y, make_float2(sTX[e], sTY[e]), make_float2(sget(cl, sm, cTX, b, g - 1), 0.f),
                                    make_float2(0.f, sget(cl, sm, cTY, b, g - w)), ru[j], ub,
                                    make_float2(riu[j], riz[j]), rex[j], kc.lambda);
      float uo;
      float2 vo;
      primal_px(code, ss.y, ss.z, make_float2(rpx[j], rpy[j]), make_float4(sQX[e], sQY[e], sQZ[e], sQW[e]),
                make_float4(sget(cl, sm, cQX, b, g - 1), 0.f, 0.f, sget(cl, sm, cQW, b, g - 1)),
                make_float4(0.f, sget(cl, sm, cQY, b, g - w), sget(cl, sm, cQZ, b, g - w), 0.f), un, ub,
                make_float2(sVX[e], sVY[e]), make_float3(ra[j], rb[j], rc[j]), make_float3(rex[j], rey[j], rez[j]),
                kc.alpha0, kc.alpha1, &uo, &vo);
      ru[j] = un;
      sUB[e] = uo;
      sVX[e] = vo.x;
      sVY[e] = vo.y;
    }
    csync(cl, single);
  }

  // ---- medianFilter + computeOpticalFlowWithClamp (Python/vfs.py:518-521)
#pragma unroll
  for (int j = 0; j < kCJ; ++j) {
    const int e = threadIdx.x + j * kCNT;
    if (e < npx) sU[e] = ru[j];
  }
  csync(cl, single);
#pragma unroll
  for (int j = 0; j < kCJ; ++j) {
    const int e = threadIdx.x + j * kCNT;
    if (e >= npx) continue;
    const long g = b.f0 + e;
    st.ub[g] = sUB[e];  // u_ carries over to the next warp
    if (!((uint8_t)rcode[j] & kSelf)) continue;
    const int Y = (int)(g / w), X = (int)(g - (long)Y * w);
    float v[25];
#pragma unroll
    for (int jj = 0; jj < 5; jj++) {
      const int yy = min(max(Y + jj - 2, 0), h - 1);
#pragma unroll
      for (int ii = 0; ii < 5; ii++) {
        const int xx = min(max(X + ii - 2, 0), w - 1);
        v[jj * 5 + ii] = sget(cl, sm, cU, b, (long)yy * w + xx);
      }
    }
#pragma unroll
    for (int a = 0; a < 13; a++) {
#pragma unroll
      for (int i = a + 1; i < 25; i++) {
        const float x = v[a], y = v[i];
        const bool sw = x > y;
        v[a] = sw ? y : x;
        v[i] = sw ? x : y;
      }
    }
    const float delta = fminf(v[12] - ubefore.at(X, Y), limit);
    ubefore.at(X, Y) += delta;
    const float2 tv = tvec.at(X, Y);
    float2 o = warp.at(X, Y);
    o.x = fmaf(delta, tv.x, o.x);
    o.y = fmaf(delta, tv.y, o.y);
    warp.at(X, Y) = o;
  }
  csync(cl, single);  // keep every CTA's shared memory alive until remote reads are done
}

}  // namespace

int tgv_cluster_size(int h, int w, int max_cluster) {
  // the smallest band count whose bands fit in a CTA: every extra CTA adds
  // cluster-barrier cost to each of the two phases of every iteration, and a
  // level that fits one CTA runs with CTA barriers only
  if (h <= 0 || w <= 0 || w > kCMaxPx) return 0;
  for (int cs = 1; cs <= max_cluster; cs *= 2)
    if ((long)((h + cs - 1) / cs) * w <= kCMaxPx) return cs;
  return 0;
}

cudaError_t tgv_cluster_prepare(int* max_cluster) {
  cudaError_t e = cudaFuncSetAttribute(k_tgv_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClusterSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_tgv_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  // the largest cluster the device can co-schedule with this kernel's resources
  int best = 0;
  for (int cs = 16; cs >= 1; cs /= 2) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kCNT);
    cfg.dynamicSmemBytes = kClusterSmem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_tgv_cluster, &cfg) == cudaSuccess && n > 0) {
      best = cs;
      break;
    }
    cudaGetLastError();
  }
  *max_cluster = best;
  return cudaSuccess;
}

cudaError_t launch_tgv_cluster(int cluster, const TgvState& st, const TgvConsts& c, const float3* sched, int niter,
                               const SolverConsts& kc, Plane<float2> warp, Plane<float> ubefore,
                               Plane<const float2> tvec, float limit, int h, int w, cudaStream_t s) {
  const int rows = (h + cluster - 1) / cluster;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(cluster);
  cfg.blockDim = dim3(kCNT);
  cfg.dynamicSmemBytes = kClusterSmem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_tgv_cluster, st, c, sched, niter, kc, warp, ubefore, tvec, limit, h, w, rows);
}

}  // namespace vfs
