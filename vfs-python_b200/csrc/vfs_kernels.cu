// Per-level and per-warp kernels of the stereo solver, one kernel per
// reference kernel (Python/vfs.cu, Python/template_cam.cu), plus the fused
// variants the solve path uses.  Launch shape: 32x8 threads, one pixel per
// thread; these run once per level or once per warp, so they are a small
// share of a solve next to the TGV iterations (vfs_tgv.cu).
#include "vfs_camera.cuh"
#include "vfs_kernels.cuh"
#include "vfs_sample.cuh"

namespace vfs {
namespace {

constexpr int kBX = 32, kBY = 8;
inline dim3 grid2d(int h, int w) { return dim3((w + kBX - 1) / kBX, (h + kBY - 1) / kBY); }
const dim3 kBlock(kBX, kBY);

#define VFS_PIXEL_PROLOGUE                         \
  const int X = blockIdx.x * blockDim.x + threadIdx.x; \
  const int Y = blockIdx.y * blockDim.y + threadIdx.y; \
  if (X >= w || Y >= h) return;

// castAndScale, Python/vfs.cu:145-156.
__global__ void k_cast_and_scale(Plane<float> out, Plane<const uint8_t> in, int h, int w) {
  VFS_PIXEL_PROLOGUE
  out.at(X, Y) = static_cast<float>(in.at(X, Y)) / static_cast<float>(256);
}

// downSamplingImage / downSamplingVectorField / downSamplingMask,
// Python/vfs.cu:171-184.
__global__ void k_downsample_image(Plane<float> out, cudaTextureObject_t src, int h, int w) {
  VFS_PIXEL_PROLOGUE
  out.at(X, Y) = box4_f(src, X, Y, h, w);
}
__global__ void k_downsample_field(Plane<float2> out, cudaTextureObject_t src, int h, int w) {
  VFS_PIXEL_PROLOGUE
  out.at(X, Y) = box4_f2(src, X, Y, h, w);
}
__global__ void k_downsample_mask(Plane<uint8_t> out, cudaTextureObject_t src, int h, int w) {
  VFS_PIXEL_PROLOGUE
  out.at(X, Y) = centre<unsigned char>(src, X, Y, h, w);
}

// warpingImage, Python/vfs.cu:186-202.
__global__ void k_warp_image(Plane<float> out, Plane<const float2> warp, cudaTextureObject_t src, int h, int w) {
  VFS_PIXEL_PROLOGUE
  const float2 d = warp.at(X, Y);
  out.at(X, Y) = displaced<float>(src, X, Y, d.x, d.y, h, w);
}

// findWarpingVector, Python/vfs.cu:283-302.
__global__ void k_find_warping_vector(Plane<float2> out, Plane<const float2> warp, cudaTextureObject_t src, int h,
                                      int w) {
  VFS_PIXEL_PROLOGUE
  const float2 d = warp.at(X, Y);
  out.at(X, Y) = displaced<float2>(src, X, Y, d.x, d.y, h, w);
}

// findWarpingVector + warpingImage in one pass (Python/vfs.py:480-483): both
// sample at the same displaced coordinate.
__global__ void k_warp_prologue(Plane<float2> tvec, Plane<float> warped, Plane<const float2> warp,
                                cudaTextureObject_t tdir, cudaTextureObject_t tother, int h, int w) {
  VFS_PIXEL_PROLOGUE
  const float2 d = warp.at(X, Y);
  tvec.at(X, Y) = displaced<float2>(tdir, X, Y, d.x, d.y, h, w);
  warped.at(X, Y) = displaced<float>(tother, X, Y, d.x, d.y, h, w);
}

// gaussianMasked, Python/vfs.cu:204-226.
__global__ void k_gaussian_masked(Plane<float> out, cudaTextureObject_t src, Plane<const uint8_t> mask, int h,
                                  int w) {
  VFS_PIXEL_PROLOGUE
  out.at(X, Y) = mask_at(mask, X, Y, h, w) ? binomial3(src, X, Y, h, w) : 0.f;
}

// computeTensorEtaMasked, Python/vfs.cu:239-281.
__global__ void k_tensor_eta(Plane<float3> abc, Plane<float3> eta, cudaTextureObject_t src,
                             Plane<const uint8_t> mask, SolverConsts k, int h, int w) {
  VFS_PIXEL_PROLOGUE
  if (!mask_at(mask, X, Y, h, w)) {
    abc.at(X, Y) = eta.at(X, Y) = make_float3(0, 0, 0);
    return;
  }
  float3 a, e;
  tensor_from_grad(forward_grad(src, X, Y, h, w), k, &a, &e);
  abc.at(X, Y) = a;
  eta.at(X, Y) = e;
}

// computeDerivatives, Python/vfs.cu:304-324.
__global__ void k_derivatives(Plane<float2> out, cudaTextureObject_t tref, cudaTextureObject_t tother,
                              cudaTextureObject_t tdir, int h, int w) {
  VFS_PIXEL_PROLOGUE
  out.at(X, Y) = epipolar_derivs(tref, tother, tdir, X, Y, h, w);
}

// Flat-index read, 0 outside [0, n): the reference reads index+-1 and
// index+-width without bounds checks; inside the buffer that is the
// row-major neighbour (wrapping across rows), outside it is not defined, and
// this build returns 0 there.
template <typename T>
__device__ __forceinline__ T flat_ld(const T* a, long i, long n) {
  if (i < 0 || i >= n) {
    T z;
    memset(&z, 0, sizeof(T));
    return z;
  }
  return a[i];
}

// updateDualVariables, Python/vfs.cu:326-419 (in place on p and q).
__global__ void k_dual_step(float2* p, float2* tp, float4* q, float sigma, const float* __restrict__ u,
                            const float2* __restrict__ v, const float3* __restrict__ abc, Plane<const uint8_t> mask,
                            SolverConsts k, int h, int w) {
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X, n = (long)h * w;
  const uint8_t code = mask_code(mask, X, Y, h, w);
  if (!(code & kSelf)) {
    p[i] = tp[i] = make_float2(0, 0);
    q[i] = make_float4(0, 0, 0, 0);
    return;
  }
  float2 pv = p[i], tpv;
  float4 qv = q[i];
  const float scaleP = k.alpha1 * sigma / k.etaP;
  const float scaleQ = k.alpha0 * sigma / k.etaQ;
  dual_px(code, u[i], v[i], flat_ld(u, i + 1, n), flat_ld(v, i + 1, n), flat_ld(u, i - 1, n), flat_ld(v, i - 1, n),
          flat_ld(u, i + w, n), flat_ld(v, i + w, n), flat_ld(u, i - w, n), flat_ld(v, i - w, n), abc[i], scaleP,
          scaleQ, &pv, &tpv, &qv);
  p[i] = pv;
  tp[i] = tpv;
  q[i] = qv;
}

// l1Thresholding, Python/vfs.cu:421-505.
__global__ void k_threshold_step(float* out, float tau, const float2* __restrict__ tp, const float* __restrict__ u,
                                 const float* __restrict__ ub, const float2* __restrict__ deriv,
                                 const float3* __restrict__ eta, Plane<const uint8_t> mask, SolverConsts k, int h,
                                 int w) {
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X, n = (long)h * w;
  const uint8_t code = mask_code(mask, X, Y, h, w);
  if (!(code & kSelf)) {
    out[i] = 0;
    return;
  }
  out[i] = threshold_px(code, tau, tp[i], flat_ld(tp, i - 1, n), flat_ld(tp, i - w, n), u[i], ub[i], deriv[i],
                        eta[i].x, k.lambda);
}

// updatePrimalVariables, Python/vfs.cu:507-581.
__global__ void k_primal_step(float* uo, float2* vo, float tau, float mu, const float2* __restrict__ p,
                              const float4* __restrict__ q, const float* __restrict__ u, const float* __restrict__ ub,
                              const float2* __restrict__ vb, const float3* __restrict__ abc,
                              const float3* __restrict__ eta, Plane<const uint8_t> mask, SolverConsts k, int h,
                              int w) {
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X, n = (long)h * w;
  const uint8_t code = mask_code(mask, X, Y, h, w);
  if (!(code & kSelf)) {
    uo[i] = 0;
    vo[i] = make_float2(0, 0);
    return;
  }
  float uu;
  float2 vv;
  primal_px(code, tau, mu, p[i], q[i], flat_ld(q, i - 1, n), flat_ld(q, i - w, n), u[i], ub[i], vb[i], abc[i], eta[i],
            k.alpha0, k.alpha1, &uu, &vv);
  uo[i] = uu;
  vo[i] = vv;
}

// 5x5 median with clamp-to-edge neighbours, Python/vfs.cu:583-631.  The
// reference finds the 13th smallest of 25 values by a partial selection
// sort; the value selected is the same as any exact order statistic, so this
// uses a register-resident exchange network over the first 13 positions.
__device__ __forceinline__ float median25(const Plane<const float>& in, int X, int Y, int h, int w) {
  float v[25];
#pragma unroll
  for (int j = 0; j < 5; j++) {
    const int yy = min(max(Y + j - 2, 0), h - 1);
#pragma unroll
    for (int i = 0; i < 5; i++) {
      const int xx = min(max(X + i - 2, 0), w - 1);
      v[j * 5 + i] = in.at(xx, yy);
    }
  }
#pragma unroll
  for (int j = 0; j < 13; j++) {
#pragma unroll
    for (int i = j + 1; i < 25; i++) {
      const float a = v[j], b = v[i];
      const bool sw = a > b;
      v[j] = sw ? b : a;
      v[i] = sw ? a : b;
    }
  }
  return v[12];
}

__global__ void k_median(Plane<float> out, Plane<const float> in, Plane<const uint8_t> mask, int h, int w) {
  VFS_PIXEL_PROLOGUE
  out.at(X, Y) = mask_at(mask, X, Y, h, w) ? median25(in, X, Y, h, w) : in.at(X, Y);
}

// computeOpticalFlowWithClamp, Python/vfs.cu:641-676 (in place).
__device__ __forceinline__ void clamp_px(Plane<float2>& warp, Plane<float>& ub, float umed, float2 tv, float limit,
                                         int X, int Y) {
  const float delta = fminf(umed - ub.at(X, Y), limit);
  ub.at(X, Y) += delta;
  float2 o = warp.at(X, Y);
  o.x = fmaf(delta, tv.x, o.x);
  o.y = fmaf(delta, tv.y, o.y);
  warp.at(X, Y) = o;
}

__global__ void k_clamp_flow(Plane<float2> warp, Plane<float> ub, Plane<const float> umed, Plane<const float2> tvec,
                             Plane<const uint8_t> mask, float limit, int h, int w) {
  VFS_PIXEL_PROLOGUE
  if (!mask_at(mask, X, Y, h, w)) return;
  clamp_px(warp, ub, umed.at(X, Y), tvec.at(X, Y), limit, X, Y);
}

// medianFilter + computeOpticalFlowWithClamp in one pass (Python/vfs.py:518-521).
__global__ void k_median_clamp(Plane<float2> warp, Plane<float> ub, Plane<const float> u, Plane<const float2> tvec,
                               Plane<const uint8_t> mask, float limit, int h, int w) {
  VFS_PIXEL_PROLOGUE
  if (!mask_at(mask, X, Y, h, w)) return;
  clamp_px(warp, ub, median25(u, X, Y, h, w), tvec.at(X, Y), limit, X, Y);
}

// upSamplingVectorField1 / upSamplingVectorField, Python/vfs.cu:69-79, 678-705.
__global__ void k_upsample1(Plane<float> out, cudaTextureObject_t src, float scale, int h, int w) {
  VFS_PIXEL_PROLOGUE
  out.at(X, Y) = scale * centre<float>(src, X, Y, h, w);
}
__global__ void k_upsample2(Plane<float2> out, cudaTextureObject_t src, float scale, int h, int w) {
  VFS_PIXEL_PROLOGUE
  out.at(X, Y) = f2scale(scale, centre<float2>(src, X, Y, h, w));
}

// warpUV_ref[masks[0] == 0, :] = 0, Python/vfs.py:531.
__global__ void k_mask_flow(Plane<float2> warp, Plane<const uint8_t> mask, int h, int w) {
  VFS_PIXEL_PROLOGUE
  if (mask.at(X, Y) == 0) warp.at(X, Y) = make_float2(0, 0);
}

__global__ void k_mask_code(Plane<uint8_t> code, Plane<const uint8_t> mask, int h, int w) {
  VFS_PIXEL_PROLOGUE
  code.at(X, Y) = mask_code(mask, X, Y, h, w);
}

// LSQ: least-squares triangulation along the reference ray (all of t)
// instead of the reference's x-only formula.
template <bool LSQ>
__device__ __forceinline__ float3 triangulate_any(float3 rr, float3 ro, float tx, float ty, float tz) {
  return LSQ ? triangulate_lsq_px(rr, ro, tx, ty, tz) : triangulate_px(rr, ro, tx, tz);
}

template <bool LSQ>
__global__ void k_triangulate(float3* out, const float3* __restrict__ rays, const float3* __restrict__ rays_o,
                              float tx, float ty, float tz, Plane<const uint8_t> mask, int h, int w) {
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X;
  out[i] = mask_at(mask, X, Y, h, w) ? triangulate_any<LSQ>(rays[i], rays_o[i], tx, ty, tz) : make_float3(0, 0, -1);
}

// Python/vfs.py:535-559 in one pass: getRays at the pixel, getXYZFromUV at
// pixel + flow (float32 add, as `uv + self.warpUV`), then triangulateRays.
template <bool LSQ>
__global__ void k_triangulate_flow(float3* out, Plane<const float2> warp, Cam cam, float tx, float ty, float tz,
                                   Plane<const uint8_t> mask, int h, int w) {
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X;
  if (!mask_at(mask, X, Y, h, w)) {
    out[i] = make_float3(0, 0, -1);
    return;
  }
  const float2 d = warp.at(X, Y);
  const float3 rr = cam_unproject(cam, make_float2((float)X, (float)Y));
  const float3 ro = cam_unproject(cam, make_float2((float)X + d.x, (float)Y + d.y));
  out[i] = triangulate_any<LSQ>(rr, ro, tx, ty, tz);
}

__global__ void k_get_rays(float3* out, Cam cam, int h, int w) {
  VFS_PIXEL_PROLOGUE
  out[(long)Y * w + X] = cam_unproject(cam, make_float2(X, Y));
}

__global__ void k_get_thetas(float3* out, const float3* __restrict__ rays, int h, int w) {
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X;
  const float3 r = rays[i];
  out[i] = make_float3(atan2f(r.x, r.z), atan2f(r.y, r.z), atan2f(hypotf(r.x, r.y), r.z));
}

__global__ void k_project(float2* out, const float3* __restrict__ xyz, Cam cam, int h, int w) {
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X;
  out[i] = cam_project(cam, xyz[i]);
}

__global__ void k_unproject(float3* out, const float2* __restrict__ uv, Cam cam, int h, int w) {
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X;
  out[i] = cam_unproject(cam, uv[i]);
}

__global__ void k_xyz_from_distance(float3* out, const float3* __restrict__ rays, const float* __restrict__ dist,
                                    Plane<const uint8_t> mask, int h, int w) {
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X;
  if (mask.at(X, Y) == 0) {
    out[i] = make_float3(0, 0, -1);
    return;
  }
  const float3 r = rays[i];
  const float d = dist[i];
  out[i] = make_float3(d * r.x, d * r.y, d * r.z);
}

// get_vector_fields, Python/vector_field.py:28-56, for one pixel of the grid
// (grid = integer pixel coordinates + grid_offset).  The reference runs this
// as a chain of camera kernels and CuPy array operations; here it is one
// pass.  Norms are formed as sqrt of the float32 sum of squares.
__global__ void k_vector_fields(float2* tvf, float2* cvf, Cam cr, Cam co, FieldPose pose, float off, int h, int w) {
  const float* Rm = pose.R;
  const float* sf = pose.st_fwd;
  const float* sb = pose.st_bwd;
  VFS_PIXEL_PROLOGUE
  const long i = (long)Y * w + X;
  const float2 g = make_float2((float)X + off, (float)Y + off);
  float3 P = cam_unproject(cr, g);
  const float n = sqrtf(P.x * P.x + P.y * P.y + P.z * P.z);
  P = make_float3(P.x / n, P.y / n, P.z / n);
  const float2 f = cam_project(cr, make_float3(P.x + sf[0], P.y + sf[1], P.z + sf[2]));
  const float2 b = cam_project(cr, make_float3(P.x - sb[0], P.y - sb[1], P.z - sb[2]));
  float2 t = make_float2((f.x - b.x) / 2, (f.y - b.y) / 2);
  const float tn = sqrtf(t.x * t.x + t.y * t.y);
  tvf[i] = make_float2(t.x / tn, t.y / tn);
  // (XYZ . R^T)_j = sum_k XYZ_k R[j][k]
  const float3 RP = make_float3(fmaf(P.z, Rm[2], fmaf(P.y, Rm[1], P.x * Rm[0])),
                                fmaf(P.z, Rm[5], fmaf(P.y, Rm[4], P.x * Rm[3])),
                                fmaf(P.z, Rm[8], fmaf(P.y, Rm[7], P.x * Rm[6])));
  const float2 uv = cam_project(co, RP);
  cvf[i] = make_float2(uv.x - g.x, uv.y - g.y);
}

}  // namespace

#define VFS_LAUNCH(kern, h, w, s, ...)                          \
  do {                                                          \
    if ((h) <= 0 || (w) <= 0) return cudaSuccess;               \
    kern<<<grid2d(h, w), kBlock, 0, s>>>(__VA_ARGS__);          \
    return cudaGetLastError();                                  \
  } while (0)

cudaError_t launch_cast_and_scale(Plane<float> out, Plane<const uint8_t> in, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_cast_and_scale, h, w, s, out, in, h, w);
}
cudaError_t launch_downsample_image(Plane<float> out, cudaTextureObject_t src, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_downsample_image, h, w, s, out, src, h, w);
}
cudaError_t launch_downsample_field(Plane<float2> out, cudaTextureObject_t src, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_downsample_field, h, w, s, out, src, h, w);
}
cudaError_t launch_downsample_mask(Plane<uint8_t> out, cudaTextureObject_t src, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_downsample_mask, h, w, s, out, src, h, w);
}
cudaError_t launch_warp_image(Plane<float> out, Plane<const float2> warp, cudaTextureObject_t src, int h, int w,
                              cudaStream_t s) {
  VFS_LAUNCH(k_warp_image, h, w, s, out, warp, src, h, w);
}
cudaError_t launch_find_warping_vector(Plane<float2> out, Plane<const float2> warp, cudaTextureObject_t src, int h,
                                       int w, cudaStream_t s) {
  VFS_LAUNCH(k_find_warping_vector, h, w, s, out, warp, src, h, w);
}
cudaError_t launch_warp_prologue(Plane<float2> tvec, Plane<float> warped, Plane<const float2> warp,
                                 cudaTextureObject_t tdir, cudaTextureObject_t tother, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_warp_prologue, h, w, s, tvec, warped, warp, tdir, tother, h, w);
}
cudaError_t launch_gaussian_masked(Plane<float> out, cudaTextureObject_t src, Plane<const uint8_t> mask, int h, int w,
                                   cudaStream_t s) {
  VFS_LAUNCH(k_gaussian_masked, h, w, s, out, src, mask, h, w);
}
cudaError_t launch_tensor_eta(Plane<float3> abc, Plane<float3> eta, cudaTextureObject_t src,
                              Plane<const uint8_t> mask, const SolverConsts& k, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_tensor_eta, h, w, s, abc, eta, src, mask, k, h, w);
}
cudaError_t launch_derivatives(Plane<float2> out, cudaTextureObject_t tref, cudaTextureObject_t tother,
                               cudaTextureObject_t tdir, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_derivatives, h, w, s, out, tref, tother, tdir, h, w);
}
cudaError_t launch_dual_step(float2* p, float2* tp, float4* q, float sigma, const float* u, const float2* v,
                             const float3* abc, Plane<const uint8_t> mask, const SolverConsts& k, int h, int w,
                             cudaStream_t s) {
  VFS_LAUNCH(k_dual_step, h, w, s, p, tp, q, sigma, u, v, abc, mask, k, h, w);
}
cudaError_t launch_threshold_step(float* out, float tau, const float2* tp, const float* u, const float* ub,
                                  const float2* deriv, const float3* eta, Plane<const uint8_t> mask,
                                  const SolverConsts& k, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_threshold_step, h, w, s, out, tau, tp, u, ub, deriv, eta, mask, k, h, w);
}
cudaError_t launch_primal_step(float* uo, float2* vo, float tau, float mu, const float2* p, const float4* q,
                               const float* u, const float* ub, const float2* vb, const float3* abc,
                               const float3* eta, Plane<const uint8_t> mask, const SolverConsts& k, int h, int w,
                               cudaStream_t s) {
  VFS_LAUNCH(k_primal_step, h, w, s, uo, vo, tau, mu, p, q, u, ub, vb, abc, eta, mask, k, h, w);
}
cudaError_t launch_median(Plane<float> out, Plane<const float> in, Plane<const uint8_t> mask, int h, int w,
                          cudaStream_t s) {
  VFS_LAUNCH(k_median, h, w, s, out, in, mask, h, w);
}
cudaError_t launch_clamp_flow(Plane<float2> warp, Plane<float> ubefore, Plane<const float> umed,
                              Plane<const float2> tvec, Plane<const uint8_t> mask, float limit, int h, int w,
                              cudaStream_t s) {
  VFS_LAUNCH(k_clamp_flow, h, w, s, warp, ubefore, umed, tvec, mask, limit, h, w);
}
cudaError_t launch_median_clamp(Plane<float2> warp, Plane<float> ubefore, Plane<const float> u,
                                Plane<const float2> tvec, Plane<const uint8_t> mask, float limit, int h, int w,
                                cudaStream_t s) {
  VFS_LAUNCH(k_median_clamp, h, w, s, warp, ubefore, u, tvec, mask, limit, h, w);
}
cudaError_t launch_upsample1(Plane<float> out, cudaTextureObject_t src, float scale, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_upsample1, h, w, s, out, src, scale, h, w);
}
cudaError_t launch_upsample2(Plane<float2> out, cudaTextureObject_t src, float scale, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_upsample2, h, w, s, out, src, scale, h, w);
}
cudaError_t launch_mask_flow(Plane<float2> warp, Plane<const uint8_t> mask, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_mask_flow, h, w, s, warp, mask, h, w);
}
cudaError_t launch_mask_code(Plane<uint8_t> code, Plane<const uint8_t> mask, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_mask_code, h, w, s, code, mask, h, w);
}
cudaError_t launch_triangulate(float3* out, const float3* rays, const float3* rays_o, float tx, float ty, float tz,
                               Plane<const uint8_t> mask, int h, int w, cudaStream_t s, bool lsq) {
  if (lsq) VFS_LAUNCH(k_triangulate<true>, h, w, s, out, rays, rays_o, tx, ty, tz, mask, h, w);
  VFS_LAUNCH(k_triangulate<false>, h, w, s, out, rays, rays_o, tx, ty, tz, mask, h, w);
}
cudaError_t launch_triangulate_flow(float3* out, Plane<const float2> warp, Cam cam, float tx, float ty, float tz,
                                    Plane<const uint8_t> mask, int h, int w, cudaStream_t s, bool lsq) {
  if (lsq) VFS_LAUNCH(k_triangulate_flow<true>, h, w, s, out, warp, cam, tx, ty, tz, mask, h, w);
  VFS_LAUNCH(k_triangulate_flow<false>, h, w, s, out, warp, cam, tx, ty, tz, mask, h, w);
}
cudaError_t launch_get_rays(float3* out, Cam cam, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_get_rays, h, w, s, out, cam, h, w);
}
cudaError_t launch_get_thetas(float3* out, const float3* rays, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_get_thetas, h, w, s, out, rays, h, w);
}
cudaError_t launch_project(float2* out, const float3* xyz, Cam cam, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_project, h, w, s, out, xyz, cam, h, w);
}
cudaError_t launch_unproject(float3* out, const float2* uv, Cam cam, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_unproject, h, w, s, out, uv, cam, h, w);
}
cudaError_t launch_xyz_from_distance(float3* out, const float3* rays, const float* dist, Plane<const uint8_t> mask,
                                     int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_xyz_from_distance, h, w, s, out, rays, dist, mask, h, w);
}
cudaError_t launch_vector_fields(float2* tvf, float2* cvf, Cam cam_ref, Cam cam_other, const FieldPose& pose,
                                 float grid_offset, int h, int w, cudaStream_t s) {
  VFS_LAUNCH(k_vector_fields, h, w, s, tvf, cvf, cam_ref, cam_other, pose, grid_offset, h, w);
}

}  // namespace vfs
