// Kernel declarations shared by the C-ABI layer (vfs_capi.cu) and the kernel
// translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "vfs_pixel.cuh"

namespace vfs {

// Camera intrinsics passed by value (the reference keeps them in __constant__
// memory, Python/equidistant_cam.cuh:28).
struct Cam {
  float f, u0, v0;
};

// Rotation (row-major) and the two scaled translations of
// Python/vector_field.py:36-52, as float32.
struct FieldPose {
  float R[9];
  float st_fwd[3];
  float st_bwd[3];
};

// A 2-D plane: base pointer and row pitch in bytes.
template <typename T>
struct Plane {
  T* ptr;
  size_t pitch;
  __device__ __forceinline__ T* row(int y) const { return (T*)((char*)ptr + (size_t)y * pitch); }
  __device__ __forceinline__ T& at(int x, int y) const { return row(y)[x]; }
};

// Mask read as the reference's point-sampled, mirror-addressed texture reads it
// at X, X+-1, Y, Y+-1: the edge texel outside the image.
__device__ __forceinline__ bool mask_at(Plane<const uint8_t> m, int x, int y, int h, int w) {
  x = min(max(x, 0), w - 1);
  y = min(max(y, 0), h - 1);
  return m.at(x, y) != 0;
}

__device__ __forceinline__ uint8_t mask_code(Plane<const uint8_t> m, int x, int y, int h, int w) {
  uint8_t c = 0;
  if (mask_at(m, x, y, h, w)) c |= kSelf;
  if (mask_at(m, x + 1, y, h, w)) c |= kE;
  if (mask_at(m, x - 1, y, h, w)) c |= kW;
  if (mask_at(m, x, y + 1, h, w)) c |= kS;
  if (mask_at(m, x, y - 1, h, w)) c |= kN;
  return c;
}

// ---- launch helpers (vfs_kernels.cu)
cudaError_t launch_cast_and_scale(Plane<float> out, Plane<const uint8_t> in, int h, int w, cudaStream_t s);
cudaError_t launch_downsample_image(Plane<float> out, cudaTextureObject_t src, int h, int w, cudaStream_t s);
cudaError_t launch_downsample_field(Plane<float2> out, cudaTextureObject_t src, int h, int w, cudaStream_t s);
cudaError_t launch_downsample_mask(Plane<uint8_t> out, cudaTextureObject_t src, int h, int w, cudaStream_t s);
cudaError_t launch_warp_image(Plane<float> out, Plane<const float2> warp, cudaTextureObject_t src, int h, int w,
                              cudaStream_t s);
cudaError_t launch_find_warping_vector(Plane<float2> out, Plane<const float2> warp, cudaTextureObject_t src, int h,
                                       int w, cudaStream_t s);
cudaError_t launch_warp_prologue(Plane<float2> tvec, Plane<float> warped, Plane<const float2> warp,
                                 cudaTextureObject_t tdir, cudaTextureObject_t tother, int h, int w, cudaStream_t s);
cudaError_t launch_gaussian_masked(Plane<float> out, cudaTextureObject_t src, Plane<const uint8_t> mask, int h, int w,
                                   cudaStream_t s);
cudaError_t launch_tensor_eta(Plane<float3> abc, Plane<float3> eta, cudaTextureObject_t src,
                              Plane<const uint8_t> mask, const SolverConsts& k, int h, int w, cudaStream_t s);
cudaError_t launch_derivatives(Plane<float2> out, cudaTextureObject_t tref, cudaTextureObject_t tother,
                               cudaTextureObject_t tdir, int h, int w, cudaStream_t s);
cudaError_t launch_dual_step(float2* p, float2* tp, float4* q, float sigma, const float* u, const float2* v,
                             const float3* abc, Plane<const uint8_t> mask, const SolverConsts& k, int h, int w,
                             cudaStream_t s);
cudaError_t launch_threshold_step(float* out, float tau, const float2* tp, const float* u, const float* ub,
                                  const float2* deriv, const float3* eta, Plane<const uint8_t> mask,
                                  const SolverConsts& k, int h, int w, cudaStream_t s);
cudaError_t launch_primal_step(float* uo, float2* vo, float tau, float mu, const float2* p, const float4* q,
                               const float* u, const float* ub, const float2* vb, const float3* abc,
                               const float3* eta, Plane<const uint8_t> mask, const SolverConsts& k, int h, int w,
                               cudaStream_t s);
cudaError_t launch_median(Plane<float> out, Plane<const float> in, Plane<const uint8_t> mask, int h, int w,
                          cudaStream_t s);
cudaError_t launch_clamp_flow(Plane<float2> warp, Plane<float> ubefore, Plane<const float> umed,
                              Plane<const float2> tvec, Plane<const uint8_t> mask, float limit, int h, int w,
                              cudaStream_t s);
cudaError_t launch_median_clamp(Plane<float2> warp, Plane<float> ubefore, Plane<const float> u,
                                Plane<const float2> tvec, Plane<const uint8_t> mask, float limit, int h, int w,
                                cudaStream_t s);
cudaError_t launch_upsample1(Plane<float> out, cudaTextureObject_t src, float scale, int h, int w, cudaStream_t s);
cudaError_t launch_upsample2(Plane<float2> out, cudaTextureObject_t src, float scale, int h, int w, cudaStream_t s);
cudaError_t launch_mask_flow(Plane<float2> warp, Plane<const uint8_t> mask, int h, int w, cudaStream_t s);
cudaError_t launch_mask_code(Plane<uint8_t> code, Plane<const uint8_t> mask, int h, int w, cudaStream_t s);
// lsq: least-squares triangulation along the reference ray instead of the
// reference's x-only formula (triangulate_lsq_px, vfs_camera.cuh)
cudaError_t launch_triangulate(float3* out, const float3* rays, const float3* rays_o, float tx, float ty, float tz,
                               Plane<const uint8_t> mask, int h, int w, cudaStream_t s, bool lsq = false);
cudaError_t launch_triangulate_flow(float3* out, Plane<const float2> warp, Cam cam, float tx, float ty, float tz,
                                    Plane<const uint8_t> mask, int h, int w, cudaStream_t s, bool lsq = false);
cudaError_t launch_get_rays(float3* out, Cam cam, int h, int w, cudaStream_t s);
cudaError_t launch_get_thetas(float3* out, const float3* rays, int h, int w, cudaStream_t s);
cudaError_t launch_project(float2* out, const float3* xyz, Cam cam, int h, int w, cudaStream_t s);
cudaError_t launch_unproject(float3* out, const float2* uv, Cam cam, int h, int w, cudaStream_t s);
cudaError_t launch_xyz_from_distance(float3* out, const float3* rays, const float* dist, Plane<const uint8_t> mask,
                                     int h, int w, cudaStream_t s);
cudaError_t launch_vector_fields(float2* tvf, float2* cvf, Cam cam_ref, Cam cam_other, const FieldPose& pose,
                                 float grid_offset, int h, int w, cudaStream_t s);

}  // namespace vfs
