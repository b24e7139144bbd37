// Equidistant fisheye camera and ray triangulation for one pixel, shared by
// the forward kernels (vfs_kernels.cu) and the reverse-mode kernels
// (vfs_grad.cu).
#pragma once
#include <cuda_runtime.h>

#include "vfs_kernels.cuh"

namespace vfs {

// ---- camera (Python/equidistant_cam.cuh:32-59, Python/template_cam.cu:25-112)
__device__ __forceinline__ float2 cam_project(const Cam& c, float3 X) {
  const float R = hypotf(X.x, X.y);
  const float theta = atan2f(R, X.z);
  const float phi = atan2f(X.y, X.x);
  float2 uv;
  sincosf(phi, &(uv.y), &(uv.x));
  uv.x = fmaf(c.f * theta, uv.x, c.u0);
  uv.y = fmaf(c.f * theta, uv.y, c.v0);
  return uv;
}

__device__ __forceinline__ float3 cam_unproject(const Cam& c, float2 x) {
  const float2 xy = make_float2(x.x - c.u0, x.y - c.v0);
  const float theta = hypotf(xy.x, xy.y) / c.f;
  const float phi = atan2f(xy.y, xy.x);
  float3 X;
  sincosf(phi, &(X.y), &(X.x));
  float2 sc;
  sincosf(theta, &(sc.x), &(sc.y));
  X.x *= sc.x;
  X.y *= sc.x;
  X.z = sc.y;
  return X;
}

// triangulateRays, Python/vfs.cu:707-735.
__device__ __forceinline__ float3 triangulate_px(float3 rr, float3 ro, float tx, float tz) {
  const float2 xyRef = make_float2(rr.x / rr.z, rr.y / rr.z);
  const float2 xyOther = make_float2(ro.x / ro.z, ro.y / ro.z);
  const float ZRef = fmaf(-tz, xyOther.x, tx) / fmaf(-1, xyRef.x, xyOther.x);
  return make_float3(ZRef * xyRef.x, ZRef * xyRef.y, ZRef);
}

}  // namespace vfs
