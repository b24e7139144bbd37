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

// Least-squares triangulation along the reference ray, using all three
// components of t (an option beside triangulate_px, which uses only t.x and
// t.z, Python/vfs.cu:728-734, and is ill-conditioned when t is mostly along
// y or z).  Same convention as the reference: the other camera sees X at
// X + t, so its centre sits at -t and its ray is -t + s*ro.  The result is
// the point lambda*rr on the reference ray closest to that ray:
//   lambda = ((-t) x ro) . (rr x ro) / |rr x ro|^2.
// The cross products keep the small parallax angle accurate in float32 (a
// dot-product form would cancel in 1 - cos^2).  Parallel rays (epipole,
// infinite depth) divide by zero, as the reference formula does.
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(fmaf(a.y, b.z, -a.z * b.y), fmaf(a.z, b.x, -a.x * b.z), fmaf(a.x, b.y, -a.y * b.x));
}
__device__ __forceinline__ float dot3(float3 a, float3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }

__device__ __forceinline__ float3 triangulate_lsq_px(float3 rr, float3 ro, float tx, float ty, float tz) {
  const float3 n = cross3(rr, ro);
  const float3 m = cross3(make_float3(-tx, -ty, -tz), ro);
  const float lam = dot3(m, n) / dot3(n, n);
  return make_float3(lam * rr.x, lam * rr.y, lam * rr.z);
}

}  // namespace vfs
