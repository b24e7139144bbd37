// Texture sampling with the reference's coordinate arithmetic.
//
// The reference samples images, vector fields and masks through bindless
// texture objects with normalised coordinates and mirror addressing, linear
// filtering for data and point filtering for masks (Python/vfs.py:96-98,
// 169-171).  The B200 build keeps the hardware texture path for these
// per-level and per-warp gathers, bound directly to pitch-linear device
// buffers (no cudaArray copies); a probe on B200 showed pitch-linear and
// cudaArray textures return bit-identical samples for f32, f32x2 and u8
// data.  Each function forms the sample coordinates with the same float32
// operations as the reference functor it follows, so fetches land on exactly
// the same texture coordinates.
#pragma once
#include <cuda_runtime.h>

namespace vfs {

__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 f2scale(float a, float2 b) { return make_float2(a * b.x, a * b.y); }

template <typename T>
__device__ __forceinline__ T tex_at(cudaTextureObject_t t, float x, float y) { return tex2D<T>(t, x, y); }

// Bilinear<T>::get, Python/vfs.cu:35-49: mean of four taps a quarter texel
// (of the output grid) left/right/up/down of the output pixel centre.
__device__ __forceinline__ float box4_f(cudaTextureObject_t t, int X, int Y, int h, int w) {
  float dx = 1.0f / w;
  float dy = 1.0f / h;
  const float x = (X + 0.5f) * dx;
  const float y = (Y + 0.5f) * dy;
  dx *= 0.25f;
  dy *= 0.25f;
  return 0.25f * (tex_at<float>(t, x - dx, y) + tex_at<float>(t, x + dx, y) + tex_at<float>(t, x, y - dy) +
                  tex_at<float>(t, x, y + dy));
}
__device__ __forceinline__ float2 box4_f2(cudaTextureObject_t t, int X, int Y, int h, int w) {
  float dx = 1.0f / w;
  float dy = 1.0f / h;
  const float x = (X + 0.5f) * dx;
  const float y = (Y + 0.5f) * dy;
  dx *= 0.25f;
  dy *= 0.25f;
  return f2scale(0.25f, f2add(f2add(f2add(tex_at<float2>(t, x - dx, y), tex_at<float2>(t, x + dx, y)),
                                    tex_at<float2>(t, x, y - dy)),
                              tex_at<float2>(t, x, y + dy)));
}

// NearestNeighbor<T>::get at the pixel centre, Python/vfs.cu:54-59.
template <typename T>
__device__ __forceinline__ T centre(cudaTextureObject_t t, int X, int Y, int h, int w) {
  const float x = (X + 0.5f) / w;
  const float y = (Y + 0.5f) / h;
  return tex_at<T>(t, x, y);
}

// NearestNeighbor<T>::get displaced by a warp vector, Python/vfs.cu:61-66.
template <typename T>
__device__ __forceinline__ T displaced(cudaTextureObject_t t, int X, int Y, float wx, float wy, int h, int w) {
  const float x = (X + wx + 0.5f) / w;
  const float y = (Y + wy + 0.5f) / h;
  return tex_at<T>(t, x, y);
}

// Gaussian<float>::get, Python/vfs.cu:81-102.  The middle weight is a double
// literal in the reference, which promotes the sum to double before the
// final rounding to float; the same promotion is written out here.
__device__ __forceinline__ float binomial3(cudaTextureObject_t t, int X, int Y, int h, int w) {
  const float dx = 1.f / w;
  const float dy = 1.f / h;
  const float x = (X + 0.5f) * dx;
  const float y = (Y + 0.5f) * dy;
  float c0 = tex_at<float>(t, x, y);
  float diag = tex_at<float>(t, x - dx, y - dy);
  diag += tex_at<float>(t, x - dx, y + dy);
  diag += tex_at<float>(t, x + dx, y - dy);
  diag += tex_at<float>(t, x + dx, y + dy);
  float edge = tex_at<float>(t, x - dx, y);
  edge += tex_at<float>(t, x + dx, y);
  edge += tex_at<float>(t, x, y - dy);
  edge += tex_at<float>(t, x, y + dy);
  return (float)((.25f * c0) + (.0625 * diag) + (.125f * edge));
}

// Derivative::get (one texture), Python/vfs.cu:106-118: forward differences
// at the pixel's lower-right neighbour.
__device__ __forceinline__ float2 forward_grad(cudaTextureObject_t t, int X, int Y, int h, int w) {
  const float dx = 1.f / w;
  const float dy = 1.f / h;
  const float x = (X + 0.5f) * dx;
  const float y = (Y + 0.5f) * dy;
  float g0 = tex_at<float>(t, x + dx, y + dy);
  g0 -= tex_at<float>(t, x, y + dy);
  float g1 = tex_at<float>(t, x + dx, y + dy);
  g1 -= tex_at<float>(t, x + dx, y);
  return make_float2(g0, g1);
}

// Derivative::get (three textures), Python/vfs.cu:120-142: five-tap
// derivative along the epipolar direction, averaged over the reference and
// the warped second image, and the temporal difference.
__device__ __forceinline__ float2 epipolar_derivs(cudaTextureObject_t tref, cudaTextureObject_t tother,
                                                  cudaTextureObject_t tdir, int X, int Y, int h, int w) {
  const float x = (X + 0.5f) / w;
  const float y = (Y + 0.5f) / h;
  const float2 vec = tex_at<float2>(tdir, x, y);
  const float norm = hypotf(vec.x, vec.y);
  const float dx = vec.x / norm / w;
  const float dy = vec.y / norm / h;
  float r = tex_at<float>(tref, x - 2 * dx, y - 2 * dy);
  r -= tex_at<float>(tref, x - dx, y - dy) * 8;
  r += tex_at<float>(tref, x + dx, y + dy) * 8;
  r -= tex_at<float>(tref, x + 2 * dx, y + 2 * dy);
  float o = tex_at<float>(tother, x - 2 * dx, y - 2 * dy);
  o -= tex_at<float>(tother, x - dx, y - dy) * 8;
  o += tex_at<float>(tother, x + dx, y + dy) * 8;
  o -= tex_at<float>(tother, x + 2 * dx, y + 2 * dy);
  const float rc = tex_at<float>(tref, x, y);
  const float oc = tex_at<float>(tother, x, y);
  return make_float2((r + o) / 24, oc - rc);
}

}  // namespace vfs
