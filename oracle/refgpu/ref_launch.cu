// Test infrastructure, not product code: a thin launch layer around the
// reference's own CUDA kernels.
//
// The reference (eshibusawa/VFS-Python) compiles Python/vfs.cu and
// Python/equidistant_cam.cuh + Python/template_cam.cu at run time with NVRTC
// after substituting VFS_* tokens (Python/vfs.py:57-68) and CameraModel
// (Python/equidistant_cam.py:62).  This file is compiled by the Makefile beside
// it with nvcc, with those tokens given as -D macros and the reference sources
// pulled in by #include from where they lie, so the kernels that run are the
// reference's, unmodified.  The host functions below only replace CuPy:
// texture objects are made the way Python/texture.py:27-55 makes them
// (cudaArray copy + bindless texture object), the camera intrinsics are
// uploaded the way Python/util_cuda.py:27-30 does (a __constant__ write), and
// every kernel is launched with the reference's block (32,32) and grid
// (ceil(W/32), ceil(H/32)) (e.g. Python/vfs.py:101-112).
#include <cuda_runtime.h>
#include <cstdint>

#include REF_VFS_CU
#include REF_CAM_CUH
#include REF_CAM_CU

namespace {
inline dim3 ref_grid(int h, int w) { return dim3((w + 31) / 32, (h + 31) / 32); }
const dim3 kBlock(32, 32);
inline int status() { return (int)cudaGetLastError(); }
}

extern "C" {

// ---- texture objects, as Python/texture.py:27-55 -------------------------
// kind: 0 = u8, 1 = s16, 2 = f32 (1 channel), 3 = f32 x2.
int ref_tex_create(const void* src, int height, int width, int kind, int address_mode, int filter_mode,
                   int read_mode, int normalized, unsigned long long* tex_out, void** array_out) {
  cudaChannelFormatDesc cd;
  size_t esz;
  switch (kind) {
    case 0: cd = cudaCreateChannelDesc(8, 0, 0, 0, cudaChannelFormatKindUnsigned); esz = 1; break;
    case 1: cd = cudaCreateChannelDesc(16, 0, 0, 0, cudaChannelFormatKindSigned); esz = 2; break;
    case 2: cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat); esz = 4; break;
    case 3: cd = cudaCreateChannelDesc(32, 32, 0, 0, cudaChannelFormatKindFloat); esz = 8; break;
    default: return -1;
  }
  cudaArray_t arr = nullptr;
  cudaError_t e = cudaMallocArray(&arr, &cd, width, height);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemcpy2DToArray(arr, 0, 0, src, width * esz, width * esz, height, cudaMemcpyDeviceToDevice);
  if (e != cudaSuccess) { cudaFreeArray(arr); return (int)e; }
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = arr;
  cudaTextureDesc td = {};
  td.addressMode[0] = (cudaTextureAddressMode)address_mode;
  td.addressMode[1] = (cudaTextureAddressMode)address_mode;
  td.filterMode = (cudaTextureFilterMode)filter_mode;
  td.readMode = (cudaTextureReadMode)read_mode;
  td.normalizedCoords = normalized;
  cudaTextureObject_t to = 0;
  e = cudaCreateTextureObject(&to, &rd, &td, nullptr);
  if (e != cudaSuccess) { cudaFreeArray(arr); return (int)e; }
  *tex_out = (unsigned long long)to;
  *array_out = arr;
  return 0;
}

int ref_tex_destroy(unsigned long long tex, void* array) {
  cudaError_t e1 = cudaDestroyTextureObject((cudaTextureObject_t)tex);
  cudaError_t e2 = cudaFreeArray((cudaArray_t)array);
  return e1 != cudaSuccess ? (int)e1 : (int)e2;
}

// ---- camera intrinsics, as Python/util_cuda.py:27-30 ---------------------
int ref_cam_set_intrinsics(float f, float u0, float v0) {
  float p[3] = {f, u0, v0};
  return (int)cudaMemcpyToSymbol(EquidistantCameraIntrinsics, p, sizeof(p));
}

int ref_sync() { return (int)cudaDeviceSynchronize(); }

// ---- Python/vfs.cu kernels ------------------------------------------------
int ref_castAndScale(float* out, unsigned char* in, int h, int w) {
  castAndScale<<<ref_grid(h, w), kBlock>>>(out, in, h, w); return status(); }
int ref_downSamplingImage(float* out, unsigned long long t, int h, int w) {
  downSamplingImage<<<ref_grid(h, w), kBlock>>>(out, t, h, w); return status(); }
int ref_downSamplingMask(unsigned char* out, unsigned long long t, int h, int w) {
  downSamplingMask<<<ref_grid(h, w), kBlock>>>(out, t, h, w); return status(); }
int ref_downSamplingVectorField(float2* out, unsigned long long t, int h, int w) {
  downSamplingVectorField<<<ref_grid(h, w), kBlock>>>(out, t, h, w); return status(); }
int ref_warpingImage(float* out, const float2* warp, unsigned long long t, int h, int w) {
  warpingImage<<<ref_grid(h, w), kBlock>>>(out, warp, t, h, w); return status(); }
int ref_gaussianMasked(float* out, unsigned long long t, unsigned long long tm, int h, int w) {
  gaussianMasked<<<ref_grid(h, w), kBlock>>>(out, t, tm, h, w); return status(); }
int ref_computeTensorEtaMasked(float3* abc, float3* eta, unsigned long long t, unsigned long long tm, int h, int w) {
  computeTensorEtaMasked<<<ref_grid(h, w), kBlock>>>(abc, eta, t, tm, h, w); return status(); }
int ref_findWarpingVector(float2* out, const float2* warp, unsigned long long t, int h, int w) {
  findWarpingVector<<<ref_grid(h, w), kBlock>>>(out, warp, t, h, w); return status(); }
int ref_computeDerivatives(float2* out, unsigned long long tr, unsigned long long to, unsigned long long tt, int h, int w) {
  computeDerivatives<<<ref_grid(h, w), kBlock>>>(out, tr, to, tt, h, w); return status(); }
int ref_updateDualVariables(float2* p, float2* tp, float4* q, float sigma, const float* u, const float2* v,
                            const float3* abc, unsigned long long tm, int h, int w) {
  updateDualVariables<<<ref_grid(h, w), kBlock>>>(p, tp, q, sigma, u, v, abc, tm, h, w); return status(); }
int ref_l1Thresholding(float* out, float tau, const float2* tp, const float* u, const float* u_,
                       const float2* deriv, const float3* eta, unsigned long long tm, int h, int w) {
  l1Thresholding<<<ref_grid(h, w), kBlock>>>(out, tau, tp, u, u_, deriv, eta, tm, h, w); return status(); }
int ref_updatePrimalVariables(float* uo, float2* vo, float tau, float mu, const float2* p, const float4* q,
                              const float* u, const float* u_, const float2* v_, const float3* abc,
                              const float3* eta, unsigned long long tm, int h, int w) {
  updatePrimalVariables<<<ref_grid(h, w), kBlock>>>(uo, vo, tau, mu, p, q, u, u_, v_, abc, eta, tm, h, w);
  return status(); }
int ref_medianFilter(float* out, const float* in, unsigned long long tm, int h, int w) {
  medianFilter<<<ref_grid(h, w), kBlock>>>(out, in, tm, h, w); return status(); }
int ref_computeOpticalFlowWithClamp(float2* of, float* clamped, const float* in, const float2* tv,
                                    unsigned long long tm, int h, int w) {
  computeOpticalFlowWithClamp<<<ref_grid(h, w), kBlock>>>(of, clamped, in, tv, tm, h, w); return status(); }
int ref_upSamplingVectorField(float2* out, unsigned long long t, int h, int w) {
  upSamplingVectorField<<<ref_grid(h, w), kBlock>>>(out, t, h, w); return status(); }
int ref_upSamplingVectorField1(float* out, unsigned long long t, int h, int w) {
  upSamplingVectorField1<<<ref_grid(h, w), kBlock>>>(out, t, h, w); return status(); }
int ref_triangulateRays(float3* out, const float3* rr, const float3* ro, const float3* t, unsigned long long tm,
                        int h, int w) {
  triangulateRays<<<ref_grid(h, w), kBlock>>>(out, rr, ro, t, tm, h, w); return status(); }

// ---- Python/template_cam.cu kernels ---------------------------------------
int ref_getRays(float3* out, int h, int w) { getRays<<<ref_grid(h, w), kBlock>>>(out, h, w); return status(); }
int ref_getThetas(float3* out, const float3* rays, int h, int w) {
  getThetas<<<ref_grid(h, w), kBlock>>>(out, rays, h, w); return status(); }
int ref_getUVFromXYZ(float2* out, const float3* xyz, int h, int w) {
  getUVFromXYZ<<<ref_grid(h, w), kBlock>>>(out, xyz, h, w); return status(); }
int ref_getXYZFromUV(float3* out, const float2* uv, int h, int w) {
  getXYZFromUV<<<ref_grid(h, w), kBlock>>>(out, uv, h, w); return status(); }
int ref_getXYZFromDistance(float3* out, const float3* rays, const float* d, unsigned long long tm, int h, int w) {
  getXYZFromDistance<<<ref_grid(h, w), kBlock>>>(out, rays, d, tm, h, w); return status(); }

}  // extern "C"
