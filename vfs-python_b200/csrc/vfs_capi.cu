// C ABI: texture objects, error reporting and one entry point per reference
// kernel (the per-step hooks that mirror Python/vfs.py:220-458 and
// Python/equidistant_cam.py).  Declarations and contracts: include/vfs_b200.h.
#include <cstring>
#include <string>

#include "vfs_api_util.cuh"
#include "vfs_kernels.cuh"

namespace vfs {
namespace {
thread_local std::string g_last_error;
}
void set_error(const std::string& msg) { g_last_error = msg; }
}  // namespace vfs

using namespace vfs;

namespace {

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

int check_hw(int h, int w) {
  if (h <= 0 || w <= 0) return fail(VFS_ERR_ARG, "height and width must be positive");
  return VFS_OK;
}

int check_prm(const VfsParams* prm, SolverConsts* k) {
  std::string why;
  if (!valid_params(prm, &why)) return fail(VFS_ERR_ARG, why);
  *k = make_consts(prm);
  return VFS_OK;
}

Plane<const uint8_t> mplane(const uint8_t* m, size_t pitch, int w) { return {m, pitch ? pitch : (size_t)w}; }

#define VFS_NONNULL(...)                                                        \
  do {                                                                          \
    const void* ps_[] = {__VA_ARGS__};                                          \
    for (const void* p_ : ps_)                                                  \
      if (!p_) return fail(VFS_ERR_ARG, "NULL pointer argument");               \
  } while (0)

}  // namespace

extern "C" {

const char* vfs_last_error(void) { return g_last_error.c_str(); }
int vfs_version(void) { return 1; }

int vfs_texture_create(const void* ptr, int height, int width, size_t pitch_bytes, int kind, int linear,
                       uint64_t* tex_out) {
  VFS_NONNULL(ptr, tex_out);
  VFS_TRY(check_hw(height, width));
  cudaChannelFormatDesc cd;
  size_t esz;
  switch (kind) {
    case VFS_TEX_U8: cd = cudaCreateChannelDesc(8, 0, 0, 0, cudaChannelFormatKindUnsigned); esz = 1; break;
    case VFS_TEX_F32: cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat); esz = 4; break;
    case VFS_TEX_F32X2: cd = cudaCreateChannelDesc(32, 32, 0, 0, cudaChannelFormatKindFloat); esz = 8; break;
    default: return fail(VFS_ERR_ARG, "unknown texture kind");
  }
  if (reinterpret_cast<uintptr_t>(ptr) % 512 != 0) return fail(VFS_ERR_ALIGN, "texture base must be 512-byte aligned");
  if (pitch_bytes % 32 != 0 || pitch_bytes < (size_t)width * esz)
    return fail(VFS_ERR_ALIGN, "texture pitch must be a multiple of 32 bytes and cover a row");
  cudaResourceDesc rd;
  memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypePitch2D;
  rd.res.pitch2D.devPtr = const_cast<void*>(ptr);
  rd.res.pitch2D.desc = cd;
  rd.res.pitch2D.width = width;
  rd.res.pitch2D.height = height;
  rd.res.pitch2D.pitchInBytes = pitch_bytes;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  td.addressMode[0] = cudaAddressModeMirror;
  td.addressMode[1] = cudaAddressModeMirror;
  td.filterMode = linear ? cudaFilterModeLinear : cudaFilterModePoint;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 1;
  cudaTextureObject_t t = 0;
  VFS_TRY_CUDA(cudaCreateTextureObject(&t, &rd, &td, nullptr), "cudaCreateTextureObject");
  *tex_out = (uint64_t)t;
  return VFS_OK;
}

int vfs_texture_destroy(uint64_t tex) {
  VFS_TRY_CUDA(cudaDestroyTextureObject((cudaTextureObject_t)tex), "cudaDestroyTextureObject");
  return VFS_OK;
}

int vfs_cast_and_scale(float* out, const uint8_t* in, int h, int w, void* s) {
  VFS_NONNULL(out, in);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_cast_and_scale({out, (size_t)w * 4}, {in, (size_t)w}, h, w, S(s)), "castAndScale");
  return VFS_OK;
}

int vfs_downsample_image(float* out, uint64_t src, int h, int w, void* s) {
  VFS_NONNULL(out);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_downsample_image({out, (size_t)w * 4}, (cudaTextureObject_t)src, h, w, S(s)),
               "downSamplingImage");
  return VFS_OK;
}

int vfs_downsample_vector_field(float* out, uint64_t src, int h, int w, void* s) {
  VFS_NONNULL(out);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_downsample_field({(float2*)out, (size_t)w * 8}, (cudaTextureObject_t)src, h, w, S(s)),
               "downSamplingVectorField");
  return VFS_OK;
}

int vfs_downsample_mask(uint8_t* out, uint64_t src, int h, int w, void* s) {
  VFS_NONNULL(out);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_downsample_mask({out, (size_t)w}, (cudaTextureObject_t)src, h, w, S(s)), "downSamplingMask");
  return VFS_OK;
}

int vfs_warping_image(float* out, const float* warp, uint64_t src, int h, int w, void* s) {
  VFS_NONNULL(out, warp);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_warp_image({out, (size_t)w * 4}, {(const float2*)warp, (size_t)w * 8}, (cudaTextureObject_t)src,
                                 h, w, S(s)),
               "warpingImage");
  return VFS_OK;
}

int vfs_gaussian(float* out, uint64_t src, const uint8_t* mask, size_t mp, int h, int w, void* s) {
  VFS_NONNULL(out, mask);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_gaussian_masked({out, (size_t)w * 4}, (cudaTextureObject_t)src, mplane(mask, mp, w), h, w, S(s)),
               "gaussianMasked");
  return VFS_OK;
}

int vfs_compute_tensor_eta(float* abc, float* eta, uint64_t src, const uint8_t* mask, size_t mp, const VfsParams* prm,
                           int h, int w, void* s) {
  VFS_NONNULL(abc, eta, mask);
  VFS_TRY(check_hw(h, w));
  SolverConsts k;
  VFS_TRY(check_prm(prm, &k));
  VFS_TRY_CUDA(launch_tensor_eta({(float3*)abc, (size_t)w * 12}, {(float3*)eta, (size_t)w * 12},
                                 (cudaTextureObject_t)src, mplane(mask, mp, w), k, h, w, S(s)),
               "computeTensorEtaMasked");
  return VFS_OK;
}

int vfs_find_warping_vector(float* out, const float* warp, uint64_t field, int h, int w, void* s) {
  VFS_NONNULL(out, warp);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_find_warping_vector({(float2*)out, (size_t)w * 8}, {(const float2*)warp, (size_t)w * 8},
                                          (cudaTextureObject_t)field, h, w, S(s)),
               "findWarpingVector");
  return VFS_OK;
}

int vfs_compute_derivatives(float* out, uint64_t tref, uint64_t tother, uint64_t tfield, int h, int w, void* s) {
  VFS_NONNULL(out);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_derivatives({(float2*)out, (size_t)w * 8}, (cudaTextureObject_t)tref,
                                  (cudaTextureObject_t)tother, (cudaTextureObject_t)tfield, h, w, S(s)),
               "computeDerivatives");
  return VFS_OK;
}

int vfs_update_dual_variables(float* p, float* tp, float* q, float sigma, const float* u, const float* v,
                              const float* abc, const uint8_t* mask, size_t mp, const VfsParams* prm, int h, int w,
                              void* s) {
  VFS_NONNULL(p, tp, q, u, v, abc, mask);
  VFS_TRY(check_hw(h, w));
  SolverConsts k;
  VFS_TRY(check_prm(prm, &k));
  VFS_TRY_CUDA(launch_dual_step((float2*)p, (float2*)tp, (float4*)q, sigma, u, (const float2*)v, (const float3*)abc,
                                mplane(mask, mp, w), k, h, w, S(s)),
               "updateDualVariables");
  return VFS_OK;
}

int vfs_l1_thresholding(float* out, float tau, const float* tp, const float* u, const float* ub, const float* deriv,
                        const float* eta, const uint8_t* mask, size_t mp, const VfsParams* prm, int h, int w,
                        void* s) {
  VFS_NONNULL(out, tp, u, ub, deriv, eta, mask);
  VFS_TRY(check_hw(h, w));
  SolverConsts k;
  VFS_TRY(check_prm(prm, &k));
  VFS_TRY_CUDA(launch_threshold_step(out, tau, (const float2*)tp, u, ub, (const float2*)deriv, (const float3*)eta,
                                     mplane(mask, mp, w), k, h, w, S(s)),
               "l1Thresholding");
  return VFS_OK;
}

int vfs_update_primal_variables(float* uo, float* vo, float tau, float mu, const float* p, const float* q,
                                const float* u, const float* ub, const float* vb, const float* abc, const float* eta,
                                const uint8_t* mask, size_t mp, const VfsParams* prm, int h, int w, void* s) {
  VFS_NONNULL(uo, vo, p, q, u, ub, vb, abc, eta, mask);
  VFS_TRY(check_hw(h, w));
  SolverConsts k;
  VFS_TRY(check_prm(prm, &k));
  VFS_TRY_CUDA(launch_primal_step(uo, (float2*)vo, tau, mu, (const float2*)p, (const float4*)q, u, ub,
                                  (const float2*)vb, (const float3*)abc, (const float3*)eta, mplane(mask, mp, w), k, h,
                                  w, S(s)),
               "updatePrimalVariables");
  return VFS_OK;
}

int vfs_median_filter(float* out, const float* in, const uint8_t* mask, size_t mp, int h, int w, void* s) {
  VFS_NONNULL(out, in, mask);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_median({out, (size_t)w * 4}, {in, (size_t)w * 4}, mplane(mask, mp, w), h, w, S(s)),
               "medianFilter");
  return VFS_OK;
}

int vfs_compute_optical_flow_with_clamp(float* warp, float* ubefore, const float* ufilt, const float* tvec,
                                        const uint8_t* mask, size_t mp, const VfsParams* prm, int h, int w, void* s) {
  VFS_NONNULL(warp, ubefore, ufilt, tvec, mask);
  VFS_TRY(check_hw(h, w));
  SolverConsts k;
  VFS_TRY(check_prm(prm, &k));
  VFS_TRY_CUDA(launch_clamp_flow({(float2*)warp, (size_t)w * 8}, {ubefore, (size_t)w * 4}, {ufilt, (size_t)w * 4},
                                 {(const float2*)tvec, (size_t)w * 8}, mplane(mask, mp, w), k.upperLimit, h, w, S(s)),
               "computeOpticalFlowWithClamp");
  return VFS_OK;
}

int vfs_upsampling_vector_field1(float* out, uint64_t src, const VfsParams* prm, int h, int w, void* s) {
  VFS_NONNULL(out);
  VFS_TRY(check_hw(h, w));
  SolverConsts k;
  VFS_TRY(check_prm(prm, &k));
  VFS_TRY_CUDA(launch_upsample1({out, (size_t)w * 4}, (cudaTextureObject_t)src, k.fscale, h, w, S(s)),
               "upSamplingVectorField1");
  return VFS_OK;
}

int vfs_upsampling_vector_field(float* out, uint64_t src, const VfsParams* prm, int h, int w, void* s) {
  VFS_NONNULL(out);
  VFS_TRY(check_hw(h, w));
  SolverConsts k;
  VFS_TRY(check_prm(prm, &k));
  VFS_TRY_CUDA(launch_upsample2({(float2*)out, (size_t)w * 8}, (cudaTextureObject_t)src, k.fscale, h, w, S(s)),
               "upSamplingVectorField");
  return VFS_OK;
}

int vfs_triangulate_rays(float* out, const float* rays, const float* rays_o, const float* t, const uint8_t* mask,
                         size_t mp, int h, int w, void* s) {
  VFS_NONNULL(out, rays, rays_o, t, mask);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_triangulate((float3*)out, (const float3*)rays, (const float3*)rays_o, t[0], t[1], t[2],
                                  mplane(mask, mp, w), h, w, S(s)),
               "triangulateRays");
  return VFS_OK;
}

int vfs_triangulate_rays_lsq(float* out, const float* rays, const float* rays_o, const float* t, const uint8_t* mask,
                             size_t mp, int h, int w, void* s) {
  VFS_NONNULL(out, rays, rays_o, t, mask);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_triangulate((float3*)out, (const float3*)rays, (const float3*)rays_o, t[0], t[1], t[2],
                                  mplane(mask, mp, w), h, w, S(s), true),
               "triangulateRays (least squares)");
  return VFS_OK;
}

int vfs_cam_get_rays(float* out, float f, float u0, float v0, int h, int w, void* s) {
  VFS_NONNULL(out);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_get_rays((float3*)out, Cam{f, u0, v0}, h, w, S(s)), "getRays");
  return VFS_OK;
}

int vfs_cam_get_uvs(float* out, const float* xyz, float f, float u0, float v0, int h, int w, void* s) {
  VFS_NONNULL(out, xyz);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_project((float2*)out, (const float3*)xyz, Cam{f, u0, v0}, h, w, S(s)), "getUVFromXYZ");
  return VFS_OK;
}

int vfs_cam_get_xyzs(float* out, const float* uv, float f, float u0, float v0, int h, int w, void* s) {
  VFS_NONNULL(out, uv);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_unproject((float3*)out, (const float2*)uv, Cam{f, u0, v0}, h, w, S(s)), "getXYZFromUV");
  return VFS_OK;
}

int vfs_cam_get_thetas(float* out, const float* rays, int h, int w, void* s) {
  VFS_NONNULL(out, rays);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_get_thetas((float3*)out, (const float3*)rays, h, w, S(s)), "getThetas");
  return VFS_OK;
}

int vfs_cam_xyz_from_distance(float* out, const float* rays, const float* dist, const uint8_t* mask, size_t mp, int h,
                              int w, void* s) {
  VFS_NONNULL(out, rays, dist, mask);
  VFS_TRY(check_hw(h, w));
  VFS_TRY_CUDA(launch_xyz_from_distance((float3*)out, (const float3*)rays, dist, mplane(mask, mp, w), h, w, S(s)),
               "getXYZFromDistance");
  return VFS_OK;
}

int vfs_vector_fields(float* tvf, float* cvf, float fr, float u0r, float v0r, float fo, float u0o, float v0o,
                      const double* R, const double* t, const double* t_scale, float grid_offset, int h, int w,
                      void* s) {
  VFS_NONNULL(tvf, cvf, R, t, t_scale);
  VFS_TRY(check_hw(h, w));
  FieldPose pose;
  for (int i = 0; i < 9; ++i) pose.R[i] = (float)R[i];
  for (int i = 0; i < 3; ++i) {
    pose.st_fwd[i] = (float)(t_scale[0] * t[i]);
    pose.st_bwd[i] = (float)(t_scale[1] * t[i]);
  }
  VFS_TRY_CUDA(launch_vector_fields((float2*)tvf, (float2*)cvf, Cam{fr, u0r, v0r}, Cam{fo, u0o, v0o}, pose,
                                    grid_offset, h, w, S(s)),
               "vector fields");
  return VFS_OK;
}

int vfs_step_schedule(int n, double time_step_lambda, float* out3) {
  VFS_NONNULL(out3);
  if (n < 0) return fail(VFS_ERR_ARG, "n must be >= 0");
  step_schedule(n, time_step_lambda, out3);
  return VFS_OK;
}

}  // extern "C"
