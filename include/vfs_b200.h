/*
 * vfs_b200.h — C ABI of the B200 variational fisheye stereo library
 * (libvfs_b200.so).
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (cudaStream_t passed as void*), enqueues its work on that stream without
 * synchronising, allocates no device memory, and returns an int status
 * (VFS_OK or one of VFS_ERR_*).  vfs_last_error() returns a message for the
 * last failure on the calling thread.
 *
 * Layouts follow the reference (eshibusawa/VFS-Python): C-contiguous arrays,
 * float2 (H, W, 2), float3 (H, W, 3) array-of-structures, u8 masks (nonzero =
 * valid).  Each entry point names the reference interface it replaces.
 */
#ifndef VFS_B200_H_
#define VFS_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define VFS_API __attribute__((visibility("default")))
#else
#define VFS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define VFS_OK 0
#define VFS_ERR_ARG 1       /* bad pointer, size, shape or parameter */
#define VFS_ERR_ALIGN 2     /* pointer or pitch misaligned for a texture */
#define VFS_ERR_WORKSPACE 3 /* workspace missing or too small */
#define VFS_ERR_CUDA 4      /* a CUDA call failed; see vfs_last_error() */
#define VFS_ERR_STATE 5     /* call order violated (e.g. solve before set_mask) */

/* Solver parameters: the attributes of the reference's vfs_params
 * (Python/vfs_params.py:25-43).  All values are run-time arguments; the
 * reference bakes most of them into its CUDA source (Python/vfs.py:57-68). */
typedef struct VfsParams {
  int width, height;
  double beta, gamma, alpha0, alpha1, timeStepLambda, Lambda, fScale, limitRange;
  int nLevel, nWarpIters, nSolverIters;
} VfsParams;

/* Texture kinds for vfs_texture_create. */
#define VFS_TEX_U8 0
#define VFS_TEX_F32 2
#define VFS_TEX_F32X2 3

VFS_API const char* vfs_last_error(void);
VFS_API int vfs_version(void);

/* ---- texture objects ------------------------------------------------------
 * Replaces create_texture_object (Python/texture.py:27-55).  The texture is
 * bound to the caller's pitch-linear buffer (no copy); `ptr` must be
 * 512-byte aligned and `pitch_bytes` a multiple of 32.  Addressing is mirror
 * with normalised coordinates, linear filtering when `linear` is nonzero
 * (point otherwise), as Python/vfs.py:96-98 and :169-171 set up. */
VFS_API int vfs_texture_create(const void* ptr, int height, int width, size_t pitch_bytes, int kind, int linear,
                       uint64_t* tex_out);
VFS_API int vfs_texture_destroy(uint64_t tex);

/* ---- one entry per reference kernel (Python/vfs.cu) -------------------------
 * Outputs and non-texture inputs are C-contiguous; `mask` is a u8 plane with
 * row pitch `mask_pitch` bytes.  Names follow the VFS methods that launch
 * the kernels (Python/vfs.py:93-559). */
/* castAndScale, Python/vfs.py:127-144 */
VFS_API int vfs_cast_and_scale(float* out, const uint8_t* in, int h, int w, void* stream);
/* downSamplingImage / downSamplingVectorField / downSamplingMask,
 * Python/vfs.py:100-115, 164-181, 195-211; h, w are the coarse size */
VFS_API int vfs_downsample_image(float* out, uint64_t src_tex, int h, int w, void* stream);
VFS_API int vfs_downsample_vector_field(float* out_hw2, uint64_t src_tex, int h, int w, void* stream);
VFS_API int vfs_downsample_mask(uint8_t* out, uint64_t src_tex, int h, int w, void* stream);
/* warpingImage, Python/vfs.py:220-236 */
VFS_API int vfs_warping_image(float* out, const float* warp_hw2, uint64_t src_tex, int h, int w, void* stream);
/* gaussianMasked, Python/vfs.py:238-253 */
VFS_API int vfs_gaussian(float* out, uint64_t src_tex, const uint8_t* mask, size_t mask_pitch, int h, int w, void* stream);
/* computeTensorEtaMasked, Python/vfs.py:255-275 */
VFS_API int vfs_compute_tensor_eta(float* abc_hw3, float* eta_hw3, uint64_t src_tex, const uint8_t* mask, size_t mask_pitch,
                           const VfsParams* prm, int h, int w, void* stream);
/* findWarpingVector, Python/vfs.py:277-293 */
VFS_API int vfs_find_warping_vector(float* out_hw2, const float* warp_hw2, uint64_t field_tex, int h, int w, void* stream);
/* computeDerivatives, Python/vfs.py:295-313 */
VFS_API int vfs_compute_derivatives(float* out_hw2, uint64_t ref_tex, uint64_t other_tex, uint64_t field_tex, int h, int w,
                            void* stream);
/* updateDualVariables, Python/vfs.py:315-335 (p, q updated in place) */
VFS_API int vfs_update_dual_variables(float* p_hw2, float* tp_hw2, float* q_hw4, float sigma, const float* u,
                              const float* v_hw2, const float* abc_hw3, const uint8_t* mask, size_t mask_pitch,
                              const VfsParams* prm, int h, int w, void* stream);
/* l1Thresholding, Python/vfs.py:337-357 */
VFS_API int vfs_l1_thresholding(float* out, float tau, const float* tp_hw2, const float* u, const float* u_,
                        const float* deriv_hw2, const float* eta_hw3, const uint8_t* mask, size_t mask_pitch,
                        const VfsParams* prm, int h, int w, void* stream);
/* updatePrimalVariables, Python/vfs.py:359-382 */
VFS_API int vfs_update_primal_variables(float* u_out, float* v_out_hw2, float tau, float mu, const float* p_hw2,
                                const float* q_hw4, const float* u, const float* u_, const float* v_hw2,
                                const float* abc_hw3, const float* eta_hw3, const uint8_t* mask, size_t mask_pitch,
                                const VfsParams* prm, int h, int w, void* stream);
/* medianFilter, Python/vfs.py:384-400 */
VFS_API int vfs_median_filter(float* out, const float* in, const uint8_t* mask, size_t mask_pitch, int h, int w,
                      void* stream);
/* computeOpticalFlowWithClamp, Python/vfs.py:402-418 (warp, u_before in place) */
VFS_API int vfs_compute_optical_flow_with_clamp(float* warp_hw2, float* u_before, const float* u_filtered,
                                        const float* tvec_hw2, const uint8_t* mask, size_t mask_pitch,
                                        const VfsParams* prm, int h, int w, void* stream);
/* upSamplingVectorField1 / upSamplingVectorField, Python/vfs.py:420-458;
 * h, w are the fine size */
VFS_API int vfs_upsampling_vector_field1(float* out, uint64_t src_tex, const VfsParams* prm, int h, int w, void* stream);
VFS_API int vfs_upsampling_vector_field(float* out_hw2, uint64_t src_tex, const VfsParams* prm, int h, int w, void* stream);
/* triangulateRays, Python/vfs.py:535-559 (t: 3 floats, host memory) */
VFS_API int vfs_triangulate_rays(float* out_hw3, const float* rays_hw3, const float* rays_other_hw3, const float* t,
                         const uint8_t* mask, size_t mask_pitch, int h, int w, void* stream);
/* Option beside triangulateRays (same arguments and masked output (0, 0, -1)):
 * least-squares triangulation that uses all three components of t.  The
 * reference's formula (Python/vfs.cu:728-734) uses only t.x and t.z and is
 * ill-conditioned when the baseline is mostly along y or z.  Same convention
 * (the other camera sees X at X + t); the result is the point on the
 * reference ray closest to the other camera's ray,
 * lambda * r, lambda = ((-t) x r_o) . (r x r_o) / |r x r_o|^2. */
VFS_API int vfs_triangulate_rays_lsq(float* out_hw3, const float* rays_hw3, const float* rays_other_hw3,
                                     const float* t, const uint8_t* mask, size_t mask_pitch, int h, int w,
                                     void* stream);

/* ---- equidistant camera (Python/equidistant_cam.py, Python/template_cam.cu) */
/* getRays, Python/equidistant_cam.py:72-92 */
VFS_API int vfs_cam_get_rays(float* out_hw3, float f, float u0, float v0, int h, int w, void* stream);
/* getUVFromXYZ, Python/equidistant_cam.py:94-114 */
VFS_API int vfs_cam_get_uvs(float* out_hw2, const float* xyz_hw3, float f, float u0, float v0, int h, int w, void* stream);
/* getXYZFromUV, Python/equidistant_cam.py:116-136 */
VFS_API int vfs_cam_get_xyzs(float* out_hw3, const float* uv_hw2, float f, float u0, float v0, int h, int w, void* stream);
/* getThetas, Python/equidistant_cam.py:138-159 */
VFS_API int vfs_cam_get_thetas(float* out_hw3, const float* rays_hw3, int h, int w, void* stream);
/* getXYZFromDistance, Python/equidistant_cam.py:180-206 */
VFS_API int vfs_cam_xyz_from_distance(float* out_hw3, const float* rays_hw3, const float* dist, const uint8_t* mask,
                              size_t mask_pitch, int h, int w, void* stream);
/* get_vector_fields, Python/vector_field.py:28-56, for the grid of integer
 * pixel coordinates + grid_offset (0: get_grid_zero, 1: get_grid_one).
 * R: 9 floats row-major, t: 3 floats, t_scale: 2 floats (host memory). */
VFS_API int vfs_vector_fields(float* tvf_hw2, float* cvf_hw2, float f_ref, float u0_ref, float v0_ref, float f_other,
                      float u0_other, float v0_other, const double* R, const double* t, const double* t_scale,
                      float grid_offset, int h, int w, void* stream);

/* ---- whole solve (Python/vfs.py:84-559) ----------------------------------
 * A plan owns no memory: the caller provides a workspace of
 * vfs_plan_workspace_size() bytes (256-byte aligned) that lives as long as
 * the plan.  Call order mirrors the reference driver
 * (Python/main_equidistant.py:71-78): set_mask (create_mask_pyramid), then
 * set_vector_fields (create_vector_field_pyramid), then solve (solve_stereo),
 * then triangulate (triangulate_flow). */
typedef struct VfsPlan VfsPlan;

VFS_API int vfs_plan_workspace_size(const VfsParams* prm, size_t* bytes);
VFS_API int vfs_plan_create(const VfsParams* prm, void* workspace, size_t workspace_bytes, VfsPlan** plan_out);
VFS_API int vfs_plan_destroy(VfsPlan* plan);
/* pyramid sizes (compute_pyramid_sizes, Python/vfs.py:84-91): hw_out gets
 * 2*nLevel ints (h0, w0, h1, w1, ...) */
VFS_API int vfs_plan_sizes(const VfsPlan* plan, int* hw_out);
/* create_mask_pyramid, Python/vfs.py:159-187 */
VFS_API int vfs_plan_set_mask(VfsPlan* plan, const uint8_t* mask, size_t mask_pitch, void* stream);
/* create_vector_field_pyramid, Python/vfs.py:189-218 */
VFS_API int vfs_plan_set_vector_fields(VfsPlan* plan, const float* tvf_hw2, const float* cvf_hw2, void* stream);
/* solve_stereo, Python/vfs.py:460-533; images u8 C-contiguous (H, W);
 * warp_out (H, W, 2) receives the masked flow */
VFS_API int vfs_plan_solve(VfsPlan* plan, const uint8_t* img_ref, const uint8_t* img_other, float* warp_out_hw2,
                   void* stream);
/* triangulate_flow, Python/vfs.py:535-559, for the flow of the last solve */
VFS_API int vfs_plan_triangulate(VfsPlan* plan, float f, float u0, float v0, const float* t, float* xyz_out_hw3,
                         void* stream);
/* vfs_plan_triangulate with the least-squares rule of vfs_triangulate_rays_lsq */
VFS_API int vfs_plan_triangulate_lsq(VfsPlan* plan, float f, float u0, float v0, const float* t,
                                     float* xyz_out_hw3, void* stream);
/* The per-iteration step sizes (sigma, tau, mu) the solve uses, as the
 * reference's host loop computes them (Python/vfs.py:494-515, NumPy >= 2
 * scalar rules); out3 receives 3*n floats.  Host-only, no GPU needed. */
VFS_API int vfs_step_schedule(int n, double time_step_lambda, float* out3);
/* Replay the whole solve as one CUDA graph (captured on the first solve after
 * enabling, on a stream the plan owns, ordered after `stream`). */
VFS_API int vfs_plan_set_graph(VfsPlan* plan, int enable);
/* Record an event pair around each warp's TGV launches (for measurement). */
VFS_API int vfs_plan_set_timing(VfsPlan* plan, int enable);
typedef struct VfsSolveStats {
  long long kernels_per_solve; /* kernels one solve launches */
  double tgv_ms;               /* summed device time of the TGV launches (timing on) */
  double tgv_alg_bytes;        /* their algorithmic bytes: 113 per pixel-iteration */
  long long tgv_launches;      /* number of TGV kernel launches timed */
  int tgv_intervals;           /* event pairs summed */
  double tgv_ms_level[16];     /* tgv_ms split by pyramid level (0 = finest) */
  double recompute_ms;         /* reverse mode: device time of the checkpoint intervals' recomputation */
} VfsSolveStats;
/* Statistics of the last solve; synchronise its stream first. */
VFS_API int vfs_plan_stats(VfsPlan* plan, VfsSolveStats* out);
/* ---- batched solve of many pairs ------------------------------------------
 * No counterpart in the reference (one pair per solve_stereo call).  Pairs of
 * uneven resolution share the solver parameters (prm's width/height are
 * ignored; heights[i] x widths[i] is pair i).  The pairs advance level by
 * level in lockstep and every TGV pass is one launch over the tiles of all
 * pairs; per pair the result is bit-identical to vfs_plan_solve.  The caller
 * provides one workspace of vfs_batch_workspace_size() bytes. */
typedef struct VfsBatch VfsBatch;
VFS_API int vfs_batch_workspace_size(const VfsParams* prm, int n, const int* heights, const int* widths,
                                     size_t* bytes);
VFS_API int vfs_batch_create(const VfsParams* prm, int n, const int* heights, const int* widths, void* workspace,
                             size_t workspace_bytes, VfsBatch** batch_out);
VFS_API int vfs_batch_destroy(VfsBatch* batch);
/* mask (u8, pitch bytes), tvf and cvf (H, W, 2) of pair i */
VFS_API int vfs_batch_set_pair(VfsBatch* batch, int i, const uint8_t* mask, size_t mask_pitch, const float* tvf_hw2,
                               const float* cvf_hw2, void* stream);
/* host arrays of n device pointers each */
VFS_API int vfs_batch_solve(VfsBatch* batch, const uint8_t* const* img_refs, const uint8_t* const* img_others,
                            float* const* warps_out_hw2, void* stream);
VFS_API int vfs_batch_triangulate(VfsBatch* batch, int i, float f, float u0, float v0, const float* t,
                                  float* xyz_out_hw3, void* stream);
/* vfs_batch_triangulate with the least-squares rule of vfs_triangulate_rays_lsq */
VFS_API int vfs_batch_triangulate_lsq(VfsBatch* batch, int i, float f, float u0, float v0, const float* t,
                                      float* xyz_out_hw3, void* stream);
/* per-level TGV kernel of the batched launches (a 1xx register-owned variant) */
VFS_API int vfs_batch_set_level_variant(VfsBatch* batch, int level, int variant);
/* Working-set budget of a batched TGV launch group: per level, consecutive
 * pairs whose solver state (113 bytes a pixel) sums to at most `bytes` share
 * one launch per pass, and a group's passes all run before the next group's,
 * so a group's state can stay in L2 between passes.  0 (the default) puts all
 * pairs of a level in one launch per pass.  Results do not depend on it. */
VFS_API int vfs_batch_set_group_bytes(VfsBatch* batch, size_t bytes);
VFS_API int vfs_batch_set_graph(VfsBatch* batch, int enable);
VFS_API int vfs_batch_set_timing(VfsBatch* batch, int enable);
VFS_API int vfs_batch_stats(VfsBatch* batch, VfsSolveStats* out);

/* ---- whole solve with no device allocation --------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (a real-time loop with a fixed memory budget, a host callback, a foreign
 * runtime that owns no CUDA allocator): the same solve as vfs_plan_create +
 * vfs_plan_set_mask + vfs_plan_set_vector_fields + vfs_plan_solve, with the
 * workspace taken from a scratch array of vfs_static_scratch_bytes() (32 MiB)
 * compiled into the library and held by every GPU that loads it until the
 * process exits.  Sizes whose workspace does not fit (see
 * vfs_plan_workspace_size) are rejected with VFS_ERR_WORKSPACE.  The first call
 * on a device (and the first after a parameter change) sets up a plan over the
 * scratch and uploads the step sizes with a synchronous copy, so make it
 * before any stream capture.  A call that changes the parameters first waits
 * until the previous call's kernels on the device have finished (it blocks),
 * so calls are safe back to back on one stream across parameter changes.  All
 * calls on a device share the scratch: calls with the same parameters whose
 * GPU work overlaps (different, unordered streams) race, so issue them on one
 * stream or order them. */
VFS_API size_t vfs_static_scratch_bytes(void);
VFS_API int vfs_solve_stereo_static(const VfsParams* prm, const uint8_t* mask, size_t mask_pitch,
                                    const float* tvf_hw2, const float* cvf_hw2, const uint8_t* img_ref,
                                    const uint8_t* img_other, float* warp_out_hw2, void* stream);
/* Compiled fused-TGV kernel variants: returns their number and writes up to
 * `cap` ids and their iterations per launch. */
VFS_API int vfs_tgv_variants(int* ids, int cap, int* iters_per_launch);
/* Run levels that fit in one thread-block cluster with the cluster-resident
 * kernel (all iterations, median and clamp in one launch) unless a per-level
 * variant is set; off by default. */
VFS_API int vfs_plan_set_cluster(VfsPlan* plan, int enable);
/* Per-level TGV kernel: a variant id, VFS_TGV_CLUSTER for the cluster-resident
 * kernel (used where the level fits in one cluster), or 0 for the plan's
 * variant.  Level 0 is the finest. */
#define VFS_TGV_CLUSTER 1000
VFS_API int vfs_plan_set_level_variant(VfsPlan* plan, int level, int variant);
/* Cluster size the cluster-resident kernel would use for a level (0: does not fit). */
VFS_API int vfs_plan_level_cluster(const VfsPlan* plan, int level);
/* Select the fused TGV kernel variant by id (see vfs_tgv_variants). */
VFS_API int vfs_plan_set_tgv_variant(VfsPlan* plan, int iters_per_launch);

/* ---- Reverse mode (no counterpart in the reference, which is forward only).
 * A gradient plan wraps a VfsPlan and differentiates
 *   depth = triangulate_flow(solve_stereo(I_ref, I_other), t)[..., 2]
 * with respect to both images, the translation t (which also moves the
 * epipolar field get_vector_fields(grid, cam, cam, I, t, t_scale)) and
 * theta = (Lambda, alpha0, alpha1, beta, gamma).  Images are float (h, w) in
 * the u8 range (castAndScale divides by 256 inside).  vfs_grad_forward records
 * a tape (flow, u, u_ at each warp's start and the solver state every
 * `ckpt_every` iterations) in the workspace; vfs_grad_backward recomputes each
 * checkpoint interval and runs the hand-written adjoint.  g_scalars receives
 * 8 doubles on the device: dt0 dt1 dt2 dLambda dalpha0 dalpha1 dbeta dgamma.
 * Set the mask on vfs_grad_plan(gp) before the first forward; per-level TGV
 * variants set there are used by the forward (the cluster kernel is not). */
typedef struct VfsGradPlan VfsGradPlan;
VFS_API int vfs_grad_workspace_size(const VfsParams* prm, int ckpt_every, size_t* bytes);
VFS_API int vfs_grad_create(const VfsParams* prm, int ckpt_every, float f, float u0, float v0, double t_scale,
                            void* workspace, size_t workspace_bytes, VfsGradPlan** plan_out);
VFS_API int vfs_grad_destroy(VfsGradPlan* plan);
VFS_API VfsPlan* vfs_grad_plan(VfsGradPlan* plan);
VFS_API int vfs_grad_forward(VfsGradPlan* plan, const float* img_ref, const float* img_other, const double* t,
                             const double* theta, float* depth_out, void* stream);
VFS_API int vfs_grad_backward(VfsGradPlan* plan, const float* g_depth, float* g_ref, float* g_other,
                              double* g_scalars, void* stream);
/* Backward kernels: fused_reverse selects how an iteration is reversed:
 * 11..20 and 22..25 (default 11) two to four iterations per launch, cotangent state on chip
 * (11: 2 iterations, 24x16 tiles; 12: 2, 16x16; 13: 3, 16x16; 14: 4, 16x8;
 * 15: 2, 8x8; 16: 4, 8x8; 17: 3, 24x12; 18: 2, 32x12; 19: 3, 20x15;
 * 20: 2, 28x16; 22: 2, 24x20; 23: 2, 24x21; 24: 3, 20x18; 25: 3, 20x17), 1..5 one
 * iteration per launch in one tiled kernel
 * (1: 32x16; 2: 32x8; 3: 64x8; 4: 32x32; 5: 28x16), 0 three gather kernels.
 * trace_variant selects the TGV variant that recomputes checkpoint intervals
 * (0: automatic, -1: one iteration per launch).  With ckpt_every 1 the
 * forward records every state and nothing is recomputed. */
VFS_API int vfs_grad_set_options(VfsGradPlan* plan, int fused_reverse, int trace_variant);
/* Reverse-step kernel form for one level (0: the plan's, from
 * vfs_grad_set_options; default 11).  Level 0 is the finest. */
VFS_API int vfs_grad_set_level_form(VfsGradPlan* plan, int level, int form);
/* Triangulation rule of the depth map and of its reverse: 0 the reference's
 * (Python/vfs.cu:728-734, default), 1 least squares along the reference ray
 * (vfs_triangulate_rays_lsq).  A forward must follow a change. */
VFS_API int vfs_grad_set_triangulation(VfsGradPlan* plan, int lsq);
/* Event timing of the reverse TGV launches of each backward (off by default).
 * vfs_grad_stats (after synchronising) fills tgv_ms, tgv_alg_bytes (241 per
 * pixel and reversed iteration: state before 40, p and q after 24, cotangent
 * in 40 and out 40, constants 33, constant cotangents read and written 64),
 * tgv_launches, tgv_intervals and tgv_ms_level for the last backward;
 * kernels_per_solve is 0. */
VFS_API int vfs_grad_set_timing(VfsGradPlan* plan, int enable);
VFS_API int vfs_grad_stats(VfsGradPlan* plan, VfsSolveStats* out);

#ifdef __cplusplus
}
#endif
#endif /* VFS_B200_H_ */
