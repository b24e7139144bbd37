// Whole-solve path: a plan that carves a caller-provided workspace into the
// pyramids, per-warp constants and ping-pong solver state, binds texture
// objects to the sampled planes once, and enqueues a complete solve_stereo
// (Python/vfs.py:460-533) on one stream with no host synchronisation.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "vfs_plan_impl.cuh"
#include "vfs_sample.cuh"

namespace vfs {
namespace {

constexpr size_t kAlign = 512;      // texture base alignment on B200
constexpr size_t kPitchAlign = 128; // row pitch (texture pitch alignment is 32)

inline size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
inline size_t pitch_of(int w, size_t esz) { return round_up((size_t)w * esz, kPitchAlign); }

// Bump allocator over the workspace (or a size counter when base is null).
struct Carver {
  char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t bytes) {
    off = round_up(off, kAlign);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += bytes;
    return p;
  }
};

constexpr int kBX = 32, kBY = 8;
inline dim3 grid2d(int h, int w) { return dim3((w + kBX - 1) / kBX, (h + kBY - 1) / kBY); }

// computeTensorEtaMasked (Python/vfs.cu:239-281) writing the per-warp
// constant planes of the fused solver (structure of arrays) and the mask
// code of each pixel.
__global__ void k_tensor_soa(TgvConsts out, uint8_t* code, cudaTextureObject_t src, Plane<const uint8_t> mask,
                             SolverConsts k, int h, int w) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x;
  const int Y = blockIdx.y * blockDim.y + threadIdx.y;
  if (X >= w || Y >= h) return;
  const long i = (long)Y * w + X;
  const uint8_t c = mask_code(mask, X, Y, h, w);
  code[i] = c;
  float3 a = make_float3(0, 0, 0), e = make_float3(0, 0, 0);
  if (c & kSelf) tensor_from_grad(forward_grad(src, X, Y, h, w), k, &a, &e);
  const_cast<float*>(out.a)[i] = a.x;
  const_cast<float*>(out.b)[i] = a.y;
  const_cast<float*>(out.c)[i] = a.z;
  const_cast<float*>(out.ex)[i] = e.x;
  const_cast<float*>(out.ey)[i] = e.y;
  const_cast<float*>(out.ez)[i] = e.z;
  if (out.rec) {
    float4* r = const_cast<float4*>(out.rec) + 2 * i;
    r[0] = make_float4(a.x, a.y, a.z, e.x);
    *reinterpret_cast<float2*>(r + 1) = make_float2(e.y, e.z);
  }
}

// computeDerivatives (Python/vfs.cu:304-324) plus the per-warp solver reset
// of Python/vfs.py:489-497: p, q, v_ <- 0, u <- u_before, u_ carried over.
__global__ void k_derivs_init(TgvConsts out, TgvState st, Plane<const float> ubefore, Plane<const float> ub_src,
                              cudaTextureObject_t tref, cudaTextureObject_t tother, cudaTextureObject_t tdir, int h,
                              int w) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x;
  const int Y = blockIdx.y * blockDim.y + threadIdx.y;
  if (X >= w || Y >= h) return;
  const long i = (long)Y * w + X;
  const float2 d = epipolar_derivs(tref, tother, tdir, X, Y, h, w);
  const_cast<float*>(out.iu)[i] = d.x;
  const_cast<float*>(out.iz)[i] = d.y;
  if (out.rec) reinterpret_cast<float2*>(const_cast<float4*>(out.rec) + 2 * i + 1)[1] = d;
  const float ubv = ub_src.at(X, Y);
  st.u[i] = ubefore.at(X, Y);
  st.ub[i] = ubv;
  st.vbx[i] = st.vby[i] = 0.f;
  st.px[i] = st.py[i] = 0.f;
  st.qx[i] = st.qy[i] = st.qz[i] = st.qw[i] = 0.f;
}

}  // namespace

cudaError_t launch_tensor_soa(const TgvConsts& out, uint8_t* code, cudaTextureObject_t smooth,
                              Plane<const uint8_t> mask, const SolverConsts& k, int h, int w, cudaStream_t s) {
  if (h <= 0 || w <= 0) return cudaSuccess;
  k_tensor_soa<<<grid2d(h, w), dim3(kBX, kBY), 0, s>>>(out, code, smooth, mask, k, h, w);
  return cudaGetLastError();
}

cudaError_t launch_derivs_init(const TgvConsts& out, const TgvState& st, Plane<const float> ubefore,
                               Plane<const float> ub_src, cudaTextureObject_t tref, cudaTextureObject_t twarped,
                               cudaTextureObject_t tdir, int h, int w, cudaStream_t s) {
  if (h <= 0 || w <= 0) return cudaSuccess;
  k_derivs_init<<<grid2d(h, w), dim3(kBX, kBY), 0, s>>>(out, st, ubefore, ub_src, tref, twarped, tdir, h, w);
  return cudaGetLastError();
}

}  // namespace vfs

using namespace vfs;

namespace {

int make_tex(VfsPlan* pl, const void* ptr, int h, int w, size_t pitch, int kind, int linear, cudaTextureObject_t* out) {
  uint64_t t = 0;
  int rc = vfs_texture_create(ptr, h, w, pitch, kind, linear, &t);
  if (rc != VFS_OK) return rc;
  *out = (cudaTextureObject_t)t;
  pl->textures.push_back(*out);
  return VFS_OK;
}

// Lays out (or, with base == nullptr, measures) every buffer of a plan.
size_t layout(VfsPlan* pl, char* base) {
  Carver cv{base};
  const int L = pl->L;
  for (int l = 0; l < L; ++l) {
    auto& v = pl->lv[l];
    v.ref = {cv.take<float>(pitch_of(v.w, 4) * v.h), pitch_of(v.w, 4)};
    v.other = {cv.take<float>(pitch_of(v.w, 4) * v.h), pitch_of(v.w, 4)};
    v.tvf = {cv.take<float2>(pitch_of(v.w, 8) * v.h), pitch_of(v.w, 8)};
    v.mask = {cv.take<uint8_t>(pitch_of(v.w, 1) * v.h), pitch_of(v.w, 1)};
    v.code = cv.take<uint8_t>((size_t)v.h * v.w);
  }
  const int h0 = pl->lv[0].h, w0 = pl->lv[0].w;
  const size_t n0 = (size_t)h0 * w0;
  pl->other0 = {cv.take<float>(pitch_of(w0, 4) * h0), pitch_of(w0, 4)};
  pl->calib = {cv.take<float2>(n0 * 8), (size_t)w0 * 8};
  pl->smooth = {cv.take<float>(pitch_of(w0, 4) * h0), pitch_of(w0, 4)};
  pl->warped = {cv.take<float>(pitch_of(w0, 4) * h0), pitch_of(w0, 4)};
  pl->tvec = {cv.take<float2>(n0 * 8), 0};
  for (int i = 0; i < 8; ++i) pl->cplanes[i] = cv.take<float>(n0 * 4);
  pl->crec = cv.take<float4>(n0 * 32);
  for (int b = 0; b < 2; ++b) {
    float** f[10] = {&pl->st[b].u, &pl->st[b].ub, &pl->st[b].vbx, &pl->st[b].vby, &pl->st[b].px,
                     &pl->st[b].py, &pl->st[b].qx, &pl->st[b].qy, &pl->st[b].qz, &pl->st[b].qw};
    for (auto* pp : f) *pp = cv.take<float>(n0 * 4);
    pl->ubefore[b] = {cv.take<float>(pitch_of(w0, 4) * h0), pitch_of(w0, 4)};
    pl->warp[b] = {cv.take<float2>(pitch_of(w0, 8) * h0), pitch_of(w0, 8)};
  }
  pl->sched = cv.take<float3>(sizeof(float3) * std::max(1, pl->prm.nSolverIters));
  pl->dscale = cv.take<float2>(sizeof(float2) * std::max(1, pl->prm.nSolverIters));
  pl->stage_ref = cv.take<uint8_t>(n0);
  pl->stage_other = cv.take<uint8_t>(n0);
  pl->cst = {pl->cplanes[0], pl->cplanes[1], pl->cplanes[2], pl->cplanes[3], pl->cplanes[4],
             pl->cplanes[5], pl->cplanes[6], pl->cplanes[7], nullptr, pl->crec};
  return cv.off + kAlign;
}

void init_levels(VfsPlan* pl) {
  pl->L = pl->prm.nLevel;
  pl->lv.resize(pl->L);
  // compute_pyramid_sizes, Python/vfs.py:84-91: int(prev / fScale)
  int h = pl->prm.height, w = pl->prm.width;
  for (int l = 0; l < pl->L; ++l) {
    pl->lv[l].h = h;
    pl->lv[l].w = w;
    h = (int)(h / pl->prm.fScale);
    w = (int)(w / pl->prm.fScale);
  }
}

}  // namespace

namespace vfs {

cudaError_t plan_set_dual_scales(VfsPlan* pl, cudaStream_t s) {
  const int n = std::max(1, pl->prm.nSolverIters);
  std::vector<float> sched(3 * n, 0.f);
  step_schedule(pl->prm.nSolverIters, pl->prm.timeStepLambda, sched.data());
  pl->dscale_host.assign(2 * n, 0.f);
  dual_scales(pl->kc, sched.data(), n, pl->dscale_host.data());
  pl->kc.dscale = pl->dscale;
  const size_t bytes = pl->dscale_host.size() * sizeof(float);
  return s ? cudaMemcpyAsync(pl->dscale, pl->dscale_host.data(), bytes, cudaMemcpyHostToDevice, s)
           : cudaMemcpy(pl->dscale, pl->dscale_host.data(), bytes, cudaMemcpyHostToDevice);
}

// create_image_pyramid, Python/vfs.py:121-157, from the staged images.
int plan_pyramids(VfsPlan* pl, cudaStream_t s, long long* nk) {
  const int L = pl->L;
  auto& v0 = pl->lv[0];
  VFS_TRY_CUDA(launch_cast_and_scale(v0.ref, {pl->stage_ref, (size_t)v0.w}, v0.h, v0.w, s), "castAndScale");
  VFS_TRY_CUDA(launch_cast_and_scale(pl->other0, {pl->stage_other, (size_t)v0.w}, v0.h, v0.w, s), "castAndScale");
  *nk += 2;
  for (int l = 1; l < L; ++l, ++*nk)
    VFS_TRY_CUDA(launch_downsample_image(pl->lv[l].ref, pl->lv[l - 1].ref_tex, pl->lv[l].h, pl->lv[l].w, s),
                 "downSamplingImage");
  VFS_TRY_CUDA(launch_warp_image(v0.other, {pl->calib.ptr, pl->calib.pitch}, pl->other0_tex, v0.h, v0.w, s),
               "warpingImage");
  ++*nk;
  for (int l = 1; l < L; ++l, ++*nk)
    VFS_TRY_CUDA(launch_downsample_image(pl->lv[l].other, pl->lv[l - 1].other_tex, pl->lv[l].h, pl->lv[l].w, s),
                 "downSamplingImage");
  return VFS_OK;
}

// Start of a level: kernel choice, the coarsest level's zero state
// (Python/vfs.py:466-469), gaussian + tensor (Python/vfs.py:474-475).
int plan_level_begin(VfsPlan* pl, int l, LevelCtx* c, cudaStream_t s, long long* nk) {
  auto& v = pl->lv[l];
  c->l = l;
  c->h = v.h;
  c->w = v.w;
  c->b = l % 2;
  // TGV kernel for this level: the plan's variant, a per-level choice (the
  // autotuner's), or the cluster-resident kernel where the level fits
  int var = pl->level_variant[l] ? pl->level_variant[l] : pl->variant;
  int cs = 0;
  if (var == VFS_TGV_CLUSTER || (pl->level_variant[l] == 0 && pl->use_cluster)) {
    cs = tgv_cluster_size(v.h, v.w, pl->max_cluster);
    if (var == VFS_TGV_CLUSTER) var = pl->variant;
  }
  c->var = var;
  c->cs = cs;
  c->K = tgv_max_iters_per_launch(var);
  c->npass = (pl->prm.nSolverIters + c->K - 1) / c->K;
  const int h = v.h, w = v.w, b = c->b;
  if (l == pl->L - 1) {
    VFS_TRY_CUDA(cudaMemset2DAsync(pl->ubefore[b].ptr, pl->ubefore[b].pitch, 0, (size_t)w * 4, h, s), "memset");
    VFS_TRY_CUDA(cudaMemset2DAsync(pl->warp[b].ptr, pl->warp[b].pitch, 0, (size_t)w * 8, h, s), "memset");
  }
  c->ub_src = {pl->ubefore[b].ptr, pl->ubefore[b].pitch};
  c->mask = {v.mask.ptr, v.mask.pitch};
  VFS_TRY_CUDA(launch_gaussian_masked(pl->smooth, v.ref_tex, c->mask, h, w, s), "gaussianMasked");
  c->cst = pl->cst;
  c->cst.code = v.code;
  k_tensor_soa<<<grid2d(h, w), dim3(kBX, kBY), 0, s>>>(c->cst, v.code, v.smooth_tex, c->mask, pl->kc, h, w);
  VFS_TRY_CUDA(cudaGetLastError(), "tensor");
  *nk += 2;
  return VFS_OK;
}

// findWarpingVector + warpingImage (Python/vfs.py:480-483), then
// computeDerivatives + the solver reset (Python/vfs.py:486-497) into st[0].
int plan_warp_pre(VfsPlan* pl, LevelCtx* c, cudaStream_t s, long long* nk) {
  auto& v = pl->lv[c->l];
  const int h = c->h, w = c->w, b = c->b;
  VFS_TRY_CUDA(launch_warp_prologue(Plane<float2>{pl->tvec.ptr, (size_t)w * 8}, pl->warped,
                                    {pl->warp[b].ptr, pl->warp[b].pitch}, v.tvf_tex, v.other_tex, h, w, s),
               "warp prologue");
  k_derivs_init<<<grid2d(h, w), dim3(kBX, kBY), 0, s>>>(c->cst, pl->st[0], {pl->ubefore[b].ptr, pl->ubefore[b].pitch},
                                                        c->ub_src, v.ref_tex, v.warped_tex, v.tvf_tex, h, w);
  VFS_TRY_CUDA(cudaGetLastError(), "derivatives");
  *nk += 2;
  return VFS_OK;
}

// The solver iterations of one warp (Python/vfs.py:498-515), with optional
// timing events around them.
int plan_warp_tgv(VfsPlan* pl, LevelCtx* c, cudaStream_t s, long long* nk, unsigned ev_flags) {
  const int h = c->h, w = c->w, b = c->b;
  const int nIt = pl->prm.nSolverIters;
  const int launches = c->cs > 0 ? 1 : c->npass;
  const bool timed = pl->timing && launches > 0;
  int pair = -1;
  if (timed) {
    pair = pl->tev_used++;
    while ((int)pl->tev.size() < 2 * (pair + 1)) {
      cudaEvent_t e;
      VFS_TRY_CUDA(cudaEventCreate(&e), "event create");
      pl->tev.push_back(e);
    }
    if ((int)pl->tev_bytes.size() < pair + 1) {
      pl->tev_bytes.resize(pair + 1);
      pl->tev_launches.resize(pair + 1);
      pl->tev_level.resize(pair + 1);
    }
    VFS_TRY_CUDA(cudaEventRecordWithFlags(pl->tev[2 * pair], s, ev_flags), "event record");
  }
  if (c->cs > 0) {
    // the whole level in one cluster: iterations + median + clamp
    VFS_TRY_CUDA(launch_tgv_cluster(c->cs, pl->st[0], c->cst, pl->sched, nIt, pl->kc,
                                    {pl->warp[b].ptr, pl->warp[b].pitch}, pl->ubefore[b],
                                    {pl->tvec.ptr, (size_t)w * 8}, pl->kc.upperLimit, h, w, s),
                 "tgv cluster");
    ++*nk;
  } else {
    for (int j = 0; j < c->npass; ++j) {
      const int it0 = j * c->K;
      VFS_TRY_CUDA(launch_tgv_block(c->var, pl->st[j % 2], pl->st[(j + 1) % 2], c->cst, pl->sched, it0,
                                    std::min(c->K, nIt - it0), pl->kc, h, w, s),
                   "tgv");
    }
    *nk += c->npass;
  }
  if (timed) {
    VFS_TRY_CUDA(cudaEventRecordWithFlags(pl->tev[2 * pair + 1], s, ev_flags), "event record");
    // algorithmic bytes: 113 per pixel per iteration (state in and out,
    // per-warp constants in)
    pl->tev_bytes[pair] = 113.0 * (double)h * w * nIt;
    pl->tev_launches[pair] = launches;
    pl->tev_level[pair] = c->l;
  }
  return VFS_OK;
}

// medianFilter + computeOpticalFlowWithClamp (Python/vfs.py:518-521); the
// cluster kernel does them itself.
int plan_warp_post(VfsPlan* pl, LevelCtx* c, cudaStream_t s, long long* nk) {
  const int h = c->h, w = c->w, b = c->b;
  if (c->cs > 0) {
    c->ub_src = {pl->st[0].ub, (size_t)w * 4};
    return VFS_OK;
  }
  const TgvState& fin = pl->st[c->npass % 2];
  VFS_TRY_CUDA(launch_median_clamp({pl->warp[b].ptr, pl->warp[b].pitch}, pl->ubefore[b], {fin.u, (size_t)w * 4},
                                   {pl->tvec.ptr, (size_t)w * 8}, c->mask, pl->kc.upperLimit, h, w, s),
               "median/clamp");
  ++*nk;
  c->ub_src = {fin.ub, (size_t)w * 4};
  return VFS_OK;
}

// Up-sampling to the next finer level, Python/vfs.py:523-528.
int plan_level_end(VfsPlan* pl, LevelCtx* c, cudaStream_t s, long long* nk) {
  const int l = c->l;
  if (l == 0) return VFS_OK;
  auto& v = pl->lv[l];
  auto& f = pl->lv[l - 1];
  const int nb = (l - 1) % 2;
  VFS_TRY_CUDA(launch_upsample1(pl->ubefore[nb], v.ubefore_tex, pl->kc.fscale, f.h, f.w, s), "upSampling1");
  VFS_TRY_CUDA(launch_upsample2(pl->warp[nb], v.warp_tex, pl->kc.fscale, f.h, f.w, s), "upSampling");
  *nk += 2;
  return VFS_OK;
}

// warpUV_ref[masks[0] == 0, :] = 0, Python/vfs.py:531.
int plan_finish(VfsPlan* pl, cudaStream_t s, long long* nk) {
  auto& v0 = pl->lv[0];
  VFS_TRY_CUDA(launch_mask_flow(pl->warp[0], {v0.mask.ptr, v0.mask.pitch}, v0.h, v0.w, s), "mask flow");
  ++*nk;
  return VFS_OK;
}

}  // namespace vfs

namespace {

// Enqueues one complete solve on `s` from the staged images into warp[0].
int enqueue_solve(VfsPlan* pl, cudaStream_t s) {
  long long nk = 0;
  pl->tev_used = 0;
  // timing events: external event nodes when captured into a graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  VFS_TRY_CUDA(cudaStreamIsCapturing(s, &cap), "capture status");
  const unsigned ev_flags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
  VFS_TRY(plan_pyramids(pl, s, &nk));
  for (int l = pl->L - 1; l >= 0; --l) {
    LevelCtx c;
    VFS_TRY(plan_level_begin(pl, l, &c, s, &nk));
    for (int wi = 0; wi < pl->prm.nWarpIters; ++wi) {
      VFS_TRY(plan_warp_pre(pl, &c, s, &nk));
      VFS_TRY(plan_warp_tgv(pl, &c, s, &nk, ev_flags));
      VFS_TRY(plan_warp_post(pl, &c, s, &nk));
    }
    VFS_TRY(plan_level_end(pl, &c, s, &nk));
  }
  VFS_TRY(plan_finish(pl, s, &nk));
  pl->kernels_per_solve = nk;
  return VFS_OK;
}

}  // namespace

extern "C" {

int vfs_plan_workspace_size(const VfsParams* prm, size_t* bytes) {
  std::string why;
  if (!valid_params(prm, &why)) return fail(VFS_ERR_ARG, why);
  if (!bytes) return fail(VFS_ERR_ARG, "bytes is NULL");
  VfsPlan tmp;
  tmp.prm = *prm;
  init_levels(&tmp);
  for (auto& v : tmp.lv)
    if (v.h <= 0 || v.w <= 0) return fail(VFS_ERR_ARG, "pyramid level has zero size; reduce nLevel");
  *bytes = layout(&tmp, nullptr);
  return VFS_OK;
}

int vfs_plan_create(const VfsParams* prm, void* workspace, size_t workspace_bytes, VfsPlan** plan_out) {
  std::string why;
  if (!valid_params(prm, &why)) return fail(VFS_ERR_ARG, why);
  if (!plan_out) return fail(VFS_ERR_ARG, "plan_out is NULL");
  size_t need = 0;
  VFS_TRY(vfs_plan_workspace_size(prm, &need));
  if (!workspace || workspace_bytes < need)
    return fail(VFS_ERR_WORKSPACE, "workspace of " + std::to_string(need) + " bytes required");
  VfsPlan* pl = new (std::nothrow) VfsPlan();
  if (!pl) return fail(VFS_ERR_ARG, "out of host memory");
  pl->prm = *prm;
  pl->kc = make_consts(prm);
  init_levels(pl);
  char* base = reinterpret_cast<char*>(round_up(reinterpret_cast<uintptr_t>(workspace), kAlign));
  layout(pl, base);
  // step sizes, Python/vfs.py:494-515
  std::vector<float> sched(3 * std::max(1, prm->nSolverIters), 0.f);
  step_schedule(prm->nSolverIters, prm->timeStepLambda, sched.data());
  cudaError_t e = cudaMemcpy(pl->sched, sched.data(), sched.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = plan_set_dual_scales(pl, nullptr);
  if (e != cudaSuccess) {
    delete pl;
    return cuda_status(e, "schedule upload");
  }
  int rc = VFS_OK;
  for (int l = 0; l < pl->L && rc == VFS_OK; ++l) {
    auto& v = pl->lv[l];
    if (rc == VFS_OK) rc = make_tex(pl, v.ref.ptr, v.h, v.w, v.ref.pitch, VFS_TEX_F32, 1, &v.ref_tex);
    if (rc == VFS_OK) rc = make_tex(pl, v.other.ptr, v.h, v.w, v.other.pitch, VFS_TEX_F32, 1, &v.other_tex);
    if (rc == VFS_OK) rc = make_tex(pl, v.tvf.ptr, v.h, v.w, v.tvf.pitch, VFS_TEX_F32X2, 1, &v.tvf_tex);
    if (rc == VFS_OK) rc = make_tex(pl, v.mask.ptr, v.h, v.w, v.mask.pitch, VFS_TEX_U8, 0, &v.mask_tex);
    if (rc == VFS_OK) rc = make_tex(pl, pl->smooth.ptr, v.h, v.w, pl->smooth.pitch, VFS_TEX_F32, 1, &v.smooth_tex);
    if (rc == VFS_OK) rc = make_tex(pl, pl->warped.ptr, v.h, v.w, pl->warped.pitch, VFS_TEX_F32, 1, &v.warped_tex);
    if (rc == VFS_OK)
      rc = make_tex(pl, pl->ubefore[l % 2].ptr, v.h, v.w, pl->ubefore[l % 2].pitch, VFS_TEX_F32, 1, &v.ubefore_tex);
    if (rc == VFS_OK)
      rc = make_tex(pl, pl->warp[l % 2].ptr, v.h, v.w, pl->warp[l % 2].pitch, VFS_TEX_F32X2, 1, &v.warp_tex);
  }
  if (rc == VFS_OK) rc = cuda_status(tgv_prepare(), "tgv kernel attributes");
  if (rc == VFS_OK) rc = cuda_status(tgv_cluster_prepare(&pl->max_cluster), "cluster kernel attributes");
  if (rc == VFS_OK)
    rc = make_tex(pl, pl->other0.ptr, pl->lv[0].h, pl->lv[0].w, pl->other0.pitch, VFS_TEX_F32, 1, &pl->other0_tex);
  if (rc != VFS_OK) {
    vfs_plan_destroy(pl);
    return rc;
  }
  *plan_out = pl;
  return VFS_OK;
}

int vfs_plan_destroy(VfsPlan* pl) {
  if (!pl) return VFS_OK;
  for (auto t : pl->textures) cudaDestroyTextureObject(t);
  pl->drop_graph();
  if (pl->gstream) cudaStreamDestroy(pl->gstream);
  if (pl->ev_in) cudaEventDestroy(pl->ev_in);
  if (pl->ev_out) cudaEventDestroy(pl->ev_out);
  for (auto e : pl->tev) cudaEventDestroy(e);
  delete pl;
  return VFS_OK;
}

int vfs_plan_sizes(const VfsPlan* pl, int* hw) {
  if (!pl || !hw) return fail(VFS_ERR_ARG, "NULL argument");
  for (int l = 0; l < pl->L; ++l) {
    hw[2 * l] = pl->lv[l].h;
    hw[2 * l + 1] = pl->lv[l].w;
  }
  return VFS_OK;
}

int vfs_plan_set_tgv_variant(VfsPlan* pl, int k) {
  if (!pl) return fail(VFS_ERR_ARG, "plan is NULL");
  if (tgv_max_iters_per_launch(k) == 0) return fail(VFS_ERR_ARG, "unknown TGV kernel variant");
  if (pl->variant != k) pl->drop_graph();
  pl->variant = k;
  return VFS_OK;
}

int vfs_plan_set_mask(VfsPlan* pl, const uint8_t* mask, size_t mask_pitch, void* stream) {
  if (!pl || !mask) return fail(VFS_ERR_ARG, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  auto& v0 = pl->lv[0];
  if (mask_pitch == 0) mask_pitch = (size_t)v0.w;
  VFS_TRY_CUDA(cudaMemcpy2DAsync(v0.mask.ptr, v0.mask.pitch, mask, mask_pitch, v0.w, v0.h, cudaMemcpyDeviceToDevice, s),
               "mask copy");
  // create_mask_pyramid, Python/vfs.py:159-187
  for (int l = 1; l < pl->L; ++l) {
    auto& v = pl->lv[l];
    VFS_TRY_CUDA(launch_downsample_mask(v.mask, pl->lv[l - 1].mask_tex, v.h, v.w, s), "downSamplingMask");
  }
  pl->mask_set = true;
  return VFS_OK;
}

int vfs_plan_set_vector_fields(VfsPlan* pl, const float* tvf, const float* cvf, void* stream) {
  if (!pl || !tvf || !cvf) return fail(VFS_ERR_ARG, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  auto& v0 = pl->lv[0];
  VFS_TRY_CUDA(cudaMemcpy2DAsync(v0.tvf.ptr, v0.tvf.pitch, tvf, (size_t)v0.w * 8, (size_t)v0.w * 8, v0.h,
                                 cudaMemcpyDeviceToDevice, s),
               "vector field copy");
  VFS_TRY_CUDA(cudaMemcpyAsync(pl->calib.ptr, cvf, (size_t)v0.w * v0.h * 8, cudaMemcpyDeviceToDevice, s),
               "calibration copy");
  // create_vector_field_pyramid, Python/vfs.py:189-218
  for (int l = 1; l < pl->L; ++l) {
    auto& v = pl->lv[l];
    VFS_TRY_CUDA(launch_downsample_field(v.tvf, pl->lv[l - 1].tvf_tex, v.h, v.w, s), "downSamplingVectorField");
  }
  pl->fields_set = true;
  return VFS_OK;
}

int vfs_plan_solve(VfsPlan* pl, const uint8_t* img_ref, const uint8_t* img_other, float* warp_out, void* stream) {
  if (!pl || !img_ref || !img_other || !warp_out) return fail(VFS_ERR_ARG, "NULL argument");
  if (!pl->mask_set || !pl->fields_set)
    return fail(VFS_ERR_STATE, "set_mask and set_vector_fields must precede solve");
  cudaStream_t s = (cudaStream_t)stream;
  auto& v0 = pl->lv[0];
  const size_t n0 = (size_t)v0.h * v0.w;
  VFS_TRY_CUDA(cudaMemcpyAsync(pl->stage_ref, img_ref, n0, cudaMemcpyDeviceToDevice, s), "image copy");
  VFS_TRY_CUDA(cudaMemcpyAsync(pl->stage_other, img_other, n0, cudaMemcpyDeviceToDevice, s), "image copy");
  if (pl->use_graph) {
    if (!pl->gstream) VFS_TRY_CUDA(cudaStreamCreateWithFlags(&pl->gstream, cudaStreamNonBlocking), "stream");
    if (!pl->ev_in) VFS_TRY_CUDA(cudaEventCreateWithFlags(&pl->ev_in, cudaEventDisableTiming), "event");
    if (!pl->ev_out) VFS_TRY_CUDA(cudaEventCreateWithFlags(&pl->ev_out, cudaEventDisableTiming), "event");
    if (!pl->gexec) {
      VFS_TRY_CUDA(cudaStreamBeginCapture(pl->gstream, cudaStreamCaptureModeThreadLocal), "begin capture");
      int rc = enqueue_solve(pl, pl->gstream);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(pl->gstream, &g);
      if (rc != VFS_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      VFS_TRY_CUDA(e, "end capture");
      e = cudaGraphInstantiate(&pl->gexec, g, 0);
      cudaGraphDestroy(g);
      VFS_TRY_CUDA(e, "graph instantiate");
    }
    VFS_TRY_CUDA(cudaEventRecord(pl->ev_in, s), "event record");
    VFS_TRY_CUDA(cudaStreamWaitEvent(pl->gstream, pl->ev_in, 0), "stream wait");
    VFS_TRY_CUDA(cudaGraphLaunch(pl->gexec, pl->gstream), "graph launch");
    VFS_TRY_CUDA(cudaEventRecord(pl->ev_out, pl->gstream), "event record");
    VFS_TRY_CUDA(cudaStreamWaitEvent(s, pl->ev_out, 0), "stream wait");
  } else {
    VFS_TRY(enqueue_solve(pl, s));
  }
  VFS_TRY_CUDA(cudaMemcpy2DAsync(warp_out, (size_t)v0.w * 8, pl->warp[0].ptr, pl->warp[0].pitch, (size_t)v0.w * 8,
                                 v0.h, cudaMemcpyDeviceToDevice, s),
               "flow copy");
  pl->solved = true;
  return VFS_OK;
}

int vfs_plan_set_graph(VfsPlan* pl, int enable) {
  if (!pl) return fail(VFS_ERR_ARG, "plan is NULL");
  if ((bool)enable != pl->use_graph) pl->drop_graph();
  pl->use_graph = enable != 0;
  return VFS_OK;
}

int vfs_plan_set_timing(VfsPlan* pl, int enable) {
  if (!pl) return fail(VFS_ERR_ARG, "plan is NULL");
  if ((bool)enable != pl->timing) pl->drop_graph();
  pl->timing = enable != 0;
  if (pl->timing) {  // one event pair per warp, created before any capture
    const size_t need = 2 * (size_t)pl->L * std::max(1, pl->prm.nWarpIters);
    while (pl->tev.size() < need) {
      cudaEvent_t e;
      VFS_TRY_CUDA(cudaEventCreate(&e), "event create");
      pl->tev.push_back(e);
    }
    pl->tev_bytes.resize(need / 2);
    pl->tev_level.resize(need / 2);
    pl->tev_launches.resize(need / 2);
  }
  return VFS_OK;
}

int vfs_plan_stats(VfsPlan* pl, VfsSolveStats* out) {
  if (!pl || !out) return fail(VFS_ERR_ARG, "NULL argument");
  memset(out, 0, sizeof(*out));
  out->kernels_per_solve = pl->kernels_per_solve;
  if (!pl->timing) return VFS_OK;
  double ms = 0, bytes = 0;
  long long launches = 0;
  for (int i = 0; i < pl->tev_used; ++i) {
    float t = 0;
    VFS_TRY_CUDA(cudaEventElapsedTime(&t, pl->tev[2 * i], pl->tev[2 * i + 1]), "event elapsed (synchronise first)");
    ms += t;
    bytes += pl->tev_bytes[i];
    launches += pl->tev_launches[i];
    const int lvl = pl->tev_level[i];
    if (lvl >= 0 && lvl < 16) out->tgv_ms_level[lvl] += t;
  }
  out->tgv_ms = ms;
  out->tgv_alg_bytes = bytes;
  out->tgv_launches = launches;
  out->tgv_intervals = pl->tev_used;
  return VFS_OK;
}

static int plan_triangulate(VfsPlan* pl, float f, float u0, float v0f, const float* t, float* xyz_out, void* stream,
                            bool lsq) {
  if (!pl || !t || !xyz_out) return fail(VFS_ERR_ARG, "NULL argument");
  if (!pl->solved) return fail(VFS_ERR_STATE, "triangulate needs a solve first");
  auto& v0 = pl->lv[0];
  VFS_TRY_CUDA(launch_triangulate_flow(reinterpret_cast<float3*>(xyz_out), {pl->warp[0].ptr, pl->warp[0].pitch},
                                       Cam{f, u0, v0f}, t[0], t[1], t[2], {v0.mask.ptr, v0.mask.pitch}, v0.h, v0.w,
                                       (cudaStream_t)stream, lsq),
               "triangulate");
  return VFS_OK;
}

int vfs_plan_triangulate(VfsPlan* pl, float f, float u0, float v0f, const float* t, float* xyz_out, void* stream) {
  return plan_triangulate(pl, f, u0, v0f, t, xyz_out, stream, false);
}

int vfs_plan_triangulate_lsq(VfsPlan* pl, float f, float u0, float v0f, const float* t, float* xyz_out,
                             void* stream) {
  return plan_triangulate(pl, f, u0, v0f, t, xyz_out, stream, true);
}

}  // extern "C"

extern "C" int vfs_tgv_variants(int* ids, int cap, int* iters_per_launch) {
  const int n = tgv_variant_list(ids, cap);
  if (ids && iters_per_launch)
    for (int i = 0; i < n && i < cap; ++i) iters_per_launch[i] = tgv_max_iters_per_launch(ids[i]);
  return n;
}

extern "C" int vfs_plan_set_cluster(VfsPlan* pl, int enable) {
  if (!pl) return fail(VFS_ERR_ARG, "plan is NULL");
  if ((bool)enable != pl->use_cluster) pl->drop_graph();
  pl->use_cluster = enable != 0;
  return VFS_OK;
}

extern "C" int vfs_plan_set_level_variant(VfsPlan* pl, int level, int variant) {
  if (!pl) return fail(VFS_ERR_ARG, "plan is NULL");
  if (level < 0 || level >= pl->L) return fail(VFS_ERR_ARG, "level out of range");
  if (variant != 0 && variant != VFS_TGV_CLUSTER && tgv_max_iters_per_launch(variant) == 0)
    return fail(VFS_ERR_ARG, "unknown TGV kernel variant");
  if (pl->level_variant[level] != variant) pl->drop_graph();
  pl->level_variant[level] = variant;
  return VFS_OK;
}

extern "C" int vfs_plan_level_cluster(const VfsPlan* pl, int level) {
  if (!pl || level < 0 || level >= pl->L) return 0;
  return tgv_cluster_size(pl->lv[level].h, pl->lv[level].w, pl->max_cluster);
}
