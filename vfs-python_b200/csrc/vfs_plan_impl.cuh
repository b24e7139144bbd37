// Internal view of a plan, shared by the single-pair solve (vfs_plan.cu) and
// the batched multi-pair solve (vfs_batch.cu).
#pragma once
#include <vector>

#include "vfs_api_util.cuh"
#include "vfs_kernels.cuh"
#include "vfs_tgv.cuh"

struct VfsPlan {
  VfsParams prm;
  vfs::SolverConsts kc;
  int L = 0;
  struct Level {
    int h, w;
    vfs::Plane<float> ref, other;
    vfs::Plane<float2> tvf;
    vfs::Plane<uint8_t> mask;
    uint8_t* code;
    cudaTextureObject_t ref_tex = 0, other_tex = 0, tvf_tex = 0, mask_tex = 0, smooth_tex = 0, warped_tex = 0,
                        ubefore_tex = 0, warp_tex = 0;
  };
  std::vector<Level> lv;
  vfs::Plane<float> other0;
  cudaTextureObject_t other0_tex = 0;
  vfs::Plane<float2> calib;
  vfs::Plane<float> smooth, warped;
  vfs::Plane<float2> tvec;
  vfs::TgvConsts cst;
  float* cplanes[8];
  float4* crec = nullptr;  // the constants as records (TgvConsts::rec)
  vfs::TgvState st[2];
  vfs::Plane<float> ubefore[2];
  vfs::Plane<float2> warp[2];
  float3* sched = nullptr;
  float2* dscale = nullptr;          // dual-step scales for kc (dual_scales)
  std::vector<float> dscale_host;    // their source for the last upload
  int variant = 134;
  int level_variant[32] = {0};  // 0: the plan's variant; VFS_TGV_CLUSTER: cluster kernel
  bool mask_set = false, fields_set = false, solved = false;
  std::vector<cudaTextureObject_t> textures;
  // input staging (workspace), so a captured graph has fixed pointers
  uint8_t* stage_ref = nullptr;
  uint8_t* stage_other = nullptr;
  // graph replay
  bool use_graph = false;
  cudaStream_t gstream = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // instrumentation: an event pair around each warp's TGV launches
  bool timing = false;
  std::vector<cudaEvent_t> tev;
  std::vector<double> tev_bytes;
  std::vector<long long> tev_launches;
  std::vector<int> tev_level;
  int tev_used = 0;
  long long kernels_per_solve = 0;
  // cluster-resident solve for levels that fit one cluster
  bool use_cluster = false;
  int max_cluster = 0;

  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
  }
};

namespace vfs {

// Per-level state of a solve in progress.
struct LevelCtx {
  int l = 0, h = 0, w = 0, b = 0;
  int var = 0;     // TGV kernel variant
  int cs = 0;      // cluster size (cluster-resident kernel) or 0
  int K = 1;       // iterations per TGV launch
  int npass = 0;   // TGV launches per warp (when cs == 0)
  TgvConsts cst;
  Plane<const uint8_t> mask;
  Plane<const float> ub_src;  // u_ at the start of the next warp
};

// The steps of solve_stereo (Python/vfs.py:460-533), enqueued on `s`; nk
// counts kernel launches.
int plan_pyramids(VfsPlan* pl, cudaStream_t s, long long* nk);
// Forms the dual-step scales of pl->kc (dual_scales), uploads them to
// pl->dscale (synchronous copy when s is null, else ordered on s) and points
// pl->kc.dscale at them.  Called whenever pl->kc is (re)built.
cudaError_t plan_set_dual_scales(VfsPlan* pl, cudaStream_t s);
int plan_level_begin(VfsPlan* pl, int l, LevelCtx* c, cudaStream_t s, long long* nk);
int plan_warp_pre(VfsPlan* pl, LevelCtx* c, cudaStream_t s, long long* nk);
int plan_warp_tgv(VfsPlan* pl, LevelCtx* c, cudaStream_t s, long long* nk, unsigned ev_flags);
int plan_warp_post(VfsPlan* pl, LevelCtx* c, cudaStream_t s, long long* nk);
int plan_level_end(VfsPlan* pl, LevelCtx* c, cudaStream_t s, long long* nk);
int plan_finish(VfsPlan* pl, cudaStream_t s, long long* nk);

// computeTensorEtaMasked into the solver's constant planes plus the mask
// code (Python/vfs.cu:239-281), and computeDerivatives plus the per-warp
// solver reset (Python/vfs.cu:304-324, Python/vfs.py:486-497).
cudaError_t launch_tensor_soa(const TgvConsts& out, uint8_t* code, cudaTextureObject_t smooth,
                              Plane<const uint8_t> mask, const SolverConsts& k, int h, int w, cudaStream_t s);
cudaError_t launch_derivs_init(const TgvConsts& out, const TgvState& st, Plane<const float> ubefore,
                               Plane<const float> ub_src, cudaTextureObject_t tref, cudaTextureObject_t twarped,
                               cudaTextureObject_t tdir, int h, int w, cudaStream_t s);

}  // namespace vfs
