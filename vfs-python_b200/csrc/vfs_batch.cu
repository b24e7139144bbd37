// Batched solve of many stereo pairs of uneven resolution on one stream.
//
// Each pair has its own plan (pyramids, state, textures) carved from one
// workspace; all pairs share the solver parameters and so the number of
// levels, warps and iterations.  The pairs advance through the coarse-to-fine
// solve in lockstep: per level and warp, each pair's small per-warp kernels
// run, then each TGV pass is one launch whose blocks cover the tiles of all
// pairs (a (pair, tile) work list of up to 32 pairs, passed as the launch's
// parameter; larger batches take one launch per 32 pairs), so small coarse
// levels of many pairs fill the GPU together.  Optionally (vfs_batch_set_group_bytes)
// the pairs of a level are cut into groups whose solver working set (two
// state sets and the per-warp constants, 113 bytes a pixel) fits a budget:
// a group's passes then all run before the next group's, each launch
// covering the group's tiles.  (On a B200, one 800x800 pair per group did
// not bring an 8-pair batch's finest level back to the single-pair time, so
// the default is one group.)  The whole batch can be captured and replayed
// as one CUDA graph.  No
// counterpart in the reference, whose solver handles one pair per call
// (Python/vfs.py:460-533); per pair the results are bit-identical to a
// single-pair solve, whatever the grouping.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "vfs_plan_impl.cuh"

using namespace vfs;

struct VfsBatch {
  VfsParams prm;
  int n = 0, L = 0;
  std::vector<VfsPlan*> plans;
  std::vector<TgvBatchItem> items;  // L x n, passed to the launches as parameters
  std::vector<int> total_tiles;   // per level
  // per level: groups of consecutive pairs launched together (first pair,
  // pair count, first tile, tile count)
  struct Group {
    int p0, np, bid0, ntiles;
  };
  std::vector<std::vector<Group>> groups;
  size_t group_bytes = 0;  // 0: all pairs of a level in one launch per pass
  int level_variant[32];
  bool use_graph = false;
  cudaStream_t gstream = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  bool timing = false;
  std::vector<cudaEvent_t> tev;
  std::vector<int> tev_level;
  std::vector<double> tev_bytes;
  std::vector<long long> tev_launches;
  int tev_used = 0;
  long long kernels_per_solve = 0;
  void drop_graph() {
    if (gexec) cudaGraphExecDestroy(gexec);
    gexec = nullptr;
  }
};

namespace {

constexpr size_t kBatchAlign = 512;
inline size_t rup(size_t v, size_t a) { return (v + a - 1) / a * a; }

VfsParams pair_params(const VfsParams* prm, int h, int w) {
  VfsParams p = *prm;
  p.height = h;
  p.width = w;
  return p;
}

int layout_sizes(const VfsParams* prm, int n, const int* hs, const int* ws, std::vector<size_t>* offs, size_t* total) {
  std::string why;
  if (!valid_params(prm, &why)) return fail(VFS_ERR_ARG, why);
  if (n <= 0 || !hs || !ws) return fail(VFS_ERR_ARG, "a batch needs n > 0 pairs and their sizes");
  size_t off = 0;
  offs->clear();
  for (int i = 0; i < n; ++i) {
    VfsParams p = pair_params(prm, hs[i], ws[i]);
    size_t b = 0;
    VFS_TRY(vfs_plan_workspace_size(&p, &b));
    offs->push_back(off);
    off = rup(off + b, kBatchAlign);
  }
  *total = off + kBatchAlign;
  return VFS_OK;
}

// The (pair, tile) work lists of every level for the chosen kernels.
int upload_items(VfsBatch* bt) {
  std::vector<TgvBatchItem>& host = bt->items;
  host.assign((size_t)bt->L * bt->n, TgvBatchItem{});
  bt->total_tiles.assign(bt->L, 0);
  for (int l = 0; l < bt->L; ++l) {
    int tx = 32, ty = 32;
    if (!tgv_tile_shape(bt->level_variant[l], &tx, &ty)) return fail(VFS_ERR_ARG, "batched solves need a 1xx kernel");
    int base = 0;
    for (int i = 0; i < bt->n; ++i) {
      VfsPlan* pl = bt->plans[i];
      TgvBatchItem& it = host[(size_t)l * bt->n + i];
      it.st[0] = pl->st[0];
      it.st[1] = pl->st[1];
      it.cst = pl->cst;
      it.cst.code = pl->lv[l].code;
      it.h = pl->lv[l].h;
      it.w = pl->lv[l].w;
      it.tiles_x = (it.w + tx - 1) / tx;
      it.tile_base = base;
      base += it.tiles_x * ((it.h + ty - 1) / ty);
    }
    bt->total_tiles[l] = base;
  }
  // groups of consecutive pairs within the working-set budget
  bt->groups.assign(bt->L, {});
  for (int l = 0; l < bt->L; ++l) {
    int i = 0;
    while (i < bt->n) {
      const TgvBatchItem& first = host[(size_t)l * bt->n + i];
      VfsBatch::Group g{i, 0, first.tile_base, 0};
      double bytes = 0;
      while (i < bt->n) {
        const TgvBatchItem& it = host[(size_t)l * bt->n + i];
        const double b = 113.0 * it.h * it.w;
        if (g.np > 0 && bt->group_bytes > 0 && bytes + b > (double)bt->group_bytes) break;
        if (g.np == kBatchParamItems) break;  // a launch's work list holds at most this many
        bytes += b;
        ++g.np;
        ++i;
      }
      const int end = i < bt->n ? host[(size_t)l * bt->n + i].tile_base : bt->total_tiles[l];
      g.ntiles = end - g.bid0;
      bt->groups[l].push_back(g);
    }
  }
  return VFS_OK;
}

int enqueue_batch(VfsBatch* bt, cudaStream_t s) {
  long long nk = 0;
  bt->tev_used = 0;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  VFS_TRY_CUDA(cudaStreamIsCapturing(s, &cap), "capture status");
  const unsigned ev_flags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
  const int n = bt->n;
  const int nIt = bt->prm.nSolverIters;
  for (int i = 0; i < n; ++i) VFS_TRY(plan_pyramids(bt->plans[i], s, &nk));
  std::vector<LevelCtx> ctx(n);
  for (int l = bt->L - 1; l >= 0; --l) {
    for (int i = 0; i < n; ++i) VFS_TRY(plan_level_begin(bt->plans[i], l, &ctx[i], s, &nk));
    const int var = bt->level_variant[l];
    const int K = tgv_max_iters_per_launch(var);
    const int npass = (nIt + K - 1) / K;
    double px = 0;
    for (int i = 0; i < n; ++i) px += (double)ctx[i].h * ctx[i].w;
    for (int wi = 0; wi < bt->prm.nWarpIters; ++wi) {
      for (int i = 0; i < n; ++i) VFS_TRY(plan_warp_pre(bt->plans[i], &ctx[i], s, &nk));
      int pair = -1;
      if (bt->timing && npass > 0) {
        pair = bt->tev_used++;
        VFS_TRY_CUDA(cudaEventRecordWithFlags(bt->tev[2 * pair], s, ev_flags), "event record");
      }
      for (const auto& g : bt->groups[l]) {
        TgvBatchParams P;
        P.n_items = g.np;
        P.bid0 = g.bid0;
        for (int i = 0; i < g.np; ++i) P.items[i] = bt->items[(size_t)l * n + g.p0 + i];
        for (int j = 0; j < npass; ++j) {
          const int it0 = j * K;
          VFS_TRY_CUDA(launch_tgv_batch(var, P, g.ntiles, j % 2, bt->plans[0]->sched, it0, std::min(K, nIt - it0),
                                        bt->plans[0]->kc, s),
                       "batched tgv");
        }
        nk += npass;
      }
      if (pair >= 0) {
        VFS_TRY_CUDA(cudaEventRecordWithFlags(bt->tev[2 * pair + 1], s, ev_flags), "event record");
        bt->tev_level[pair] = l;
        bt->tev_bytes[pair] = 113.0 * px * nIt;
        bt->tev_launches[pair] = npass * (long long)bt->groups[l].size();
      }
      for (int i = 0; i < n; ++i) {
        ctx[i].npass = npass;  // the batched launches' parity decides the final state set
        ctx[i].cs = 0;
        VFS_TRY(plan_warp_post(bt->plans[i], &ctx[i], s, &nk));
      }
    }
    for (int i = 0; i < n; ++i) VFS_TRY(plan_level_end(bt->plans[i], &ctx[i], s, &nk));
  }
  for (int i = 0; i < n; ++i) VFS_TRY(plan_finish(bt->plans[i], s, &nk));
  bt->kernels_per_solve = nk;
  return VFS_OK;
}

}  // namespace

extern "C" {

int vfs_batch_workspace_size(const VfsParams* prm, int n, const int* heights, const int* widths, size_t* bytes) {
  if (!bytes) return fail(VFS_ERR_ARG, "bytes is NULL");
  std::vector<size_t> offs;
  return layout_sizes(prm, n, heights, widths, &offs, bytes);
}

int vfs_batch_destroy(VfsBatch* bt) {
  if (!bt) return VFS_OK;
  for (auto* p : bt->plans) vfs_plan_destroy(p);
  bt->drop_graph();
  if (bt->gstream) cudaStreamDestroy(bt->gstream);
  if (bt->ev_in) cudaEventDestroy(bt->ev_in);
  if (bt->ev_out) cudaEventDestroy(bt->ev_out);
  for (auto e : bt->tev) cudaEventDestroy(e);
  delete bt;
  return VFS_OK;
}

int vfs_batch_create(const VfsParams* prm, int n, const int* heights, const int* widths, void* workspace,
                     size_t workspace_bytes, VfsBatch** out) {
  if (!out) return fail(VFS_ERR_ARG, "out is NULL");
  std::vector<size_t> offs;
  size_t need = 0;
  VFS_TRY(layout_sizes(prm, n, heights, widths, &offs, &need));
  if (!workspace || workspace_bytes < need)
    return fail(VFS_ERR_WORKSPACE, "workspace of " + std::to_string(need) + " bytes required");
  char* base = reinterpret_cast<char*>(rup(reinterpret_cast<uintptr_t>(workspace), kBatchAlign));
  VfsBatch* bt = new (std::nothrow) VfsBatch();
  if (!bt) return fail(VFS_ERR_ARG, "out of host memory");
  bt->prm = *prm;
  bt->n = n;
  bt->L = prm->nLevel;
  for (int l = 0; l < 32; ++l) bt->level_variant[l] = 134;
  for (int i = 0; i < n; ++i) {
    VfsParams p = pair_params(prm, heights[i], widths[i]);
    VfsPlan* pl = nullptr;
    size_t b = 0;
    vfs_plan_workspace_size(&p, &b);
    const int rc = vfs_plan_create(&p, base + offs[i], b, &pl);
    if (rc != VFS_OK) {
      vfs_batch_destroy(bt);
      return rc;
    }
    bt->plans.push_back(pl);
  }
  const int rc = upload_items(bt);
  if (rc != VFS_OK) {
    vfs_batch_destroy(bt);
    return rc;
  }
  *out = bt;
  return VFS_OK;
}

int vfs_batch_set_pair(VfsBatch* bt, int i, const uint8_t* mask, size_t mask_pitch, const float* tvf,
                       const float* cvf, void* stream) {
  if (!bt || i < 0 || i >= bt->n) return fail(VFS_ERR_ARG, "pair index out of range");
  VFS_TRY(vfs_plan_set_mask(bt->plans[i], mask, mask_pitch, stream));
  return vfs_plan_set_vector_fields(bt->plans[i], tvf, cvf, stream);
}

int vfs_batch_set_level_variant(VfsBatch* bt, int level, int variant) {
  if (!bt || level < 0 || level >= bt->L) return fail(VFS_ERR_ARG, "level out of range");
  int tx, ty;
  if (!tgv_tile_shape(variant, &tx, &ty)) return fail(VFS_ERR_ARG, "batched solves need a 1xx kernel variant");
  if (bt->level_variant[level] == variant) return VFS_OK;
  bt->level_variant[level] = variant;
  bt->drop_graph();
  return upload_items(bt);
}

int vfs_batch_set_group_bytes(VfsBatch* bt, size_t bytes) {
  if (!bt) return fail(VFS_ERR_ARG, "batch is NULL");
  if (bt->group_bytes == bytes) return VFS_OK;
  bt->group_bytes = bytes;
  bt->drop_graph();
  return upload_items(bt);
}

int vfs_batch_set_graph(VfsBatch* bt, int enable) {
  if (!bt) return fail(VFS_ERR_ARG, "batch is NULL");
  if ((bool)enable != bt->use_graph) bt->drop_graph();
  bt->use_graph = enable != 0;
  return VFS_OK;
}

int vfs_batch_set_timing(VfsBatch* bt, int enable) {
  if (!bt) return fail(VFS_ERR_ARG, "batch is NULL");
  if ((bool)enable != bt->timing) bt->drop_graph();
  bt->timing = enable != 0;
  if (bt->timing) {
    const size_t need = 2 * (size_t)bt->L * std::max(1, bt->prm.nWarpIters);
    while (bt->tev.size() < need) {
      cudaEvent_t e;
      VFS_TRY_CUDA(cudaEventCreate(&e), "event create");
      bt->tev.push_back(e);
    }
    bt->tev_level.resize(need / 2);
    bt->tev_bytes.resize(need / 2);
    bt->tev_launches.resize(need / 2);
  }
  return VFS_OK;
}

int vfs_batch_solve(VfsBatch* bt, const uint8_t* const* img_refs, const uint8_t* const* img_others,
                    float* const* warps_out, void* stream) {
  if (!bt || !img_refs || !img_others || !warps_out) return fail(VFS_ERR_ARG, "NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  for (int i = 0; i < bt->n; ++i) {
    VfsPlan* pl = bt->plans[i];
    if (!pl->mask_set || !pl->fields_set) return fail(VFS_ERR_STATE, "set every pair before solving");
    if (!img_refs[i] || !img_others[i] || !warps_out[i]) return fail(VFS_ERR_ARG, "NULL image or output");
    const size_t n0 = (size_t)pl->lv[0].h * pl->lv[0].w;
    VFS_TRY_CUDA(cudaMemcpyAsync(pl->stage_ref, img_refs[i], n0, cudaMemcpyDeviceToDevice, s), "image copy");
    VFS_TRY_CUDA(cudaMemcpyAsync(pl->stage_other, img_others[i], n0, cudaMemcpyDeviceToDevice, s), "image copy");
  }
  if (bt->use_graph) {
    if (!bt->gstream) VFS_TRY_CUDA(cudaStreamCreateWithFlags(&bt->gstream, cudaStreamNonBlocking), "stream");
    if (!bt->ev_in) VFS_TRY_CUDA(cudaEventCreateWithFlags(&bt->ev_in, cudaEventDisableTiming), "event");
    if (!bt->ev_out) VFS_TRY_CUDA(cudaEventCreateWithFlags(&bt->ev_out, cudaEventDisableTiming), "event");
    if (!bt->gexec) {
      VFS_TRY_CUDA(cudaStreamBeginCapture(bt->gstream, cudaStreamCaptureModeThreadLocal), "begin capture");
      const int rc = enqueue_batch(bt, bt->gstream);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(bt->gstream, &g);
      if (rc != VFS_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      VFS_TRY_CUDA(e, "end capture");
      e = cudaGraphInstantiate(&bt->gexec, g, 0);
      cudaGraphDestroy(g);
      VFS_TRY_CUDA(e, "graph instantiate");
    }
    VFS_TRY_CUDA(cudaEventRecord(bt->ev_in, s), "event record");
    VFS_TRY_CUDA(cudaStreamWaitEvent(bt->gstream, bt->ev_in, 0), "stream wait");
    VFS_TRY_CUDA(cudaGraphLaunch(bt->gexec, bt->gstream), "graph launch");
    VFS_TRY_CUDA(cudaEventRecord(bt->ev_out, bt->gstream), "event record");
    VFS_TRY_CUDA(cudaStreamWaitEvent(s, bt->ev_out, 0), "stream wait");
  } else {
    VFS_TRY(enqueue_batch(bt, s));
  }
  for (int i = 0; i < bt->n; ++i) {
    VfsPlan* pl = bt->plans[i];
    auto& v0 = pl->lv[0];
    VFS_TRY_CUDA(cudaMemcpy2DAsync(warps_out[i], (size_t)v0.w * 8, pl->warp[0].ptr, pl->warp[0].pitch,
                                   (size_t)v0.w * 8, v0.h, cudaMemcpyDeviceToDevice, s),
                 "flow copy");
    pl->solved = true;
  }
  return VFS_OK;
}

int vfs_batch_triangulate(VfsBatch* bt, int i, float f, float u0, float v0, const float* t, float* xyz_out,
                          void* stream) {
  if (!bt || i < 0 || i >= bt->n) return fail(VFS_ERR_ARG, "pair index out of range");
  return vfs_plan_triangulate(bt->plans[i], f, u0, v0, t, xyz_out, stream);
}

int vfs_batch_triangulate_lsq(VfsBatch* bt, int i, float f, float u0, float v0, const float* t, float* xyz_out,
                              void* stream) {
  if (!bt || i < 0 || i >= bt->n) return fail(VFS_ERR_ARG, "pair index out of range");
  return vfs_plan_triangulate_lsq(bt->plans[i], f, u0, v0, t, xyz_out, stream);
}

int vfs_batch_stats(VfsBatch* bt, VfsSolveStats* out) {
  if (!bt || !out) return fail(VFS_ERR_ARG, "NULL argument");
  memset(out, 0, sizeof(*out));
  out->kernels_per_solve = bt->kernels_per_solve;
  if (!bt->timing) return VFS_OK;
  for (int i = 0; i < bt->tev_used; ++i) {
    float t = 0;
    VFS_TRY_CUDA(cudaEventElapsedTime(&t, bt->tev[2 * i], bt->tev[2 * i + 1]), "event elapsed (synchronise first)");
    out->tgv_ms += t;
    out->tgv_alg_bytes += bt->tev_bytes[i];
    out->tgv_launches += bt->tev_launches[i];
    const int lvl = bt->tev_level[i];
    if (lvl >= 0 && lvl < 16) out->tgv_ms_level[lvl] += t;
  }
  out->tgv_intervals = bt->tev_used;
  return VFS_OK;
}

}  // extern "C"
