// Whole solve without any device allocation, for callers that cannot call
// cudaMalloc: code running where allocation is not allowed or not wanted (a
// real-time loop with a fixed memory budget, a host callback, a foreign-
// language runtime that hands over device pointers but owns no CUDA
// allocator).  vfs_plan_solve needs a workspace from its caller; this entry
// point instead uses a fixed scratch array compiled into the library, so the
// caller passes only inputs and outputs.
//
// The scratch is a file-scope __device__ array of kStaticScratchBytes.  Every
// GPU that loads the library holds it (in every context, until the process
// exits).  Host code cannot use the array's name as a device address, so on
// the first call on each device, with that device current, the entry point
// asks the runtime for the address (cudaGetSymbolAddress) and builds a plan
// over it; later calls with the same parameters reuse that plan, and a call
// with different parameters rebuilds it (texture objects only; no memory is
// allocated or freed).  The first call on a device (and the first after a
// parameter change) also uploads the step-size schedule with a synchronous
// copy, so it must come before any stream capture.
//
// A rebuild blocks the calling thread: it first waits (on an event recorded
// after every call's work) until the previous call's kernels on this device
// have finished, whatever stream they ran on, because they still read the
// old plan's texture objects and the schedule in the scratch.  So calls that
// change the parameters are safe back to back on one stream, or on several.
//
// Every call shares the one array per device: a call overwrites what the
// previous call left there, and everything a solve reads is recomputed or
// cleared by that solve.  Calls with the same parameters whose GPU work
// overlaps (on different streams, or from threads that do not order their
// streams) race on the array; issue them on one stream or order them.
#include <cstring>
#include <mutex>
#include <string>

#include "vfs_api_util.cuh"

namespace {

constexpr size_t kStaticScratchBytes = 32ull << 20;  // 32 MiB per device
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_vfs_static_scratch[kStaticScratchBytes];

struct StaticSlot {
  void* scratch = nullptr;  // device address of g_vfs_static_scratch on this device
  VfsPlan* plan = nullptr;
  VfsParams prm;
  cudaEvent_t done = nullptr;  // recorded after each call's work on its stream
};
StaticSlot g_slots[kMaxDevices];
std::mutex g_mutex;

// Plain == on the doubles: vfs_plan_workspace_size (called first) rejects
// non-finite parameters, so a NaN never reaches here and forces a rebuild.
bool same_params(const VfsParams& a, const VfsParams& b) {
  return a.width == b.width && a.height == b.height && a.beta == b.beta && a.gamma == b.gamma &&
         a.alpha0 == b.alpha0 && a.alpha1 == b.alpha1 && a.timeStepLambda == b.timeStepLambda &&
         a.Lambda == b.Lambda && a.fScale == b.fScale && a.limitRange == b.limitRange && a.nLevel == b.nLevel &&
         a.nWarpIters == b.nWarpIters && a.nSolverIters == b.nSolverIters;
}

}  // namespace

using namespace vfs;

extern "C" {

size_t vfs_static_scratch_bytes(void) { return kStaticScratchBytes; }

int vfs_solve_stereo_static(const VfsParams* prm, const uint8_t* mask, size_t mask_pitch, const float* tvf_hw2,
                            const float* cvf_hw2, const uint8_t* img_ref, const uint8_t* img_other,
                            float* warp_out_hw2, void* stream) {
  if (!prm || !mask || !tvf_hw2 || !cvf_hw2 || !img_ref || !img_other || !warp_out_hw2)
    return fail(VFS_ERR_ARG, "NULL argument");
  size_t need = 0;
  VFS_TRY(vfs_plan_workspace_size(prm, &need));
  if (need > kStaticScratchBytes)
    return fail(VFS_ERR_WORKSPACE, "this size needs " + std::to_string(need) + " bytes of scratch; the static scratch "
                "holds " + std::to_string(kStaticScratchBytes) + " (use vfs_plan_create with a workspace)");
  int dev = 0;
  VFS_TRY_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(VFS_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_mutex);
  StaticSlot& slot = g_slots[dev];
  if (!slot.scratch) {
    void* p = nullptr;
    VFS_TRY_CUDA(cudaGetSymbolAddress(&p, g_vfs_static_scratch), "cudaGetSymbolAddress");
    slot.scratch = p;
  }
  if (!slot.done) VFS_TRY_CUDA(cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming), "event create");
  if (slot.plan && !same_params(slot.prm, *prm)) {
    // the previous call's kernels may still read this plan's textures and
    // the schedule in the scratch: let them finish before both change
    VFS_TRY_CUDA(cudaEventSynchronize(slot.done), "wait for the previous call");
    vfs_plan_destroy(slot.plan);
    slot.plan = nullptr;
  }
  if (!slot.plan) {
    VFS_TRY(vfs_plan_create(prm, slot.scratch, kStaticScratchBytes, &slot.plan));
    slot.prm = *prm;
  }
  VFS_TRY(vfs_plan_set_mask(slot.plan, mask, mask_pitch, stream));
  VFS_TRY(vfs_plan_set_vector_fields(slot.plan, tvf_hw2, cvf_hw2, stream));
  VFS_TRY(vfs_plan_solve(slot.plan, img_ref, img_other, warp_out_hw2, stream));
  VFS_TRY_CUDA(cudaEventRecord(slot.done, (cudaStream_t)stream), "event record");
  return VFS_OK;
}

}  // extern "C"
