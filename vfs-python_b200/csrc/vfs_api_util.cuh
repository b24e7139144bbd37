// Helpers shared by the C-ABI translation units: status codes, the
// per-thread error message, parameter conversion and the step schedule.
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/vfs_b200.h"
#include "vfs_pixel.cuh"

namespace vfs {

void set_error(const std::string& msg);

inline int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}

inline int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return VFS_OK;
  return fail(VFS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define VFS_TRY_CUDA(expr, what)                 \
  do {                                           \
    cudaError_t e_ = (expr);                     \
    if (e_ != cudaSuccess) return cuda_status(e_, what); \
  } while (0)

#define VFS_TRY(expr)              \
  do {                             \
    int rc_ = (expr);              \
    if (rc_ != VFS_OK) return rc_; \
  } while (0)

inline bool valid_params(const VfsParams* p, std::string* why) {
  if (!p) { *why = "params is NULL"; return false; }
  if (p->width <= 0 || p->height <= 0) { *why = "width/height must be positive"; return false; }
  if (p->nLevel <= 0 || p->nLevel > 32) { *why = "nLevel must be in [1, 32]"; return false; }
  if (p->nWarpIters < 0 || p->nSolverIters < 0) { *why = "iteration counts must be >= 0"; return false; }
  if (!(p->fScale > 1.0)) { *why = "fScale must be > 1"; return false; }
  if (!std::isfinite(p->beta) || !std::isfinite(p->gamma) || !std::isfinite(p->alpha0) ||
      !std::isfinite(p->alpha1) || !std::isfinite(p->Lambda) || !std::isfinite(p->timeStepLambda) ||
      !std::isfinite(p->limitRange)) {
    *why = "parameters must be finite";
    return false;
  }
  return true;
}

// Constants as the reference's compile-time substitution produces them
// (Python/vfs.py:52-68 with the `static const float` declarations of
// Python/vfs.cu:230-231, 243-246, 334-337, 429-430).
inline SolverConsts make_consts(const VfsParams* p) {
  SolverConsts k;
  k.alpha0 = (float)p->alpha0;
  k.alpha1 = (float)p->alpha1;
  k.lambda = (float)p->Lambda;
  k.etaP = 3.0f;
  k.etaQ = 2.0f;
  k.beta = (float)p->beta;
  k.gamma = (float)p->gamma;
  k.minGrad = (float)1e-8;
  k.minTensor = (float)1e-8;
  k.a004 = (float)(4 * p->alpha0 * p->alpha0);
  k.a11 = (float)(p->alpha1 * p->alpha1);
  k.fscale = (float)p->fScale;
  k.upperLimit = (float)p->limitRange;
  k.dscale = nullptr;
  return k;
}

// The dual step's scales for each iteration of a (sigma, tau, mu) schedule:
// alpha1 * sigma / etaP and alpha0 * sigma / etaQ, the float32 multiply then
// divide of the dual step (Python/vfs.cu:370-371).  IEEE single-precision
// multiply and divide round the same on the host as on the device, so these
// equal the kernels' own evaluation bit for bit.
inline void dual_scales(const SolverConsts& k, const float* sched3, int n, float* out2) {
  for (int i = 0; i < n; ++i) {
    const float sigma = sched3[3 * i];
    const float a1s = k.alpha1 * sigma, a0s = k.alpha0 * sigma;
    out2[2 * i] = a1s / k.etaP;
    out2[2 * i + 1] = a0s / k.etaQ;
  }
}

// (sigma, tau, mu) for each solver iteration, as the reference's host loop
// computes them (Python/vfs.py:494-515) under NumPy >= 2 scalar rules: the
// first iteration's mu comes from a float64 square root rounded to float32;
// after it sigma and tau are NumPy float32 scalars, so every operation, the
// Python float constants included, is float32.
inline void step_schedule(int n, double time_step_lambda, float* out3) {
  float sigma = 1.0f, tau = 1.0f;
  for (int i = 0; i < n; ++i) {
    float mu;
    if (i == 0) {
      mu = 1.0f / (float)std::sqrt(1.0 + 0.7 * 1.0 * time_step_lambda);
    } else if (sigma < 1000.0f) {
      volatile float t = 0.7f * tau;
      t = t * (float)time_step_lambda;
      volatile float s = 1.0f + t;
      mu = 1.0f / std::sqrt((float)s);
    } else {
      mu = 1.0f;
    }
    out3[3 * i + 0] = sigma;
    out3[3 * i + 1] = tau;
    out3[3 * i + 2] = mu;
    volatile float ns = sigma / mu;
    volatile float nt = tau * mu;
    sigma = ns;
    tau = nt;
  }
}

}  // namespace vfs
