// Per-pixel arithmetic of the variational fisheye stereo solver.
//
// Every function here computes, for one pixel, exactly the float32 operations
// of the corresponding reference kernel in Python/vfs.cu (cited per function),
// in the same order and with the same explicit fmaf calls, so that results are
// bit-identical to the reference on the same inputs.  The functions take
// values, not memory, so the one-kernel-per-step entry points and the fused,
// temporally blocked solver share them.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace vfs {

// Mask-code bits for a pixel: its own mask and the mask at its E/W/S/N
// neighbours as the reference reads them (point-sampled, mirror-addressed
// texture at X+-1 / Y+-1, which returns the edge texel outside the image;
// Python/vfs.cu:345, 359, 371, 448-467, 537-553).
enum : uint8_t { kSelf = 1, kE = 2, kW = 4, kS = 8, kN = 16 };
// the code of an unmasked pixel whose four neighbours are unmasked
constexpr uint8_t kAllSides = kSelf | kE | kW | kS | kN;

// Run-time solver constants.  The reference bakes these into the source text
// (Python/vfs.py:57-68); the float members hold the values as the reference's
// `static const float x(LITERAL)` declarations round them, the derived ones
// are evaluated in double first as the reference's constant initialisers are.
struct SolverConsts {
  float alpha0, alpha1, lambda, etaP, etaQ;
  float beta, gamma, minGrad, minTensor;
  float a004, a11;  // 4*alpha0*alpha0 and alpha1*alpha1 (double, then float)
  float fscale, upperLimit;
  // per solver iteration, (alpha1 sigma / etaP, alpha0 sigma / etaQ): the
  // dual step's scales, formed once on the host (device memory; read by the
  // register-owned TGV kernels and the blocked reverse)
  const float2* dscale;
};

// ---------------------------------------------------------------- K7 tensor
// computeEta, Python/vfs.cu:228-237.
__device__ __forceinline__ float3 compute_eta(float a, float b, float c, float a11, float a004) {
  return make_float3(
      fmaf(a11, (fmaf(a, a, b * b) + 2 * c * c), fmaf(a11, fmaf(a + c, a + c, fmaf((b + c), (b + c), 0)), 0)),
      fmaf(a11, fmaf(b, b, c * c), a004),
      fmaf(a11, fmaf(a, a, c * c), a004));
}

// computeTensorEtaMasked_ body after the gradient fetch, Python/vfs.cu:260-275.
__device__ __forceinline__ void tensor_from_grad(float2 grad, const SolverConsts& k, float3* abc, float3* eta) {
  const float normGrad = hypotf(grad.x, grad.y);
  float2 n = make_float2(grad.x / normGrad, grad.y / normGrad);
  if (normGrad < k.minGrad) n = make_float2(1, 0);
  const float2 nT = make_float2(n.y, -n.x);
  const float weight = fmaxf(expf(-k.beta * powf(normGrad, k.gamma)), k.minTensor);
  const float a = weight * n.x * n.x + nT.x * nT.x;
  const float b = weight * n.y * n.y + nT.y * nT.y;
  const float c = weight * n.x * n.y + nT.x * nT.y;
  *abc = make_float3(a, b, c);
  *eta = compute_eta(a, b, c, k.a11, k.a004);
}

// ---------------------------------------------------------------- K10 dual
// updateDualVariables_ for an unmasked pixel, Python/vfs.cu:352-408.
// uc/vc: u_ and v_ at the pixel; uE,vE / uW,vW / uS,vS / uN,vN: at the flat
// neighbours index+-1, index+-width.  `scaleP` = alpha1*sigma/etaP and
// `scaleQ` = alpha0*sigma/etaQ, formed by the caller as the reference does.
__device__ __forceinline__ void dual_px(uint8_t code, float uc, float2 vc, float uE, float2 vE, float uW, float2 vW,
                                        float uS, float2 vS, float uN, float2 vN, float3 abc, float scaleP,
                                        float scaleQ, float2* p, float2* tp, float4* q) {
  float2 gradU = make_float2(0, 0);
  float4 gradV = make_float4(0, 0, 0, 0);
  if (code & kE) {
    gradU.x = uE - uc - vc.x;
    gradV.x = vE.x - vc.x;
    gradV.w = vE.y - vc.y;
  } else {
    gradU.x = uc - uW - vc.x;
    gradV.x = vc.x - vW.x;
    gradV.w = vc.y - vW.y;
  }
  if (code & kS) {
    gradU.y = uS - uc - vc.y;
    gradV.y = vS.y - vc.y;
    gradV.z = vS.x - vc.x;
  } else {
    gradU.y = uc - uN - vc.y;
    gradV.y = vc.y - vN.y;
    gradV.z = vc.x - vN.x;
  }
  const float2 tu = make_float2(fmaf(abc.x, gradU.x, abc.z * gradU.y), fmaf(abc.z, gradU.x, abc.y * gradU.y));
  const float2 up = make_float2(fmaf(scaleP, tu.x, p->x), fmaf(scaleP, tu.y, p->y));
  // Projection onto the unit ball: norm = max(|up|, 1), p = up / norm.  When
  // the L1 norm is <= 0.99 the Euclidean norm (and hypotf's result, accurate
  // to a few ulp) is below 1, so norm is exactly 1 and up / 1 == up: the
  // shortcut skips hypotf and the divisions with bit-identical results.  The
  // same holds when norm comes out exactly 1 (NaNs take the full path).
  float2 pn;
  if (fabsf(up.x) + fabsf(up.y) <= 0.99f) {
    pn = up;
  } else {
    const float norm = fmaxf(hypotf(up.x, up.y), 1.0f);
    pn = (norm == 1.0f && up.x == up.x && up.y == up.y) ? up : make_float2(up.x / norm, up.y / norm);
  }
  *p = pn;
  *tp = make_float2(fmaf(abc.x, pn.x, abc.z * pn.y), fmaf(abc.z, pn.x, abc.y * pn.y));
  const float4 uq = make_float4(fmaf(scaleQ, gradV.x, q->x), fmaf(scaleQ, gradV.y, q->y),
                                fmaf(scaleQ, gradV.z, q->z), fmaf(scaleQ, gradV.w, q->w));
  if (fabsf(uq.x) + fabsf(uq.y) + fabsf(uq.z) + fabsf(uq.w) <= 0.99f) {
    *q = uq;
  } else {
    const float norm = fmaxf(norm4df(uq.x, uq.y, uq.z, uq.w), 1.0f);
    *q = (norm == 1.0f && uq.x == uq.x && uq.y == uq.y && uq.z == uq.z && uq.w == uq.w)
             ? uq
             : make_float4(uq.x / norm, uq.y / norm, uq.z / norm, uq.w / norm);
  }
}

// ---------------------------------------------------------------- K11 threshold
// l1Thresholding_ for an unmasked pixel, Python/vfs.cu:444-494.
__device__ __forceinline__ float threshold_px(uint8_t code, float tau, float2 tpc, float2 tpW, float2 tpN, float u,
                                              float ub, float2 deriv, float etax, float lambda) {
  const float eps = 1E-7f;
  float2 gradTp = make_float2(0, 0);
  const bool e = code & kE, w = code & kW, s = code & kS, n = code & kN;
  if (e && w) gradTp.x = tpc.x - tpW.x;
  else if (!e) gradTp.x = -tpW.x;
  else gradTp.x = tpc.x;
  if (s && n) gradTp.y = tpc.y - tpN.y;
  else if (!s) gradTp.y = -tpN.y;
  else gradTp.y = tpc.y;
  const float dIu = deriv.x, dIz = deriv.y;
  const float tauEtaU = (fabsf(etax) < eps) ? tau : tau / etax;
  const float uTauGtp = ub + tauEtaU * (gradTp.x + gradTp.y);
  const float rho = dIu * (uTauGtp - u) + dIz;
  const float bound = lambda * tauEtaU * dIu * dIu;
  float du = 0.f;
  if ((rho <= bound) && (rho >= -bound)) {
    du = (fabsf(dIu) < eps) ? ((uTauGtp - u)) : ((uTauGtp - u) - rho / dIu);
  } else if (rho < -bound) {
    du = (uTauGtp - u) + lambda * tauEtaU * dIu;
  } else if (rho > bound) {
    du = (uTauGtp - u) - lambda * tauEtaU * dIu;
  }
  return u + du;
}

// ---------------------------------------------------------------- K12 primal
// updatePrimalVariables_ for an unmasked pixel, Python/vfs.cu:533-569.
// un: the thresholded u of this iteration; ub, vb: the previous bar iterates.
__device__ __forceinline__ void primal_px(uint8_t code, float tau, float mu, float2 pc, float4 qc, float4 qW,
                                          float4 qN, float un, float ub, float2 vb, float3 abc, float3 eta,
                                          float alpha0, float alpha1, float* u_out, float2* v_out) {
  const float eps = 1E-7f;
  float4 gradQ = make_float4(0, 0, 0, 0);
  if (code & kE) {
    gradQ.x = qc.x;
    gradQ.w = qc.w;
  }
  if (code & kW) {
    gradQ.x -= qW.x;
    gradQ.w -= qW.w;
  }
  if (code & kS) {
    gradQ.y = qc.y;
    gradQ.z = qc.z;
  }
  if (code & kN) {
    gradQ.y -= qN.y;
    gradQ.z -= qN.z;
  }
  const float2 tu = make_float2(fmaf(abc.x, pc.x, abc.z * pc.y), fmaf(abc.z, pc.x, abc.y * pc.y));
  const float tauEta1 = (fabsf(eta.y) < eps) ? tau : (tau / eta.y);
  const float tauEta2 = (fabsf(eta.z) < eps) ? tau : (tau / eta.z);
  const float2 updatedV = make_float2(fmaf(tauEta1, fmaf(alpha1, tu.x, alpha0 * (gradQ.x + gradQ.z)), vb.x),
                                      fmaf(tauEta2, fmaf(alpha1, tu.y, alpha0 * (gradQ.w + gradQ.y)), vb.y));
  *u_out = fmaf(mu, un - ub, un);
  v_out->x = fmaf(mu, updatedV.x - vb.x, updatedV.x);
  v_out->y = fmaf(mu, updatedV.y - vb.y, updatedV.y);
}

}  // namespace vfs
