// Reverse mode of the coarse-to-fine stereo solve.  The reference is forward
// only; this has no counterpart there.
//
// vfs_grad_forward runs a plan's solve (Python/vfs.py:460-533) on float
// images and a translation t, then the depth map of triangulate_flow
// (Python/vfs.py:535-559), recording a tape: per warp the flow, u and u_ at
// its start, and the solver state at the end of every `ckpt`-iteration
// interval (with ckpt 1, every state, written by the recording form of the
// blocked TGV kernel).  vfs_grad_backward takes the cotangent of the depth
// map and returns the cotangents of both images, of t and of theta =
// (Lambda, alpha0, alpha1, beta, gamma).
//
// Backward schedule, per level from fine to coarse and per warp from last to
// first: recompute the warp's constants and tvec from the tape, reverse the
// median/clamp, then for each checkpoint interval from last to first
// recompute the states between its ends (recording kernel) and reverse its
// iterations.  An iteration reverses in three phases: primal and threshold
// adjoints (pixel-local), the dual adjoint (gathers phase-1 values at the E
// and S flat neighbours), the transposed gradients of u_ and v_ (gathers
// phase-2 values at the four flat neighbours).  The default form,
// k_rev_block, runs them for 2-4 iterations per launch on shared-memory
// tiles; k_rev_tile (one iteration per launch) and k_rev1/2/3 (one kernel
// per phase) are the simpler forms, kept selectable and tested against it.
// The outer stages have one kernel each; transposed texture fetches scatter
// with float atomics.  Scalar cotangents are block-reduced and added to a
// device double[8] (t0 t1 t2 Lambda alpha0 alpha1 beta gamma).
//
// Rules at the non-smooth points: a texture fetch differentiates exact
// bilinear interpolation at the fetch coordinate (the hardware's 8-bit
// weights are passed straight through); the median routes its cotangent to
// the tap the exchange network selected; min(., limitRange) routes to its
// first argument unless the limit is taken; the L1 shrink and the unit-ball
// projections take the branch the forward took.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "vfs_camera.cuh"
#include "vfs_plan_impl.cuh"
#include "vfs_sample.cuh"

namespace vfs {
namespace {

constexpr int kGX = 32, kGY = 8;
inline dim3 g2d(int h, int w) { return dim3((w + kGX - 1) / kGX, (h + kGY - 1) / kGY); }
const dim3 kGB(kGX, kGY);

enum { G_T0 = 0, G_T1, G_T2, G_LAMBDA, G_ALPHA0, G_ALPHA1, G_BETA, G_GAMMA, G_NSCAL };

#define GRAD_PIXEL                                     \
  const int X = blockIdx.x * blockDim.x + threadIdx.x; \
  const int Y = blockIdx.y * blockDim.y + threadIdx.y; \
  const bool inside = X < w && Y < h;                  \
  const long i = (long)Y * w + X;

__device__ __forceinline__ int mirror_ix(int i, int n) {
  const int m = 2 * n;
  i %= m;
  if (i < 0) i += m;
  return i >= n ? m - 1 - i : i;
}

template <typename T>
__device__ __forceinline__ T ld0(const T* a, long i, long n) {
  return (i >= 0 && i < n) ? a[i] : T(0);
}

// A cotangent contribution that is not finite is dropped.  The forward can
// leave a few pixels with NaN state (beside an epipole, the epipolar
// direction is undefined; the reference's kernels give the same NaNs); a
// NaN state times a finite (even zero) cotangent is NaN, and the stencil
// would carry it to every cotangent within a few iterations.  Such pixels
// are treated as passing no gradient: every cotangent a reverse kernel
// writes, and every scalar it accumulates, goes through fin0.
__device__ __forceinline__ float fin0(float x) { return isfinite(x) ? x : 0.f; }

// Sum of N per-thread values over the block (at most 1024 threads), added to
// out[0..N).  Every thread of the block must call it.
template <int N>
__device__ __forceinline__ void block_sum_to(const float (&v)[N], double* out) {
  __shared__ float red[N][32];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    float s = fin0(v[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[k][wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x * blockDim.y) >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      float s = lane < nw ? red[k][lane] : 0.f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0 && s != 0.f) atomicAdd(out + k, (double)s);
    }
  }
}

// ---------------------------------------------------------------- transposed fetches
// A linear, mirror-addressed fetch at texel coordinate (u, v) (normalised
// coordinate * size - 0.5): its four texels and exact weights.
struct Bilin {
  int i0, i1, j0, j1;
  float a, b;
  bool ok;
};

// Mirror addressing has period 2n, so the texel of any finite coordinate is
// found from floor(u) mod 2n (exact in float for integer values).  A
// non-finite coordinate gets zero weights: no cotangent and no derivative.
__device__ __forceinline__ void mirror_pair(float u, int n, int* i0, int* i1, float* frac) {
  const float fu = floorf(u);
  *frac = u - fu;
  float r = fmodf(fu, 2.f * n);
  if (r < 0.f) r += 2.f * n;
  const int iu = min((int)r, 2 * n - 1);
  *i0 = mirror_ix(iu, n);
  *i1 = mirror_ix(iu + 1, n);
}

__device__ __forceinline__ Bilin bilin(float u, float v, int h, int w) {
  Bilin r;
  if (!isfinite(u) || !isfinite(v)) {
    r.i0 = r.i1 = r.j0 = r.j1 = 0;
    r.a = r.b = 0.f;
    r.ok = false;
    return r;
  }
  mirror_pair(u, w, &r.i0, &r.i1, &r.a);
  mirror_pair(v, h, &r.j0, &r.j1, &r.b);
  r.ok = true;
  return r;
}

__device__ __forceinline__ void scatter1(float* g, int w, const Bilin& B, float val) {
  if (val == 0.f || !B.ok) return;
  atomicAdd(g + (long)B.j0 * w + B.i0, (1.f - B.a) * (1.f - B.b) * val);
  atomicAdd(g + (long)B.j0 * w + B.i1, B.a * (1.f - B.b) * val);
  atomicAdd(g + (long)B.j1 * w + B.i0, (1.f - B.a) * B.b * val);
  atomicAdd(g + (long)B.j1 * w + B.i1, B.a * B.b * val);
}

__device__ __forceinline__ void scatter2(float2* g, int w, const Bilin& B, float2 val) {
  if (!B.ok) return;
  float* f = reinterpret_cast<float*>(g);
  const float wt[4] = {(1.f - B.a) * (1.f - B.b), B.a * (1.f - B.b), (1.f - B.a) * B.b, B.a * B.b};
  const long ix[4] = {(long)B.j0 * w + B.i0, (long)B.j0 * w + B.i1, (long)B.j1 * w + B.i0, (long)B.j1 * w + B.i1};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (val.x != 0.f) atomicAdd(f + 2 * ix[k], wt[k] * val.x);
    if (val.y != 0.f) atomicAdd(f + 2 * ix[k] + 1, wt[k] * val.y);
  }
}

// d(fetch)/du, d(fetch)/dv of a one-channel plane.
__device__ __forceinline__ float2 bilin_d1(Plane<const float> T, const Bilin& B) {
  if (!B.ok) return make_float2(0.f, 0.f);
  const float t00 = T.at(B.i0, B.j0), t01 = T.at(B.i1, B.j0), t10 = T.at(B.i0, B.j1), t11 = T.at(B.i1, B.j1);
  return make_float2((1.f - B.b) * (t01 - t00) + B.b * (t11 - t10), (1.f - B.a) * (t10 - t00) + B.a * (t11 - t01));
}

// g . d(fetch)/du, g . d(fetch)/dv of a two-channel plane.
__device__ __forceinline__ float2 bilin_d2(Plane<const float2> T, const Bilin& B, float2 g) {
  if (!B.ok) return make_float2(0.f, 0.f);
  const float2 t00 = T.at(B.i0, B.j0), t01 = T.at(B.i1, B.j0), t10 = T.at(B.i0, B.j1), t11 = T.at(B.i1, B.j1);
  const float dux = (1.f - B.b) * (t01.x - t00.x) + B.b * (t11.x - t10.x);
  const float duy = (1.f - B.b) * (t01.y - t00.y) + B.b * (t11.y - t10.y);
  const float dvx = (1.f - B.a) * (t10.x - t00.x) + B.a * (t11.x - t01.x);
  const float dvy = (1.f - B.a) * (t10.y - t00.y) + B.a * (t11.y - t01.y);
  return make_float2(g.x * dux + g.y * duy, g.x * dvx + g.y * dvy);
}

// ---------------------------------------------------------------- forward helpers
__global__ void k_g_to_plane(Plane<float> out, const float* __restrict__ in, float s, int h, int w) {
  GRAD_PIXEL
  if (inside) out.at(X, Y) = in[i] * s;
}

__global__ void k_g_scale(float* out, const float* __restrict__ in, float s, int h, int w) {
  GRAD_PIXEL
  if (inside) out[i] = in[i] * s;
}

// z of triangulate_flow's xyz (Python/vfs.py:535-559, Python/vfs.cu:707-745;
// LSQ: the least-squares rule, triangulate_lsq_px).
template <bool LSQ>
__global__ void k_g_depth(float* depth, Plane<const float2> warp, Cam cam, float tx, float ty, float tz,
                          Plane<const uint8_t> mask, int h, int w) {
  GRAD_PIXEL
  if (!inside) return;
  if (mask.at(X, Y) == 0) {
    depth[i] = -1.f;
    return;
  }
  const float2 d = warp.at(X, Y);
  const float3 rr = cam_unproject(cam, make_float2((float)X, (float)Y));
  const float3 ro = cam_unproject(cam, make_float2((float)X + d.x, (float)Y + d.y));
  depth[i] = LSQ ? triangulate_lsq_px(rr, ro, tx, ty, tz).z : triangulate_px(rr, ro, tx, tz).z;
}

// ---------------------------------------------------------------- triangulation
// d depth / d flow and d depth / d (t0, t2).  xo = x tan(rho/f) / rho is the
// x/z of the unprojected ray at (X, Y) + flow, relative to the principal point.
__global__ void k_g_tri(const float* __restrict__ gdepth, Plane<const float2> warp, Cam cam, float tx, float tz,
                        Plane<const uint8_t> mask, float2* gwarp, double* scal, int h, int w) {
  GRAD_PIXEL
  float acc[3] = {0.f, 0.f, 0.f};
  if (inside) {
    float2 gw = make_float2(0.f, 0.f);
    const float g = gdepth[i];
    if (mask.at(X, Y) != 0 && g != 0.f) {
      const float2 d = warp.at(X, Y);
      const float3 rr = cam_unproject(cam, make_float2((float)X, (float)Y));
      const float xr = rr.x / rr.z;
      const float2 uv = make_float2((float)X + d.x, (float)Y + d.y);
      const float3 ro = cam_unproject(cam, uv);
      const float xo = ro.x / ro.z;
      const float x = uv.x - cam.u0, y = uv.y - cam.v0;
      const float rho = hypotf(x, y);
      const float th = rho / cam.f;
      float G, Gpr;  // tan(th)/rho and (d/drho of it)/rho
      if (th < 0.05f) {
        const float t2 = th * th;
        G = (1.f + t2 * (1.f / 3.f + t2 * (2.f / 15.f))) / cam.f;
        Gpr = (2.f / 3.f + t2 * (8.f / 15.f + t2 * (102.f / 315.f))) / (cam.f * cam.f * cam.f);
      } else {
        const float tn = tanf(th), c = cosf(th);
        G = tn / rho;
        Gpr = (rho / (cam.f * c * c) - tn) / (rho * rho * rho);
      }
      const float D = xo - xr;
      const float gx = g * (tz * xr - tx) / (D * D);
      gw = make_float2(gx * fmaf(x * x, Gpr, G), gx * x * y * Gpr);
      acc[0] = g / D;
      acc[2] = -g * xo / D;
    }
    gwarp[i] = gw;
  }
  block_sum_to<3>(acc, scal + G_T0);
}

// d depth / d flow and d depth / d t for the least-squares rule:
// depth = lambda r_z, lambda = (m . n) / (n . n), n = r x o, m = (-t) x o,
// o = unproject((X, Y) + flow).  With x, y relative to the principal point,
// rho = |(x, y)|, theta = rho / f, S = sin(theta) / rho, o = (S x, S y,
// cos theta) and d o / d(x, y) = [[S + x^2 S', x y S'], [x y S', S + y^2 S'],
// [-S x / f, -S y / f]] with S' = (dS/drho) / rho (series below theta 0.05).
__global__ void k_g_tri_lsq(const float* __restrict__ gdepth, Plane<const float2> warp, Cam cam, float tx, float ty,
                            float tz, Plane<const uint8_t> mask, float2* gwarp, double* scal, int h, int w) {
  GRAD_PIXEL
  float acc[3] = {0.f, 0.f, 0.f};
  if (inside) {
    float2 gw = make_float2(0.f, 0.f);
    const float g = gdepth[i];
    if (mask.at(X, Y) != 0 && g != 0.f) {
      const float2 d = warp.at(X, Y);
      const float3 rr = cam_unproject(cam, make_float2((float)X, (float)Y));
      const float2 uv = make_float2((float)X + d.x, (float)Y + d.y);
      const float3 ro = cam_unproject(cam, uv);
      const float3 mt = make_float3(-tx, -ty, -tz);
      const float3 n = cross3(rr, ro), m = cross3(mt, ro);
      const float inn = 1.f / dot3(n, n);
      const float lam = dot3(m, n) * inn;
      const float gl = g * rr.z * inn;
      const float3 gm = make_float3(gl * n.x, gl * n.y, gl * n.z);
      const float3 gn = make_float3(gl * (m.x - 2.f * lam * n.x), gl * (m.y - 2.f * lam * n.y),
                                    gl * (m.z - 2.f * lam * n.z));
      const float3 gt = cross3(gm, ro);  // -(o x gm)
      const float3 a = cross3(gm, mt), b = cross3(gn, rr);
      const float3 go = make_float3(a.x + b.x, a.y + b.y, a.z + b.z);
      const float x = uv.x - cam.u0, y = uv.y - cam.v0;
      const float rho = hypotf(x, y);
      const float th = rho / cam.f;
      float S, Sp;
      if (th < 0.05f) {
        const float t2 = th * th;
        S = (1.f - t2 * (1.f / 6.f - t2 * (1.f / 120.f))) / cam.f;
        Sp = (-1.f / 3.f + t2 * (1.f / 30.f - t2 * (1.f / 840.f))) / (cam.f * cam.f * cam.f);
      } else {
        float sn, cs;
        sincosf(th, &sn, &cs);
        S = sn / rho;
        Sp = (rho * cs / cam.f - sn) / (rho * rho * rho);
      }
      const float jxy = x * y * Sp;
      gw.x = go.x * fmaf(x * x, Sp, S) + go.y * jxy - go.z * S * x / cam.f;
      gw.y = go.x * jxy + go.y * fmaf(y * y, Sp, S) - go.z * S * y / cam.f;
      acc[0] = gt.x;
      acc[1] = gt.y;
      acc[2] = gt.z;
    }
    gwarp[i] = gw;
  }
  block_sum_to<3>(acc, scal + G_T0);
}

// ---------------------------------------------------------------- median / clamp
// medianFilter + computeOpticalFlowWithClamp (Python/vfs.cu:583-676) reversed:
// gu is the cotangent of u_before after the update on entry and before it on
// exit; the median's share goes to the selected tap of uT (atomically into
// guT); gtvec is the cotangent of tvec.  The exchange network is the
// forward's, carrying tap indices.
__global__ void k_g_post(float2* __restrict__ gwarp, float* __restrict__ gu, float* guT, const float* __restrict__ uT,
                         const float* __restrict__ u_in, const float2* __restrict__ tvec, Plane<const uint8_t> mask,
                         float limit, float2* __restrict__ gtvec, int h, int w) {
  GRAD_PIXEL
  if (!inside) return;
  if (!mask_at(mask, X, Y, h, w)) {
    gtvec[i] = make_float2(0.f, 0.f);
    return;
  }
  float v[25];
  int ix[25];
#pragma unroll
  for (int j = 0; j < 5; j++) {
    const int yy = min(max(Y + j - 2, 0), h - 1);
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const int xx = min(max(X + k - 2, 0), w - 1);
      v[j * 5 + k] = uT[(long)yy * w + xx];
      ix[j * 5 + k] = yy * w + xx;
    }
  }
#pragma unroll
  for (int j = 0; j < 13; j++) {
#pragma unroll
    for (int k = j + 1; k < 25; k++) {
      const float a = v[j], b = v[k];
      const int ia = ix[j], ib = ix[k];
      const bool sw = a > b;
      v[j] = sw ? b : a;
      v[k] = sw ? a : b;
      ix[j] = sw ? ib : ia;
      ix[k] = sw ? ia : ib;
    }
  }
  const float raw = v[12] - u_in[i];
  const float delta = fminf(raw, limit);
  const float2 gw = gwarp[i];
  const float2 tv = tvec[i];
  const float gd = fin0(gu[i] + gw.x * tv.x + gw.y * tv.y);
  gtvec[i] = make_float2(fin0(delta * gw.x), fin0(delta * gw.y));
  if (raw < limit) {
    gu[i] -= gd;
    atomicAdd(guT + ix[12], gd);
  }
}

// ---------------------------------------------------------------- TGV iteration reversed
struct RevArgs {
  TgvState s0, s1;  // state before / after the iteration
  TgvState g1, g0;  // cotangent of s1 (in) / of s0 (out)
  TgvConsts c;
  float* gc[8];  // cotangents of a b c ex ey ez iu iz (accumulated)
  float* A[3];   // k_rev1 -> k_rev2: t1*alpha0*gVx, t2*alpha0*gVy, te*g(ut)
  float* C[6];   // k_rev2 -> k_rev3: cotangents of gradU (2) and gradV (4)
  float sigma, tau, mu;
  SolverConsts k;
  int h, w;
  double* scal;
};

// Primal (updatePrimalVariables, Python/vfs.cu:507-581) and threshold
// (l1Thresholding, Python/vfs.cu:421-505) reversed at one pixel.  Writes the
// final cotangent of u, the pixel-local parts of those of u_ and v_, and the
// values k_rev2 gathers.
__global__ void __launch_bounds__(kGX* kGY) k_rev1(RevArgs r) {
  const int w = r.w, h = r.h;
  GRAD_PIXEL
  const long n = (long)h * w;
  float acc[3] = {0.f, 0.f, 0.f};  // Lambda, alpha0, alpha1
  if (inside) {
    const uint8_t c = r.c.code[i];
    float gu = 0.f, gubl = 0.f, gvx = 0.f, gvy = 0.f, Ax = 0.f, Ay = 0.f, Bv = 0.f;
    if (c & kSelf) {
      const float eps = 1E-7f;
      const float mu = r.mu, tau = r.tau, al0 = r.k.alpha0, al1 = r.k.alpha1, lam = r.k.lambda;
      const float gubn = r.g1.ub[i];
      const float gvbx = r.g1.vbx[i], gvby = r.g1.vby[i];
      const float gun = r.g1.u[i] + (1.f + mu) * gubn;
      const float gVx = (1.f + mu) * gvbx, gVy = (1.f + mu) * gvby;
      const float a = r.c.a[i], b = r.c.b[i], cc = r.c.c[i];
      // primal: divergence of q (after the iteration) with the mask rules
      const float gQx = ((c & kE) ? r.s1.qx[i] : 0.f) - ((c & kW) ? ld0(r.s1.qx, i - 1, n) : 0.f);
      const float gQw = ((c & kE) ? r.s1.qw[i] : 0.f) - ((c & kW) ? ld0(r.s1.qw, i - 1, n) : 0.f);
      const float gQy = ((c & kS) ? r.s1.qy[i] : 0.f) - ((c & kN) ? ld0(r.s1.qy, i - w, n) : 0.f);
      const float gQz = ((c & kS) ? r.s1.qz[i] : 0.f) - ((c & kN) ? ld0(r.s1.qz, i - w, n) : 0.f);
      const float px = r.s1.px[i], py = r.s1.py[i];
      const float tpx = fmaf(a, px, cc * py), tpy = fmaf(cc, px, b * py);
      const float ex = r.c.ex[i], ey = r.c.ey[i], ez = r.c.ez[i];
      const bool sx = fabsf(ex) < eps, sy = fabsf(ey) < eps, sz = fabsf(ez) < eps;
      const float t1 = sy ? tau : tau / ey, t2 = sz ? tau : tau / ez;
      const float inx = fmaf(al1, tpx, al0 * (gQx + gQz));
      const float iny = fmaf(al1, tpy, al0 * (gQw + gQy));
      const float gey = sy ? 0.f : -t1 / ey * inx * gVx;
      const float gez = sz ? 0.f : -t2 / ez * iny * gVy;
      acc[2] += t1 * tpx * gVx + t2 * tpy * gVy;
      acc[1] += t1 * (gQx + gQz) * gVx + t2 * (gQw + gQy) * gVy;
      Ax = t1 * al0 * gVx;
      Ay = t2 * al0 * gVy;
      // threshold: divergence of tp = T^(1/2) p with the mask rules
      const float tpWx = fmaf(ld0(r.c.a, i - 1, n), ld0(r.s1.px, i - 1, n), ld0(r.c.c, i - 1, n) * ld0(r.s1.py, i - 1, n));
      const float tpNy = fmaf(ld0(r.c.c, i - w, n), ld0(r.s1.px, i - w, n), ld0(r.c.b, i - w, n) * ld0(r.s1.py, i - w, n));
      const bool e = c & kE, wv = c & kW, s = c & kS, nn = c & kN;
      const float gTx = (e && wv) ? tpx - tpWx : (!e ? -tpWx : tpx);
      const float gTy = (s && nn) ? tpy - tpNy : (!s ? -tpNy : tpy);
      const float Iu = r.c.iu[i], Iz = r.c.iz[i];
      const float te = sx ? tau : tau / ex;
      const float u = r.s0.u[i], ub = r.s0.ub[i];
      const float ut = ub + te * (gTx + gTy);
      const float rho = Iu * (ut - u) + Iz;
      const float Bd = lam * te * Iu * Iu;
      float gut = 0.f, gte = 0.f, giu = 0.f, giz = 0.f;
      if ((rho <= Bd) && (rho >= -Bd)) {
        if (fabsf(Iu) >= eps) {  // u + du = u - Iz / Iu
          gu += gun;
          giz = -gun / Iu;
          giu = gun * Iz / (Iu * Iu);
        } else {
          gut = gun;
        }
      } else if (rho < -Bd) {
        gut = gun;
        acc[0] += te * Iu * gun;
        gte = lam * Iu * gun;
        giu = lam * te * gun;
      } else if (rho > Bd) {
        gut = gun;
        acc[0] -= te * Iu * gun;
        gte = -lam * Iu * gun;
        giu = -lam * te * gun;
      } else {
        gu += gun;
      }
      gte += (gTx + gTy) * gut;
      Bv = te * gut;
      const float gex = sx ? 0.f : -te / ex * gte;
      gubl = -mu * gubn + gut;
      gvx = gVx - mu * gvbx;
      gvy = gVy - mu * gvby;
      r.gc[3][i] += fin0(gex);
      r.gc[4][i] += fin0(gey);
      r.gc[5][i] += fin0(gez);
      r.gc[6][i] += fin0(giu);
      r.gc[7][i] += fin0(giz);
    }
    r.g0.u[i] = fin0(gu);
    r.g0.ub[i] = fin0(gubl);
    r.g0.vbx[i] = fin0(gvx);
    r.g0.vby[i] = fin0(gvy);
    r.A[0][i] = Ax;
    r.A[1][i] = Ay;
    r.A[2][i] = Bv;
  }
  block_sum_to<3>(acc, r.scal + G_LAMBDA);
}

// Dual update (updateDualVariables, Python/vfs.cu:326-419) reversed at one
// pixel: gathers k_rev1's values from the pixel and its flat E and S
// neighbours (the transposes of the W/N reads of the threshold and primal
// divergences), back-projects through the unit-ball projections, writes the
// final cotangents of p and q and the cotangents of gradU/gradV for k_rev3.
__global__ void __launch_bounds__(kGX* kGY) k_rev2(RevArgs r) {
  const int w = r.w, h = r.h;
  GRAD_PIXEL
  const long n = (long)h * w;
  float acc[2] = {0.f, 0.f};  // alpha0, alpha1
  if (inside) {
    const uint8_t c = r.c.code[i];
    float gP0 = 0.f, gP1 = 0.f, gQ[4] = {0.f, 0.f, 0.f, 0.f}, Cv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (c & kSelf) {
      const float eps = 1E-7f;
      const float mu = r.mu, tau = r.tau, sigma = r.sigma, al0 = r.k.alpha0, al1 = r.k.alpha1;
      const float Ax = r.A[0][i], Ay = r.A[1][i], Bv = r.A[2][i];
      const bool hasE = i + 1 < n, hasS = i + w < n;
      const uint8_t cE = hasE ? r.c.code[i + 1] : 0, cS = hasS ? r.c.code[i + w] : 0;
      const float AxE = hasE ? r.A[0][i + 1] : 0.f, AyE = hasE ? r.A[1][i + 1] : 0.f, BE = hasE ? r.A[2][i + 1] : 0.f;
      const float AxS = hasS ? r.A[0][i + w] : 0.f, AyS = hasS ? r.A[1][i + w] : 0.f, BS = hasS ? r.A[2][i + w] : 0.f;
      const float gVx = (1.f + mu) * r.g1.vbx[i], gVy = (1.f + mu) * r.g1.vby[i];
      const float ey = r.c.ey[i], ez = r.c.ez[i];
      const float t1 = fabsf(ey) < eps ? tau : tau / ey, t2 = fabsf(ez) < eps ? tau : tau / ez;
      const float gtpx = t1 * al1 * gVx + ((c & kE) ? Bv : 0.f) - (((cE & kW) || !(cE & kE)) ? BE : 0.f);
      const float gtpy = t2 * al1 * gVy + ((c & kS) ? Bv : 0.f) - (((cS & kN) || !(cS & kS)) ? BS : 0.f);
      float gq0 = r.g1.qx[i] + ((c & kE) ? Ax : 0.f) - ((cE & kW) ? AxE : 0.f);
      float gq3 = r.g1.qw[i] + ((c & kE) ? Ay : 0.f) - ((cE & kW) ? AyE : 0.f);
      float gq1 = r.g1.qy[i] + ((c & kS) ? Ay : 0.f) - ((cS & kN) ? AyS : 0.f);
      float gq2 = r.g1.qz[i] + ((c & kS) ? Ax : 0.f) - ((cS & kN) ? AxS : 0.f);
      const float a = r.c.a[i], b = r.c.b[i], cc = r.c.c[i];
      const float pnx = r.s1.px[i], pny = r.s1.py[i];
      const float gpx = r.g1.px[i] + fmaf(a, gtpx, cc * gtpy);
      const float gpy = r.g1.py[i] + fmaf(cc, gtpx, b * gtpy);
      float ga = pnx * gtpx, gb = pny * gtpy, gcc = pny * gtpx + pnx * gtpy;
      // the dual step's inputs, as dual_px forms them
      const float uc = r.s0.ub[i];
      const float2 vc = make_float2(r.s0.vbx[i], r.s0.vby[i]);
      float gUx, gUy, gVxx, gVyy, gVz, gVw;
      if (c & kE) {
        gUx = ld0(r.s0.ub, i + 1, n) - uc - vc.x;
        gVxx = ld0(r.s0.vbx, i + 1, n) - vc.x;
        gVw = ld0(r.s0.vby, i + 1, n) - vc.y;
      } else {
        gUx = uc - ld0(r.s0.ub, i - 1, n) - vc.x;
        gVxx = vc.x - ld0(r.s0.vbx, i - 1, n);
        gVw = vc.y - ld0(r.s0.vby, i - 1, n);
      }
      if (c & kS) {
        gUy = ld0(r.s0.ub, i + w, n) - uc - vc.y;
        gVyy = ld0(r.s0.vby, i + w, n) - vc.y;
        gVz = ld0(r.s0.vbx, i + w, n) - vc.x;
      } else {
        gUy = uc - ld0(r.s0.ub, i - w, n) - vc.y;
        gVyy = vc.y - ld0(r.s0.vby, i - w, n);
        gVz = vc.x - ld0(r.s0.vbx, i - w, n);
      }
      const float scaleP = al1 * sigma / r.k.etaP;
      const float scaleQ = al0 * sigma / r.k.etaQ;
      const float tux = fmaf(a, gUx, cc * gUy), tuy = fmaf(cc, gUx, b * gUy);
      const float upx = fmaf(scaleP, tux, r.s0.px[i]), upy = fmaf(scaleP, tuy, r.s0.py[i]);
      const float nP = hypotf(upx, upy);
      if (nP > 1.f) {
        const float dt = pnx * gpx + pny * gpy;
        gP0 = (gpx - pnx * dt) / nP;
        gP1 = (gpy - pny * dt) / nP;
      } else {
        gP0 = gpx;
        gP1 = gpy;
      }
      const float uq0 = fmaf(scaleQ, gVxx, r.s0.qx[i]), uq1 = fmaf(scaleQ, gVyy, r.s0.qy[i]);
      const float uq2 = fmaf(scaleQ, gVz, r.s0.qz[i]), uq3 = fmaf(scaleQ, gVw, r.s0.qw[i]);
      const float nQ = norm4df(uq0, uq1, uq2, uq3);
      if (nQ > 1.f) {
        const float q0 = r.s1.qx[i], q1 = r.s1.qy[i], q2 = r.s1.qz[i], q3 = r.s1.qw[i];
        const float dt = q0 * gq0 + q1 * gq1 + q2 * gq2 + q3 * gq3;
        gq0 = (gq0 - q0 * dt) / nQ;
        gq1 = (gq1 - q1 * dt) / nQ;
        gq2 = (gq2 - q2 * dt) / nQ;
        gq3 = (gq3 - q3 * dt) / nQ;
      }
      gQ[0] = gq0;
      gQ[1] = gq1;
      gQ[2] = gq2;
      gQ[3] = gq3;
      acc[0] += sigma / r.k.etaQ * (gVxx * gq0 + gVyy * gq1 + gVz * gq2 + gVw * gq3);
      acc[1] += sigma / r.k.etaP * (tux * gP0 + tuy * gP1);
      const float gtux = scaleP * gP0, gtuy = scaleP * gP1;
      ga += gUx * gtux;
      gb += gUy * gtuy;
      gcc += gUy * gtux + gUx * gtuy;
      Cv[0] = fmaf(a, gtux, cc * gtuy);
      Cv[1] = fmaf(cc, gtux, b * gtuy);
      Cv[2] = scaleQ * gq0;
      Cv[3] = scaleQ * gq1;
      Cv[4] = scaleQ * gq2;
      Cv[5] = scaleQ * gq3;
      r.gc[0][i] += fin0(ga);
      r.gc[1][i] += fin0(gb);
      r.gc[2][i] += fin0(gcc);
    }
    r.g0.px[i] = fin0(gP0);
    r.g0.py[i] = fin0(gP1);
    r.g0.qx[i] = fin0(gQ[0]);
    r.g0.qy[i] = fin0(gQ[1]);
    r.g0.qz[i] = fin0(gQ[2]);
    r.g0.qw[i] = fin0(gQ[3]);
#pragma unroll
    for (int k = 0; k < 6; ++k) r.C[k][i] = Cv[k];
  }
  block_sum_to<2>(acc, r.scal + G_ALPHA0);
}

// Transposed gradients of u_ and v_ (the dual step's forward/backward
// differences with the mask rules): gathers k_rev2's values from the pixel
// and its four flat neighbours.
__global__ void __launch_bounds__(kGX* kGY) k_rev3(RevArgs r) {
  const int w = r.w, h = r.h;
  GRAD_PIXEL
  if (!inside) return;
  const long n = (long)h * w;
  const uint8_t c = r.c.code[i];
  float gub = r.g0.ub[i], gvx = r.g0.vbx[i], gvy = r.g0.vby[i];
  if (c & kSelf) {
    const float u0 = r.C[0][i], u1 = r.C[1][i];
    const float v0 = r.C[2][i], v1 = r.C[3][i], v2 = r.C[4][i], v3 = r.C[5][i];
    gub += ((c & kE) ? -u0 : u0) + ((c & kS) ? -u1 : u1);
    gvx += -u0 + ((c & kE) ? -v0 : v0) + ((c & kS) ? -v2 : v2);
    gvy += -u1 + ((c & kE) ? -v3 : v3) + ((c & kS) ? -v1 : v1);
  }
  if (i - 1 >= 0 && (r.c.code[i - 1] & kE)) {
    gub += r.C[0][i - 1];
    gvx += r.C[2][i - 1];
    gvy += r.C[5][i - 1];
  }
  if (i + 1 < n && !(r.c.code[i + 1] & kE)) {
    gub -= r.C[0][i + 1];
    gvx -= r.C[2][i + 1];
    gvy -= r.C[5][i + 1];
  }
  if (i - w >= 0 && (r.c.code[i - w] & kS)) {
    gub += r.C[1][i - w];
    gvx += r.C[4][i - w];
    gvy += r.C[3][i - w];
  }
  if (i + w < n && !(r.c.code[i + w] & kS)) {
    gub -= r.C[1][i + w];
    gvx -= r.C[4][i + w];
    gvy -= r.C[3][i + w];
  }
  r.g0.ub[i] = fin0(gub);
  r.g0.vbx[i] = fin0(gvx);
  r.g0.vby[i] = fin0(gvy);
}

// The three phases above in one kernel over a TX x TY tile.  The window is
// the tile plus 2 pixels on every side in flat addressing (window pixel
// (wx, wy) is flat index (y0-2+wy)*w + (x0-2+wx), so window neighbours are the
// flat neighbours, row wrap included).  Phase 1 runs on the window minus its
// first row and column, phase 2 on the tile plus 1 pixel, phase 3 on the
// tile; the values passed between phases stay in shared memory.
enum RevPlane { qUB, qVX, qVY, qPX, qPY, qQX, qQY, qQZ, qQW, qA, qB, qC, aX, aY, aB, c0, c1, c2, c3, c4, c5, lUB, lVX,
                lVY, kRevPlanes };

template <int TX, int TY>
struct RevGeom {
  static constexpr int WX = TX + 4, WY = TY + 4, N = WX * WY;
  static constexpr size_t smem_bytes() { return (size_t)kRevPlanes * N * sizeof(float) + ((N + 15) / 16) * 16; }
};

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) k_rev_tile(RevArgs r) {
  using G = RevGeom<TX, TY>;
  constexpr int WX = G::WX, WY = G::WY, N = G::N;
  extern __shared__ float4 smem_raw[];
  float* const sm = reinterpret_cast<float*>(smem_raw);
  uint8_t* const scode = reinterpret_cast<uint8_t*>(sm + (size_t)kRevPlanes * N);
  auto P = [&](int plane) { return sm + (size_t)plane * N; };
  const int w = r.w, h = r.h;
  const long n = (long)h * w;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const long base = (long)(y0 - 2) * w + (x0 - 2);
  const float eps = 1E-7f;
  const float mu = r.mu, tau = r.tau, sigma = r.sigma, al0 = r.k.alpha0, al1 = r.k.alpha1, lam = r.k.lambda;
  const float* __restrict__ const S0U = r.s0.u;
  const float* __restrict__ const S0UB = r.s0.ub;
  const float* __restrict__ const S0VX = r.s0.vbx;
  const float* __restrict__ const S0VY = r.s0.vby;
  const float* __restrict__ const S0PX = r.s0.px;
  const float* __restrict__ const S0PY = r.s0.py;
  const float* __restrict__ const S0QX = r.s0.qx;
  const float* __restrict__ const S0QY = r.s0.qy;
  const float* __restrict__ const S0QZ = r.s0.qz;
  const float* __restrict__ const S0QW = r.s0.qw;
  const float* __restrict__ const S1PX = r.s1.px;
  const float* __restrict__ const S1PY = r.s1.py;
  const float* __restrict__ const S1QX = r.s1.qx;
  const float* __restrict__ const S1QY = r.s1.qy;
  const float* __restrict__ const S1QZ = r.s1.qz;
  const float* __restrict__ const S1QW = r.s1.qw;
  const float* __restrict__ const G1U = r.g1.u;
  const float* __restrict__ const G1UB = r.g1.ub;
  const float* __restrict__ const G1VX = r.g1.vbx;
  const float* __restrict__ const G1VY = r.g1.vby;
  const float* __restrict__ const G1PX = r.g1.px;
  const float* __restrict__ const G1PY = r.g1.py;
  const float* __restrict__ const G1QX = r.g1.qx;
  const float* __restrict__ const G1QY = r.g1.qy;
  const float* __restrict__ const G1QZ = r.g1.qz;
  const float* __restrict__ const G1QW = r.g1.qw;
  float* __restrict__ const G0U = r.g0.u;
  float* __restrict__ const G0UB = r.g0.ub;
  float* __restrict__ const G0VX = r.g0.vbx;
  float* __restrict__ const G0VY = r.g0.vby;
  float* __restrict__ const G0PX = r.g0.px;
  float* __restrict__ const G0PY = r.g0.py;
  float* __restrict__ const G0QX = r.g0.qx;
  float* __restrict__ const G0QY = r.g0.qy;
  float* __restrict__ const G0QZ = r.g0.qz;
  float* __restrict__ const G0QW = r.g0.qw;
  const float* __restrict__ const CA = r.c.a;
  const float* __restrict__ const CB = r.c.b;
  const float* __restrict__ const CC = r.c.c;
  const float* __restrict__ const CEX = r.c.ex;
  const float* __restrict__ const CEY = r.c.ey;
  const float* __restrict__ const CEZ = r.c.ez;
  const float* __restrict__ const CIU = r.c.iu;
  const float* __restrict__ const CIZ = r.c.iz;
  const uint8_t* __restrict__ const CCODE = r.c.code;
  float* __restrict__ const GC0 = r.gc[0];
  float* __restrict__ const GC1 = r.gc[1];
  float* __restrict__ const GC2 = r.gc[2];
  float* __restrict__ const GC3 = r.gc[3];
  float* __restrict__ const GC4 = r.gc[4];
  float* __restrict__ const GC5 = r.gc[5];
  float* __restrict__ const GC6 = r.gc[6];
  float* __restrict__ const GC7 = r.gc[7];
  float acc[3] = {0.f, 0.f, 0.f};  // Lambda, alpha0, alpha1

#pragma unroll
  for (int j = 0; j < (N + NT - 1) / NT; ++j) {
    const int e = threadIdx.x + j * NT;
    if (e >= N) continue;
    const int wy = e / WX, wx = e - wy * WX;
    const long f = base + (long)wy * w + wx;
    const bool ok = f >= 0 && f < n;
    P(qUB)[e] = ok ? S0UB[f] : 0.f;
    P(qVX)[e] = ok ? S0VX[f] : 0.f;
    P(qVY)[e] = ok ? S0VY[f] : 0.f;
    P(qPX)[e] = ok ? S1PX[f] : 0.f;
    P(qPY)[e] = ok ? S1PY[f] : 0.f;
    P(qQX)[e] = ok ? S1QX[f] : 0.f;
    P(qQY)[e] = ok ? S1QY[f] : 0.f;
    P(qQZ)[e] = ok ? S1QZ[f] : 0.f;
    P(qQW)[e] = ok ? S1QW[f] : 0.f;
    P(qA)[e] = ok ? CA[f] : 0.f;
    P(qB)[e] = ok ? CB[f] : 0.f;
    P(qC)[e] = ok ? CC[f] : 0.f;
    scode[e] = ok ? CCODE[f] : 0;
  }
  __syncthreads();

  // phase 1: primal and threshold reversed, on [1, WX) x [1, WY)
#pragma unroll
  for (int j = 0; j < (N + NT - 1) / NT; ++j) {
    const int e = threadIdx.x + j * NT;
    if (e >= N) continue;
    const int wy = e / WX, wx = e - wy * WX;
    if (wx < 1 || wy < 1) continue;
    const long f = base + (long)wy * w + wx;
    const uint8_t c = scode[e];
    const bool core = wx >= 2 && wx < TX + 2 && wy >= 2 && wy < TY + 2 && x0 + wx - 2 < w && y0 + wy - 2 < h;
    float gu = 0.f, gubl = 0.f, gvx = 0.f, gvy = 0.f, Ax = 0.f, Ay = 0.f, Bv = 0.f;
    if (f >= 0 && f < n && (c & kSelf)) {
      const float gubn = G1UB[f];
      const float gvbx = G1VX[f], gvby = G1VY[f];
      const float gun = G1U[f] + (1.f + mu) * gubn;
      const float gVx = (1.f + mu) * gvbx, gVy = (1.f + mu) * gvby;
      const float a = P(qA)[e], b = P(qB)[e], cc = P(qC)[e];
      const float gQx = ((c & kE) ? P(qQX)[e] : 0.f) - ((c & kW) ? P(qQX)[e - 1] : 0.f);
      const float gQw = ((c & kE) ? P(qQW)[e] : 0.f) - ((c & kW) ? P(qQW)[e - 1] : 0.f);
      const float gQy = ((c & kS) ? P(qQY)[e] : 0.f) - ((c & kN) ? P(qQY)[e - WX] : 0.f);
      const float gQz = ((c & kS) ? P(qQZ)[e] : 0.f) - ((c & kN) ? P(qQZ)[e - WX] : 0.f);
      const float px = P(qPX)[e], py = P(qPY)[e];
      const float tpx = fmaf(a, px, cc * py), tpy = fmaf(cc, px, b * py);
      const float ex = CEX[f], ey = CEY[f], ez = CEZ[f];
      const bool sx = fabsf(ex) < eps, sy = fabsf(ey) < eps, sz = fabsf(ez) < eps;
      const float t1 = sy ? tau : tau / ey, t2 = sz ? tau : tau / ez;
      Ax = t1 * al0 * gVx;
      Ay = t2 * al0 * gVy;
      const float tpWx = fmaf(P(qA)[e - 1], P(qPX)[e - 1], P(qC)[e - 1] * P(qPY)[e - 1]);
      const float tpNy = fmaf(P(qC)[e - WX], P(qPX)[e - WX], P(qB)[e - WX] * P(qPY)[e - WX]);
      const bool E_ = c & kE, W_ = c & kW, S_ = c & kS, N_ = c & kN;
      const float gTx = (E_ && W_) ? tpx - tpWx : (!E_ ? -tpWx : tpx);
      const float gTy = (S_ && N_) ? tpy - tpNy : (!S_ ? -tpNy : tpy);
      const float Iu = CIU[f], Iz = CIZ[f];
      const float te = sx ? tau : tau / ex;
      const float u = S0U[f], ub = P(qUB)[e];
      const float ut = ub + te * (gTx + gTy);
      const float rho = Iu * (ut - u) + Iz;
      const float Bd = lam * te * Iu * Iu;
      float gut = 0.f, gte = 0.f, giu = 0.f, giz = 0.f, gl = 0.f;
      if ((rho <= Bd) && (rho >= -Bd)) {
        if (fabsf(Iu) >= eps) {
          gu += gun;
          giz = -gun / Iu;
          giu = gun * Iz / (Iu * Iu);
        } else {
          gut = gun;
        }
      } else if (rho < -Bd) {
        gut = gun;
        gl = te * Iu * gun;
        gte = lam * Iu * gun;
        giu = lam * te * gun;
      } else if (rho > Bd) {
        gut = gun;
        gl = -te * Iu * gun;
        gte = -lam * Iu * gun;
        giu = -lam * te * gun;
      } else {
        gu += gun;
      }
      gte += (gTx + gTy) * gut;
      Bv = te * gut;
      gubl = -mu * gubn + gut;
      gvx = gVx - mu * gvbx;
      gvy = gVy - mu * gvby;
      if (core) {
        const float inx = fmaf(al1, tpx, al0 * (gQx + gQz));
        const float iny = fmaf(al1, tpy, al0 * (gQw + gQy));
        GC3[f] += fin0(sx ? 0.f : -te / ex * gte);
        GC4[f] += fin0(sy ? 0.f : -t1 / ey * inx * gVx);
        GC5[f] += fin0(sz ? 0.f : -t2 / ez * iny * gVy);
        GC6[f] += fin0(giu);
        GC7[f] += fin0(giz);
        acc[0] += gl;
        acc[1] += t1 * (gQx + gQz) * gVx + t2 * (gQw + gQy) * gVy;
        acc[2] += t1 * tpx * gVx + t2 * tpy * gVy;
      }
    }
    P(aX)[e] = Ax;
    P(aY)[e] = Ay;
    P(aB)[e] = Bv;
    if (core) {
      G0U[f] = fin0(gu);
      P(lUB)[e] = gubl;
      P(lVX)[e] = gvx;
      P(lVY)[e] = gvy;
    }
  }
  __syncthreads();

  // phase 2: dual step reversed, on [1, WX - 1) x [1, WY - 1)
#pragma unroll
  for (int j = 0; j < (N + NT - 1) / NT; ++j) {
    const int e = threadIdx.x + j * NT;
    if (e >= N) continue;
    const int wy = e / WX, wx = e - wy * WX;
    if (wx < 1 || wy < 1 || wx >= WX - 1 || wy >= WY - 1) continue;
    const long f = base + (long)wy * w + wx;
    const uint8_t c = scode[e];
    const bool core = wx >= 2 && wx < TX + 2 && wy >= 2 && wy < TY + 2 && x0 + wx - 2 < w && y0 + wy - 2 < h;
    float Cv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (f >= 0 && f < n && (c & kSelf)) {
      const uint8_t cE = scode[e + 1], cS = scode[e + WX];
      const float Bv = P(aB)[e];
      const float gVx = (1.f + mu) * G1VX[f], gVy = (1.f + mu) * G1VY[f];
      const float ey = CEY[f], ez = CEZ[f];
      const float t1 = fabsf(ey) < eps ? tau : tau / ey, t2 = fabsf(ez) < eps ? tau : tau / ez;
      const float gtpx = t1 * al1 * gVx + ((c & kE) ? Bv : 0.f) - (((cE & kW) || !(cE & kE)) ? P(aB)[e + 1] : 0.f);
      const float gtpy = t2 * al1 * gVy + ((c & kS) ? Bv : 0.f) - (((cS & kN) || !(cS & kS)) ? P(aB)[e + WX] : 0.f);
      const float Ax = P(aX)[e], Ay = P(aY)[e];
      float gq0 = G1QX[f] + ((c & kE) ? Ax : 0.f) - ((cE & kW) ? P(aX)[e + 1] : 0.f);
      float gq3 = G1QW[f] + ((c & kE) ? Ay : 0.f) - ((cE & kW) ? P(aY)[e + 1] : 0.f);
      float gq1 = G1QY[f] + ((c & kS) ? Ay : 0.f) - ((cS & kN) ? P(aY)[e + WX] : 0.f);
      float gq2 = G1QZ[f] + ((c & kS) ? Ax : 0.f) - ((cS & kN) ? P(aX)[e + WX] : 0.f);
      const float a = P(qA)[e], b = P(qB)[e], cc = P(qC)[e];
      const float pnx = P(qPX)[e], pny = P(qPY)[e];
      const float gpx = G1PX[f] + fmaf(a, gtpx, cc * gtpy);
      const float gpy = G1PY[f] + fmaf(cc, gtpx, b * gtpy);
      float ga = pnx * gtpx, gb = pny * gtpy, gcc = pny * gtpx + pnx * gtpy;
      const float uc = P(qUB)[e], vcx = P(qVX)[e], vcy = P(qVY)[e];
      float gUx, gUy, gVxx, gVyy, gVz, gVw;
      if (c & kE) {
        gUx = P(qUB)[e + 1] - uc - vcx;
        gVxx = P(qVX)[e + 1] - vcx;
        gVw = P(qVY)[e + 1] - vcy;
      } else {
        gUx = uc - P(qUB)[e - 1] - vcx;
        gVxx = vcx - P(qVX)[e - 1];
        gVw = vcy - P(qVY)[e - 1];
      }
      if (c & kS) {
        gUy = P(qUB)[e + WX] - uc - vcy;
        gVyy = P(qVY)[e + WX] - vcy;
        gVz = P(qVX)[e + WX] - vcx;
      } else {
        gUy = uc - P(qUB)[e - WX] - vcy;
        gVyy = vcy - P(qVY)[e - WX];
        gVz = vcx - P(qVX)[e - WX];
      }
      const float scaleP = al1 * sigma / r.k.etaP;
      const float scaleQ = al0 * sigma / r.k.etaQ;
      const float tux = fmaf(a, gUx, cc * gUy), tuy = fmaf(cc, gUx, b * gUy);
      const float upx = fmaf(scaleP, tux, S0PX[f]), upy = fmaf(scaleP, tuy, S0PY[f]);
      const float nP = hypotf(upx, upy);
      float gP0 = gpx, gP1 = gpy;
      if (nP > 1.f) {
        const float dt = pnx * gpx + pny * gpy;
        gP0 = (gpx - pnx * dt) / nP;
        gP1 = (gpy - pny * dt) / nP;
      }
      const float uq0 = fmaf(scaleQ, gVxx, S0QX[f]), uq1 = fmaf(scaleQ, gVyy, S0QY[f]);
      const float uq2 = fmaf(scaleQ, gVz, S0QZ[f]), uq3 = fmaf(scaleQ, gVw, S0QW[f]);
      const float nQ = norm4df(uq0, uq1, uq2, uq3);
      if (nQ > 1.f) {
        const float q0 = P(qQX)[e], q1 = P(qQY)[e], q2 = P(qQZ)[e], q3 = P(qQW)[e];
        const float dt = q0 * gq0 + q1 * gq1 + q2 * gq2 + q3 * gq3;
        gq0 = (gq0 - q0 * dt) / nQ;
        gq1 = (gq1 - q1 * dt) / nQ;
        gq2 = (gq2 - q2 * dt) / nQ;
        gq3 = (gq3 - q3 * dt) / nQ;
      }
      const float gtux = scaleP * gP0, gtuy = scaleP * gP1;
      Cv[0] = fmaf(a, gtux, cc * gtuy);
      Cv[1] = fmaf(cc, gtux, b * gtuy);
      Cv[2] = scaleQ * gq0;
      Cv[3] = scaleQ * gq1;
      Cv[4] = scaleQ * gq2;
      Cv[5] = scaleQ * gq3;
      if (core) {
        ga += gUx * gtux;
        gb += gUy * gtuy;
        gcc += gUy * gtux + gUx * gtuy;
        GC0[f] += fin0(ga);
        GC1[f] += fin0(gb);
        GC2[f] += fin0(gcc);
        acc[1] += sigma / r.k.etaQ * (gVxx * gq0 + gVyy * gq1 + gVz * gq2 + gVw * gq3);
        acc[2] += sigma / r.k.etaP * (tux * gP0 + tuy * gP1);
        G0PX[f] = fin0(gP0);
        G0PY[f] = fin0(gP1);
        G0QX[f] = fin0(gq0);
        G0QY[f] = fin0(gq1);
        G0QZ[f] = fin0(gq2);
        G0QW[f] = fin0(gq3);
      }
    } else if (core) {
      G0PX[f] = fin0(G0PY[f] = 0.f);
      G0QX[f] = fin0(G0QY[f] = G0QZ[f] = G0QW[f] = 0.f);
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) P(c0 + k)[e] = Cv[k];
  }
  __syncthreads();

  // phase 3: transposed gradients of u_ and v_, on the tile
#pragma unroll
  for (int j = 0; j < (N + NT - 1) / NT; ++j) {
    const int e = threadIdx.x + j * NT;
    if (e >= N) continue;
    const int wy = e / WX, wx = e - wy * WX;
    if (wx < 2 || wy < 2 || wx >= TX + 2 || wy >= TY + 2 || x0 + wx - 2 >= w || y0 + wy - 2 >= h) continue;
    const long f = base + (long)wy * w + wx;
    const uint8_t c = scode[e];
    float gub = P(lUB)[e], gvx = P(lVX)[e], gvy = P(lVY)[e];
    if (c & kSelf) {
      const float u0 = P(c0)[e], u1 = P(c1)[e];
      const float v0 = P(c2)[e], v1 = P(c3)[e], v2 = P(c4)[e], v3 = P(c5)[e];
      gub += ((c & kE) ? -u0 : u0) + ((c & kS) ? -u1 : u1);
      gvx += -u0 + ((c & kE) ? -v0 : v0) + ((c & kS) ? -v2 : v2);
      gvy += -u1 + ((c & kE) ? -v3 : v3) + ((c & kS) ? -v1 : v1);
    }
    if (scode[e - 1] & kE) {
      gub += P(c0)[e - 1];
      gvx += P(c2)[e - 1];
      gvy += P(c5)[e - 1];
    }
    if (!(scode[e + 1] & kE)) {
      gub -= P(c0)[e + 1];
      gvx -= P(c2)[e + 1];
      gvy -= P(c5)[e + 1];
    }
    if (scode[e - WX] & kS) {
      gub += P(c1)[e - WX];
      gvx += P(c4)[e - WX];
      gvy += P(c3)[e - WX];
    }
    if (!(scode[e + WX] & kS)) {
      gub -= P(c1)[e + WX];
      gvx -= P(c4)[e + WX];
      gvy -= P(c3)[e + WX];
    }
    G0UB[f] = fin0(gub);
    G0VX[f] = fin0(gvx);
    G0VY[f] = fin0(gvy);
  }
  block_sum_to<3>(acc, r.scal + G_LAMBDA);
}

// Tile shapes of the reverse step, selected by vfs_grad_set_options.
#define VFS_REV_SHAPES(X) \
  X(1, 32, 16, 512)       \
  X(2, 32, 8, 256)        \
  X(3, 64, 8, 512)        \
  X(4, 32, 32, 1024)      \
  X(5, 28, 16, 640)

cudaError_t launch_rev_tile(int shape, const RevArgs& r, cudaStream_t s) {
  switch (shape) {
#define VFS_REV_L(id, TX, TY, NT)                                                      \
  case id: {                                                                           \
    dim3 grid((r.w + TX - 1) / TX, (r.h + TY - 1) / TY);                               \
    k_rev_tile<TX, TY, NT><<<grid, NT, RevGeom<TX, TY>::smem_bytes(), s>>>(r);         \
    return cudaGetLastError();                                                         \
  }
    VFS_REV_SHAPES(VFS_REV_L)
#undef VFS_REV_L
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t prepare_rev_tile() {
  cudaError_t e = cudaSuccess;
#define VFS_REV_P(id, TX, TY, NT)                                                                         \
  if (e == cudaSuccess)                                                                                   \
    e = cudaFuncSetAttribute(k_rev_tile<TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                             (int)RevGeom<TX, TY>::smem_bytes());
  VFS_REV_SHAPES(VFS_REV_P)
#undef VFS_REV_P
  return e;
}

bool rev_shape_ok(int shape) {
  switch (shape) {
#define VFS_REV_OK(id, TX, TY, NT) \
  case id: return true;
    VFS_REV_SHAPES(VFS_REV_OK)
#undef VFS_REV_OK
    default: return false;
  }
}

// ---------------------------------------------------------------- blocked reverse
// k (<= K) reverse iterations per launch: from the cotangent of S_{i0+k} to
// that of S_{i0}, reading the recorded states S_{i0} .. S_{i0+k}.  The same
// three phases per step as k_rev_tile.  Each thread owns one window pixel:
// its cotangent state and, on the tile, its constant cotangents stay in the
// thread's registers, so cotangents and constants cross HBM once per launch
// instead of once per iteration.  The recorded states stream into three
// shared-memory buffers with cp.async: while step m runs on S_{i0+k-m} and
// S_{i0+k-m+1}, the state of step m+1 is already loading.  Two barriers per
// step: phase 3 and the next step's phase 1 share one interval.
//
// Geometry.  Step m (1..k) produces a valid cotangent on O_m = [-(k-m),
// T + 2(k-m)) in tile coordinates (phase 3 there; phase 2 on O_m grown by 1,
// phase 1 on O_m grown by 1 low and 2 high) and reads S_{i0+k-m} on O_m
// grown by 2, so the window is the tile plus K+1 pixels low and 2K high, in
// the flat addressing of k_rev_tile.
//
// Quotients that only scale cotangents use the fast divide; tau / eta uses a
// reciprocal of eta formed once per launch (the branch of the L1 shrink is
// the forward's except where rho is within an ulp of the bound).
struct RevBlockArgs {
  const TgvState* states;  // states[0..k]: S_{i0} .. S_{i0+k}
  TgvState g_in, g_out;    // cotangent of S_{i0+k} (in), of S_{i0} (out)
  TgvConsts c;
  float* gc[8];
  const float3* sched;
  int i0, niter;
  SolverConsts k;
  int h, w;
  double* scal;
};

// state buffer planes
enum { sUB, sVX, sVY, sU, sPX, sPY, sQX, sQY, sQZ, sQW, kStPlanes };
enum RbPlane { bS0 = 0, bAX = 3 * kStPlanes, bAY, bAB, bC0, bCA = bC0 + 6, bCB, bCC, bREX, bREY, bREZ, bIU, bIZ,
               kRbPlanes };

// The window starts LHX >= K+1 columns left of the tile, rounded to a
// multiple of 4, and is a multiple of 4 wide: with a row stride divisible by
// 4 every window row then starts on a 16-byte boundary and the recorded
// states load as 16-byte chunks.
template <int K, int TX, int TY>
struct RbGeom {
  static_assert(TX % 4 == 0, "tile width must be a multiple of 4");
  static constexpr int LH = K + 1;
  static constexpr int LHX = (K + 1 + 3) / 4 * 4;
  static constexpr int WX = (TX + LHX + 2 * K + 3) / 4 * 4, WY = TY + 3 * K + 1, N = WX * WY;
  static constexpr size_t smem_bytes() {
    // planes, mask codes, then (sigma, tau, mu, scaleP, scaleQ) of each of
    // the launch's iterations
    return (size_t)kRbPlanes * N * 4 + ((N + 15) / 16) * 16 + 5 * K * 4;
  }
};


template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 1) k_rev_block(RevBlockArgs r) {
  using G = RbGeom<K, TX, TY>;
  static_assert(G::N <= NT, "one window pixel per thread");
  constexpr int WX = G::WX, N = G::N, LH = G::LH, LHX = G::LHX, J = (N + NT - 1) / NT;
  extern __shared__ float4 smem_raw[];
  float* const sm = reinterpret_cast<float*>(smem_raw);
  uint8_t* const scode = reinterpret_cast<uint8_t*>(sm + (size_t)kRbPlanes * N);
  float* const sSch = reinterpret_cast<float*>(scode + ((N + 15) / 16) * 16);
  auto P = [&](int plane) { return sm + (size_t)plane * N; };
  const int w = r.w, h = r.h;
  const long n = (long)h * w;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const long base = (long)(y0 - LH) * w + (x0 - LHX);
  const bool vec4 = (w % 4) == 0;
  const int k = r.niter < K ? r.niter : K;
  const float eps = 1E-7f;
  const float al0 = r.k.alpha0, al1 = r.k.alpha1, lam = r.k.lambda;
  float acc[3] = {0.f, 0.f, 0.f};  // Lambda, alpha0, alpha1
  // constant cotangents of the thread's tile pixel over this launch's steps
  // (one window pixel per thread: J == 1)
  static_assert(J == 1, "one window pixel per thread");
  float gca[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};

  float gU[J], gUB[J], gVX[J], gVY[J], gPX[J], gPY[J], gQ0[J], gQ1[J], gQ2[J], gQ3[J];
  int rx[J], ry[J];

  // state S_{i0+q} into buffer b over O_m grown by 2 (m = k - q; the whole
  // window for q = k)
  auto load_state = [&](int q, int b) {
    const TgvState S = r.states[q];
    const float* src[kStPlanes] = {S.ub, S.vbx, S.vby, S.u, S.px, S.py, S.qx, S.qy, S.qz, S.qw};
    const int m = k - q;
    const int lo = m == 0 ? -LH : -(k - m) - 2, hiX = m == 0 ? TX + 2 * K : TX + 2 * (k - m) + 2,
              hiY = m == 0 ? TY + 2 * K : TY + 2 * (k - m) + 2;
    if (vec4) {
      // 16-byte chunks along rows (a chunk is wholly inside or outside
      // [0, n) since n and the chunk start are multiples of 4)
      for (int c = threadIdx.x; c < N / 4; c += NT) {
        const int e0 = 4 * c;
        const int wy = e0 / WX, wx0 = e0 - wy * WX;
        const int cx = wx0 - LHX, cy = wy - LH;
        if (cy < lo || cy >= hiY || cx + 3 < lo || cx >= hiX) continue;
        const long f = base + (long)wy * w + wx0;
        const bool ok = f >= 0 && f < n;
#pragma unroll
        for (int pl = 0; pl < kStPlanes; ++pl)
          cp_async16(P(bS0 + b * kStPlanes + pl) + e0, ok ? src[pl] + f : src[pl], ok);
      }
    } else {
#pragma unroll
      for (int j = 0; j < J; ++j) {
        if (rx[j] < lo || rx[j] >= hiX || ry[j] < lo || ry[j] >= hiY) continue;
        const int e = threadIdx.x + j * NT;
        const long f = base + (long)(ry[j] + LH) * w + (rx[j] + LHX);
        const bool ok = f >= 0 && f < n;
#pragma unroll
        for (int pl = 0; pl < kStPlanes; ++pl)
          cp_async4(P(bS0 + b * kStPlanes + pl) + e, ok ? src[pl] + f : src[pl], ok);
      }
    }
    cp_async_commit();
  };

#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int e = threadIdx.x + j * NT;
    const int wy = e / WX, wx = e - wy * WX;
    rx[j] = wx - LHX;
    ry[j] = e < N ? wy - LH : (1 << 20);
  }
  load_state(k, 0);
  if (k >= 1) load_state(k - 1, 1);
  if (k >= 2) load_state(k - 2, 2);
  // a launch that follows another reverse launch may start before it ends:
  // everything above and the constants below are recorded data; the
  // cotangent it wrote is read only after griddepcontrol.wait
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  if (threadIdx.x < 5 * k) {  // this launch's step sizes and dual-step scales
    const int t = threadIdx.x / 5, c = threadIdx.x - 5 * t;
    sSch[threadIdx.x] = c < 3 ? reinterpret_cast<const float*>(r.sched + r.i0 + t)[c]
                              : reinterpret_cast<const float*>(r.k.dscale + r.i0 + t)[c - 3];
  }
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int e = threadIdx.x + j * NT;
    const long f = base + (long)(ry[j] + LH) * w + (rx[j] + LHX);
    const bool ok = e < N && f >= 0 && f < n;
    if (e < N) {
      // the constants as two 16-byte records per pixel (a, b, c, ex), (ey, ez, iu, iz)
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 c0 = ok ? r.c.rec[2 * f] : z, c1 = ok ? r.c.rec[2 * f + 1] : z;
      P(bCA)[e] = c0.x;
      P(bCB)[e] = c0.y;
      P(bCC)[e] = c0.z;
      P(bREX)[e] = fabsf(c0.w) < eps ? 0.f : 1.f / c0.w;
      P(bREY)[e] = fabsf(c1.x) < eps ? 0.f : 1.f / c1.x;
      P(bREZ)[e] = fabsf(c1.y) < eps ? 0.f : 1.f / c1.y;
      P(bIU)[e] = c1.z;
      P(bIZ)[e] = c1.w;
      scode[e] = ok ? r.c.code[f] : 0;
    }
  }
  // with the tile and a one-pixel ring around it all masked, every phase-2
  // value the tile gathers is zero and so is its cotangent: write that
  int live = 0;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int e = threadIdx.x + j * NT;
    if (e < N && rx[j] >= -1 && rx[j] <= TX && ry[j] >= -1 && ry[j] <= TY && (scode[e] & kSelf)) live = 1;
  }
  live = __syncthreads_or(live);
  // a warp whose pixels and their four neighbours are all unmasked with
  // all four neighbours unmasked (most of the image) takes the phases
  // compiled for that code: no code tests, no neighbour-code loads (not
  // for tiles below 16x16, which measured faster without it)
  bool wfull = false;
  if constexpr (TX * TY >= 256) {
    const int e = threadIdx.x;
    const bool ring = e >= WX && e + WX < N && scode[e] == kAllSides && scode[e - 1] == kAllSides &&
                      scode[e + 1] == kAllSides && scode[e - WX] == kAllSides && scode[e + WX] == kAllSides;
    wfull = __all_sync(0xffffffffu, ring);
  }
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  if (!live) {
#pragma unroll
    for (int j = 0; j < J; ++j) {
      if (rx[j] < 0 || rx[j] >= TX || ry[j] < 0 || ry[j] >= TY) continue;
      const int X = x0 + rx[j], Y = y0 + ry[j];
      if (X >= w || Y >= h) continue;
      const long f = (long)Y * w + X;
      r.g_out.u[f] = r.g_out.ub[f] = r.g_out.vbx[f] = r.g_out.vby[f] = r.g_out.px[f] = r.g_out.py[f] = 0.f;
      r.g_out.qx[f] = r.g_out.qy[f] = r.g_out.qz[f] = r.g_out.qw[f] = 0.f;
    }
    cp_async_wait<0>();
    return;
  }
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int e = threadIdx.x + j * NT;
    const long f = base + (long)(ry[j] + LH) * w + (rx[j] + LHX);
    const bool ok = e < N && f >= 0 && f < n;
    gU[j] = ok ? r.g_in.u[f] : 0.f;
    gUB[j] = ok ? r.g_in.ub[f] : 0.f;
    gVX[j] = ok ? r.g_in.vbx[f] : 0.f;
    gVY[j] = ok ? r.g_in.vby[f] : 0.f;
    gPX[j] = ok ? r.g_in.px[f] : 0.f;
    gPY[j] = ok ? r.g_in.py[f] : 0.f;
    gQ0[j] = ok ? r.g_in.qx[f] : 0.f;
    gQ1[j] = ok ? r.g_in.qy[f] : 0.f;
    gQ2[j] = ok ? r.g_in.qz[f] : 0.f;
    gQ3[j] = ok ? r.g_in.qw[f] : 0.f;
  }
  if (k >= 2) cp_async_wait<1>(); else cp_async_wait<0>();
  __syncthreads();

  for (int m = 1; m <= k; ++m) {
    const float* const sc = sSch + 5 * (k - m);
    const float sigma = sc[0], tau = sc[1], mu = sc[2];
    const float sQe = __fdividef(sigma, r.k.etaQ), sPe = __fdividef(sigma, r.k.etaP);  // gradient scales only
    const float2 dsc = make_float2(sc[3], sc[4]);  // the forward's dual-step scales
    const int lo = -(k - m), hiX = TX + 2 * (k - m), hiY = TY + 2 * (k - m);
    const int L0 = bS0 + (m % 3) * kStPlanes, H0 = bS0 + ((m - 1) % 3) * kStPlanes;  // later / earlier state
    // phase 1: primal and threshold reversed on [lo - 1, hi + 2)
    float nU[J], lUB[J], lVX[J], lVY[J];
#pragma unroll
    for (int j = 0; j < J; ++j) {
      nU[j] = lUB[j] = lVX[j] = lVY[j] = 0.f;
      if (rx[j] < lo - 1 || rx[j] >= hiX + 2 || ry[j] < lo - 1 || ry[j] >= hiY + 2) continue;
      const int e = threadIdx.x + j * NT;
      const long f = base + (long)(ry[j] + LH) * w + (rx[j] + LHX);
      const bool core = rx[j] >= 0 && rx[j] < TX && ry[j] >= 0 && ry[j] < TY && x0 + rx[j] < w && y0 + ry[j] < h;
      auto phase1 = [&](const uint8_t c) {
      float Ax = 0.f, Ay = 0.f, Bv = 0.f;
      if (f >= 0 && f < n && (c & kSelf)) {
        const float gubn = gUB[j], gvbx = gVX[j], gvby = gVY[j];
        const float gun = gU[j] + (1.f + mu) * gubn;
        const float gVx = (1.f + mu) * gvbx, gVy = (1.f + mu) * gvby;
        const float* hq = P(H0 + sQX);
        const float gQx = ((c & kE) ? hq[e] : 0.f) - ((c & kW) ? hq[e - 1] : 0.f);
        const float gQw = ((c & kE) ? P(H0 + sQW)[e] : 0.f) - ((c & kW) ? P(H0 + sQW)[e - 1] : 0.f);
        const float gQy = ((c & kS) ? P(H0 + sQY)[e] : 0.f) - ((c & kN) ? P(H0 + sQY)[e - WX] : 0.f);
        const float gQz = ((c & kS) ? P(H0 + sQZ)[e] : 0.f) - ((c & kN) ? P(H0 + sQZ)[e - WX] : 0.f);
        const float a = P(bCA)[e], b = P(bCB)[e], cc = P(bCC)[e];
        const float px = P(H0 + sPX)[e], py = P(H0 + sPY)[e];
        const float tpx = fmaf(a, px, cc * py), tpy = fmaf(cc, px, b * py);
        const float tpWx = fmaf(P(bCA)[e - 1], P(H0 + sPX)[e - 1], P(bCC)[e - 1] * P(H0 + sPY)[e - 1]);
        const float tpNy = fmaf(P(bCC)[e - WX], P(H0 + sPX)[e - WX], P(bCB)[e - WX] * P(H0 + sPY)[e - WX]);
        const float rex = P(bREX)[e], rey = P(bREY)[e], rez = P(bREZ)[e];
        const float t1 = rey == 0.f ? tau : tau * rey, t2 = rez == 0.f ? tau : tau * rez;
        Ax = t1 * al0 * gVx;
        Ay = t2 * al0 * gVy;
        const bool E_ = c & kE, W_ = c & kW, S_ = c & kS, N_ = c & kN;
        const float gTx = (E_ && W_) ? tpx - tpWx : (!E_ ? -tpWx : tpx);
        const float gTy = (S_ && N_) ? tpy - tpNy : (!S_ ? -tpNy : tpy);
        const float Iu = P(bIU)[e], Iz = P(bIZ)[e];
        const float te = rex == 0.f ? tau : tau * rex;
        const float u = P(L0 + sU)[e], ub = P(L0 + sUB)[e];
        const float ut = ub + te * (gTx + gTy);
        const float rho = Iu * (ut - u) + Iz;
        const float Bd = lam * te * Iu * Iu;
        float gu = 0.f, gut = 0.f, gte = 0.f, giu = 0.f, giz = 0.f, gl = 0.f;
        if ((rho <= Bd) && (rho >= -Bd)) {
          if (fabsf(Iu) >= eps) {
            const float ri = __fdividef(1.f, Iu);
            gu = gun;
            giz = -gun * ri;
            giu = gun * Iz * ri * ri;
          } else {
            gut = gun;
          }
        } else if (rho < -Bd) {
          gut = gun;
          gl = te * Iu * gun;
          gte = lam * Iu * gun;
          giu = lam * te * gun;
        } else if (rho > Bd) {
          gut = gun;
          gl = -te * Iu * gun;
          gte = -lam * Iu * gun;
          giu = -lam * te * gun;
        } else {
          gu = gun;
        }
        gte += (gTx + gTy) * gut;
        Bv = te * gut;
        nU[j] = gu;
        lUB[j] = -mu * gubn + gut;
        lVX[j] = gVx - mu * gvbx;
        lVY[j] = gVy - mu * gvby;
        if (core) {
          const float inx = fmaf(al1, tpx, al0 * (gQx + gQz));
          const float iny = fmaf(al1, tpy, al0 * (gQw + gQy));
          gca[3] -= te * rex * gte;
          gca[4] -= t1 * rey * inx * gVx;
          gca[5] -= t2 * rez * iny * gVy;
          gca[6] += giu;
          gca[7] += giz;
          acc[0] += gl;
          acc[1] += t1 * (gQx + gQz) * gVx + t2 * (gQw + gQy) * gVy;
          acc[2] += t1 * tpx * gVx + t2 * tpy * gVy;
        }
      }
      P(bAX)[e] = Ax;
      P(bAY)[e] = Ay;
      P(bAB)[e] = Bv;
      };
      if (wfull) phase1(kAllSides);
      else phase1(scode[e]);
    }
    __syncthreads();
    // phase 2: dual step reversed on [lo - 1, hi + 1)
    float nPX[J], nPY[J], nQ0[J], nQ1[J], nQ2[J], nQ3[J];
#pragma unroll
    for (int j = 0; j < J; ++j) {
      nPX[j] = nPY[j] = nQ0[j] = nQ1[j] = nQ2[j] = nQ3[j] = 0.f;
      if (rx[j] < lo - 1 || rx[j] >= hiX + 1 || ry[j] < lo - 1 || ry[j] >= hiY + 1) continue;
      const int e = threadIdx.x + j * NT;
      const long f = base + (long)(ry[j] + LH) * w + (rx[j] + LHX);
      const bool core = rx[j] >= 0 && rx[j] < TX && ry[j] >= 0 && ry[j] < TY && x0 + rx[j] < w && y0 + ry[j] < h;
      auto phase2 = [&](const uint8_t c, const bool full) {
      float Cv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (f >= 0 && f < n && (c & kSelf)) {
        const uint8_t cE = full ? kAllSides : scode[e + 1], cS = full ? kAllSides : scode[e + WX];
        const float Bv = P(bAB)[e];
        const float gVx = (1.f + mu) * gVX[j], gVy = (1.f + mu) * gVY[j];
        const float rey = P(bREY)[e], rez = P(bREZ)[e];
        const float t1 = rey == 0.f ? tau : tau * rey, t2 = rez == 0.f ? tau : tau * rez;
        const float gtpx = t1 * al1 * gVx + ((c & kE) ? Bv : 0.f) - (((cE & kW) || !(cE & kE)) ? P(bAB)[e + 1] : 0.f);
        const float gtpy = t2 * al1 * gVy + ((c & kS) ? Bv : 0.f) - (((cS & kN) || !(cS & kS)) ? P(bAB)[e + WX] : 0.f);
        const float Ax = P(bAX)[e], Ay = P(bAY)[e];
        float gq0 = gQ0[j] + ((c & kE) ? Ax : 0.f) - ((cE & kW) ? P(bAX)[e + 1] : 0.f);
        float gq3 = gQ3[j] + ((c & kE) ? Ay : 0.f) - ((cE & kW) ? P(bAY)[e + 1] : 0.f);
        float gq1 = gQ1[j] + ((c & kS) ? Ay : 0.f) - ((cS & kN) ? P(bAY)[e + WX] : 0.f);
        float gq2 = gQ2[j] + ((c & kS) ? Ax : 0.f) - ((cS & kN) ? P(bAX)[e + WX] : 0.f);
        const float a = P(bCA)[e], b = P(bCB)[e], cc = P(bCC)[e];
        const float pnx = P(H0 + sPX)[e], pny = P(H0 + sPY)[e];
        const float gpx = gPX[j] + fmaf(a, gtpx, cc * gtpy);
        const float gpy = gPY[j] + fmaf(cc, gtpx, b * gtpy);
        const float ga = pnx * gtpx, gb = pny * gtpy, gcc = pny * gtpx + pnx * gtpy;
        const float* lub = P(L0 + sUB);
        const float* lvx = P(L0 + sVX);
        const float* lvy = P(L0 + sVY);
        const float uc = lub[e], vcx = lvx[e], vcy = lvy[e];
        float gUx, gUy, gVxx, gVyy, gVz, gVw;
        if (c & kE) {
          gUx = lub[e + 1] - uc - vcx;
          gVxx = lvx[e + 1] - vcx;
          gVw = lvy[e + 1] - vcy;
        } else {
          gUx = uc - lub[e - 1] - vcx;
          gVxx = vcx - lvx[e - 1];
          gVw = vcy - lvy[e - 1];
        }
        if (c & kS) {
          gUy = lub[e + WX] - uc - vcy;
          gVyy = lvy[e + WX] - vcy;
          gVz = lvx[e + WX] - vcx;
        } else {
          gUy = uc - lub[e - WX] - vcy;
          gVyy = vcy - lvy[e - WX];
          gVz = vcx - lvx[e - WX];
        }
        const float scaleP = dsc.x, scaleQ = dsc.y;
        const float tux = fmaf(a, gUx, cc * gUy), tuy = fmaf(cc, gUx, b * gUy);
        const float upx = fmaf(scaleP, tux, P(L0 + sPX)[e]), upy = fmaf(scaleP, tuy, P(L0 + sPY)[e]);
        // A projection was active where the recorded result differs from its
        // recomputed argument: the forward returns an inactive argument bit
        // for bit, an active one divided by a norm > 1.  NaN arguments count
        // as inactive (the forward's norm > 1 is false for them).  The
        // reciprocal norm only scales cotangents: rsqrt of the squared norm.
        float gP0 = gpx, gP1 = gpy;
        if ((pnx != upx || pny != upy) && upx == upx && upy == upy) {
          const float dt = pnx * gpx + pny * gpy, rn = rsqrtf(fmaf(upx, upx, upy * upy));
          gP0 = (gpx - pnx * dt) * rn;
          gP1 = (gpy - pny * dt) * rn;
        }
        const float uq0 = fmaf(scaleQ, gVxx, P(L0 + sQX)[e]), uq1 = fmaf(scaleQ, gVyy, P(L0 + sQY)[e]);
        const float uq2 = fmaf(scaleQ, gVz, P(L0 + sQZ)[e]), uq3 = fmaf(scaleQ, gVw, P(L0 + sQW)[e]);
        const float q0 = P(H0 + sQX)[e], q1 = P(H0 + sQY)[e], q2 = P(H0 + sQZ)[e], q3 = P(H0 + sQW)[e];
        if ((q0 != uq0 || q1 != uq1 || q2 != uq2 || q3 != uq3) && uq0 == uq0 && uq1 == uq1 && uq2 == uq2 &&
            uq3 == uq3) {
          const float dt = q0 * gq0 + q1 * gq1 + q2 * gq2 + q3 * gq3,
                      rn = rsqrtf(fmaf(uq0, uq0, fmaf(uq1, uq1, fmaf(uq2, uq2, uq3 * uq3))));
          gq0 = (gq0 - q0 * dt) * rn;
          gq1 = (gq1 - q1 * dt) * rn;
          gq2 = (gq2 - q2 * dt) * rn;
          gq3 = (gq3 - q3 * dt) * rn;
        }
        const float gtux = scaleP * gP0, gtuy = scaleP * gP1;
        Cv[0] = fmaf(a, gtux, cc * gtuy);
        Cv[1] = fmaf(cc, gtux, b * gtuy);
        Cv[2] = scaleQ * gq0;
        Cv[3] = scaleQ * gq1;
        Cv[4] = scaleQ * gq2;
        Cv[5] = scaleQ * gq3;
        nPX[j] = gP0;
        nPY[j] = gP1;
        nQ0[j] = gq0;
        nQ1[j] = gq1;
        nQ2[j] = gq2;
        nQ3[j] = gq3;
        if (core) {
          gca[0] += ga + gUx * gtux;
          gca[1] += gb + gUy * gtuy;
          gca[2] += gcc + gUy * gtux + gUx * gtuy;
          acc[1] += sQe * (gVxx * gq0 + gVyy * gq1 + gVz * gq2 + gVw * gq3);
          acc[2] += sPe * (tux * gP0 + tuy * gP1);
        }
      }
#pragma unroll
      for (int q = 0; q < 6; ++q) P(bC0 + q)[e] = Cv[q];
      };
      if (wfull) phase2(kAllSides, true);
      else phase2(scode[e], false);
    }
    // phase 3 and the next step's phase 1 share one barrier interval: the
    // state that phase 1 reads first (loaded a step ahead) is waited for here
    if (m < k) cp_async_wait<0>();
    __syncthreads();
    // the later state's buffer is no longer read: the state of step m + 2
    // starts loading into it
    if (m + 2 <= k) load_state(k - m - 2, (m + 2) % 3);
    // phase 3: transposed gradients of u_ and v_ on [lo, hi); commit the step.
    // It reads the phase-2 results only; the next phase 1 writes the phase-1
    // planes (last read in phase 2) and reads states waited for above.
#pragma unroll
    for (int j = 0; j < J; ++j) {
      if (rx[j] < lo || rx[j] >= hiX || ry[j] < lo || ry[j] >= hiY) continue;
      const int e = threadIdx.x + j * NT;
      float gub = lUB[j], gvx = lVX[j], gvy = lVY[j];
      auto phase3 = [&](const uint8_t c, const uint8_t cW, const uint8_t cE, const uint8_t cN, const uint8_t cS) {
      if (c & kSelf) {
        const float u0 = P(bC0)[e], u1 = P(bC0 + 1)[e];
        const float v0 = P(bC0 + 2)[e], v1 = P(bC0 + 3)[e], v2 = P(bC0 + 4)[e], v3 = P(bC0 + 5)[e];
        gub += ((c & kE) ? -u0 : u0) + ((c & kS) ? -u1 : u1);
        gvx += -u0 + ((c & kE) ? -v0 : v0) + ((c & kS) ? -v2 : v2);
        gvy += -u1 + ((c & kE) ? -v3 : v3) + ((c & kS) ? -v1 : v1);
      }
      if (cW & kE) {
        gub += P(bC0)[e - 1];
        gvx += P(bC0 + 2)[e - 1];
        gvy += P(bC0 + 5)[e - 1];
      }
      if (!(cE & kE)) {
        gub -= P(bC0)[e + 1];
        gvx -= P(bC0 + 2)[e + 1];
        gvy -= P(bC0 + 5)[e + 1];
      }
      if (cN & kS) {
        gub += P(bC0 + 1)[e - WX];
        gvx += P(bC0 + 4)[e - WX];
        gvy += P(bC0 + 3)[e - WX];
      }
      if (!(cS & kS)) {
        gub -= P(bC0 + 1)[e + WX];
        gvx -= P(bC0 + 4)[e + WX];
        gvy -= P(bC0 + 3)[e + WX];
      }
      };
      if (wfull) phase3(kAllSides, kAllSides, kAllSides, kAllSides, kAllSides);
      else phase3(scode[e], scode[e - 1], scode[e + 1], scode[e - WX], scode[e + WX]);
      gU[j] = nU[j];
      gUB[j] = gub;
      gVX[j] = gvx;
      gVY[j] = gvy;
      gPX[j] = nPX[j];
      gPY[j] = nPY[j];
      gQ0[j] = nQ0[j];
      gQ1[j] = nQ1[j];
      gQ2[j] = nQ2[j];
      gQ3[j] = nQ3[j];
    }
  }

  // cotangent of S_{i0} on the tile; constant cotangents added to HBM once
#pragma unroll
  for (int j = 0; j < J; ++j) {
    if (rx[j] < 0 || rx[j] >= TX || ry[j] < 0 || ry[j] >= TY) continue;
    const int X = x0 + rx[j], Y = y0 + ry[j];
    if (X >= w || Y >= h) continue;
    const long f = (long)Y * w + X;
    r.g_out.u[f] = fin0(gU[j]);
    r.g_out.ub[f] = fin0(gUB[j]);
    r.g_out.vbx[f] = fin0(gVX[j]);
    r.g_out.vby[f] = fin0(gVY[j]);
    r.g_out.px[f] = fin0(gPX[j]);
    r.g_out.py[f] = fin0(gPY[j]);
    r.g_out.qx[f] = fin0(gQ0[j]);
    r.g_out.qy[f] = fin0(gQ1[j]);
    r.g_out.qz[f] = fin0(gQ2[j]);
    r.g_out.qw[f] = fin0(gQ3[j]);
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (gca[q] != 0.f) r.gc[q][f] += fin0(gca[q]);
  }
  block_sum_to<3>(acc, r.scal + G_LAMBDA);
}

// Blocked reverse configurations: id -> (iterations per launch, tile, threads).
// One CTA per SM (registers and shared memory): 19 covers a 200^2 level
// with 140 tiles, one wave on the 148 SMs, where 17 needs 153; 23 (window
// 32x28, 896 threads at 72 registers, the most that one pixel per thread
// allows) recomputes 1.78 window pixels per tile pixel (22: 1.80, 20: 1.85,
// 11: 1.92) and is the fastest at the 800^2 and 400^2 levels; 24 and 25 are
// three-iteration forms of the same window size.
// One iteration per launch with wider tiles (28x20, 32x18, 24x24 at 864-896
// threads: 1.54 window pixels per tile pixel) measured 1.5x slower at
// 800x800 than these forms: the constants, cotangents and states are then
// loaded and the cotangents of the constants written back once per
// iteration.
#define VFS_REVB_SHAPES(X) \
  X(11, 2, 24, 16, 736)    \
  X(12, 2, 16, 16, 576)    \
  X(13, 3, 16, 16, 736)    \
  X(14, 4, 16, 8, 672)     \
  X(15, 2, 8, 8, 256)      \
  X(16, 4, 8, 8, 512)      \
  X(17, 3, 24, 12, 800)    \
  X(18, 2, 32, 12, 768)    \
  X(19, 3, 20, 15, 800)    \
  X(20, 2, 28, 16, 832)    \
  X(22, 2, 24, 20, 864)    \
  X(23, 2, 24, 21, 896)    \
  X(24, 3, 20, 18, 896)    \
  X(25, 3, 20, 17, 864)

// pdl: may start as a programmatic dependent of the previous launch (only
// when that launch wrote none of the recorded states this one reads before
// its griddepcontrol.wait, i.e. not right after a recomputation).
cudaError_t launch_rev_block(int shape, const RevBlockArgs& r, cudaStream_t s, bool pdl) {
  if (!r.k.dscale || !r.c.rec) return cudaErrorInvalidValue;  // dual-step scales or constant records missing
  switch (shape) {
#define VFS_REVB_L(ID, K, TX, TY, NT)                                              \
  case ID: {                                                                       \
    if (r.niter > K) return cudaErrorInvalidValue;                                 \
    cudaLaunchConfig_t cfg = {};                                                   \
    cfg.gridDim = dim3((r.w + TX - 1) / TX, (r.h + TY - 1) / TY);                  \
    cfg.blockDim = dim3(NT);                                                       \
    cfg.dynamicSmemBytes = RbGeom<K, TX, TY>::smem_bytes();                        \
    cfg.stream = s;                                                                \
    cudaLaunchAttribute at[1];                                                     \
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;                 \
    at[0].val.programmaticStreamSerializationAllowed = 1;                          \
    cfg.attrs = at;                                                                \
    cfg.numAttrs = pdl ? 1 : 0;                                                    \
    return cudaLaunchKernelEx(&cfg, k_rev_block<K, TX, TY, NT>, r);                \
  }
    VFS_REVB_SHAPES(VFS_REVB_L)
#undef VFS_REVB_L
    default: return cudaErrorInvalidValue;
  }
}

int rev_block_iters(int shape) {
  switch (shape) {
#define VFS_REVB_K(id, K, TX, TY, NT) \
  case id: return K;
    VFS_REVB_SHAPES(VFS_REVB_K)
#undef VFS_REVB_K
    default: return 0;
  }
}

cudaError_t prepare_rev_block() {
  cudaError_t e = cudaSuccess;
#define VFS_REVB_P(id, K, TX, TY, NT)                                                                 \
  if (e == cudaSuccess)                                                                               \
    e = cudaFuncSetAttribute(k_rev_block<K, TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             (int)RbGeom<K, TX, TY>::smem_bytes());
  VFS_REVB_SHAPES(VFS_REVB_P)
#undef VFS_REVB_P
  return e;
}

// ---------------------------------------------------------------- warp prologue reversed
// computeDerivatives (Python/vfs.cu:120-142, 304-324) reversed: the
// cotangents of (Iu, Iz) go to the reference level image, the warped image
// and (through the tap direction) the translation field at the pixel.
__global__ void k_g_derivs(const float* __restrict__ giu, const float* __restrict__ giz, Plane<const float2> tvf,
                           Plane<const float> ref, Plane<const float> warped, float* gref, float* gwarped,
                           float2* gtvf, int h, int w) {
  GRAD_PIXEL
  if (!inside) return;
  const float gI = giu[i] * (1.f / 24.f), gZ = giz[i];
  if (gI == 0.f && gZ == 0.f) return;
  const float2 vec = tvf.at(X, Y);
  const float nv = hypotf(vec.x, vec.y);
  const float dxn = vec.x / nv, dyn = vec.y / nv;
  float gdx = 0.f, gdy = 0.f;
  const int ks[4] = {-2, -1, 1, 2};
  const float cs[4] = {1.f, -8.f, 8.f, -1.f};
  if (gI != 0.f) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const float u = X + ks[t] * dxn, v = Y + ks[t] * dyn;
      const Bilin B = bilin(u, v, h, w);
      const float gv = cs[t] * gI;
      scatter1(gref, w, B, gv);
      scatter1(gwarped, w, B, gv);
      const float2 dr = bilin_d1(ref, B), dw = bilin_d1(warped, B);
      gdx += ks[t] * gv * (dr.x + dw.x);
      gdy += ks[t] * gv * (dr.y + dw.y);
    }
  }
  if (gZ != 0.f) {
    atomicAdd(gref + i, -gZ);
    atomicAdd(gwarped + i, gZ);
  }
  const float n3 = nv * nv * nv;
  float2 gt = gtvf[i];
  gt.x += (gdx * vec.y * vec.y - gdy * vec.x * vec.y) / n3;
  gt.y += (gdy * vec.x * vec.x - gdx * vec.x * vec.y) / n3;
  gtvf[i] = gt;
}

// findWarpingVector + warpingImage (Python/vfs.cu:186-202, 283-302) reversed,
// and the start of the warp: u at the start of the warp gets the solver's
// cotangent of its initial u, u_ carries the solver's cotangent of its
// initial u_.
__global__ void k_g_fetches(const float* __restrict__ gwarped, const float2* __restrict__ gtvec,
                            const float2* __restrict__ warp_in, Plane<const float> other, Plane<const float2> tvf,
                            float* gother, float2* gtvf, float2* __restrict__ gwarp, float* __restrict__ gu,
                            float* __restrict__ gub, const float* __restrict__ Gu, const float* __restrict__ Gub, int h,
                            int w) {
  GRAD_PIXEL
  if (!inside) return;
  gu[i] += Gu[i];
  gub[i] = Gub[i];
  const float2 d = warp_in[i];
  const Bilin B = bilin(X + d.x, Y + d.y, h, w);
  float2 gw = gwarp[i];
  const float gv = gwarped[i];
  if (gv != 0.f) {
    scatter1(gother, w, B, gv);
    const float2 dd = bilin_d1(other, B);
    gw.x += gv * dd.x;
    gw.y += gv * dd.y;
  }
  const float2 gt = gtvec[i];
  if (gt.x != 0.f || gt.y != 0.f) {
    scatter2(gtvf, w, B, gt);
    const float2 dd = bilin_d2(tvf, B, gt);
    gw.x += dd.x;
    gw.y += dd.y;
  }
  gwarp[i] = gw;
}

// ---------------------------------------------------------------- per-level reversed
// computeTensorEtaMasked (Python/vfs.cu:228-281) reversed: cotangents of
// (a, b, c, eta) go to the smoothed image (the forward differences at the
// lower-right neighbour) and to alpha0, alpha1, beta, gamma.
__global__ void k_g_tensor(const float* __restrict__ ga_, const float* __restrict__ gb_,
                           const float* __restrict__ gc_, const float* __restrict__ ge0_,
                           const float* __restrict__ ge1_, const float* __restrict__ ge2_,
                           const uint8_t* __restrict__ code, Plane<const float> sm, SolverConsts k, float* gsm,
                           double* scal, int h, int w) {
  GRAD_PIXEL
  float acc[4] = {0.f, 0.f, 0.f, 0.f};  // alpha0, alpha1, beta, gamma
  if (inside && (code[i] & kSelf)) {
    const int x1 = mirror_ix(X + 1, w), y1 = mirror_ix(Y + 1, h);
    const float t11 = sm.at(x1, y1);
    const float g0 = t11 - sm.at(X, y1);
    const float g1 = t11 - sm.at(x1, Y);
    const float ng = hypotf(g0, g1);
    const bool small = ng < k.minGrad;
    const float n0 = small ? 1.f : g0 / ng, n1 = small ? 0.f : g1 / ng;
    const float ngg = ng > 0.f ? powf(ng, k.gamma) : 0.f;
    const float e = expf(-k.beta * ngg);
    const bool live = e > k.minTensor;
    const float wt = live ? e : k.minTensor;
    const float a = wt * n0 * n0 + n1 * n1;
    const float b = wt * n1 * n1 + n0 * n0;
    const float c = wt * n0 * n1 - n0 * n1;
    float ga = ga_[i], gb = gb_[i], gc = gc_[i];
    const float ge0 = ge0_[i], ge1 = ge1_[i], ge2 = ge2_[i];
    const float a11 = k.a11;
    ga += a11 * (ge0 * (2.f * a + 2.f * (a + c)) + ge2 * 2.f * a);
    gb += a11 * (ge0 * (2.f * b + 2.f * (b + c)) + ge1 * 2.f * b);
    gc += a11 * (ge0 * (4.f * c + 2.f * (a + c) + 2.f * (b + c)) + (ge1 + ge2) * 2.f * c);
    const float g_a11 = ge0 * (a * a + b * b + 2.f * c * c + (a + c) * (a + c) + (b + c) * (b + c)) +
                        ge1 * (b * b + c * c) + ge2 * (a * a + c * c);
    acc[1] = g_a11 * 2.f * k.alpha1;
    acc[0] = (ge1 + ge2) * 8.f * k.alpha0;
    const float gw = ga * n0 * n0 + gb * n1 * n1 + gc * n0 * n1;
    const float gn0 = ga * 2.f * wt * n0 + gb * 2.f * n0 + gc * (wt - 1.f) * n1;
    const float gn1 = ga * 2.f * n1 + gb * 2.f * wt * n1 + gc * (wt - 1.f) * n0;
    const float gE = live ? gw * e : 0.f;
    acc[2] = -gE * ngg;
    acc[3] = ng > 0.f ? -gE * k.beta * ngg * logf(ng) : 0.f;
    float gg0 = 0.f, gg1 = 0.f;
    if (!small) {
      const float gng = -gE * k.beta * k.gamma * ngg / ng;
      const float dt = gn0 * n0 + gn1 * n1;
      gg0 = (gn0 - n0 * dt) / ng + gng * n0;
      gg1 = (gn1 - n1 * dt) / ng + gng * n1;
    }
    if (gg0 + gg1 != 0.f) atomicAdd(gsm + (long)y1 * w + x1, gg0 + gg1);
    if (gg0 != 0.f) atomicAdd(gsm + (long)y1 * w + X, -gg0);
    if (gg1 != 0.f) atomicAdd(gsm + (long)Y * w + x1, -gg1);
  }
  block_sum_to<4>(acc, scal + G_ALPHA0);
}

// gaussianMasked (Python/vfs.cu:81-102, 204-226) reversed.
__global__ void k_g_gauss(const float* __restrict__ gsm, Plane<const uint8_t> mask, float* gref, int h, int w) {
  GRAD_PIXEL
  if (!inside || !mask_at(mask, X, Y, h, w)) return;
  const float g = gsm[i];
  if (g == 0.f) return;
#pragma unroll
  for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx) {
      const float wt = (dx == 0 && dy == 0) ? 0.25f : (dx != 0 && dy != 0) ? 0.0625f : 0.125f;
      atomicAdd(gref + (long)mirror_ix(Y + dy, h) * w + mirror_ix(X + dx, w), wt * g);
    }
  }
}

// upSamplingVectorField1 / upSamplingVectorField (Python/vfs.cu:69-79,
// 678-705) reversed: from the fine level's start (u = u_ = up(u), flow =
// up(flow)) to the coarse level's end.
__global__ void k_g_up(const float* __restrict__ gu, const float* __restrict__ gub, const float2* __restrict__ gwarp,
                       float* guc, float2* gwarpc, float scale, int hc, int wc, int h, int w) {
  GRAD_PIXEL
  if (!inside) return;
  const float u = (X + 0.5f) / w * wc - 0.5f, v = (Y + 0.5f) / h * hc - 0.5f;
  const Bilin B = bilin(u, v, hc, wc);
  scatter1(guc, wc, B, scale * (gu[i] + gub[i]));
  const float2 gw = gwarp[i];
  scatter2(gwarpc, wc, B, make_float2(scale * gw.x, scale * gw.y));
}

// downSamplingImage / downSamplingVectorField (Python/vfs.cu:35-49, 171-184)
// reversed: coarse (h, w) cotangents onto the fine (hf, wf) level.
template <int C>
__global__ void k_g_down(const float* __restrict__ gc, float* gf, int hf, int wf, int h, int w) {
  GRAD_PIXEL
  if (!inside) return;
  const float x = (X + 0.5f) / w, y = (Y + 0.5f) / h;
  const float dx = 0.25f / w, dy = 0.25f / h;
  const float xs[4] = {x - dx, x + dx, x, x};
  const float ys[4] = {y, y, y - dy, y + dy};
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const Bilin B = bilin(xs[t] * wf - 0.5f, ys[t] * hf - 0.5f, hf, wf);
    if (C == 1) {
      scatter1(gf, wf, B, 0.25f * gc[i]);
    } else {
      const float2 g = reinterpret_cast<const float2*>(gc)[i];
      scatter2(reinterpret_cast<float2*>(gf), wf, B, make_float2(0.25f * g.x, 0.25f * g.y));
    }
  }
}

// The calibration warp of the second image (Python/vfs.py:130-131) and the
// castAndScale of both images reversed: cotangents onto the input images.
__global__ void k_g_calib(const float* __restrict__ gother0, const float2* __restrict__ cvf, float* gimg, float s,
                          int h, int w) {
  GRAD_PIXEL
  if (!inside) return;
  const float2 d = cvf[i];
  scatter1(gimg, w, bilin(X + d.x, Y + d.y, h, w), s * gother0[i]);
}

// d project / d X for the equidistant camera (Python/equidistant_cam.cuh:32-45).
__device__ __forceinline__ void proj_jac(const Cam& cam, float3 P, float J[2][3]) {
  const float R = hypotf(P.x, P.y);
  const float th = atan2f(R, P.z);
  const float R2Z2 = fmaf(R, R, P.z * P.z);
  const float kk = R > 0.f ? cam.f * th / R : cam.f / P.z;
  float D;
  if (P.z > 0.f && R < 0.05f * P.z) {
    const float s2 = (R / P.z) * (R / P.z);
    D = cam.f / (P.z * P.z * P.z) * (-2.f / 3.f + s2 * (0.8f - s2 * (6.f / 7.f)));
  } else {
    D = cam.f * (P.z * R / R2Z2 - th) / (R * R * R);
  }
  const float dz = -cam.f / R2Z2;
  J[0][0] = fmaf(P.x * D, P.x, kk);
  J[0][1] = P.x * D * P.y;
  J[0][2] = P.x * dz;
  J[1][0] = P.y * D * P.x;
  J[1][1] = fmaf(P.y * D, P.y, kk);
  J[1][2] = P.y * dz;
}

// get_vector_fields' translation field (Python/vector_field.py:28-50)
// reversed to the translation: tvf = normalise((project(P + s t) -
// project(P - s t)) / 2) per pixel.
__global__ void k_g_vf(const float2* __restrict__ gtvf, Cam cam, float3 st, float s, double* scal, int h, int w) {
  GRAD_PIXEL
  float acc[3] = {0.f, 0.f, 0.f};
  if (inside) {
    const float2 g = gtvf[i];
    if (g.x != 0.f || g.y != 0.f) {
      float3 P = cam_unproject(cam, make_float2((float)X, (float)Y));
      const float nn = sqrtf(P.x * P.x + P.y * P.y + P.z * P.z);
      P = make_float3(P.x / nn, P.y / nn, P.z / nn);
      const float3 Pf = make_float3(P.x + st.x, P.y + st.y, P.z + st.z);
      const float3 Pb = make_float3(P.x - st.x, P.y - st.y, P.z - st.z);
      const float2 f = cam_project(cam, Pf), b = cam_project(cam, Pb);
      const float2 tv = make_float2((f.x - b.x) / 2, (f.y - b.y) / 2);
      const float tn = sqrtf(tv.x * tv.x + tv.y * tv.y);
      const float2 d = make_float2(tv.x / tn, tv.y / tn);
      const float dt = g.x * d.x + g.y * d.y;
      const float2 gtv = make_float2((g.x - d.x * dt) / tn * 0.5f * s, (g.y - d.y * dt) / tn * 0.5f * s);
      float Jf[2][3], Jb[2][3];
      proj_jac(cam, Pf, Jf);
      proj_jac(cam, Pb, Jb);
#pragma unroll
      for (int k = 0; k < 3; ++k) acc[k] = gtv.x * (Jf[0][k] + Jb[0][k]) + gtv.y * (Jf[1][k] + Jb[1][k]);
    }
  }
  block_sum_to<3>(acc, scal + G_T0);
}

}  // namespace
}  // namespace vfs

using namespace vfs;

// ---------------------------------------------------------------- host side
struct VfsGradPlan {
  VfsPlan* pl = nullptr;
  int ckpt = 10;
  int nint = 1;  // checkpoint intervals per warp
  Cam cam{};
  double t_scale = 1.0;
  double t[3] = {0, 0, 0};
  std::vector<float> sched;  // host copy of (sigma, tau, mu) per iteration
  bool recorded = false;
  struct Warp {
    float* u_in;
    float* ub_in;
    float2* warp_in;
    std::vector<TgvState> ck;  // state after iterations ckpt, 2 ckpt, ..., nSolverIters
    TgvState* d_seg;           // per checkpoint interval, its states (segment_lists)
  };
  std::vector<std::vector<Warp>> tape;
  float2 *tvf0 = nullptr, *cvf0 = nullptr;
  // backward buffers (level-0 sized, flat)
  std::vector<TgvState> slot;
  TgvState G[2];
  float* A[3];
  float* C[6];
  float* gcp[8];
  float *gu[2], *gub[2], *gwarped, *gsm;
  float2 *gwarp[2], *gtvec;
  std::vector<float*> gref, gother;
  std::vector<float2*> gtvf;
  double* scal = nullptr;
  int fused_reverse = 11;  // reverse-step kernel form (vfs_grad_set_options)
  // instrumentation: an event pair around each interval's reverse launches
  bool timing = false;
  std::vector<cudaEvent_t> tev;
  std::vector<double> tev_bytes;
  std::vector<long long> tev_launches;
  std::vector<int> tev_level;
  int tev_used = 0;
  int level_form[32] = {0};  // per level: 0 = fused_reverse
  int trace_variant = 0;  // 0: the level's forward variant if it records, else 134
  bool tri_lsq = false;   // least-squares triangulation (vfs_grad_set_triangulation)
};

namespace {

constexpr size_t kGAlign = 512;
inline size_t gru(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct GCarver {
  char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t bytes) {
    off = gru(off, kGAlign);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += bytes;
    return p;
  }
};

void take_state(GCarver& cv, TgvState* s, size_t n) {
  float** f[10] = {&s->u, &s->ub, &s->vbx, &s->vby, &s->px, &s->py, &s->qx, &s->qy, &s->qz, &s->qw};
  for (auto* pp : f) *pp = cv.take<float>(n * 4);
}

// Entries of a warp's interval state lists: with ckpt 1 one list of all
// nSolverIters + 1 states, else (ckpt + 1) per interval.
size_t seg_entries(const VfsGradPlan* gp, const VfsParams* p) {
  return gp->ckpt == 1 ? (size_t)p->nSolverIters + 1 : (size_t)gp->nint * (gp->ckpt + 1);
}

std::vector<std::pair<int, int>> level_sizes(const VfsParams* p) {
  std::vector<std::pair<int, int>> s;
  int h = p->height, w = p->width;
  for (int l = 0; l < p->nLevel; ++l) {
    s.push_back({h, w});
    h = (int)(h / p->fScale);
    w = (int)(w / p->fScale);
  }
  return s;
}

// Lays out (or, with base == nullptr, measures) the tape and the backward
// buffers of a gradient plan.
size_t grad_layout(VfsGradPlan* gp, const VfsParams* p, char* base) {
  GCarver cv{base};
  const auto sz = level_sizes(p);
  const size_t n0 = (size_t)sz[0].first * sz[0].second;
  const int nW = std::max(0, p->nWarpIters);
  const int nck = gp->nint;
  gp->tape.assign(sz.size(), {});
  for (size_t l = 0; l < sz.size(); ++l) {
    const size_t n = (size_t)sz[l].first * sz[l].second;
    gp->tape[l].resize(nW);
    for (auto& wt : gp->tape[l]) {
      wt.u_in = cv.take<float>(n * 4);
      wt.ub_in = cv.take<float>(n * 4);
      wt.warp_in = cv.take<float2>(n * 8);
      wt.ck.resize(std::max(0, nck));
      for (auto& s : wt.ck) take_state(cv, &s, n);
      wt.d_seg = cv.take<TgvState>(seg_entries(gp, p) * sizeof(TgvState));
    }
  }
  gp->tvf0 = cv.take<float2>(n0 * 8);
  gp->cvf0 = cv.take<float2>(n0 * 8);
  gp->slot.resize(gp->ckpt + 1);
  for (auto& s : gp->slot) take_state(cv, &s, n0);
  for (auto& s : gp->G) take_state(cv, &s, n0);
  for (auto& a : gp->A) a = cv.take<float>(n0 * 4);
  for (auto& c : gp->C) c = cv.take<float>(n0 * 4);
  for (auto& c : gp->gcp) c = cv.take<float>(n0 * 4);
  for (int b = 0; b < 2; ++b) {
    gp->gu[b] = cv.take<float>(n0 * 4);
    gp->gub[b] = cv.take<float>(n0 * 4);
    gp->gwarp[b] = cv.take<float2>(n0 * 8);
  }
  gp->gwarped = cv.take<float>(n0 * 4);
  gp->gsm = cv.take<float>(n0 * 4);
  gp->gtvec = cv.take<float2>(n0 * 8);
  gp->gref.resize(sz.size());
  gp->gother.resize(sz.size());
  gp->gtvf.resize(sz.size());
  for (size_t l = 0; l < sz.size(); ++l) {
    const size_t n = (size_t)sz[l].first * sz[l].second;
    gp->gref[l] = cv.take<float>(n * 4);
    gp->gother[l] = cv.take<float>(n * 4);
    gp->gtvf[l] = cv.take<float2>(n * 8);
  }
  gp->scal = cv.take<double>(G_NSCAL * sizeof(double));
  return cv.off + kGAlign;
}

int plan_bytes(const VfsParams* p, size_t* b) { return vfs_plan_workspace_size(p, b); }

// The states of checkpoint interval j: its first (the warp's initial state
// or the previous interval's last), those recomputed into the slots, and
// its last (from the tape).
std::vector<TgvState> interval_states(const VfsGradPlan* gp, const VfsGradPlan::Warp& wt, int j, int nI) {
  const int nj = std::max(0, std::min(gp->ckpt, nI - j * gp->ckpt));
  std::vector<TgvState> S(nj + 1);
  S[0] = j == 0 ? gp->slot[0] : wt.ck[j - 1];
  for (int q = 1; q < nj; ++q) S[q] = gp->slot[q];
  if (nj > 0) S[nj] = wt.ck[j];
  return S;
}

// The distance in floats between consecutive state sets v[i0 .. i0 + m),
// when every plane moves by the same amount (the recording kernel's trace
// layout); false if they do not.
bool record_stride(const std::vector<TgvState>& v, int i0, int m, long* stride) {
  *stride = 0;
  if (i0 < 0 || m < 1 || i0 + m > (int)v.size()) return false;
  if (m == 1) return true;
  const long d = v[i0 + 1].u - v[i0].u;
  for (int r = i0; r + 1 < i0 + m; ++r) {
    const TgvState &a = v[r], &b = v[r + 1];
    const float* pa[10] = {a.u, a.ub, a.vbx, a.vby, a.px, a.py, a.qx, a.qy, a.qz, a.qw};
    const float* pb[10] = {b.u, b.ub, b.vbx, b.vby, b.px, b.py, b.qx, b.qy, b.qz, b.qw};
    for (int q = 0; q < 10; ++q)
      if (pb[q] - pa[q] != d) return false;
  }
  *stride = d;
  return true;
}

// All interval state lists of a warp, in the layout of Warp::d_seg.
std::vector<TgvState> segment_lists(const VfsGradPlan* gp, const VfsGradPlan::Warp& wt, int nI) {
  std::vector<TgvState> out;
  if (gp->ckpt == 1) {
    out.push_back(gp->slot[0]);
    for (int i = 0; i < nI; ++i) out.push_back(wt.ck[i]);
    return out;
  }
  out.resize((size_t)gp->nint * (gp->ckpt + 1));
  for (int j = 0; j < gp->nint; ++j) {
    const auto S = interval_states(gp, wt, j, nI);
    std::copy(S.begin(), S.end(), out.begin() + (size_t)j * (gp->ckpt + 1));
  }
  return out;
}

int check_grad_params(const VfsParams* p, int ckpt) {
  std::string why;
  if (!valid_params(p, &why)) return fail(VFS_ERR_ARG, why);
  if (ckpt <= 0) return fail(VFS_ERR_ARG, "ckpt_every must be >= 1");
  return VFS_OK;
}

int level_variant_of(VfsPlan* pl, int l) {
  const int v = pl->level_variant[l];
  return (v != 0 && v != VFS_TGV_CLUSTER) ? v : pl->variant;
}

TgvState other_scratch(VfsPlan* pl, const TgvState& cur) {
  return cur.u == pl->st[0].u ? pl->st[1] : pl->st[0];
}

// create_image_pyramid (Python/vfs.py:121-157) from float images already in
// the solver's scale (castAndScale's u8 / 256).
int grad_pyramids(VfsPlan* pl, const float* ref, const float* other, cudaStream_t s) {
  auto& v0 = pl->lv[0];
  k_g_to_plane<<<g2d(v0.h, v0.w), kGB, 0, s>>>(v0.ref, ref, 1.f / 256.f, v0.h, v0.w);
  k_g_to_plane<<<g2d(v0.h, v0.w), kGB, 0, s>>>(pl->other0, other, 1.f / 256.f, v0.h, v0.w);
  VFS_TRY_CUDA(cudaGetLastError(), "image staging");
  for (int l = 1; l < pl->L; ++l)
    VFS_TRY_CUDA(launch_downsample_image(pl->lv[l].ref, pl->lv[l - 1].ref_tex, pl->lv[l].h, pl->lv[l].w, s),
                 "downSamplingImage");
  VFS_TRY_CUDA(launch_warp_image(v0.other, {pl->calib.ptr, pl->calib.pitch}, pl->other0_tex, v0.h, v0.w, s),
               "warpingImage");
  for (int l = 1; l < pl->L; ++l)
    VFS_TRY_CUDA(launch_downsample_image(pl->lv[l].other, pl->lv[l - 1].other_tex, pl->lv[l].h, pl->lv[l].w, s),
                 "downSamplingImage");
  return VFS_OK;
}

void flat_copy_async(void* dst, const void* src, size_t pitch, size_t row_bytes, int h, cudaStream_t s,
                     cudaError_t* e) {
  if (*e == cudaSuccess) *e = cudaMemcpy2DAsync(dst, row_bytes, src, pitch, row_bytes, h, cudaMemcpyDeviceToDevice, s);
}

int grad_forward(VfsGradPlan* gp, const float* img_ref, const float* img_other, float* depth, cudaStream_t s) {
  VfsPlan* pl = gp->pl;
  // vector fields for t (Python/vector_field.py:28-56 with R = I) and their pyramid
  const auto& v0 = pl->lv[0];
  FieldPose pose;
  for (int k = 0; k < 9; ++k) pose.R[k] = (k % 4 == 0) ? 1.f : 0.f;
  for (int k = 0; k < 3; ++k) pose.st_fwd[k] = pose.st_bwd[k] = (float)(gp->t_scale * gp->t[k]);
  VFS_TRY_CUDA(launch_vector_fields(gp->tvf0, gp->cvf0, gp->cam, gp->cam, pose, 0.f, v0.h, v0.w, s), "vector fields");
  VFS_TRY(vfs_plan_set_vector_fields(pl, (const float*)gp->tvf0, (const float*)gp->cvf0, s));
  VFS_TRY(grad_pyramids(pl, img_ref, img_other, s));
  long long nk = 0;
  const int nI = pl->prm.nSolverIters;
  for (int l = pl->L - 1; l >= 0; --l) {
    LevelCtx c;
    VFS_TRY(plan_level_begin(pl, l, &c, s, &nk));
    c.cs = 0;
    c.var = level_variant_of(pl, l);
    c.K = tgv_max_iters_per_launch(c.var);
    const int h = c.h, w = c.w, b = c.b;
    for (int wi = 0; wi < pl->prm.nWarpIters; ++wi) {
      auto& wt = gp->tape[l][wi];
      cudaError_t e = cudaSuccess;
      flat_copy_async(wt.u_in, pl->ubefore[b].ptr, pl->ubefore[b].pitch, (size_t)w * 4, h, s, &e);
      flat_copy_async(wt.ub_in, c.ub_src.ptr, c.ub_src.pitch, (size_t)w * 4, h, s, &e);
      flat_copy_async(wt.warp_in, pl->warp[b].ptr, pl->warp[b].pitch, (size_t)w * 8, h, s, &e);
      VFS_TRY_CUDA(e, "tape copy");
      VFS_TRY(plan_warp_pre(pl, &c, s, &nk));
      TgvState cur = pl->st[0];
      int it = 0;
      if (gp->ckpt == 1 && nI > 0) {
        // every state recorded: the recording form of the blocked kernel
        const int tv = tgv_has_trace(c.var) ? c.var : 134;
        const int K = tgv_max_iters_per_launch(tv);
        while (it < nI) {
          const int m = std::min(K, nI - it);
          long rs;
          if (!record_stride(wt.ck, it, m, &rs)) return fail(VFS_ERR_WORKSPACE, "tape records not evenly spaced");
          VFS_TRY_CUDA(launch_tgv_trace(tv, cur, wt.ck[it], rs, c.cst, pl->sched, it, m, pl->kc, h, w, s), "tgv");
          cur = wt.ck[it + m - 1];
          it += m;
        }
      }
      for (int j = 0; j < gp->nint && it < nI; ++j) {
        const int end = std::min((j + 1) * gp->ckpt, nI);
        while (it < end) {
          const int m = std::min(c.K, end - it);
          const TgvState out = (it + m == end) ? wt.ck[j] : other_scratch(pl, cur);
          VFS_TRY_CUDA(launch_tgv_block(c.var, cur, out, c.cst, pl->sched, it, m, pl->kc, h, w, s), "tgv");
          cur = out;
          it += m;
        }
      }
      VFS_TRY_CUDA(launch_median_clamp({pl->warp[b].ptr, pl->warp[b].pitch}, pl->ubefore[b], {cur.u, (size_t)w * 4},
                                       {pl->tvec.ptr, (size_t)w * 8}, c.mask, pl->kc.upperLimit, h, w, s),
                   "median/clamp");
      c.ub_src = {cur.ub, (size_t)w * 4};
    }
    VFS_TRY(plan_level_end(pl, &c, s, &nk));
  }
  VFS_TRY(plan_finish(pl, s, &nk));
  {
    auto kern = gp->tri_lsq ? k_g_depth<true> : k_g_depth<false>;
    kern<<<g2d(v0.h, v0.w), kGB, 0, s>>>(depth, {pl->warp[0].ptr, pl->warp[0].pitch}, gp->cam, (float)gp->t[0],
                                         (float)gp->t[1], (float)gp->t[2], {v0.mask.ptr, v0.mask.pitch}, v0.h, v0.w);
  }
  VFS_TRY_CUDA(cudaGetLastError(), "depth");
  pl->solved = true;
  return VFS_OK;
}

RevArgs rev_args(VfsGradPlan* gp, const TgvConsts& cst, int it, const SolverConsts& k, int h, int w) {
  RevArgs r;
  r.c = cst;
  for (int q = 0; q < 8; ++q) r.gc[q] = gp->gcp[q];
  for (int q = 0; q < 3; ++q) r.A[q] = gp->A[q];
  for (int q = 0; q < 6; ++q) r.C[q] = gp->C[q];
  r.sigma = gp->sched[3 * it];
  r.tau = gp->sched[3 * it + 1];
  r.mu = gp->sched[3 * it + 2];
  r.k = k;
  r.h = h;
  r.w = w;
  r.scal = gp->scal;
  return r;
}

cudaError_t zero(void* p, size_t bytes, cudaStream_t s) { return cudaMemsetAsync(p, 0, bytes, s); }

cudaError_t zero_state(const TgvState& st, size_t n, cudaStream_t s) {
  float* f[10] = {st.u, st.ub, st.vbx, st.vby, st.px, st.py, st.qx, st.qy, st.qz, st.qw};
  for (float* p : f) {
    cudaError_t e = zero(p, n * 4, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Timing mode: opens an event pair (its first event recorded now) for a
// stretch of launches of level `level` (negative: a recomputation) with the
// given algorithmic bytes and launch count.
int timing_pair(VfsGradPlan* gp, int level, double bytes, long long launches, cudaStream_t s, int* pair) {
  *pair = gp->tev_used++;
  while ((int)gp->tev.size() < 2 * (*pair + 1)) {
    cudaEvent_t e;
    VFS_TRY_CUDA(cudaEventCreate(&e), "event create");
    gp->tev.push_back(e);
  }
  gp->tev_bytes.resize(*pair + 1);
  gp->tev_launches.resize(*pair + 1);
  gp->tev_level.resize(*pair + 1);
  gp->tev_bytes[*pair] = bytes;
  gp->tev_launches[*pair] = launches;
  gp->tev_level[*pair] = level;
  VFS_TRY_CUDA(cudaEventRecord(gp->tev[2 * *pair], s), "event record");
  return VFS_OK;
}

int grad_backward(VfsGradPlan* gp, const float* gdepth, float* g_ref, float* g_other, double* g_scalars,
                  cudaStream_t s) {
  VfsPlan* pl = gp->pl;
  gp->tev_used = 0;
  const int L = pl->L, nW = pl->prm.nWarpIters, nI = pl->prm.nSolverIters;
  const auto& v0 = pl->lv[0];
  const size_t n0 = (size_t)v0.h * v0.w;
  VFS_TRY_CUDA(zero(gp->scal, G_NSCAL * sizeof(double), s), "memset");
  for (int l = 0; l < L; ++l) {
    const size_t n = (size_t)pl->lv[l].h * pl->lv[l].w;
    VFS_TRY_CUDA(zero(gp->gref[l], n * 4, s), "memset");
    VFS_TRY_CUDA(zero(gp->gother[l], n * 4, s), "memset");
    VFS_TRY_CUDA(zero(gp->gtvf[l], n * 8, s), "memset");
  }
  int cb = 0;  // which of the gu/gub/gwarp pairs holds the current level
  VFS_TRY_CUDA(zero(gp->gu[cb], n0 * 4, s), "memset");
  VFS_TRY_CUDA(zero(gp->gub[cb], n0 * 4, s), "memset");
  if (gp->tri_lsq)
    k_g_tri_lsq<<<g2d(v0.h, v0.w), kGB, 0, s>>>(gdepth, {pl->warp[0].ptr, pl->warp[0].pitch}, gp->cam,
                                                 (float)gp->t[0], (float)gp->t[1], (float)gp->t[2],
                                                 {v0.mask.ptr, v0.mask.pitch}, gp->gwarp[cb], gp->scal, v0.h, v0.w);
  else
    k_g_tri<<<g2d(v0.h, v0.w), kGB, 0, s>>>(gdepth, {pl->warp[0].ptr, pl->warp[0].pitch}, gp->cam, (float)gp->t[0],
                                             (float)gp->t[2], {v0.mask.ptr, v0.mask.pitch}, gp->gwarp[cb], gp->scal,
                                             v0.h, v0.w);
  VFS_TRY_CUDA(cudaGetLastError(), "triangulate backward");
  for (int l = 0; l < L; ++l) {
    auto& v = pl->lv[l];
    const int h = v.h, w = v.w;
    const size_t n = (size_t)h * w;
    const Plane<const uint8_t> mask{v.mask.ptr, v.mask.pitch};
    // the level's constants: gaussian + tensor
    VFS_TRY_CUDA(launch_gaussian_masked(pl->smooth, v.ref_tex, mask, h, w, s), "gaussianMasked");
    TgvConsts cst = pl->cst;
    cst.code = v.code;
    VFS_TRY_CUDA(launch_tensor_soa(cst, v.code, v.smooth_tex, mask, pl->kc, h, w, s), "tensor");
    for (int q = 0; q < 6; ++q) VFS_TRY_CUDA(zero(gp->gcp[q], n * 4, s), "memset");
    // recording kernel for the recomputation (0: one iteration per launch)
    int tv = gp->trace_variant;
    if (tv == 0) {
      const int fv = level_variant_of(pl, l);
      tv = tgv_has_trace(fv) ? fv : 134;
    } else if (tv < 0 || !tgv_has_trace(tv)) {
      tv = 0;
    }
    for (int wi = nW - 1; wi >= 0; --wi) {
      auto& wt = gp->tape[l][wi];
      // the warp's tvec, warped image, derivatives and initial state
      VFS_TRY_CUDA(launch_warp_prologue(Plane<float2>{pl->tvec.ptr, (size_t)w * 8}, pl->warped,
                                        {wt.warp_in, (size_t)w * 8}, v.tvf_tex, v.other_tex, h, w, s),
                   "warp prologue");
      VFS_TRY_CUDA(launch_derivs_init(cst, gp->slot[0], {wt.u_in, (size_t)w * 4}, {wt.ub_in, (size_t)w * 4},
                                      v.ref_tex, v.warped_tex, v.tvf_tex, h, w, s),
                   "derivatives");
      VFS_TRY_CUDA(zero(gp->gcp[6], n * 4, s), "memset");
      VFS_TRY_CUDA(zero(gp->gcp[7], n * 4, s), "memset");
      int gi = 0;
      // cotangent of the final state: u from the median/clamp, u_ from the
      // next warp (or zero), v, p, q zero
      const TgvState fin = nI > 0 ? wt.ck[gp->nint - 1] : gp->slot[0];
      VFS_TRY_CUDA(zero_state(gp->G[gi], n, s), "memset");
      k_g_post<<<g2d(h, w), kGB, 0, s>>>(gp->gwarp[cb], gp->gu[cb], gp->G[gi].u, fin.u, wt.u_in, pl->tvec.ptr, mask,
                                          pl->kc.upperLimit, gp->gtvec, h, w);
      VFS_TRY_CUDA(cudaGetLastError(), "median/clamp backward");
      VFS_TRY_CUDA(cudaMemcpyAsync(gp->G[gi].ub, gp->gub[cb], n * 4, cudaMemcpyDeviceToDevice, s), "copy");
      // checkpoint intervals from last to first (with ckpt 1, one interval
      // over the whole tape)
      const int nseg = gp->ckpt == 1 ? (nI > 0 ? 1 : 0) : gp->nint;
      for (int j = nseg - 1; j >= 0; --j) {
        int it0, nj;
        std::vector<TgvState> S;
        const TgvState* dS;
        if (gp->ckpt == 1) {
          it0 = 0;
          nj = nI;
          S = segment_lists(gp, wt, nI);
          dS = wt.d_seg;
        } else {
          it0 = j * gp->ckpt;
          nj = std::max(0, std::min(gp->ckpt, nI - it0));
          S = interval_states(gp, wt, j, nI);
          dS = wt.d_seg + (size_t)j * (gp->ckpt + 1);
          // timing: the recomputation's own event pair, marked by a level of -1 - l
          int rpair = -1;
          if (gp->timing && nj > 1) {
            VFS_TRY(timing_pair(gp, -1 - l, 0.0, 0, s, &rpair));
          }
          if (tv) {
            for (int q = 0; q < nj - 1;) {
              const int m = std::min(tgv_max_iters_per_launch(tv), nj - 1 - q);
              long rs;
              if (!record_stride(gp->slot, q + 1, m, &rs))
                return fail(VFS_ERR_WORKSPACE, "recomputation slots not evenly spaced");
              VFS_TRY_CUDA(launch_tgv_trace(tv, S[q], gp->slot[q + 1], rs, cst, pl->sched, it0 + q, m, pl->kc, h, w, s),
                           "tgv recompute");
              q += m;
            }
          } else {
            for (int q = 1; q < nj; ++q)
              VFS_TRY_CUDA(launch_tgv_block(1, S[q - 1], S[q], cst, pl->sched, it0 + q - 1, 1, pl->kc, h, w, s),
                           "tgv recompute");
          }
          if (rpair >= 0) VFS_TRY_CUDA(cudaEventRecord(gp->tev[2 * rpair + 1], s), "event record");
        }
        const int form = gp->level_form[l] ? gp->level_form[l] : gp->fused_reverse;
        const int Kr = rev_block_iters(form);
        int pair = -1;
        if (gp->timing && nj > 0) {
          // algorithmic bytes of one reversed iteration, per pixel: the state
          // before (40) and the p, q after it (24), the cotangent in (40) and
          // out (40), the constants (33), the constant cotangents read and
          // written (64)
          VFS_TRY(timing_pair(gp, l, 241.0 * (double)n * nj, Kr > 0 ? (nj + Kr - 1) / Kr : (form ? nj : 3 * nj), s,
                              &pair));
        }
        if (Kr > 0) {
          for (int i1 = nj; i1 > 0;) {
            const int kk = std::min(Kr, i1);
            RevBlockArgs rb;
            rb.states = dS + (i1 - kk);
            rb.g_in = gp->G[gi];
            rb.g_out = gp->G[gi ^ 1];
            rb.c = cst;
            for (int q = 0; q < 8; ++q) rb.gc[q] = gp->gcp[q];
            rb.sched = pl->sched;
            rb.i0 = it0 + i1 - kk;
            rb.niter = kk;
            rb.k = pl->kc;
            rb.h = h;
            rb.w = w;
            rb.scal = gp->scal;
            // right after a recomputation the states were just written
            VFS_TRY_CUDA(launch_rev_block(form, rb, s, !(gp->ckpt > 1 && i1 == nj)), "tgv backward");
            gi ^= 1;
            i1 -= kk;
          }
          if (pair >= 0) VFS_TRY_CUDA(cudaEventRecord(gp->tev[2 * pair + 1], s), "event record");
          continue;
        }
        for (int q = nj - 1; q >= 0; --q) {
          RevArgs r = rev_args(gp, cst, it0 + q, pl->kc, h, w);
          r.s0 = S[q];
          r.s1 = S[q + 1];
          r.g1 = gp->G[gi];
          r.g0 = gp->G[gi ^ 1];
          if (form) {
            VFS_TRY_CUDA(launch_rev_tile(form, r, s), "tgv backward");
          } else {
            k_rev1<<<g2d(h, w), kGB, 0, s>>>(r);
            k_rev2<<<g2d(h, w), kGB, 0, s>>>(r);
            k_rev3<<<g2d(h, w), kGB, 0, s>>>(r);
            VFS_TRY_CUDA(cudaGetLastError(), "tgv backward");
          }
          gi ^= 1;
        }
        if (pair >= 0) VFS_TRY_CUDA(cudaEventRecord(gp->tev[2 * pair + 1], s), "event record");
      }
      // derivatives, then the fetches of tvec and the warped image
      VFS_TRY_CUDA(zero(gp->gwarped, n * 4, s), "memset");
      k_g_derivs<<<g2d(h, w), kGB, 0, s>>>(gp->gcp[6], gp->gcp[7], {v.tvf.ptr, v.tvf.pitch}, {v.ref.ptr, v.ref.pitch},
                                            {pl->warped.ptr, pl->warped.pitch}, gp->gref[l], gp->gwarped, gp->gtvf[l],
                                            h, w);
      k_g_fetches<<<g2d(h, w), kGB, 0, s>>>(gp->gwarped, gp->gtvec, wt.warp_in, {v.other.ptr, v.other.pitch},
                                             {v.tvf.ptr, v.tvf.pitch}, gp->gother[l], gp->gtvf[l], gp->gwarp[cb],
                                             gp->gu[cb], gp->gub[cb], gp->G[gi].u, gp->G[gi].ub, h, w);
      VFS_TRY_CUDA(cudaGetLastError(), "warp prologue backward");
    }
    // tensor and gaussian
    VFS_TRY_CUDA(zero(gp->gsm, n * 4, s), "memset");
    k_g_tensor<<<g2d(h, w), kGB, 0, s>>>(gp->gcp[0], gp->gcp[1], gp->gcp[2], gp->gcp[3], gp->gcp[4], gp->gcp[5],
                                          v.code, {pl->smooth.ptr, pl->smooth.pitch}, pl->kc, gp->gsm, gp->scal, h, w);
    k_g_gauss<<<g2d(h, w), kGB, 0, s>>>(gp->gsm, mask, gp->gref[l], h, w);
    VFS_TRY_CUDA(cudaGetLastError(), "tensor backward");
    if (l + 1 < L) {
      auto& vc = pl->lv[l + 1];
      const size_t nc = (size_t)vc.h * vc.w;
      const int nb = cb ^ 1;
      VFS_TRY_CUDA(zero(gp->gu[nb], nc * 4, s), "memset");
      VFS_TRY_CUDA(zero(gp->gub[nb], nc * 4, s), "memset");
      VFS_TRY_CUDA(zero(gp->gwarp[nb], nc * 8, s), "memset");
      k_g_up<<<g2d(h, w), kGB, 0, s>>>(gp->gu[cb], gp->gub[cb], gp->gwarp[cb], gp->gu[nb], gp->gwarp[nb],
                                        pl->kc.fscale, vc.h, vc.w, h, w);
      VFS_TRY_CUDA(cudaGetLastError(), "upsampling backward");
      cb = nb;
    }
  }
  // pyramids, coarse to fine
  for (int l = L - 1; l >= 1; --l) {
    const auto& f = pl->lv[l - 1];
    const auto& c = pl->lv[l];
    k_g_down<1><<<g2d(c.h, c.w), kGB, 0, s>>>(gp->gref[l], gp->gref[l - 1], f.h, f.w, c.h, c.w);
    k_g_down<1><<<g2d(c.h, c.w), kGB, 0, s>>>(gp->gother[l], gp->gother[l - 1], f.h, f.w, c.h, c.w);
    k_g_down<2><<<g2d(c.h, c.w), kGB, 0, s>>>((const float*)gp->gtvf[l], (float*)gp->gtvf[l - 1], f.h, f.w, c.h,
                                               c.w);
  }
  VFS_TRY_CUDA(cudaGetLastError(), "pyramid backward");
  k_g_scale<<<g2d(v0.h, v0.w), kGB, 0, s>>>(g_ref, gp->gref[0], 1.f / 256.f, v0.h, v0.w);
  VFS_TRY_CUDA(zero(g_other, n0 * 4, s), "memset");
  k_g_calib<<<g2d(v0.h, v0.w), kGB, 0, s>>>(gp->gother[0], gp->cvf0, g_other, 1.f / 256.f, v0.h, v0.w);
  const float3 st = make_float3((float)(gp->t_scale * gp->t[0]), (float)(gp->t_scale * gp->t[1]),
                                (float)(gp->t_scale * gp->t[2]));
  k_g_vf<<<g2d(v0.h, v0.w), kGB, 0, s>>>(gp->gtvf[0], gp->cam, st, (float)gp->t_scale, gp->scal, v0.h, v0.w);
  VFS_TRY_CUDA(cudaGetLastError(), "input backward");
  VFS_TRY_CUDA(cudaMemcpyAsync(g_scalars, gp->scal, G_NSCAL * sizeof(double), cudaMemcpyDeviceToDevice, s),
               "scalar copy");
  return VFS_OK;
}

}  // namespace

extern "C" {

int vfs_grad_workspace_size(const VfsParams* prm, int ckpt_every, size_t* bytes) {
  VFS_TRY(check_grad_params(prm, ckpt_every));
  if (!bytes) return fail(VFS_ERR_ARG, "bytes is NULL");
  size_t pb = 0;
  VFS_TRY(plan_bytes(prm, &pb));
  VfsGradPlan tmp;
  tmp.ckpt = ckpt_every;
  tmp.nint = std::max(1, (prm->nSolverIters + ckpt_every - 1) / ckpt_every);
  *bytes = gru(pb, kGAlign) + grad_layout(&tmp, prm, nullptr);
  return VFS_OK;
}

int vfs_grad_create(const VfsParams* prm, int ckpt_every, float f, float u0, float v0, double t_scale,
                    void* workspace, size_t workspace_bytes, VfsGradPlan** out) {
  VFS_TRY(check_grad_params(prm, ckpt_every));
  if (!out) return fail(VFS_ERR_ARG, "out is NULL");
  if (!(f > 0.f) || !std::isfinite(t_scale)) return fail(VFS_ERR_ARG, "camera focal length must be > 0");
  size_t need = 0, pb = 0;
  VFS_TRY(vfs_grad_workspace_size(prm, ckpt_every, &need));
  VFS_TRY(plan_bytes(prm, &pb));
  if (!workspace || workspace_bytes < need)
    return fail(VFS_ERR_WORKSPACE, "workspace of " + std::to_string(need) + " bytes required");
  VfsGradPlan* gp = new (std::nothrow) VfsGradPlan();
  if (!gp) return fail(VFS_ERR_ARG, "out of host memory");
  char* base = reinterpret_cast<char*>(workspace);
  int rc = vfs_plan_create(prm, base, pb, &gp->pl);
  if (rc != VFS_OK) {
    delete gp;
    return rc;
  }
  gp->ckpt = ckpt_every;
  gp->nint = std::max(1, (prm->nSolverIters + ckpt_every - 1) / ckpt_every);
  gp->cam = Cam{f, u0, v0};
  gp->t_scale = t_scale;
  gp->sched.assign(3 * std::max(1, prm->nSolverIters), 0.f);
  step_schedule(prm->nSolverIters, prm->timeStepLambda, gp->sched.data());
  char* gbase = reinterpret_cast<char*>(gru(reinterpret_cast<uintptr_t>(base + gru(pb, kGAlign)), kGAlign));
  grad_layout(gp, prm, gbase);
  cudaError_t e = cudaSuccess;
  for (auto& lvl : gp->tape)
    for (auto& wt : lvl) {
      if (e == cudaSuccess) {
        const std::vector<TgvState> seg = segment_lists(gp, wt, prm->nSolverIters);
        e = cudaMemcpy(wt.d_seg, seg.data(), seg.size() * sizeof(TgvState), cudaMemcpyHostToDevice);
      }
    }
  if (e == cudaSuccess) e = prepare_rev_block();
  if (e == cudaSuccess) e = prepare_rev_tile();
  if (e != cudaSuccess) {
    vfs_grad_destroy(gp);
    return cuda_status(e, "gradient plan setup");
  }
  *out = gp;
  return VFS_OK;
}

int vfs_grad_destroy(VfsGradPlan* gp) {
  if (!gp) return VFS_OK;
  for (auto e : gp->tev) cudaEventDestroy(e);
  vfs_plan_destroy(gp->pl);
  delete gp;
  return VFS_OK;
}

VfsPlan* vfs_grad_plan(VfsGradPlan* gp) { return gp ? gp->pl : nullptr; }

int vfs_grad_set_timing(VfsGradPlan* gp, int enable) {
  if (!gp) return fail(VFS_ERR_ARG, "plan is NULL");
  gp->timing = enable != 0;
  return VFS_OK;
}

int vfs_grad_stats(VfsGradPlan* gp, VfsSolveStats* out) {
  if (!gp || !out) return fail(VFS_ERR_ARG, "NULL argument");
  memset(out, 0, sizeof(*out));
  if (!gp->timing) return VFS_OK;
  for (int i = 0; i < gp->tev_used; ++i) {
    float t = 0;
    VFS_TRY_CUDA(cudaEventElapsedTime(&t, gp->tev[2 * i], gp->tev[2 * i + 1]), "event elapsed (synchronise first)");
    const int lvl = gp->tev_level[i];
    if (lvl < 0) {  // a recomputation
      out->recompute_ms += t;
      continue;
    }
    out->tgv_ms += t;
    out->tgv_alg_bytes += gp->tev_bytes[i];
    out->tgv_launches += gp->tev_launches[i];
    if (lvl < 16) out->tgv_ms_level[lvl] += t;
  }
  out->tgv_intervals = gp->tev_used;
  return VFS_OK;
}

int vfs_grad_set_level_form(VfsGradPlan* gp, int level, int form) {
  if (!gp) return fail(VFS_ERR_ARG, "plan is NULL");
  if (level < 0 || level >= gp->pl->L) return fail(VFS_ERR_ARG, "level out of range");
  if (form != 0 && !rev_shape_ok(form) && rev_block_iters(form) == 0)
    return fail(VFS_ERR_ARG, "unknown reverse kernel form");
  gp->level_form[level] = form;
  return VFS_OK;
}

int vfs_grad_set_triangulation(VfsGradPlan* gp, int lsq) {
  if (!gp) return fail(VFS_ERR_ARG, "plan is NULL");
  if (lsq != 0 && lsq != 1) return fail(VFS_ERR_ARG, "triangulation: 0 (reference) or 1 (least squares)");
  gp->tri_lsq = lsq == 1;
  gp->recorded = false;  // the recorded depth came from the other rule
  return VFS_OK;
}

int vfs_grad_set_options(VfsGradPlan* gp, int fused_reverse, int trace_variant) {
  if (!gp) return fail(VFS_ERR_ARG, "plan is NULL");
  if (trace_variant > 0 && !tgv_has_trace(trace_variant))
    return fail(VFS_ERR_ARG, "variant has no recording form");
  if (fused_reverse != 0 && !rev_shape_ok(fused_reverse) && rev_block_iters(fused_reverse) == 0)
    return fail(VFS_ERR_ARG, "unknown reverse kernel form");
  gp->fused_reverse = fused_reverse;
  gp->trace_variant = trace_variant;
  return VFS_OK;
}

int vfs_grad_forward(VfsGradPlan* gp, const float* img_ref, const float* img_other, const double* t,
                     const double* theta, float* depth_out, void* stream) {
  if (!gp || !img_ref || !img_other || !t || !theta || !depth_out) return fail(VFS_ERR_ARG, "NULL argument");
  VfsPlan* pl = gp->pl;
  if (!pl->mask_set) return fail(VFS_ERR_STATE, "set the mask (vfs_plan_set_mask on vfs_grad_plan) first");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(t[k])) return fail(VFS_ERR_ARG, "t must be finite");
  for (int k = 0; k < 5; ++k)
    if (!std::isfinite(theta[k])) return fail(VFS_ERR_ARG, "theta must be finite");
  VfsParams p = pl->prm;
  p.Lambda = theta[0];
  p.alpha0 = theta[1];
  p.alpha1 = theta[2];
  p.beta = theta[3];
  p.gamma = theta[4];
  pl->prm = p;
  pl->kc = make_consts(&p);
  pl->drop_graph();
  VFS_TRY_CUDA(plan_set_dual_scales(pl, (cudaStream_t)stream ? (cudaStream_t)stream : cudaStreamLegacy),
               "dual-step scales");
  for (int k = 0; k < 3; ++k) gp->t[k] = t[k];
  gp->recorded = false;
  VFS_TRY(grad_forward(gp, img_ref, img_other, depth_out, (cudaStream_t)stream));
  gp->recorded = true;
  return VFS_OK;
}

int vfs_grad_backward(VfsGradPlan* gp, const float* g_depth, float* g_ref, float* g_other, double* g_scalars,
                      void* stream) {
  if (!gp || !g_depth || !g_ref || !g_other || !g_scalars) return fail(VFS_ERR_ARG, "NULL argument");
  if (!gp->recorded) return fail(VFS_ERR_STATE, "backward needs vfs_grad_forward first");
  return grad_backward(gp, g_depth, g_ref, g_other, g_scalars, (cudaStream_t)stream);
}

}  // extern "C"
