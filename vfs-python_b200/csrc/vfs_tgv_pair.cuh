// Two-pixel lockstep variant of the temporally blocked TGV kernel (included
// by vfs_tgv.cu; same geometry, same flat addressing, same per-pixel results).
//
// Thread t owns window pixels e0 = t and e1 = t + NT and carries them through
// every step together, as the two lanes of float2 values: on sm_100 one
// FFMA2/FADD2/FMUL2 instruction performs the fused multiply-add / add /
// multiply of both lanes, each rounded exactly as the scalar instruction, so
// the arithmetic of the solver step costs half the instructions of a
// pixel-per-lane formulation while producing the same bits.
//
// Shared memory holds "pair records": the value of a quantity for both
// pixels of a thread side by side, so one 8- or 16-byte access loads both
// lanes of one or two quantities straight into a register pair.  The flat
// neighbour of a thread's pixels (e +- 1, e +- WX) is the same lane of the
// record of thread t +- 1 or t +- WX, except across the seam between the two
// halves of the window (t + 1 == NT, t + WX >= NT, t == 0, t < WX), where the
// neighbour is the other lane of the record at t +- 1 -+ NT; those loads take
// the other lane (a register move in the few threads concerned).
//
// Which pixels a step computes: the tile's cone of dependence shrinks by
// (2, 1) pixels per iteration (vfs_tgv.cu).  A thread computes both of its
// pixels whenever either is inside the current region; a pixel outside the
// region gets a value that nothing inside any later region reads, so it may
// be anything.  Pixels whose mask code is not "unmasked with all four
// neighbours unmasked" (masked pixels, the pixels along the mask border,
// pixels outside the image) take the scalar per-pixel functions of
// vfs_pixel.cuh lane by lane; the packed path handles the interior.
//
// Division.  tau / eta (eta a per-level constant of each pixel) and rho / dIu
// use r = RN(1 / y), formed once per level (eta) or per warp (dIu), and two
// corrections (Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990): q0 = RN(x r) is
// within 1.5 ulp of x / y, q1 = RN(q0 + (x - y q0) r) within an ulp, and
// q2 = RN(q1 + (x - y q1) r) is the correctly rounded quotient RN(x / y),
// the IEEE division's result, provided x, y, the quotient and the remainders
// are normal numbers.  The kernel uses it only where 2^-60 <= |x|, |y| <= 2^60
// (tau from the host's schedule is checked per iteration, rho per pixel, and
// the reciprocal of an eta or dIu outside the range is stored as NaN); any
// lane whose fast quotient is NaN is divided with '/' instead, which also
// covers NaN inputs.
#pragma once

namespace vfs {
namespace {

__device__ __forceinline__ float2 f2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b: one rounding of a + (-1 * b), the product being exact
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.f), a); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// RN(x / y) of both lanes from ny = -y and r = RN(1 / y), for x and y in
// the reciprocal range (see the file comment); the callers route other
// operands to '/'.
__device__ __forceinline__ float2 pdiv(float2 x, float2 ny, float2 r) {
  const float2 q0 = pmul(x, r);
  const float2 e0 = pfma(q0, ny, x);
  const float2 q1 = pfma(e0, r, q0);
  const float2 e1 = pfma(q1, ny, x);
  return pfma(e1, r, q1);
}

// How the reference's threshold step rounds its multiply-adds (the compiler
// fuses some of them into FMAs), established on a B200 against
// threshold_px (bit-exact with the reference kernel) over 4M random pixels
// covering all three shrink cases: uTauGtp = u_ + tauEtaU (gx + gy) and
// rho = dIu (uTauGtp - u) + dIz are fused, while in uTauGtp - u +- lambda
// tauEtaU dIu the product lambda tauEtaU dIu is rounded on its own (it is
// shared with the bound lambda tauEtaU dIu dIu).
constexpr bool kFuseUT = true, kFuseRho = true, kFuseLo = false, kFuseHi = false;

template <int K, int TX, int TY>
struct PairGeom {
  static constexpr int WX = TX + 3 * K;
  static constexpr int WY = TY + 3 * K;
  static constexpr int N = WX * WY;
};

// Shared-memory pair records of NT threads.
template <int NT>
struct PairSmem {
  float4* base;
  // (u_0, u_1, vx0, vx1), (vy0, vy1, -, -): the bar variables
  __device__ __forceinline__ float4& uvA(int t) const { return base[t]; }
  __device__ __forceinline__ float2& uvB(int t) const { return reinterpret_cast<float2*>(base + NT)[2 * t]; }
  // (qx0, qx1, qy0, qy1), (qz0, qz1, qw0, qw1)
  __device__ __forceinline__ float4& qA(int t) const { return base[2 * NT + t]; }
  __device__ __forceinline__ float4& qB(int t) const { return base[3 * NT + t]; }
  // (tpx0, tpx1, tpy0, tpy1)
  __device__ __forceinline__ float4& tp(int t) const { return base[4 * NT + t]; }
  // (-eta'.x0, -eta'.x1, rx0, rx1), the same for eta.y, eta.z, and
  // (-dIu0, -dIu1, riu0, riu1)
  __device__ __forceinline__ float4& cE(int t) const { return base[5 * NT + t]; }
  __device__ __forceinline__ float4& cY(int t) const { return base[6 * NT + t]; }
  __device__ __forceinline__ float4& cZ(int t) const { return base[7 * NT + t]; }
  __device__ __forceinline__ float4& cU(int t) const { return base[8 * NT + t]; }
  static constexpr int kRecords = 9;
};

template <int K, int TX, int TY>
constexpr size_t pair_smem_bytes(int nt) {
  return (size_t)PairSmem<1>::kRecords * nt * 16 + 5 * K * sizeof(float);
}

// The last phase (1-based: the dual step of iteration s is phase 2s-1, its
// threshold and primal steps phase 2s) whose region contains window pixel
// (wx, wy) when the launch runs k iterations; 0 if none.  The regions are
// nested, so a pixel takes part in phases 1 .. last.
template <int K, int TX, int TY>
__device__ __forceinline__ int last_phase(int wx, int wy, int k) {
  int last = 0;
  for (int s = 1; s <= k; ++s) {
    const int lo_d = 2 * K - 2 * (k - s) - 1, lo_p = lo_d + 1;
    const int hiX = 2 * K + TX + (k - s), hiY = 2 * K + TY + (k - s);
    if (wx >= lo_d && wx < hiX && wy >= lo_d && wy < hiY) last = 2 * s - 1;
    if (wx >= lo_p && wx < hiX && wy >= lo_p && wy < hiY) last = 2 * s;
  }
  return last;
}

// The dual step lane by lane with the scalar per-pixel function (pixels
// that are masked or beside masked ones), reading the pair records of the
// thread and its four neighbours.  Out of line, so that its registers do not
// weigh on the packed path.
template <int NT, int WX>
__device__ __noinline__ void pair_dual_lanes(const PairSmem<NT> S, int t, unsigned info, float2 ra, float2 rb, float2 rc,
                                             float scaleP, float scaleQ, float2& px, float2& py, float2& tpx,
                                             float2& tpy, float2& qx, float2& qy, float2& qz, float2& qw) {
  const bool seamE = t + 1 == NT, seamS = t + WX >= NT, seamW = t == 0, seamN = t < WX;
  const int tE = seamE ? 0 : t + 1, tS = seamS ? t + WX - NT : t + WX;
  const int tW = seamW ? NT - 1 : t - 1, tN = seamN ? t + NT - WX : t - WX;
  auto uv_lane = [&](int r, int lane) {
    const float4 a = S.uvA(r);
    const float2 b = S.uvB(r);
    return lane ? make_float3(a.y, a.w, b.y) : make_float3(a.x, a.z, b.x);
  };
#pragma unroll 1
  for (int j = 0; j < 2; ++j) {
    const uint8_t cd = (uint8_t)(info >> (8 * j) & 31u);
    float2 p = make_float2(j ? px.y : px.x, j ? py.y : py.x), tp = make_float2(0.f, 0.f);
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    if (cd & kSelf) {
      const int lE = seamE ? 1 : j, lS = seamS ? 1 : j, lW = seamW ? 0 : j, lN = seamN ? 0 : j;
      const float3 c = uv_lane(t, j), cE = uv_lane(tE, lE), cW = uv_lane(tW, lW);
      const float3 cS = uv_lane(tS, lS), cN = uv_lane(tN, lN);
      const float4 qa = S.qA(t), qb = S.qB(t);
      q = j ? make_float4(qa.y, qa.w, qb.y, qb.w) : make_float4(qa.x, qa.z, qb.x, qb.z);
      dual_px(cd, c.x, make_float2(c.y, c.z), cE.x, make_float2(cE.y, cE.z), cW.x, make_float2(cW.y, cW.z), cS.x,
              make_float2(cS.y, cS.z), cN.x, make_float2(cN.y, cN.z),
              j ? make_float3(ra.y, rb.y, rc.y) : make_float3(ra.x, rb.x, rc.x), scaleP, scaleQ, &p, &tp, &q);
    } else {
      p = make_float2(0.f, 0.f);
    }
    if (j) px.y = p.x, py.y = p.y, tpx.y = tp.x, tpy.y = tp.y, qx.y = q.x, qy.y = q.y, qz.y = q.z, qw.y = q.w;
    else px.x = p.x, py.x = p.y, tpx.x = tp.x, tpy.x = tp.y, qx.x = q.x, qy.x = q.y, qz.x = q.z, qw.x = q.w;
  }
}

// The threshold and primal steps lane by lane (see pair_dual_lanes).
template <int NT, int WX>
__device__ __noinline__ void pair_primal_lanes(const PairSmem<NT> S, int t, unsigned info, float2 ra, float2 rb,
                                               float2 rc, float2 iu, float2 iz, float2 u, float2 px, float2 py,
                                               float tau, float mu, float lambda, float alpha0, float alpha1,
                                               float2& un, float2& uo, float2& vxo, float2& vyo) {
  const bool seamW = t == 0, seamN = t < WX;
  const int tW = seamW ? NT - 1 : t - 1, tN = seamN ? t + NT - WX : t - WX;
  auto rec_lane = [](float4 r, int lane) { return lane ? r.y : r.x; };
  auto rec_lane2 = [](float4 r, int lane) { return lane ? r.w : r.z; };
#pragma unroll 1
  for (int j = 0; j < 2; ++j) {
    const uint8_t cd = (uint8_t)(info >> (8 * j) & 31u);
    float unj = 0.f, uoj = 0.f;
    float2 vo = make_float2(0.f, 0.f);
    if (cd & kSelf) {
      const int lW = seamW ? 0 : j, lN = seamN ? 0 : j;
      // eta' (the records hold -eta') gives the reference's result: where
      // |eta| < eps, eta' = 1 and tau / 1 == tau
      const float3 eta = make_float3(-rec_lane(S.cE(t), j), -rec_lane(S.cY(t), j), -rec_lane(S.cZ(t), j));
      const float4 tc = S.tp(t), tw = S.tp(tW), tn = S.tp(tN);
      const float4 ua = S.uvA(t);
      const float2 ubb = S.uvB(t);
      const float ub = rec_lane(ua, j);
      const float2 vb = make_float2(rec_lane2(ua, j), j ? ubb.y : ubb.x);
      unj = threshold_px(cd, tau, make_float2(rec_lane(tc, j), rec_lane2(tc, j)), make_float2(rec_lane(tw, lW), 0.f),
                         make_float2(0.f, rec_lane2(tn, lN)), j ? u.y : u.x, ub,
                         j ? make_float2(iu.y, iz.y) : make_float2(iu.x, iz.x), eta.x, lambda);
      const float4 qa = S.qA(t), qb = S.qB(t), qwa = S.qA(tW), qwb = S.qB(tW), qna = S.qA(tN), qnb = S.qB(tN);
      primal_px(cd, tau, mu, j ? make_float2(px.y, py.y) : make_float2(px.x, py.x),
                make_float4(rec_lane(qa, j), rec_lane2(qa, j), rec_lane(qb, j), rec_lane2(qb, j)),
                make_float4(rec_lane(qwa, lW), 0.f, 0.f, rec_lane2(qwb, lW)),
                make_float4(0.f, rec_lane2(qna, lN), rec_lane(qnb, lN), 0.f), unj, ub, vb,
                j ? make_float3(ra.y, rb.y, rc.y) : make_float3(ra.x, rb.x, rc.x), eta, alpha0, alpha1, &uoj, &vo);
    }
    if (j) un.y = unj, uo.y = uoj, vxo.y = vo.x, vyo.y = vo.y;
    else un.x = unj, uo.x = uoj, vxo.x = vo.x, vyo.x = vo.y;
  }
}

template <int K, int TX, int TY, int NT>
__device__ __forceinline__ void tgv_pair_tile(const TgvState& in, const TgvState& out, const TgvConsts& cst,
                                              const float3* __restrict__ sched, int it0, int niter,
                                              const SolverConsts& kc, int h, int w, int x0, int y0) {
  using G = PairGeom<K, TX, TY>;
  constexpr int WX = G::WX, N = G::N;
  static_assert(N <= 2 * NT && WX < NT, "window must fit two pixels per thread");
  static_assert(2 * K < 64, "the last phase must fit 6 bits");
  extern __shared__ float4 smem_raw[];
  const PairSmem<NT> S{smem_raw};
  float* const sSch = reinterpret_cast<float*>(smem_raw + PairSmem<NT>::kRecords * NT);

  const int t = threadIdx.x;
  const long n = (long)h * w;
  const long base = (long)(y0 - 2 * K) * w + (x0 - 2 * K);
  const int e0 = t, e1 = t + NT;

  // When launched as a programmatic dependent of the previous TGV launch this
  // CTA may start before that launch ends: the per-warp constants are read
  // first, the state (which that launch writes) only after griddepcontrol.wait.
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  const int k = niter < K ? niter : K;
  if (t < 5 * k) {  // this launch's step sizes and dual-step scales
    const int i = t / 5, c = t - 5 * i;
    sSch[t] = c < 3 ? reinterpret_cast<const float*>(sched + it0 + i)[c]
                    : reinterpret_cast<const float*>(kc.dscale + it0 + i)[c - 3];
  }

  // ---- per-warp constants of both pixels
  float2 ra, rb, rc, iu, iz;
  int code[2];
  int lastP = 0;    // the last phase either pixel takes part in
  bool fdiv = true;  // the reciprocal divisions of the packed path hold for both pixels
  {
    float4 rcp[2];
    float ex[2], ey[2], ez[2];
    const float nan = __int_as_float(0x7fffffff);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int e = j ? e1 : e0;
      const int wy = e / WX, wx = e - wy * WX;
      const long f = base + (long)wy * w + wx;
      const bool ok = e < N && f >= 0 && f < n;
      const float a = ok ? cst.a[f] : 0.f, b = ok ? cst.b[f] : 0.f, c = ok ? cst.c[f] : 0.f;
      const float du = ok ? cst.iu[f] : 0.f, dz = ok ? cst.iz[f] : 0.f;
      if (j) ra.y = a, rb.y = b, rc.y = c, iu.y = du, iz.y = dz;
      else ra.x = a, rb.x = b, rc.x = c, iu.x = du, iz.x = dz;
      ex[j] = eta_used(ok ? cst.ex[f] : 1.f);
      ey[j] = eta_used(ok ? cst.ey[f] : 1.f);
      ez[j] = eta_used(ok ? cst.ez[f] : 1.f);
      // without reciprocal records every division takes '/' (NaN reciprocals)
      rcp[j] = ok && cst.rcp ? cst.rcp[f] : make_float4(nan, nan, nan, nan);
      code[j] = ok ? cst.code[f] : 0;
      if (e < N) lastP = max(lastP, last_phase<K, TX, TY>(wx, wy, k));
      // every eta in the reciprocal range with its reciprocal formed (NaN
      // otherwise), and dIu too unless the reference never divides by it
      fdiv = fdiv && div_range(ex[j]) && div_range(ey[j]) && div_range(ez[j]) && rcp[j].x == rcp[j].x &&
             rcp[j].y == rcp[j].y && rcp[j].z == rcp[j].z &&
             (fabsf(du) < 1E-7f || (div_range(du) && rcp[j].w == rcp[j].w));
    }
    S.cE(t) = make_float4(-ex[0], -ex[1], rcp[0].x, rcp[1].x);
    S.cY(t) = make_float4(-ey[0], -ey[1], rcp[0].y, rcp[1].y);
    S.cZ(t) = make_float4(-ez[0], -ez[1], rcp[0].z, rcp[1].z);
    S.cU(t) = make_float4(-iu.x, -iu.y, rcp[0].w, rcp[1].w);
  }
  // class 0: both pixels unmasked with all four neighbours unmasked and
  // their divisors in the reciprocal range (packed path); 1: both masked
  // (zero state); 2: lane by lane with the scalar per-pixel functions.
  // info bits 0-4 / 8-12: the mask codes, 16-21: the last phase, 30-31: the class.
  const unsigned cls = (code[0] == 0x1F && code[1] == 0x1F && fdiv) ? 0u
                       : (!(code[0] & kSelf) && !(code[1] & kSelf)) ? 1u
                                                                     : 2u;
  const unsigned info = (unsigned)code[0] | (unsigned)code[1] << 8 | (unsigned)lastP << 16 | cls << 30;

  // a tile whose pixels are all masked ends with zero state (masked pixels
  // are written 0 every iteration): write that and skip the iterations
  int live = 0;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int e = j ? e1 : e0;
    const int wy = e / WX, wx = e - wy * WX;
    const int tx = wx - 2 * K, ty = wy - 2 * K;
    if (e < N && tx >= 0 && tx < TX && ty >= 0 && ty < TY && x0 + tx < w && y0 + ty < h && (code[j] & kSelf))
      live = 1;
  }
  live = __syncthreads_or(live);
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  if (!live) {
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int e = j ? e1 : e0;
      const int wy = e / WX, wx = e - wy * WX;
      const int tx = wx - 2 * K, ty = wy - 2 * K;
      if (e >= N || tx < 0 || tx >= TX || ty < 0 || ty >= TY) continue;
      const int X = x0 + tx, Y = y0 + ty;
      if (X >= w || Y >= h) continue;
      const long f = (long)Y * w + X;
      out.u[f] = out.ub[f] = out.vbx[f] = out.vby[f] = out.px[f] = out.py[f] = 0.f;
      out.qx[f] = out.qy[f] = out.qz[f] = out.qw[f] = 0.f;
    }
    return;
  }

  // ---- state of both pixels
  float2 u, px, py;
  {
    float v[2][10];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int e = j ? e1 : e0;
      const int wy = e / WX, wx = e - wy * WX;
      const long f = base + (long)wy * w + wx;
      const bool ok = e < N && f >= 0 && f < n;
      v[j][0] = ok ? in.u[f] : 0.f;
      v[j][1] = ok ? in.ub[f] : 0.f;
      v[j][2] = ok ? in.vbx[f] : 0.f;
      v[j][3] = ok ? in.vby[f] : 0.f;
      v[j][4] = ok ? in.px[f] : 0.f;
      v[j][5] = ok ? in.py[f] : 0.f;
      v[j][6] = ok ? in.qx[f] : 0.f;
      v[j][7] = ok ? in.qy[f] : 0.f;
      v[j][8] = ok ? in.qz[f] : 0.f;
      v[j][9] = ok ? in.qw[f] : 0.f;
    }
    u = make_float2(v[0][0], v[1][0]);
    px = make_float2(v[0][4], v[1][4]);
    py = make_float2(v[0][5], v[1][5]);
    S.uvA(t) = make_float4(v[0][1], v[1][1], v[0][2], v[1][2]);
    S.uvB(t) = make_float2(v[0][3], v[1][3]);
    S.qA(t) = make_float4(v[0][6], v[1][6], v[0][7], v[1][7]);
    S.qB(t) = make_float4(v[0][8], v[1][8], v[0][9], v[1][9]);
  }
  __syncthreads();

  // the bar variables (u_, v_) of a pair record, and across the seam the
  // other lane of the neighbour's record (see the file comment)
  struct UV {
    float2 u, vx, vy;
  };
  auto ld_uv = [&](int r) {
    const float4 a = S.uvA(r);
    return UV{lo2(a), hi2(a), S.uvB(r)};
  };
  auto lane_y_to_x = [](UV& v) { v.u.x = v.u.y, v.vx.x = v.vx.y, v.vy.x = v.vy.y; };
  // (recomputed where used: cheaper than keeping them in registers)
#define VFS_PAIR_NEIGHBOURS                                                              \
  const bool seamE = t + 1 == NT, seamS = t + WX >= NT, seamW = t == 0, seamN = t < WX; \
  const int tE = seamE ? 0 : t + 1, tS = seamS ? t + WX - NT : t + WX;                  \
  const int tW = seamW ? NT - 1 : t - 1, tN = seamN ? t + NT - WX : t - WX;             \
  (void)tE, (void)tS, (void)tW, (void)tN;
  const unsigned cl = info >> 30;
  const int lastPh = (int)(info >> 16 & 63u);

  for (int s = 1; s <= k; ++s) {
    const float* const sc = sSch + 5 * (s - 1);
    const float tau = sc[1], mu = sc[2];
    const float scaleP = sc[3], scaleQ = sc[4];  // alpha1 sigma / etaP, alpha0 sigma / etaQ
    // ---------------------------------------------------------------- dual step
    if (2 * s - 1 <= lastPh) {
      if (cl == 1) {
        px = py = f2(0.f);
        S.tp(t) = make_float4(0.f, 0.f, 0.f, 0.f);
        S.qA(t) = S.qB(t) = make_float4(0.f, 0.f, 0.f, 0.f);
      } else {
        VFS_PAIR_NEIGHBOURS
        float2 tpx, tpy, qx, qy, qz, qw;
        if (cl == 0) {
          UV c = ld_uv(t), cE = ld_uv(tE), cS = ld_uv(tS);
          if (seamE) lane_y_to_x(cE);
          if (seamS) lane_y_to_x(cS);
          const float4 qa = S.qA(t), qb = S.qB(t);
          // updateDualVariables with E and S unmasked (Python/vfs.cu:352-408)
          const float2 gUx = psub(psub(cE.u, c.u), c.vx);
          const float2 gVx = psub(cE.vx, c.vx), gVw = psub(cE.vy, c.vy);
          const float2 gUy = psub(psub(cS.u, c.u), c.vy);
          const float2 gVy = psub(cS.vy, c.vy), gVz = psub(cS.vx, c.vx);
          const float2 tux = pfma(ra, gUx, pmul(rc, gUy)), tuy = pfma(rc, gUx, pmul(rb, gUy));
          float2 upx = pfma(f2(scaleP), tux, px), upy = pfma(f2(scaleP), tuy, py);
          // projection onto the unit ball: a lane with |up|^2 < 0.98 has a norm
          // below 1, so max(hypot, 1) is 1 and up / 1 == up; others as the reference
          const float2 n2 = pfma(upx, upx, pmul(upy, upy));
          if (!(n2.x < 0.98f)) {
            const float nr = fmaxf(hypotf(upx.x, upy.x), 1.0f);
            upx.x = upx.x / nr, upy.x = upy.x / nr;
          }
          if (!(n2.y < 0.98f)) {
            const float nr = fmaxf(hypotf(upx.y, upy.y), 1.0f);
            upx.y = upx.y / nr, upy.y = upy.y / nr;
          }
          px = upx, py = upy;
          tpx = pfma(ra, upx, pmul(rc, upy)), tpy = pfma(rc, upx, pmul(rb, upy));
          qx = pfma(f2(scaleQ), gVx, lo2(qa)), qy = pfma(f2(scaleQ), gVy, hi2(qa));
          qz = pfma(f2(scaleQ), gVz, lo2(qb)), qw = pfma(f2(scaleQ), gVw, hi2(qb));
          const float2 m2 = pfma(qx, qx, pfma(qy, qy, pfma(qz, qz, pmul(qw, qw))));
          if (!(m2.x < 0.98f)) {
            const float nr = fmaxf(norm4df(qx.x, qy.x, qz.x, qw.x), 1.0f);
            qx.x = qx.x / nr, qy.x = qy.x / nr, qz.x = qz.x / nr, qw.x = qw.x / nr;
          }
          if (!(m2.y < 0.98f)) {
            const float nr = fmaxf(norm4df(qx.y, qy.y, qz.y, qw.y), 1.0f);
            qx.y = qx.y / nr, qy.y = qy.y / nr, qz.y = qz.y / nr, qw.y = qw.y / nr;
          }
        } else {
          // lane by lane with the scalar step: masked pixels and pixels
          // beside masked ones (out of line: its registers stay off the packed path)
          pair_dual_lanes<NT, WX>(S, t, info, ra, rb, rc, scaleP, scaleQ, px, py, tpx, tpy, qx, qy, qz, qw);
        }
        S.tp(t) = make_float4(tpx.x, tpx.y, tpy.x, tpy.y);
        S.qA(t) = make_float4(qx.x, qx.y, qy.x, qy.y);
        S.qB(t) = make_float4(qz.x, qz.y, qw.x, qw.y);
      }
    }
    __syncthreads();
    // ------------------------------------------------- threshold + primal steps
    if (2 * s <= lastPh) {
      if (cl == 1) {
        u = f2(0.f);
        S.uvA(t) = make_float4(0.f, 0.f, 0.f, 0.f);
        S.uvB(t) = f2(0.f);
      } else {
        VFS_PAIR_NEIGHBOURS
        float2 un, uo, vxo, vyo;
        if (cl == 0) {
          const float4 tc = S.tp(t);
          float4 tw = S.tp(tW), tn = S.tp(tN);
          if (seamW) tw.y = tw.x;
          if (seamN) tn.w = tn.z;
          const UV c = ld_uv(t);
          const float2 tau2 = f2(tau);
          const bool fast_tau = div_range(tau);
          // l1Thresholding with all four neighbours unmasked (Python/vfs.cu:444-494)
          const float2 gTx = psub(lo2(tc), lo2(tw)), gTy = psub(hi2(tc), hi2(tn));
          const float4 ce = S.cE(t);
          const float2 tauEtaU = fast_tau ? pdiv(tau2, lo2(ce), hi2(ce)) : make_float2(tau / -ce.x, tau / -ce.y);
          const float2 uT = kFuseUT ? pfma(tauEtaU, padd(gTx, gTy), c.u) : padd(c.u, pmul(tauEtaU, padd(gTx, gTy)));
          const float2 d = psub(uT, u);
          const float2 rho = kFuseRho ? pfma(iu, d, iz) : padd(pmul(iu, d), iz);
          const float2 t1 = pmul(f2(kc.lambda), tauEtaU);
          const float2 t2 = pmul(t1, iu);
          const float2 bound = pmul(t2, iu);
          const float4 cu = S.cU(t);
          float2 qr = pdiv(rho, lo2(cu), hi2(cu));
          if (!(div_range(rho.x) && div_range(rho.y))) {
            if (!div_range(rho.x)) qr.x = rho.x / iu.x;
            if (!div_range(rho.y)) qr.y = rho.y / iu.y;
          }
          const float2 dmid = psub(d, qr);
          const float2 dlo = kFuseLo ? pfma(t1, iu, d) : padd(d, t2);
          const float2 dhi = kFuseHi ? pfma(make_float2(-t1.x, -t1.y), iu, d) : psub(d, t2);
          float2 du;
          {
            const float eps = 1E-7f;
            const float mx = fabsf(iu.x) < eps ? d.x : dmid.x, my = fabsf(iu.y) < eps ? d.y : dmid.y;
            du.x = (rho.x <= bound.x && rho.x >= -bound.x) ? mx
                   : rho.x < -bound.x                      ? dlo.x
                   : rho.x > bound.x                       ? dhi.x
                                                           : 0.f;
            du.y = (rho.y <= bound.y && rho.y >= -bound.y) ? my
                   : rho.y < -bound.y                      ? dlo.y
                   : rho.y > bound.y                       ? dhi.y
                                                           : 0.f;
          }
          un = padd(u, du);
          // keeps the primal step's loads below this point (fewer live registers)
          asm volatile("" ::: "memory");
          // updatePrimalVariables with all four neighbours unmasked (Python/vfs.cu:533-569)
          const float4 qa = S.qA(t), qb = S.qB(t);
          float4 qwa = S.qA(tW), qwb = S.qB(tW), qna = S.qA(tN), qnb = S.qB(tN);
          if (seamW) qwa.y = qwa.x, qwb.w = qwb.z;
          if (seamN) qna.w = qna.z, qnb.y = qnb.x;
          const float2 gQx = psub(lo2(qa), lo2(qwa)), gQw = psub(hi2(qb), hi2(qwb));
          const float2 gQy = psub(hi2(qa), hi2(qna)), gQz = psub(lo2(qb), lo2(qnb));
          const float2 tux = pfma(ra, px, pmul(rc, py)), tuy = pfma(rc, px, pmul(rb, py));
          const float4 cy = S.cY(t), cz = S.cZ(t);
          const float2 te1 = fast_tau ? pdiv(tau2, lo2(cy), hi2(cy)) : make_float2(tau / -cy.x, tau / -cy.y);
          const float2 te2 = fast_tau ? pdiv(tau2, lo2(cz), hi2(cz)) : make_float2(tau / -cz.x, tau / -cz.y);
          const float2 Vx = pfma(te1, pfma(f2(kc.alpha1), tux, pmul(f2(kc.alpha0), padd(gQx, gQz))), c.vx);
          const float2 Vy = pfma(te2, pfma(f2(kc.alpha1), tuy, pmul(f2(kc.alpha0), padd(gQw, gQy))), c.vy);
          uo = pfma(f2(mu), psub(un, c.u), un);
          vxo = pfma(f2(mu), psub(Vx, c.vx), Vx), vyo = pfma(f2(mu), psub(Vy, c.vy), Vy);
        } else {
          pair_primal_lanes<NT, WX>(S, t, info, ra, rb, rc, iu, iz, u, px, py, tau, mu, kc.lambda, kc.alpha0,
                                    kc.alpha1, un, uo, vxo, vyo);
        }
        u = un;
        S.uvA(t) = make_float4(uo.x, uo.y, vxo.x, vxo.y);
        S.uvB(t) = vyo;
      }
    }
    __syncthreads();
  }

#undef VFS_PAIR_NEIGHBOURS

  // ---- write back the tile (real pixels only)
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int e = j ? e1 : e0;
    const int wy = e / WX, wx = e - wy * WX;
    const int tx = wx - 2 * K, ty = wy - 2 * K;
    if (e >= N || tx < 0 || tx >= TX || ty < 0 || ty >= TY) continue;
    const int X = x0 + tx, Y = y0 + ty;
    if (X >= w || Y >= h) continue;
    const long f = (long)Y * w + X;
    const float4 uvA = S.uvA(t), qA = S.qA(t), qB = S.qB(t);
    const float2 uvB = S.uvB(t);
    out.u[f] = j ? u.y : u.x;
    out.ub[f] = j ? uvA.y : uvA.x;
    out.vbx[f] = j ? uvA.w : uvA.z;
    out.vby[f] = j ? uvB.y : uvB.x;
    out.px[f] = j ? px.y : px.x;
    out.py[f] = j ? py.y : py.x;
    out.qx[f] = j ? qA.y : qA.x;
    out.qy[f] = j ? qA.w : qA.z;
    out.qz[f] = j ? qB.y : qB.x;
    out.qw[f] = j ? qB.w : qB.z;
  }
}

template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 1)
    k_tgv_pair(TgvState in, TgvState out, TgvConsts cst, const float3* __restrict__ sched, int it0, int niter,
               SolverConsts kc, int h, int w) {
  tgv_pair_tile<K, TX, TY, NT>(in, out, cst, sched, it0, niter, kc, h, w, blockIdx.x * TX, blockIdx.y * TY);
}

// Batched: one launch over the tiles of many images (see k_tgv_reg_batch).
template <int K, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 1)
    k_tgv_pair_batch(const TgvBatchItem* __restrict__ items, int n_items, int parity,
                     const float3* __restrict__ sched, int it0, int niter, SolverConsts kc) {
  int lo = 0, hi = n_items - 1;
  const int bid = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].tile_base <= bid) lo = mid;
    else hi = mid - 1;
  }
  const TgvBatchItem& it = items[lo];
  const int t = bid - it.tile_base;
  const int ty = t / it.tiles_x, tx = t - ty * it.tiles_x;
  tgv_pair_tile<K, TX, TY, NT>(it.st[parity], it.st[parity ^ 1], it.cst, sched, it0, niter, kc, it.h, it.w, tx * TX,
                               ty * TY);
}

}  // namespace
}  // namespace vfs
