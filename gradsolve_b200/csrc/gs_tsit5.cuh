// gs_tsit5.cuh -- adaptive Tsit5 forward with dt record, frozen-mesh replay, and the
// hand-written reverse-replay adjoint (float64).
//
// One thread integrates one trajectory; state, stages and the step-size controller live in
// registers.  The forward follows tsit5_adaptive (gradsolve/solvers/tsit5_replay.py:62-124):
// FSAL reuse of k7 on accept, WRMS error norm sc = atol + rtol*max(|y|,|y5|), accept iff
// err <= 1, dt = h * clip(0.9 * max(err,1e-10)^-0.2, 0.2, 5) after accept AND reject, last
// step clamped to h = min(dt, t1 - t), at most max_steps attempts.
//
// Memory layouts (all in HBM, all 64-bit indexed):
//   y0, y_final, gy0, ybar : (n, D) row-major float64 (the Python API's layout)
//   p, gp                   : (n, P) row-major float64
//   dt record               : chunk-interleaved, 4 steps per 32-byte sector:
//                             step s of trajectory j lives at ((s/4)*n + j)*4 + s%4.
//                             The forward kernels store each accepted dt as it comes (8
//                             bytes into its sector; L2 merges a sector's four writes before
//                             it goes to DRAM -- faster than holding four dt's in registers
//                             and writing the whole sector at once).  Entries past n_acc[j]
//                             in trajectory j's last sector are 0 (identity steps).
//   checkpoints             : slot c of trajectory j = (y after c*K accepted steps, t), at
//                             ((c*n + j) * CW) with CW = D+1 rounded up to even (16-byte
//                             aligned); slot 0 is (y0, t0).  K = ckpt_every.
//
// The adjoint walks each trajectory's record backwards in segments of K steps.  For a
// segment it takes the checkpoint (prefetched into shared memory), recomputes the K-1
// interior states into a per-thread shared-memory buffer, then applies the step VJPs in
// reverse.  Every trajectory runs whole segments
// (n_acc padded up to a multiple of K with dt = 0 identity steps, which are exact
// identities in value and gradient, gradsolve/solvers/tsit5_step.py:84-86), so the lanes of
// a warp stay in the same phase (recompute vs VJP) instead of diverging.  With K = 1 every
// state is a checkpoint and nothing is recomputed.
#pragma once
#include <cmath>

#include "gs_fields.cuh"
#include "gs_tableau.cuh"

namespace gs {

constexpr int KMAX = 64;  // largest checkpoint interval the adjoint supports

// Per-thread segment buffers of the adjoint kernels live in dynamic shared memory: element e
// of thread t sits at smem[e * blockDim + t], so a warp's accesses to one element are
// consecutive 8-byte words (no bank conflicts).  The layouts (AdjBuf, AdjStageBuf, AdjRosBuf)
// are defined with the kernels that use them.
extern __shared__ double gs_seg_smem[];

GS_HD int ckpt_width(int D) { return (D + 2) & ~1; }

GS_HD size_t rec_index(long long j, long long s, long long n) {
  return ((size_t)(s >> 2) * (size_t)n + (size_t)j) * 4u + (size_t)(s & 3);
}

// numpy's add.reduce order for a length-D array (sequential below 8 terms, 8-way pairwise
// from 8 up): the reference's np.mean((e/sc)**2).
template <int D>
__device__ __forceinline__ double wrms_sum(const double* q) {
  if constexpr (D < 8) {
    double s = q[0];
#pragma unroll
    for (int i = 1; i < D; ++i) s += q[i];
    return s;
  } else {
    double r[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = q[j];
    constexpr int full = D - (D % 8);
#pragma unroll
    for (int i = 8; i < full; i += 8)
#pragma unroll
      for (int j = 0; j < 8; ++j) r[j] += q[i + j];
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
#pragma unroll
    for (int i = full; i < D; ++i) res += q[i];
    return res;
  }
}

// ---- the controller from the mean of squares, without pow and sqrt ----------------------
// The reference computes err = sqrt(m) (m = mean((e/sc)^2)), accepts iff err <= 1 and sets
// dt = h * clip(0.9 * max(err, 1e-10)^(-1/q), 0.2, 5) with q = 5 (Tsit5) or 3 (Rosenbrock23).
//  * err <= 1  <=>  m <= 1 + 2^-52: sqrt is correctly rounded, and sqrt(1 + 2^-52) rounds to
//    1 while sqrt(1 + 2^-51) does not, so the accept test is unchanged bit for bit.
//  * 0.9 * err^(-1/q) = 0.9 * m^(-1/(2q)); the clip at 5 (resp. 0.2) is reached for
//    m <= (0.9/5)^(2q) (resp. m >= (0.9/0.2)^(2q)), which also covers the 1e-10 floor.
//  * in between, y = m^(-1/k), k = 2q, is refined from a single-precision first guess y0
//    (exp2(-log2(m)/k), ~2^-21 relative) by one second-order step of the binomial series:
//    with r = 1 - m y0^k (|r| ~ k 2^-21), y = y0 (1 - r)^(-1/k)
//    = y0 (1 + r/k + (k+1)/(2k^2) r^2 + O(r^3)), and the truncated O(r^3) term is below
//    2^-58 relative -- under an ulp, as two Newton iterations y <- y (k + 1 - m y^k) / k
//    (quadratic, ~2^-80) were, for 8 float64 operations instead of 14.
// The result agrees with 0.9 * pow(sqrt(m), -1/q) to a few ulp (checked against CUDA's pow
// by tests/test_gpu_controller.py); the reference's own Warp and numpy paths already differ
// at that level.
constexpr double kAcceptMax = 1.0000000000000002;  // 1 + 2^-52

template <int K>
__device__ __forceinline__ double pow_k(double y) {
  static_assert(K == 6 || K == 10, "inverse root order");
  const double y2 = y * y;
  const double y4 = y2 * y2;
  if constexpr (K == 6) {
    return y4 * y2;
  } else {
    return (y4 * y4) * y2;
  }
}

// The first guess uses the hardware's approximate base-2 logarithm and exponential (PTX
// lg2.approx / ex2.approx, ~2^-22 relative): m lies in the controller's unclipped range
// (about 1e-8 .. 1e8 times D), where neither leaves the normal float range.
__device__ __forceinline__ float lg2_approx(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

template <int K>
__device__ __forceinline__ double inv_root(double m) {
  const double y0 = (double)ex2_approx(lg2_approx((float)m) * (-1.0f / (float)K));
  constexpr double c1 = 1.0 / K, c2 = (K + 1.0) / (2.0 * K * K);
  const double r = fma(-m, pow_k<K>(y0), 1.0);
  return fma(y0, r * fma(c2, r, c1), y0);
}

// The kernels work with the SUM of squares S (m = fl(S / D)), which spares the division by D
// in every attempt.  The constants below are computed on the host (make_ctrl_consts) for the
// field's D and the method's root order K:
//  * accept_sum is the largest double S with fl(S / D) <= 1 + 2^-52; division by D is
//    correctly rounded and monotone, so S <= accept_sum <=> m <= 1 + 2^-52;
//  * 0.9 m^(-1/K) = scale S^(-1/K) with scale = 0.9 D^(1/K); the clips are at D 0.18^K and
//    D 4.5^K.
struct CtrlConsts {
  double accept_sum, lo, hi, scale;
};

__host__ inline CtrlConsts make_ctrl_consts(int D, int K) {
  const double A = kAcceptMax, dd = (double)D;
  double x = A * dd;  // then walk to the last double whose quotient still rounds to <= A
  while (x / dd > A) x = std::nextafter(x, 0.0);
  while (std::nextafter(x, 1e300) / dd <= A) x = std::nextafter(x, 1e300);
  CtrlConsts c;
  c.accept_sum = x;
  c.lo = dd * std::pow(0.18, K);
  c.hi = dd * std::pow(4.5, K);
  c.scale = Ctrl::SAFETY * std::pow(dd, 1.0 / K);
  return c;
}

// The same controller in float (the float32 route; the reference kernel's err = sqrtf(S / D),
// accept iff err <= 1, dt = h * clip(0.9 * max(err, 1e-10)^(-1/q), 0.2, 5), all in float):
//  * sqrtf is correctly rounded and sqrt(1 + 2^-23) = 1 + 2^-24 - 2^-49 rounds to 1 while
//    sqrt(1 + 2^-22) rounds to 1 + 2^-23, so err <= 1 <=> fl(S / D) <= 1 + 2^-23 <=>
//    S <= accept_sum, the largest float whose quotient by D still rounds to <= 1 + 2^-23;
//  * 0.9 * err^(-1/q) = scale * S^(-1/K), K = 2q, scale = 0.9 D^(1/K), from the hardware's
//    approximate lg2 / ex2 directly (a few float ulp; no refinement is needed at float
//    precision); S = 0 or below the 1e-10 floor gives a factor at or above 5 and S = +inf
//    gives 0, which the clip turns into 5 and 0.2 as the reference's max/clip does.
struct CtrlConstsF {
  float accept_sum, scale, inv_k;
};

__host__ inline CtrlConstsF make_ctrl_consts_f32(int D, int K) {
  const float A = 1.0f + 1.1920928955078125e-7f;  // 1 + 2^-23
  const float dd = (float)D;
  float x = A * dd;
  while (x / dd > A) x = std::nextafterf(x, 0.0f);
  while (std::nextafterf(x, 1e30f) / dd <= A) x = std::nextafterf(x, 1e30f);
  CtrlConstsF c;
  c.accept_sum = x;
  c.scale = (float)(Ctrl::SAFETY * std::pow((double)D, 1.0 / K));
  c.inv_k = -1.0f / (float)K;
  return c;
}

__device__ __forceinline__ float step_from_sum_f32(float S, float h, const CtrlConstsF& c) {
  float fac = c.scale * ex2_approx(lg2_approx(S) * c.inv_k);
  fac = fac > (float)Ctrl::FAC_MIN ? fac : (float)Ctrl::FAC_MIN;
  fac = (float)Ctrl::FAC_MAX < fac ? (float)Ctrl::FAC_MAX : fac;
  return h * fac;
}

// K = 10 for Tsit5 (q = 5), K = 6 for Rosenbrock23 (q = 3).  Returns the new dt from the sum
// of squares S.
template <int K>
__device__ __forceinline__ double step_from_sum(double S, double h, const CtrlConsts& c) {
  double fac;
  if (S <= c.lo) {
    fac = Ctrl::FAC_MAX;
  } else if (S >= c.hi) {
    fac = Ctrl::FAC_MIN;
  } else {
    fac = c.scale * inv_root<K>(S);
    fac = fac > Ctrl::FAC_MIN ? fac : Ctrl::FAC_MIN;
    fac = Ctrl::FAC_MAX < fac ? Ctrl::FAC_MAX : fac;
  }
  return h * fac;
}

// sum of squares (e_i / sc_i)^2 in numpy's summation order (the reference's np.mean times D).
// For D <= 4 the D quotients share one division: with P = prod sc_j, e_i / sc_i is taken as
// e_i * ((prod_{j != i} sc_j) / P), within a few ulp of the quotient (the controller and the
// accept test read it at that level only where the reference's own Warp and numpy paths
// already differ), unless P leaves the normal range, where each quotient is divided out.
template <int D>
__device__ __forceinline__ double wrms_sumsq(const double* e, const double* y, const double* yn,
                                             double rtol, double atol) {
  double sc[D], q[D];
#pragma unroll
  for (int i = 0; i < D; ++i) sc[i] = atol + rtol * fmax(fabs(y[i]), fabs(yn[i]));
  bool shared = false;
  if constexpr (D >= 2 && D <= 4) {
    double pre[D], suf[D];  // products of the scales before / after component i
    pre[0] = 1.0;
#pragma unroll
    for (int i = 1; i < D; ++i) pre[i] = pre[i - 1] * sc[i - 1];
    suf[D - 1] = 1.0;
#pragma unroll
    for (int i = D - 2; i >= 0; --i) suf[i] = suf[i + 1] * sc[i + 1];
    const double P = pre[D - 1] * sc[D - 1];
    if (P > 1e-290 && P < 1e290) {
      shared = true;
      const double r = 1.0 / P;
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const double c = e[i] * ((pre[i] * suf[i]) * r);
        q[i] = c * c;
      }
    }
  }
  if (!shared) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const double c = e[i] / sc[i];
      q[i] = c * c;
    }
  }
  return wrms_sum<D>(q);
}

// --- the shared stage arithmetic ------------------------------------------------------
// Stages 2..6 inputs and k2..k6 from (y, k1, h).  Used by the forward, the replay and the
// adjoint's recomputation so every kernel evaluates the same expressions.
template <class F, class R = double>
struct Stages {
  static constexpr int D = F::D;
  R k2[D], k3[D], k4[D], k5[D], k6[D];
};

template <class F, class R = double>
__device__ __forceinline__ void tsit5_k2_to_k6(const R* y, const R* p, const R* k1, R h,
                                               Stages<F, R>& S) {
  constexpr int D = F::D;
  using T = Tsit5;
  R s[D];
#pragma unroll
  for (int i = 0; i < D; ++i) s[i] = y[i] + h * (R(T::A21) * k1[i]);
  F::rhs(s, p, S.k2);
#pragma unroll
  for (int i = 0; i < D; ++i) s[i] = y[i] + h * (R(T::A31) * k1[i] + R(T::A32) * S.k2[i]);
  F::rhs(s, p, S.k3);
#pragma unroll
  for (int i = 0; i < D; ++i)
    s[i] = y[i] + h * (R(T::A41) * k1[i] + R(T::A42) * S.k2[i] + R(T::A43) * S.k3[i]);
  F::rhs(s, p, S.k4);
#pragma unroll
  for (int i = 0; i < D; ++i)
    s[i] = y[i] + h * (R(T::A51) * k1[i] + R(T::A52) * S.k2[i] + R(T::A53) * S.k3[i] + R(T::A54) * S.k4[i]);
  F::rhs(s, p, S.k5);
#pragma unroll
  for (int i = 0; i < D; ++i)
    s[i] = y[i] + h * (R(T::A61) * k1[i] + R(T::A62) * S.k2[i] + R(T::A63) * S.k3[i] + R(T::A64) * S.k4[i] +
                       R(T::A65) * S.k5[i]);
  F::rhs(s, p, S.k6);
}

template <class F, class R = double>
__device__ __forceinline__ void tsit5_y5(const R* y, const R* k1, const Stages<F, R>& S, R h,
                                         R* y5) {
  using T = Tsit5;
#pragma unroll
  for (int i = 0; i < F::D; ++i)
    y5[i] = y[i] + h * (R(T::B1) * k1[i] + R(T::B2) * S.k2[i] + R(T::B3) * S.k3[i] + R(T::B4) * S.k4[i] +
                        R(T::B5) * S.k5[i] + R(T::B6) * S.k6[i]);
}

// One replay step (gradsolve/solvers/tsit5_step.py:80-102).  The B7*k7 term of the
// reference is an exact +0 (B7 == 0), so k7 is not evaluated here.
template <class F, class R = double>
__device__ __forceinline__ void tsit5_replay_step(R* y, const R* p, R dt) {
  constexpr int D = F::D;
  R k1[D], yn[D];
  Stages<F, R> S;
  F::rhs(y, p, k1);
  tsit5_k2_to_k6<F, R>(y, p, k1, dt, S);
  tsit5_y5<F, R>(y, k1, S, dt, yn);
#pragma unroll
  for (int i = 0; i < D; ++i) y[i] = yn[i];
}

// Stage inputs s2..s6 of one step at (y, dt) -- the expressions of tsit5_k2_to_k6 -- and,
// with kNext, the step's result (tsit5_y5), so a pass that keeps the stages for the reverse
// sweep produces the same states as tsit5_replay_step.
template <class F, class R = double>
struct StageStates {
  static constexpr int D = F::D;
  R s2[D], s3[D], s4[D], s5[D], s6[D];
  template <int M>
  __device__ __forceinline__ void get(R* out) const {
    const R* src = M == 2 ? s2 : M == 3 ? s3 : M == 4 ? s4 : M == 5 ? s5 : s6;
#pragma unroll
    for (int i = 0; i < D; ++i) out[i] = src[i];
  }
};

template <class F, bool kNext, class R = double>
__device__ __forceinline__ void tsit5_stage_states(const R* y, const R* p, R dt,
                                                   StageStates<F, R>& S, R* ynext) {
  constexpr int D = F::D;
  using T = Tsit5;
  R k1[D], k2[D], k3[D], k4[D], k5[D];
  F::rhs(y, p, k1);
#pragma unroll
  for (int i = 0; i < D; ++i) S.s2[i] = y[i] + dt * (R(T::A21) * k1[i]);
  F::rhs(S.s2, p, k2);
#pragma unroll
  for (int i = 0; i < D; ++i) S.s3[i] = y[i] + dt * (R(T::A31) * k1[i] + R(T::A32) * k2[i]);
  F::rhs(S.s3, p, k3);
#pragma unroll
  for (int i = 0; i < D; ++i)
    S.s4[i] = y[i] + dt * (R(T::A41) * k1[i] + R(T::A42) * k2[i] + R(T::A43) * k3[i]);
  F::rhs(S.s4, p, k4);
#pragma unroll
  for (int i = 0; i < D; ++i)
    S.s5[i] = y[i] + dt * (R(T::A51) * k1[i] + R(T::A52) * k2[i] + R(T::A53) * k3[i] + R(T::A54) * k4[i]);
  F::rhs(S.s5, p, k5);
#pragma unroll
  for (int i = 0; i < D; ++i)
    S.s6[i] = y[i] + dt * (R(T::A61) * k1[i] + R(T::A62) * k2[i] + R(T::A63) * k3[i] + R(T::A64) * k4[i] +
                           R(T::A65) * k5[i]);
  if (kNext) {
    R k6[D];
    F::rhs(S.s6, p, k6);
#pragma unroll
    for (int i = 0; i < D; ++i)
      ynext[i] = y[i] + dt * (R(T::B1) * k1[i] + R(T::B2) * k2[i] + R(T::B3) * k3[i] + R(T::B4) * k4[i] +
                              R(T::B5) * k5[i] + R(T::B6) * k6[i]);
  }
}

// Reverse of one replay step at (y, dt) given its stage inputs (Src::get<M> yields s_M):
// lam <- (dy'/dy)^T lam, gp += (dy'/dp)^T lam.  Stage 7 carries weight B7 == 0, so its
// cotangent is exactly zero and it is skipped.
template <class F, class Src, class R = double>
__device__ __forceinline__ void tsit5_vjp_core(const R* y, const Src& src, const R* p, R dt,
                                               R* lam, R* gp) {
  constexpr int D = F::D;
  using T = Tsit5;
  R st[D];
  R g[D], kb1[D], kb2[D], kb3[D], kb4[D], kb5[D], kb6[D], sb[D], yb[D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    g[i] = dt * lam[i];
    yb[i] = lam[i];
    kb1[i] = R(T::B1) * g[i];
    kb2[i] = R(T::B2) * g[i];
    kb3[i] = R(T::B3) * g[i];
    kb4[i] = R(T::B4) * g[i];
    kb5[i] = R(T::B5) * g[i];
    kb6[i] = R(T::B6) * g[i];
  }
  // stage 6
  src.template get<6>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = R(0.0);
  F::vjp(st, p, kb6, sb, gp);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    yb[i] += sb[i];
    const R u = dt * sb[i];
    kb1[i] += R(T::A61) * u;
    kb2[i] += R(T::A62) * u;
    kb3[i] += R(T::A63) * u;
    kb4[i] += R(T::A64) * u;
    kb5[i] += R(T::A65) * u;
  }
  // stage 5
  src.template get<5>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = R(0.0);
  F::vjp(st, p, kb5, sb, gp);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    yb[i] += sb[i];
    const R u = dt * sb[i];
    kb1[i] += R(T::A51) * u;
    kb2[i] += R(T::A52) * u;
    kb3[i] += R(T::A53) * u;
    kb4[i] += R(T::A54) * u;
  }
  // stage 4
  src.template get<4>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = R(0.0);
  F::vjp(st, p, kb4, sb, gp);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    yb[i] += sb[i];
    const R u = dt * sb[i];
    kb1[i] += R(T::A41) * u;
    kb2[i] += R(T::A42) * u;
    kb3[i] += R(T::A43) * u;
  }
  // stage 3
  src.template get<3>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = R(0.0);
  F::vjp(st, p, kb3, sb, gp);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    yb[i] += sb[i];
    const R u = dt * sb[i];
    kb1[i] += R(T::A31) * u;
    kb2[i] += R(T::A32) * u;
  }
  // stage 2
  src.template get<2>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = R(0.0);
  F::vjp(st, p, kb2, sb, gp);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    yb[i] += sb[i];
    kb1[i] += R(T::A21) * (dt * sb[i]);
  }
  // stage 1 (s1 = y)
  F::vjp(y, p, kb1, yb, gp);
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] = yb[i];
}

// Reverse of one replay step, recomputing its stages from y.
template <class F, class R = double>
__device__ __forceinline__ void tsit5_step_vjp(const R* y, const R* p, R dt, R* lam, R* gp) {
  StageStates<F, R> S;
  tsit5_stage_states<F, false, R>(y, p, dt, S, nullptr);
  tsit5_vjp_core<F>(y, S, p, dt, lam, gp);
}

// --- kernel arguments -----------------------------------------------------------------
struct RecordArgs {
  long long n;
  const double* y0;
  const double* p;
  double t0, t1, rtol, atol, dt0;
  const double* t1v;  // per-trajectory end times or null
  int max_steps, cap, ck_every, ck_slots;
  double* rec;   // chunked dt record or null
  double* ckpt;  // checkpoints or null
  double* yf;
  int* n_acc;
  int* n_rej;
  int* status;
  CtrlConsts ctrl{};  // set by the launcher for the field's D and the method's order
  // dense output produced by the forward itself (persistent kernel only): requested times,
  // row j at ts + j * ts_ld (ts_ld = 0: one shared row), K per trajectory, states (n, K, D)
  const double* ts = nullptr;
  long long ts_ld = 0;
  int K = 0;
  double* ys = nullptr;
  CtrlConstsF ctrlf{};  // the float32 route's controller constants (set by its launcher)
};

struct AdjointArgs {
  long long n;
  const double* p;
  const double* rec;
  const int* n_acc;
  const double* ckpt;
  int ck_every;
  const double* ybar;
  double* gy0;
  double* gp;
  int cap;  // record capacity: step counts are clamped to [0, cap] before any record read
  // lane t integrates trajectory order[t] (a permutation of [0, n): lanes ordered by step
  // count keep a warp's lanes in step), or trajectory t when null
  const long long* order = nullptr;
};

// The trajectory of reverse-pass lane t; -1 (the lane idles) for an entry of `order` outside
// [0, n), so a bad permutation cannot send a lane outside the batch's arrays.
__device__ __forceinline__ long long lane_traj(const AdjointArgs& a, long long t) {
  if (!a.order) return t;
  const long long j = __ldg(a.order + t);
  return (j >= 0 && j < a.n) ? j : -1;
}

struct ReplayArgs {
  long long n;
  const double* y0;
  const double* p;
  double t0;
  const double* rec;
  const int* n_acc;
  int ck_every, ck_slots;
  double* ckpt;
  double* yf;
  int cap;  // record capacity: step counts are clamped to [0, cap] before any record read
};

// A trajectory's step count as the reverse and replay kernels use it: never outside the
// record's capacity, whatever the caller's n_acc holds (a record read past the capacity would
// leave the buffer).
__device__ __forceinline__ int steps_in_record(const int* n_acc, long long j, int cap) {
  const int na = n_acc[j];
  return na < 0 ? 0 : (na > cap ? cap : na);
}

template <int D>
__device__ __forceinline__ void store_ckpt(double* ckpt, long long n, long long j, int slot,
                                           const double* y, double t) {
  constexpr int CW = (D + 2) & ~1;
  double v[CW];
#pragma unroll
  for (int i = 0; i < D; ++i) v[i] = y[i];
  v[D] = t;
#pragma unroll
  for (int i = D + 1; i < CW; ++i) v[i] = 0.0;
  double2* dst = reinterpret_cast<double2*>(ckpt + ((size_t)slot * (size_t)n + (size_t)j) * CW);
#pragma unroll
  for (int i = 0; i < CW / 2; ++i) dst[i] = make_double2(v[2 * i], v[2 * i + 1]);
}

template <int D>
__device__ __forceinline__ double load_ckpt(const double* ckpt, long long n, long long j, int slot,
                                            double* y) {
  constexpr int CW = (D + 2) & ~1;
  const double2* src =
      reinterpret_cast<const double2*>(ckpt + ((size_t)slot * (size_t)n + (size_t)j) * CW);
  double v[CW];
#pragma unroll
  for (int i = 0; i < CW / 2; ++i) {
    const double2 w = __ldg(src + i);
    v[2 * i] = w.x;
    v[2 * i + 1] = w.y;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) y[i] = v[i];
  return v[D];
}

__device__ __forceinline__ void store_rec_chunk(double* rec, long long n, long long j, int chunk,
                                                double a, double b, double c, double d) {
  double2* dst = reinterpret_cast<double2*>(rec + ((size_t)chunk * (size_t)n + (size_t)j) * 4u);
  dst[0] = make_double2(a, b);
  dst[1] = make_double2(c, d);
}

__device__ __forceinline__ double load_rec(const double* rec, long long n, long long j,
                                           long long s) {
  return __ldg(rec + rec_index(j, s, n));
}

// --- forward adaptive solve with record --------------------------------------------------
// Per-trajectory bookkeeping of the forward, carried from attempt to attempt.
struct FwdCounters {
  double t, dt;
  int it, acc, rej, st, ck_cnt, ck_slot;
  double* rp;  // this trajectory's slots of the current record sector (rec_index, advanced)
};

// One attempt from the state (y, k1) (k1 = f(y), FSAL).  The candidate is computed into
// (yo, ko); returns true when the integration goes on from (yo, ko) -- which after a rejection
// receive a copy of (y, k1) -- and false when it stops with its state in (y, k1).  The kernel
// alternates the two register sets, so an accepted step (the common case) moves no state.
template <class F>
__device__ __forceinline__ bool tsit5_attempt(const RecordArgs& a, long long j,
                                              const double* p, double t1, bool rec_on,
                                              bool ck_on, long long rstride, FwdCounters& c,
                                              const double* y, const double* k1, double* yo,
                                              double* ko) {
  constexpr int D = F::D;
  using T = Tsit5;
  if (c.it >= a.max_steps || c.t >= t1) return false;
  ++c.it;
  const double h = (t1 - c.t < c.dt) ? (t1 - c.t) : c.dt;
  Stages<F> S;
  tsit5_k2_to_k6<F>(y, p, k1, h, S);
  tsit5_y5<F>(y, k1, S, h, yo);
  F::rhs(yo, p, ko);
  double e[D];
#pragma unroll
  for (int i = 0; i < D; ++i)
    e[i] = h * (T::E1 * k1[i] + T::E2 * S.k2[i] + T::E3 * S.k3[i] + T::E4 * S.k4[i] +
                T::E5 * S.k5[i] + T::E6 * S.k6[i] + T::E7 * ko[i]);
  const double m = wrms_sumsq<D>(e, y, yo, a.rtol, a.atol);
  if (!(m == m)) {  // NaN error: dt would turn NaN and the loop could never finish
    c.st = 1;
    return false;
  }
  if (m <= a.ctrl.accept_sum) {  // err = sqrt(m / D) <= 1
    if ((rec_on || ck_on) && c.acc >= a.cap) {
      c.st = 3;
      return false;
    }
    c.t = c.t + h;
    if (rec_on) {
      c.rp[c.acc & 3] = h;
      if ((c.acc & 3) == 3) c.rp += rstride;
    }
    ++c.acc;
    if (ck_on && ++c.ck_cnt == a.ck_every) {
      c.ck_cnt = 0;
      if (++c.ck_slot < a.ck_slots) store_ckpt<D>(a.ckpt, a.n, j, c.ck_slot, yo, c.t);
    }
  } else {
    ++c.rej;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      yo[i] = y[i];
      ko[i] = k1[i];
    }
  }
  c.dt = step_from_sum<10>(m, h, a.ctrl);
  return true;
}

// Bounded to 6 resident blocks of 128 per SM (80 registers) for D <= 4: with the
// shared-reciprocal error norm the unbounded kernel takes 84 and drops to 5 blocks; the few
// bytes it spills at 80 cost less than the lost warps (11.63 vs 11.73 ms on the Lorenz 2^20
// bench forward; 7 blocks at 72 registers: 11.35 ms).  Larger states keep their registers.
// kStore = false: the forward-only solve (no record, no checkpoints), with the store paths
// compiled out.  kMinB > 0 bounds the registers for kMinB resident blocks per SM instead
// (the instances the occupancy autotuner chooses among; same arithmetic, bit for bit).
template <class F, bool kStore = true, int kMinB = 0>
__global__ void __launch_bounds__(128, (kMinB > 0 ? kMinB : (F::D <= 4 ? 6 : 1)))
    tsit5_record_kernel(const RecordArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  double ya[D], ka[D], yb[D], kb[D], p[P];
#pragma unroll
  for (int i = 0; i < D; ++i) ya[i] = a.y0[j * D + i];
#pragma unroll
  for (int i = 0; i < P; ++i) p[i] = a.p[j * P + i];
  const double t1 = a.t1v ? a.t1v[j] : a.t1;
  const bool rec_on = kStore && a.rec != nullptr;
  const bool ck_on = kStore && a.ckpt != nullptr;
  const long long rstride = 4 * a.n;
  FwdCounters c;
  c.t = a.t0;
  c.dt = a.dt0 > 0.0 ? a.dt0 : (t1 - a.t0) / 100.0;
  c.it = c.acc = c.rej = c.st = c.ck_cnt = c.ck_slot = 0;
  c.rp = rec_on ? a.rec + j * 4 : nullptr;
  if (ck_on) store_ckpt<D>(a.ckpt, a.n, j, 0, ya, c.t);
  F::rhs(ya, p, ka);
  bool in_b = false;  // where the state is when the loop stops
  for (;;) {
    if (!tsit5_attempt<F>(a, j, p, t1, rec_on, ck_on, rstride, c, ya, ka, yb, kb)) break;
    if (!tsit5_attempt<F>(a, j, p, t1, rec_on, ck_on, rstride, c, yb, kb, ya, ka)) {
      in_b = true;
      break;
    }
  }
  if (c.st == 0 && !(c.t >= t1)) c.st = 1;
  if (rec_on) {  // zero-pad the last sector (identity steps)
    for (int s = c.acc; (s & 3) != 0; ++s) c.rp[s & 3] = 0.0;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) a.yf[j * D + i] = in_b ? yb[i] : ya[i];
  a.n_acc[j] = c.acc;
  a.n_rej[j] = c.rej;
  a.status[j] = c.st;
}

// --- frozen-mesh replay (values), optionally writing checkpoints -------------------------
template <class F>
__global__ void __launch_bounds__(128) tsit5_replay_kernel(const ReplayArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  double y[D], p[P];
#pragma unroll
  for (int i = 0; i < D; ++i) y[i] = a.y0[j * D + i];
#pragma unroll
  for (int i = 0; i < P; ++i) p[i] = a.p[j * P + i];
  const int na = steps_in_record(a.n_acc, j, a.cap);
  double t = a.t0;
  const bool ck_on = a.ckpt != nullptr;
  if (ck_on) store_ckpt<D>(a.ckpt, a.n, j, 0, y, t);
  int ck_cnt = 0, ck_slot = 0;
  for (int s = 0; s < na; ++s) {
    const double dt = load_rec(a.rec, a.n, j, s);
    tsit5_replay_step<F>(y, p, dt);
    t = t + dt;
    if (ck_on && ++ck_cnt == a.ck_every) {
      ck_cnt = 0;
      if (++ck_slot < a.ck_slots) store_ckpt<D>(a.ckpt, a.n, j, ck_slot, y, t);
    }
  }
#pragma unroll
  for (int i = 0; i < D; ++i) a.yf[j * D + i] = y[i];
}

// --- reverse-replay adjoint ---------------------------------------------------------------
// Each thread's shared memory holds its segment's K states and, double-buffered, the K dts
// and the checkpoint of a segment: while a segment is recomputed and differentiated, the
// next one's checkpoint and dts are already on their way (cp.async, global -> shared, no
// register staging), so segment starts do not wait on DRAM, and each dt is read from DRAM
// once instead of once per sweep.
//
// The dts and the checkpoint sit in 16-byte units (unit u of thread t at unit u * blockDim +
// t), so that each is fetched with 16-byte copies: a checkpoint is CW / 2 copies and, for an
// even segment start and length, a pair of dts (two 8-byte slots of one 32-byte record
// sector) is one -- half the copy instructions of 8-byte copies (Lorenz reverse pass at
// K = 2: 3.89 -> 3.78 ms per 2^18 launch).
__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gmem_src) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}
// both addresses 16-byte aligned
__device__ __forceinline__ void cp_async16(double2* smem_dst, const double* gmem_src) {
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// The segment count of the warp's longest trajectory (over the lanes executing together
// here).  The reverse passes sweep segments top-1 .. 0 in every lane, a lane idling while sg
// lies beyond its own trajectory: the lanes then work on segment sg of adjacent trajectories
// at the same time, so the checkpoint rows and dt sectors they fetch are neighbours in memory
// and share DRAM bursts, where lanes each starting from their own last segment fetch
// scattered sectors whose neighbours are evicted before their turn comes.  A warp takes as
// long as before: it always ran until its longest trajectory was done (the idle time moves
// from the end of the short trajectories to their start).
__device__ __forceinline__ int warp_top_segments(int nseg) {
  return __reduce_max_sync(__activemask(), nseg);
}

// Doubles per thread of the double-buffered dts + checkpoint area.
template <int D>
GS_HD int seg_io_doubles(int K) { return 2 * 2 * (((K + 1) >> 1) + ((D + 2) & ~1) / 2); }

template <int D>
struct SegIO {
  static constexpr int CW = (D + 2) & ~1, CU = CW / 2;  // checkpoint doubles, units
  double2* base;
  int stride, KU;  // KU: 16-byte units of dts per buffer
  // `off`: doubles per thread before the area (the block's shared memory is thread-strided
  // in 8-byte elements up to it; blockDim is a multiple of 32, so the area is 16-byte aligned)
  __device__ __forceinline__ SegIO(int off, int K)
      : base(reinterpret_cast<double2*>(gs_seg_smem + (size_t)off * blockDim.x) + threadIdx.x),
        stride(blockDim.x), KU((K + 1) >> 1) {}
  __device__ __forceinline__ double2* unit(int b, int u) { return base + (b * (KU + CU) + u) * stride; }
  __device__ __forceinline__ double& dt(int b, int q) {
    return reinterpret_cast<double*>(unit(b, q >> 1))[q & 1];
  }
  __device__ __forceinline__ double& ck(int b, int i) {
    return reinterpret_cast<double*>(unit(b, KU + (i >> 1)))[i & 1];
  }
};

// W doubles of segment state per step (D: the states; D + 1: states and step start time).
template <int D, int W = D>
GS_HD int adjoint_smem_doubles(int K) { return K * W + seg_io_doubles<D>(K); }

template <int D, int W = D>
struct AdjBuf {
  double* base;
  int stride;
  SegIO<D> io;
  __device__ __forceinline__ AdjBuf(int K)
      : base(gs_seg_smem + threadIdx.x), stride(blockDim.x), io(K * W, K) {}
  __device__ __forceinline__ double& st(int q, int i) { return base[(q * W + i) * stride]; }
  __device__ __forceinline__ double& dt(int b, int q) { return io.dt(b, q); }
  __device__ __forceinline__ double& ck(int b, int i) { return io.ck(b, i); }
};

// Start the copies of segment sg's checkpoint and dts into buffer b of buf.io (steps at or
// past na read as 0).  Record addresses: step s of trajectory j at rec_index(j, s, n), so an
// even s and s + 1 share a 16-byte aligned half sector.
// The dts of segment sg into buffer b (steps at or past na read as 0); the caller commits.
template <int D>
__device__ __forceinline__ void prefetch_dts(SegIO<D>& io, int b, const double* rec, long long n,
                                             long long j, int sg, int K, int na) {
  const int start = sg * K;
  // (the loops stay rolled: unrolled, the copies of the pair loop raised the stage-keeping
  // kernel from 90 to 118 registers)
  if (((start | K) & 1) == 0) {  // even start and length: pairs of dts, 16 bytes each
#pragma unroll 1
    for (int q = 0; q < K; q += 2) {
      const int s = start + q;
      if (s + 1 < na) {
        cp_async16(io.unit(b, q >> 1), rec + rec_index(j, s, n));
      } else {
        if (s < na)
          cp_async8(&io.dt(b, q), rec + rec_index(j, s, n));
        else
          io.dt(b, q) = 0.0;
        io.dt(b, q + 1) = 0.0;
      }
    }
  } else {
#pragma unroll 1
    for (int q = 0; q < K; ++q) {
      const int s = start + q;
      if (s < na)
        cp_async8(&io.dt(b, q), rec + rec_index(j, s, n));
      else
        io.dt(b, q) = 0.0;
    }
  }
}

template <int D, class Buf>
__device__ __forceinline__ void prefetch_segment(Buf& buf, int b, const double* ckpt,
                                                 const double* rec, long long n, long long j,
                                                 int sg, int K, int na) {
  SegIO<D>& io = buf.io;
  constexpr int CW = SegIO<D>::CW;
  const double* src = ckpt + ((size_t)sg * (size_t)n + (size_t)j) * CW;
#pragma unroll
  for (int u = 0; u < CW / 2; ++u) cp_async16(io.unit(b, io.KU + u), src + 2 * u);
  prefetch_dts<D>(io, b, rec, n, j, sg, K, na);
  cp_async_commit();
}

template <class F>
__global__ void __launch_bounds__(128) tsit5_adjoint_kernel(const AdjointArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const long long j = lane_traj(a, t);
  if (j < 0) return;
  double p[P], lam[D], gp[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    p[i] = a.p[j * P + i];
    gp[i] = 0.0;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] = a.ybar[j * D + i];
  const int na = steps_in_record(a.n_acc, j, a.cap);
  const int K = a.ck_every;
  const int nseg = (na + K - 1) / K;
  AdjBuf<D> buf(K);
  int b = 0;
  if (nseg > 0) prefetch_segment<D>(buf, b, a.ckpt, a.rec, a.n, j, nseg - 1, K, na);
  const int top = warp_top_segments(nseg);
  for (int sg = top - 1; sg >= 0; --sg) {
    if (sg >= nseg) continue;  // in step with the warp's longest trajectory
    cp_async_wait_all();  // this segment's checkpoint and dts have landed
    double y[D];
#pragma unroll
    for (int i = 0; i < D; ++i) y[i] = buf.ck(b, i);
    if (sg > 0) prefetch_segment<D>(buf, b ^ 1, a.ckpt, a.rec, a.n, j, sg - 1, K, na);
#pragma unroll
    for (int i = 0; i < D; ++i) buf.st(0, i) = y[i];
    for (int q = 1; q < K; ++q) {
      const double dt = buf.dt(b, q - 1);
      if (dt != 0.0) tsit5_replay_step<F>(y, p, dt);
#pragma unroll
      for (int i = 0; i < D; ++i) buf.st(q, i) = y[i];
    }
    for (int q = K - 1; q >= 0; --q) {
      const double dt = buf.dt(b, q);
      if (dt != 0.0) {
        double ys[D];
#pragma unroll
        for (int i = 0; i < D; ++i) ys[i] = buf.st(q, i);
        tsit5_step_vjp<F>(ys, p, dt, lam, gp);
      }
    }
    b ^= 1;
  }
  if (a.gy0) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.gy0[j * D + i] = lam[i];
  }
  if (a.gp) {
#pragma unroll
    for (int i = 0; i < P; ++i) a.gp[j * P + i] = gp[i];
  }
}

// --- reverse-replay adjoint that keeps the stage inputs -----------------------------------
// The segment's replay evaluates the stages of its first K-1 steps anyway: this variant keeps
// their inputs s2..s6 (5*D doubles per step) in the shared-memory buffer, so those steps'
// VJPs run without recomputing them; only the segment's last step, which the replay does not
// take, recomputes its stages.  Per segment: K stage evaluations instead of 2K-1, for
// (K-1)*5*D more doubles of buffer per thread.  Same states (tsit5_stage_states<F, true>
// evaluates tsit5_replay_step's expressions), the same VJP code (tsit5_vjp_core), and the
// same checkpoint/dt prefetch as tsit5_adjoint_kernel.
template <int D>
GS_HD int adjoint_stages_smem_doubles(int K) {
  return K * D + (K - 1) * 5 * D + seg_io_doubles<D>(K);
}

template <int D>
struct AdjStageBuf {
  double* base;
  int stride, K;
  SegIO<D> io;
  __device__ __forceinline__ AdjStageBuf(int k)
      : base(gs_seg_smem + threadIdx.x), stride(blockDim.x), K(k),
        io(k * D + (k - 1) * 5 * D, k) {}
  __device__ __forceinline__ double& st(int q, int i) { return base[(q * D + i) * stride]; }
  // stage input s_M (M = 2..6) of step q < K-1
  __device__ __forceinline__ double& stg(int q, int m, int i) {
    return base[(K * D + (q * 5 + (m - 2)) * D + i) * stride];
  }
  __device__ __forceinline__ double& dt(int b, int q) { return io.dt(b, q); }
  __device__ __forceinline__ double& ck(int b, int i) { return io.ck(b, i); }
};

template <class F>
struct KeptStages {  // tsit5_vjp_core's stage source: the kept inputs of step q
  static constexpr int D = F::D;
  AdjStageBuf<D>* buf;
  int q;
  template <int M>
  __device__ __forceinline__ void get(double* out) const {
#pragma unroll
    for (int i = 0; i < D; ++i) out[i] = buf->stg(q, M, i);
  }
};

// KC > 0: the segment length fixed at compile time (the autotuned K = 2 of the built-in
// fields), so the segment loops unroll and the buffer offsets are constants; KC = 0 reads K
// from the arguments.
template <class F, int KC>
__device__ __forceinline__ void tsit5_adjoint_stages_body(const AdjointArgs& a) {
  constexpr int D = F::D, P = F::P;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const long long j = lane_traj(a, t);
  if (j < 0) return;
  double p[P], lam[D], gp[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    p[i] = a.p[j * P + i];
    gp[i] = 0.0;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] = a.ybar[j * D + i];
  const int na = steps_in_record(a.n_acc, j, a.cap);
  const int K = KC > 0 ? KC : a.ck_every;
  const int nseg = (na + K - 1) / K;
  AdjStageBuf<D> buf(K);
  int b = 0;
  if (nseg > 0) prefetch_segment<D>(buf, b, a.ckpt, a.rec, a.n, j, nseg - 1, K, na);
  const int top = warp_top_segments(nseg);
  for (int sg = top - 1; sg >= 0; --sg) {
    if (sg >= nseg) continue;  // in step with the warp's longest trajectory
    cp_async_wait_all();  // this segment's checkpoint and dts have landed
    double y[D];
#pragma unroll
    for (int i = 0; i < D; ++i) y[i] = buf.ck(b, i);
    if (sg > 0) prefetch_segment<D>(buf, b ^ 1, a.ckpt, a.rec, a.n, j, sg - 1, K, na);
#pragma unroll
    for (int i = 0; i < D; ++i) buf.st(0, i) = y[i];
    for (int q = 1; q < K; ++q) {  // replay steps 0..K-2, keeping their stage inputs
      const double dt = buf.dt(b, q - 1);
      if (dt != 0.0) {
        StageStates<F> S;
        double yn[D];
        tsit5_stage_states<F, true>(y, p, dt, S, yn);
#pragma unroll
        for (int i = 0; i < D; ++i) {
          y[i] = yn[i];
          buf.stg(q - 1, 2, i) = S.s2[i];
          buf.stg(q - 1, 3, i) = S.s3[i];
          buf.stg(q - 1, 4, i) = S.s4[i];
          buf.stg(q - 1, 5, i) = S.s5[i];
          buf.stg(q - 1, 6, i) = S.s6[i];
        }
      }
#pragma unroll
      for (int i = 0; i < D; ++i) buf.st(q, i) = y[i];
    }
    {  // the segment's last step: its stages were not evaluated by the replay
      const double dt = buf.dt(b, K - 1);
      if (dt != 0.0) {
        double ys[D];
#pragma unroll
        for (int i = 0; i < D; ++i) ys[i] = buf.st(K - 1, i);
        tsit5_step_vjp<F>(ys, p, dt, lam, gp);
      }
    }
    for (int q = K - 2; q >= 0; --q) {
      const double dt = buf.dt(b, q);
      if (dt != 0.0) {
        double ys[D];
#pragma unroll
        for (int i = 0; i < D; ++i) ys[i] = buf.st(q, i);
        const KeptStages<F> src{&buf, q};
        tsit5_vjp_core<F>(ys, src, p, dt, lam, gp);
      }
    }
    b ^= 1;
  }
  if (a.gy0) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.gy0[j * D + i] = lam[i];
  }
  if (a.gp) {
#pragma unroll
    for (int i = 0; i < P; ++i) a.gp[j * P + i] = gp[i];
  }
}

template <class F>
__global__ void __launch_bounds__(128) tsit5_adjoint_stages_kernel(const AdjointArgs a) {
  tsit5_adjoint_stages_body<F, 0>(a);
}

// K = 2, bounded to 5 blocks of 128 per SM: unrolled without the bound, the segment's two
// steps interleave into 128 registers (4 blocks).  kMinB > 0 bounds it for kMinB blocks
// instead (the instances the occupancy autotuner chooses among; same arithmetic, bit for bit).
template <class F, int kMinB = 0>
__global__ void __launch_bounds__(128, (kMinB > 0 ? kMinB : 5))
    tsit5_adjoint_stages_k2_kernel(const AdjointArgs a) {
  tsit5_adjoint_stages_body<F, 2>(a);
}

}  // namespace gs
