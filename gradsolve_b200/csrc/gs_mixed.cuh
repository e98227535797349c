// gs_mixed.cuh -- Tsit5 forward/replay/adjoint with float32 stages (GS_PREC_MIXED).
//
// Float64 is kept for the time, the state y (updated with compensated summation), the
// base right-hand side k1 = f(y) (the FSAL stage, once per attempt), the error norm and the
// step-size controller.  Everything else runs in float32 in increment form:
//
//   k_i = k1 + dk_i,  dk_i = f(y + d_i) - f(y)  (F::rhs_delta: expanded, no cancellation)
//   d_i = h (c_i k1 + sum_{j=2}^{i-1} a_ij dk_j)          (c_i = sum_j a_ij)
//   y5  = y + h k1 + h sum_{i>=2} b_i dk_i                (sum_i b_i = 1)
//   e   = h sum_{i>=2} E_i dk_i                           (sum_i E_i = 0)
//
// This is the same Tsit5 step (gradsolve/solvers/tsit5_step.py:80-102) regrouped, so the
// float32 roundings act only on the increments dk_i and d_i, which are smaller than k and
// y by the factor h|J|; the embedded error estimate, whose terms cancel in float64 form,
// is computed from the increments directly.  The reverse pass applies the float32 stage
// VJPs at the stage states y + d_i and accumulates the cotangent lambda and the parameter
// gradient in float64.
#pragma once
#include "gs_fields.cuh"
#include "gs_tableau.cuh"
#include "gs_tsit5.cuh"

namespace gs {

struct Tsit5f {
  static constexpr float C2 = (float)Tsit5::C2, C3 = (float)Tsit5::C3, C4 = (float)Tsit5::C4,
                         C5 = (float)Tsit5::C5, C6 = 1.0f;
  static constexpr float A21 = (float)Tsit5::A21, A31 = (float)Tsit5::A31,
                         A32 = (float)Tsit5::A32, A41 = (float)Tsit5::A41,
                         A42 = (float)Tsit5::A42, A43 = (float)Tsit5::A43,
                         A51 = (float)Tsit5::A51, A52 = (float)Tsit5::A52,
                         A53 = (float)Tsit5::A53, A54 = (float)Tsit5::A54,
                         A61 = (float)Tsit5::A61, A62 = (float)Tsit5::A62,
                         A63 = (float)Tsit5::A63, A64 = (float)Tsit5::A64,
                         A65 = (float)Tsit5::A65;
  static constexpr float B1 = (float)Tsit5::B1, B2 = (float)Tsit5::B2, B3 = (float)Tsit5::B3,
                         B4 = (float)Tsit5::B4, B5 = (float)Tsit5::B5, B6 = (float)Tsit5::B6;
  static constexpr float E2 = (float)Tsit5::E2, E3 = (float)Tsit5::E3, E4 = (float)Tsit5::E4,
                         E5 = (float)Tsit5::E5, E6 = (float)Tsit5::E6, E7 = (float)Tsit5::E7;
};

template <class F>
struct MixedStages {
  static constexpr int D = F::D;
  float dk2[D], dk3[D], dk4[D], dk5[D], dk6[D];
};

// Increments dk2..dk6 for step h from (y, k1); yf/pf/k1f are the float copies.
template <class F>
__device__ __forceinline__ void mixed_dk2_to_dk6(const float* yf, const float* pf,
                                                 const float* k1f, float hf,
                                                 MixedStages<F>& S) {
  constexpr int D = F::D;
  using T = Tsit5f;
  float d[D];
#pragma unroll
  for (int i = 0; i < D; ++i) d[i] = hf * (T::C2 * k1f[i]);
  F::rhs_delta(yf, pf, d, S.dk2);
#pragma unroll
  for (int i = 0; i < D; ++i) d[i] = hf * (T::C3 * k1f[i] + T::A32 * S.dk2[i]);
  F::rhs_delta(yf, pf, d, S.dk3);
#pragma unroll
  for (int i = 0; i < D; ++i) d[i] = hf * (T::C4 * k1f[i] + T::A42 * S.dk2[i] + T::A43 * S.dk3[i]);
  F::rhs_delta(yf, pf, d, S.dk4);
#pragma unroll
  for (int i = 0; i < D; ++i)
    d[i] = hf * (T::C5 * k1f[i] + T::A52 * S.dk2[i] + T::A53 * S.dk3[i] + T::A54 * S.dk4[i]);
  F::rhs_delta(yf, pf, d, S.dk5);
#pragma unroll
  for (int i = 0; i < D; ++i)
    d[i] = hf * (T::C6 * k1f[i] + T::A62 * S.dk2[i] + T::A63 * S.dk3[i] + T::A64 * S.dk4[i] +
                 T::A65 * S.dk5[i]);
  F::rhs_delta(yf, pf, d, S.dk6);
}

// Full float64 increment of the step: h k1 + h sum b_i dk_i.
template <class F>
__device__ __forceinline__ void mixed_increment(const double* k1, const MixedStages<F>& S,
                                                double h, float hf, double* inc) {
  using T = Tsit5f;
#pragma unroll
  for (int i = 0; i < F::D; ++i) {
    const float s = hf * (T::B2 * S.dk2[i] + T::B3 * S.dk3[i] + T::B4 * S.dk4[i] +
                          T::B5 * S.dk5[i] + T::B6 * S.dk6[i]);
    inc[i] = fma(h, k1[i], (double)s);
  }
}

// y <- y + inc with Kahan compensation c (both float64).
template <int D>
__device__ __forceinline__ void kahan_add(double* y, double* c, const double* inc) {
#pragma unroll
  for (int i = 0; i < D; ++i) {
    const double yk = inc[i] - c[i];
    const double tt = y[i] + yk;
    c[i] = (tt - y[i]) - yk;
    y[i] = tt;
  }
}

template <class F>
__device__ __forceinline__ void to_float(const double* a, float* b) {
#pragma unroll
  for (int i = 0; i < F::D; ++i) b[i] = (float)a[i];
}

// One replay step (values), float32 stages.
template <class F>
__device__ __forceinline__ void mixed_replay_step(double* y, double* c, const double* p,
                                                  const float* pf, double dt) {
  constexpr int D = F::D;
  double k1[D], inc[D];
  float yf[D], k1f[D];
  F::rhs(y, p, k1);
  to_float<F>(y, yf);
  to_float<F>(k1, k1f);
  MixedStages<F> S;
  const float hf = (float)dt;
  mixed_dk2_to_dk6<F>(yf, pf, k1f, hf, S);
  mixed_increment<F>(k1, S, dt, hf, inc);
  kahan_add<D>(y, c, inc);
}

// Float32 inputs of one step's stages: yf = y and the stage states s_m = y + d_m (m = 2..6).
// With kNext the step's result is also produced (the expressions of mixed_replay_step, so a
// replay that keeps the stages lands on the same states).
template <class F>
struct MixedStageStates {
  static constexpr int D = F::D;
  float yf[D], s2[D], s3[D], s4[D], s5[D], s6[D];
  template <int M>
  __device__ __forceinline__ void get(float* out) const {
    const float* src = M == 1 ? yf : M == 2 ? s2 : M == 3 ? s3 : M == 4 ? s4 : M == 5 ? s5 : s6;
#pragma unroll
    for (int i = 0; i < D; ++i) out[i] = src[i];
  }
};

template <class F, bool kNext>
__device__ __forceinline__ void mixed_stage_states(const double* y, const double* p,
                                                   const float* pf, double dt,
                                                   MixedStageStates<F>& S, double* yn,
                                                   double* cn) {
  constexpr int D = F::D;
  using T = Tsit5f;
  double k1[D];
  float k1f[D];
  F::rhs(y, p, k1);
  to_float<F>(y, S.yf);
  to_float<F>(k1, k1f);
  const float hf = (float)dt;
  MixedStages<F> K;
  float d[D];
#pragma unroll
  for (int i = 0; i < D; ++i) { d[i] = hf * (T::C2 * k1f[i]); S.s2[i] = S.yf[i] + d[i]; }
  F::rhs_delta(S.yf, pf, d, K.dk2);
#pragma unroll
  for (int i = 0; i < D; ++i) { d[i] = hf * (T::C3 * k1f[i] + T::A32 * K.dk2[i]); S.s3[i] = S.yf[i] + d[i]; }
  F::rhs_delta(S.yf, pf, d, K.dk3);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    d[i] = hf * (T::C4 * k1f[i] + T::A42 * K.dk2[i] + T::A43 * K.dk3[i]);
    S.s4[i] = S.yf[i] + d[i];
  }
  F::rhs_delta(S.yf, pf, d, K.dk4);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    d[i] = hf * (T::C5 * k1f[i] + T::A52 * K.dk2[i] + T::A53 * K.dk3[i] + T::A54 * K.dk4[i]);
    S.s5[i] = S.yf[i] + d[i];
  }
  F::rhs_delta(S.yf, pf, d, K.dk5);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    d[i] = hf * (T::C6 * k1f[i] + T::A62 * K.dk2[i] + T::A63 * K.dk3[i] + T::A64 * K.dk4[i] +
                 T::A65 * K.dk5[i]);
    S.s6[i] = S.yf[i] + d[i];
  }
  if constexpr (kNext) {
    F::rhs_delta(S.yf, pf, d, K.dk6);
    double inc[D];
    mixed_increment<F>(k1, K, dt, hf, inc);
    kahan_add<D>(yn, cn, inc);
  }
}

// Reverse of one step given its float32 stage inputs (Src::get<1> yields y as float, get<M>
// s_M): lam (float64) <- (dy'/dy)^T lam; gp += (dy'/dp)^T lam.  The stage VJPs run in float32
// and their sums join lam and gp in float64.
template <class F, class Src>
__device__ __forceinline__ void mixed_vjp_core(const Src& src, const float* pf, double dt,
                                               double* lam, double* gp) {
  constexpr int D = F::D, P = F::P;
  using T = Tsit5f;
  const float hf = (float)dt;
  float st[D], g[D], kb1[D], kb2[D], kb3[D], kb4[D], kb5[D], kb6[D], sb[D], acc[D], gpf[P];
#pragma unroll
  for (int k = 0; k < P; ++k) gpf[k] = 0.0f;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    g[i] = hf * (float)lam[i];
    acc[i] = 0.0f;
    kb1[i] = T::B1 * g[i];
    kb2[i] = T::B2 * g[i];
    kb3[i] = T::B3 * g[i];
    kb4[i] = T::B4 * g[i];
    kb5[i] = T::B5 * g[i];
    kb6[i] = T::B6 * g[i];
  }
  src.template get<6>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = 0.0f;
  F::vjp(st, pf, kb6, sb, gpf);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    acc[i] += sb[i];
    const float u = hf * sb[i];
    kb1[i] += T::A61 * u; kb2[i] += T::A62 * u; kb3[i] += T::A63 * u;
    kb4[i] += T::A64 * u; kb5[i] += T::A65 * u;
  }
  src.template get<5>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = 0.0f;
  F::vjp(st, pf, kb5, sb, gpf);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    acc[i] += sb[i];
    const float u = hf * sb[i];
    kb1[i] += T::A51 * u; kb2[i] += T::A52 * u; kb3[i] += T::A53 * u; kb4[i] += T::A54 * u;
  }
  src.template get<4>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = 0.0f;
  F::vjp(st, pf, kb4, sb, gpf);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    acc[i] += sb[i];
    const float u = hf * sb[i];
    kb1[i] += T::A41 * u; kb2[i] += T::A42 * u; kb3[i] += T::A43 * u;
  }
  src.template get<3>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = 0.0f;
  F::vjp(st, pf, kb3, sb, gpf);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    acc[i] += sb[i];
    const float u = hf * sb[i];
    kb1[i] += T::A31 * u; kb2[i] += T::A32 * u;
  }
  src.template get<2>(st);
#pragma unroll
  for (int i = 0; i < D; ++i) sb[i] = 0.0f;
  F::vjp(st, pf, kb2, sb, gpf);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    acc[i] += sb[i];
    kb1[i] += T::A21 * (hf * sb[i]);
  }
  src.template get<1>(st);
  F::vjp(st, pf, kb1, acc, gpf);
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] += (double)acc[i];
#pragma unroll
  for (int k = 0; k < P; ++k) gp[k] += (double)gpf[k];
}

// Reverse of one step at (y, dt), recomputing its stages.
template <class F>
__device__ __forceinline__ void mixed_step_vjp(const double* y, const double* p, const float* pf,
                                               double dt, double* lam, double* gp) {
  MixedStageStates<F> S;
  mixed_stage_states<F, false>(y, p, pf, dt, S, nullptr, nullptr);
  mixed_vjp_core<F>(S, pf, dt, lam, gp);
}

// --- forward adaptive solve with record, float32 stages ----------------------------------
// One float32-stage attempt from the state (y, c, k1) -- c the compensated sum's carry, k1 =
// f(y) -- into (yo, co, ko), with the register-set alternation of tsit5_attempt: true when
// the integration goes on from (yo, co, ko), a copy of the state after a rejection.
template <class F>
__device__ __forceinline__ bool mixed_attempt(const RecordArgs& a, long long j, const double* p,
                                              const float* pf, double t1, bool rec_on,
                                              bool ck_on, long long rstride, FwdCounters& ct,
                                              const double* y, const double* c,
                                              const double* k1, double* yo, double* co,
                                              double* ko) {
  constexpr int D = F::D;
  using T = Tsit5f;
  if (ct.it >= a.max_steps || ct.t >= t1) return false;
  ++ct.it;
  const double h = (t1 - ct.t < ct.dt) ? (t1 - ct.t) : ct.dt;
  const float hf = (float)h;
  float yf[D], k1f[D];
  double inc[D], ed[D];
  to_float<F>(y, yf);
  to_float<F>(k1, k1f);
  MixedStages<F> S;
  mixed_dk2_to_dk6<F>(yf, pf, k1f, hf, S);
  mixed_increment<F>(k1, S, h, hf, inc);
#pragma unroll
  for (int i = 0; i < D; ++i) { yo[i] = y[i]; co[i] = c[i]; }
  kahan_add<D>(yo, co, inc);
  F::rhs(yo, p, ko);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    const float dk7 = (float)(ko[i] - k1[i]);
    ed[i] = (double)(hf * (T::E2 * S.dk2[i] + T::E3 * S.dk3[i] + T::E4 * S.dk4[i] +
                           T::E5 * S.dk5[i] + T::E6 * S.dk6[i] + T::E7 * dk7));
  }
  const double m = wrms_sumsq<D>(ed, y, yo, a.rtol, a.atol);
  if (!(m == m)) {
    ct.st = 1;
    return false;
  }
  if (m <= a.ctrl.accept_sum) {
    if ((rec_on || ck_on) && ct.acc >= a.cap) {
      ct.st = 3;
      return false;
    }
    ct.t = ct.t + h;
    if (rec_on) {
      ct.rp[ct.acc & 3] = h;
      if ((ct.acc & 3) == 3) ct.rp += rstride;
    }
    ++ct.acc;
    if (ck_on && ++ct.ck_cnt == a.ck_every) {
      ct.ck_cnt = 0;
      if (++ct.ck_slot < a.ck_slots) store_ckpt<D>(a.ckpt, a.n, j, ct.ck_slot, yo, ct.t);
    }
  } else {
    ++ct.rej;
#pragma unroll
    for (int i = 0; i < D; ++i) { yo[i] = y[i]; co[i] = c[i]; ko[i] = k1[i]; }
  }
  ct.dt = step_from_sum<10>(m, h, a.ctrl);
  return true;
}

template <class F>
__global__ void __launch_bounds__(128) tsit5_mixed_record_kernel(const RecordArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  double ya[D], ca[D], ka[D], yb[D], cb[D], kb[D], p[P];
  float pf[P];
#pragma unroll
  for (int i = 0; i < D; ++i) { ya[i] = a.y0[j * D + i]; ca[i] = 0.0; }
#pragma unroll
  for (int i = 0; i < P; ++i) { p[i] = a.p[j * P + i]; pf[i] = (float)p[i]; }
  const double t1 = a.t1v ? a.t1v[j] : a.t1;
  const bool rec_on = a.rec != nullptr;
  const bool ck_on = a.ckpt != nullptr;
  const long long rstride = 4 * a.n;
  FwdCounters ct;
  ct.t = a.t0;
  ct.dt = a.dt0 > 0.0 ? a.dt0 : (t1 - a.t0) / 100.0;
  ct.it = ct.acc = ct.rej = ct.st = ct.ck_cnt = ct.ck_slot = 0;
  ct.rp = rec_on ? a.rec + j * 4 : nullptr;
  if (ck_on) store_ckpt<D>(a.ckpt, a.n, j, 0, ya, ct.t);
  F::rhs(ya, p, ka);
  bool in_b = false;  // where the state is when the loop stops
  for (;;) {
    if (!mixed_attempt<F>(a, j, p, pf, t1, rec_on, ck_on, rstride, ct, ya, ca, ka, yb, cb, kb))
      break;
    if (!mixed_attempt<F>(a, j, p, pf, t1, rec_on, ck_on, rstride, ct, yb, cb, kb, ya, ca, ka)) {
      in_b = true;
      break;
    }
  }
  if (ct.st == 0 && !(ct.t >= t1)) ct.st = 1;
  if (rec_on) {  // zero-pad the last sector (identity steps)
    for (int s = ct.acc; (s & 3) != 0; ++s) ct.rp[s & 3] = 0.0;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) a.yf[j * D + i] = in_b ? yb[i] : ya[i];
  a.n_acc[j] = ct.acc;
  a.n_rej[j] = ct.rej;
  a.status[j] = ct.st;
}

template <class F>
__global__ void __launch_bounds__(128) tsit5_mixed_replay_kernel(const ReplayArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  double y[D], c[D], p[P];
  float pf[P];
#pragma unroll
  for (int i = 0; i < D; ++i) { y[i] = a.y0[j * D + i]; c[i] = 0.0; }
#pragma unroll
  for (int i = 0; i < P; ++i) { p[i] = a.p[j * P + i]; pf[i] = (float)p[i]; }
  const int na = steps_in_record(a.n_acc, j, a.cap);
  double t = a.t0;
  const bool ck_on = a.ckpt != nullptr;
  if (ck_on) store_ckpt<D>(a.ckpt, a.n, j, 0, y, t);
  int ck_cnt = 0, ck_slot = 0;
  for (int s = 0; s < na; ++s) {
    const double dt = load_rec(a.rec, a.n, j, s);
    mixed_replay_step<F>(y, c, p, pf, dt);
    t = t + dt;
    if (ck_on && ++ck_cnt == a.ck_every) {
      ck_cnt = 0;
      if (++ck_slot < a.ck_slots) store_ckpt<D>(a.ckpt, a.n, j, ck_slot, y, t);
    }
  }
#pragma unroll
  for (int i = 0; i < D; ++i) a.yf[j * D + i] = y[i];
}

template <class F>
__global__ void __launch_bounds__(128) tsit5_mixed_adjoint_kernel(const AdjointArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const long long j = lane_traj(a, t);
  if (j < 0) return;
  double p[P], lam[D], gp[P];
  float pf[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    p[i] = a.p[j * P + i];
    pf[i] = (float)p[i];
    gp[i] = 0.0;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] = a.ybar[j * D + i];
  const int na = steps_in_record(a.n_acc, j, a.cap);
  const int K = a.ck_every;
  const int nseg = (na + K - 1) / K;
  // segment buffer and cp.async prefetch of the next segment: as tsit5_adjoint_kernel
  AdjBuf<D> buf(K);
  int b = 0;
  if (nseg > 0) prefetch_segment<D>(buf, b, a.ckpt, a.rec, a.n, j, nseg - 1, K, na);
  const int top = warp_top_segments(nseg);
  for (int sg = top - 1; sg >= 0; --sg) {
    if (sg >= nseg) continue;  // in step with the warp's longest trajectory
    cp_async_wait_all();
    double y[D], c[D];
#pragma unroll
    for (int i = 0; i < D; ++i) { y[i] = buf.ck(b, i); c[i] = 0.0; }
    if (sg > 0) prefetch_segment<D>(buf, b ^ 1, a.ckpt, a.rec, a.n, j, sg - 1, K, na);
#pragma unroll
    for (int i = 0; i < D; ++i) buf.st(0, i) = y[i];
    for (int q = 1; q < K; ++q) {
      const double dt = buf.dt(b, q - 1);
      if (dt != 0.0) mixed_replay_step<F>(y, c, p, pf, dt);
#pragma unroll
      for (int i = 0; i < D; ++i) buf.st(q, i) = y[i];
    }
    for (int q = K - 1; q >= 0; --q) {
      const double dt = buf.dt(b, q);
      if (dt != 0.0) {
        double ys[D];
#pragma unroll
        for (int i = 0; i < D; ++i) ys[i] = buf.st(q, i);
        mixed_step_vjp<F>(ys, p, pf, dt, lam, gp);
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


// --- float32-stage reverse pass that keeps the stage inputs ---------------------------------
// The counterpart of tsit5_adjoint_stages_body: the segment's replay keeps, for each of its
// first K-1 steps, the float32 stage inputs (y and s2..s6: 6*D floats, packed two to a
// double of the shared-memory buffer), so those steps' VJPs skip the recomputation; only the
// segment's last step evaluates its stages in the reverse sweep.  Same states as
// tsit5_mixed_adjoint_kernel (mixed_stage_states<F, true> evaluates mixed_replay_step's
// expressions) and the same VJP code (mixed_vjp_core).
template <int D>
GS_HD int mixed_stages_smem_doubles(int K) {
  return K * D + (K - 1) * 3 * D + seg_io_doubles<D>(K);
}

template <int D>
struct MixedStageBuf {
  double* base;
  int stride, K;
  SegIO<D> io;
  __device__ __forceinline__ MixedStageBuf(int k)
      : base(gs_seg_smem + threadIdx.x), stride(blockDim.x), K(k),
        io(k * D + (k - 1) * 3 * D, k) {}
  __device__ __forceinline__ double& st(int q, int i) { return base[(q * D + i) * stride]; }
  // float m*D + i of step q's kept inputs (m = 0: y, m = 1..5: s2..s6), q < K-1
  __device__ __forceinline__ float& stg(int q, int m, int i) {
    const int f = m * D + i;
    return reinterpret_cast<float*>(&base[(K * D + q * 3 * D + (f >> 1)) * stride])[f & 1];
  }
  __device__ __forceinline__ double& dt(int b, int q) { return io.dt(b, q); }
  __device__ __forceinline__ double& ck(int b, int i) { return io.ck(b, i); }
};

template <class F>
struct MixedKeptStages {  // mixed_vjp_core's stage source: the kept inputs of step q
  static constexpr int D = F::D;
  MixedStageBuf<D>* buf;
  int q;
  template <int M>
  __device__ __forceinline__ void get(float* out) const {
#pragma unroll
    for (int i = 0; i < D; ++i) out[i] = buf->stg(q, M - 1, i);
  }
};

template <class F, int KC>
__device__ __forceinline__ void tsit5_mixed_adjoint_stages_body(const AdjointArgs& a) {
  constexpr int D = F::D, P = F::P;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const long long j = lane_traj(a, t);
  if (j < 0) return;
  double p[P], lam[D], gp[P];
  float pf[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    p[i] = a.p[j * P + i];
    pf[i] = (float)p[i];
    gp[i] = 0.0;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] = a.ybar[j * D + i];
  const int na = steps_in_record(a.n_acc, j, a.cap);
  const int K = KC > 0 ? KC : a.ck_every;
  const int nseg = (na + K - 1) / K;
  MixedStageBuf<D> buf(K);
  int b = 0;
  if (nseg > 0) prefetch_segment<D>(buf, b, a.ckpt, a.rec, a.n, j, nseg - 1, K, na);
  const int top = warp_top_segments(nseg);
  for (int sg = top - 1; sg >= 0; --sg) {
    if (sg >= nseg) continue;  // in step with the warp's longest trajectory
    cp_async_wait_all();  // this segment's checkpoint and dts have landed
    double y[D], c[D];
#pragma unroll
    for (int i = 0; i < D; ++i) { y[i] = buf.ck(b, i); c[i] = 0.0; }
    if (sg > 0) prefetch_segment<D>(buf, b ^ 1, a.ckpt, a.rec, a.n, j, sg - 1, K, na);
#pragma unroll
    for (int i = 0; i < D; ++i) buf.st(0, i) = y[i];
    for (int q = 1; q < K; ++q) {  // replay steps 0..K-2, keeping their stage inputs
      const double dt = buf.dt(b, q - 1);
      if (dt != 0.0) {
        MixedStageStates<F> S;
        mixed_stage_states<F, true>(y, p, pf, dt, S, y, c);
#pragma unroll
        for (int i = 0; i < D; ++i) {
          buf.stg(q - 1, 0, i) = S.yf[i];
          buf.stg(q - 1, 1, i) = S.s2[i];
          buf.stg(q - 1, 2, i) = S.s3[i];
          buf.stg(q - 1, 3, i) = S.s4[i];
          buf.stg(q - 1, 4, i) = S.s5[i];
          buf.stg(q - 1, 5, i) = S.s6[i];
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
        mixed_step_vjp<F>(ys, p, pf, dt, lam, gp);
      }
    }
    for (int q = K - 2; q >= 0; --q) {
      const double dt = buf.dt(b, q);
      if (dt != 0.0) {
        const MixedKeptStages<F> src{&buf, q};
        mixed_vjp_core<F>(src, pf, dt, lam, gp);
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
__global__ void __launch_bounds__(128) tsit5_mixed_adjoint_stages_kernel(const AdjointArgs a) {
  tsit5_mixed_adjoint_stages_body<F, 0>(a);
}

// K = 2 with the segment loops unrolled (the autotuned interval of the small built-in fields),
// bounded to 6 blocks of 128 per SM: unbounded, Lorenz's instance takes 94 registers (5 blocks)
// where the general stage-keeping kernel holds 6.  kMinB > 0 bounds it for kMinB blocks
// instead (the occupancy autotuner's instances; same arithmetic, bit for bit).
template <class F, int kMinB = 0>
__global__ void __launch_bounds__(128, (kMinB > 0 ? kMinB : 6))
    tsit5_mixed_adjoint_stages_k2_kernel(const AdjointArgs a) {
  tsit5_mixed_adjoint_stages_body<F, 2>(a);
}

}  // namespace gs
