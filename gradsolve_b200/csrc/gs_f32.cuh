// gs_f32.cuh -- the float32 route (GS_PREC_F32): forward with a float32 dt record, float32
// replay and float32 reverse pass, for Tsit5 and Rosenbrock23.
//
// The reference's precision="float32" lane records the mesh with its float32 fused kernel
// (every quantity float32: state, stages, time, error norm, controller; the record is float32,
// half the bytes of the float64 one) and replays and differentiates it in float32
// (gradsolve/warp/warp_replay.py:87-94, 140-160, 200-219, 305-325, 370-384;
// gradsolve/api.py:253-274).  These kernels
// do the same arithmetic in float, one thread per trajectory, with the step helpers of
// gs_tsit5.cuh / gs_ros23.cuh instantiated for float.  The float64 arrays of the C ABI (y0,
// p, y_final, cotangents, gradients) are read and written as float64 holding float32 values;
// rec and ckpt hold float32 data:
//   rec  : step s of trajectory j at float ((s/4)*n + j)*4 + s%4 (16-byte chunks of 4 steps)
//   ckpt : slot c of trajectory j at float (c*n + j)*CWF, CWF = D+1 rounded up to a multiple
//          of 4 (16-byte rows): the state, then the time.
// The controller is the reference kernel's, in float: err = sqrt(sum / D), accept iff
// err <= 1, dt = h * clip(0.9 * max(err, 1e-10)^(-1/q), 0.2, 5) after accept and reject --
// evaluated from the sum of squares without sqrt, pow or the division by D
// (step_from_sum_f32, gs_tsit5.cuh): the accept test is the reference's bit for bit on the
// same sum, the factor within a few float ulp of its powf.
#pragma once

#include <math_constants.h>

#include <type_traits>

#include "gs_pack.cuh"
#include "gs_ros23.cuh"
#include "gs_saveat.cuh"
#include "gs_tsit5.cuh"

namespace gs {

GS_HD int ckpt_width_f32(int D) { return (D + 4) & ~3; }

template <int D>
__device__ __forceinline__ void store_ckpt_f32(float* ckpt, long long n, long long j, int slot,
                                               const float* y, float t) {
  constexpr int CW = (D + 4) & ~3;
  float v[CW];
#pragma unroll
  for (int i = 0; i < D; ++i) v[i] = y[i];
  v[D] = t;
#pragma unroll
  for (int i = D + 1; i < CW; ++i) v[i] = 0.0f;
  float4* dst = reinterpret_cast<float4*>(ckpt + ((size_t)slot * (size_t)n + (size_t)j) * CW);
#pragma unroll
  for (int u = 0; u < CW / 4; ++u) dst[u] = make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
}

template <int D>
__device__ __forceinline__ void load_ckpt_f32(const float* ckpt, long long n, long long j, int slot,
                                              float* y) {
  constexpr int CW = (D + 4) & ~3;
  const float4* src =
      reinterpret_cast<const float4*>(ckpt + ((size_t)slot * (size_t)n + (size_t)j) * CW);
  float v[CW];
#pragma unroll
  for (int u = 0; u < CW / 4; ++u) {
    const float4 w = __ldg(src + u);
    v[4 * u] = w.x;
    v[4 * u + 1] = w.y;
    v[4 * u + 2] = w.z;
    v[4 * u + 3] = w.w;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) y[i] = v[i];
}

__device__ __forceinline__ float load_rec_f32(const float* rec, long long n, long long j,
                                              long long s) {
  return __ldg(rec + rec_index(j, s, n));
}

// Tsit5 steps on the float32 route are evaluated through F1 (gs_pack.cuh) for the fields the
// two-per-thread reverse pass covers (Packable): explicit contractions, the per-trajectory
// arithmetic of that pass, so the forward, the replay and both reverse passes see the same
// states bit for bit.  Other fields (generated ones may call sin, exp ...) keep plain float.
// (The copies in and out of the F1 arrays are register moves.)
// the fields the two-per-thread reverse pass is built for (f32_adjoint_pairs_kernel)
template <> struct Packable<Lorenz> { static constexpr bool value = true; };
template <> struct Packable<Lorenz3> { static constexpr bool value = true; };
template <> struct Packable<VdP> { static constexpr bool value = true; };
template <> struct Packable<LotkaVolterra> { static constexpr bool value = true; };
template <int DD> struct Packable<Linear<DD>> { static constexpr bool value = true; };
// (Lorenz-96 above 4 components: the pair's registers spill)
template <int DD> struct Packable<Lorenz96<DD>> { static constexpr bool value = DD <= 4; };

template <class F>
struct F32Step {
  using R = typename std::conditional<Packable<F>::value, F1, float>::type;
};

__device__ __forceinline__ float fval(F1 x) { return x.v; }
__device__ __forceinline__ float fval(float x) { return x; }

template <int N, class R>
__device__ __forceinline__ void to_f1(const float* x, R* y) {
#pragma unroll
  for (int i = 0; i < N; ++i) y[i] = R(x[i]);
}

template <int N, class R>
__device__ __forceinline__ void from_f1(const R* x, float* y) {
#pragma unroll
  for (int i = 0; i < N; ++i) y[i] = fval(x[i]);
}

template <class F>
__device__ __forceinline__ void rhs_f1(const float* y, const float* p, float* dy) {
  using R = typename F32Step<F>::R;
  R yy[F::D], pp[F::P], dd[F::D];
  to_f1<F::D>(y, yy);
  to_f1<F::P>(p, pp);
  F::rhs(yy, pp, dd);
  from_f1<F::D>(dd, dy);
}

template <class F>
__device__ __forceinline__ void tsit5_step_f1(float* y, const float* p, float dt) {
  using R = typename F32Step<F>::R;
  R yy[F::D], pp[F::P];
  to_f1<F::D>(y, yy);
  to_f1<F::P>(p, pp);
  tsit5_replay_step<F>(yy, pp, R(dt));
  from_f1<F::D>(yy, y);
}

template <class F>
__device__ __forceinline__ void tsit5_step_vjp_f1(const float* y, const float* p, float dt,
                                                  float* lam, float* gp) {
  using R = typename F32Step<F>::R;
  R yy[F::D], pp[F::P], ll[F::D], gg[F::P];
  to_f1<F::D>(y, yy);
  to_f1<F::P>(p, pp);
  to_f1<F::D>(lam, ll);
  to_f1<F::P>(gp, gg);
  tsit5_step_vjp<F>(yy, pp, R(dt), ll, gg);
  from_f1<F::D>(ll, lam);
  from_f1<F::P>(gg, gp);
}

// sum of squares (e_i / sc_i)^2, in component order.  The quotients are the hardware's
// approximate division (reciprocal and product, within 2 ulp of the rounded quotient for the
// scales' range, atol > 0 up to 2^126).
template <int D>
__device__ __forceinline__ float sumsq_f32(const float* e, const float* y, const float* yn,
                                           float rtol, float atol) {
  float acc = 0.0f;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    const float sc = atol + rtol * fmaxf(fabsf(y[i]), fabsf(yn[i]));
    const float q = __fdividef(e[i], sc);
    acc += q * q;
  }
  return acc;
}

struct F32Counters {
  float t, dt;
  int it, acc, rej, st, ck_cnt, ck_slot;
};

// method: 0 Tsit5, 1 Rosenbrock23.  kStore = false: the forward-only solve.
template <class F, int kMethod, bool kStore>
__global__ void __launch_bounds__(128) f32_record_kernel(const RecordArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  float y[D], k1[D], p[P];
#pragma unroll
  for (int i = 0; i < D; ++i) y[i] = (float)a.y0[j * D + i];
#pragma unroll
  for (int i = 0; i < P; ++i) p[i] = (float)a.p[j * P + i];
  float* rec = kStore ? reinterpret_cast<float*>(a.rec) : nullptr;
  float* ckpt = kStore ? reinterpret_cast<float*>(a.ckpt) : nullptr;
  const bool rec_on = rec != nullptr, ck_on = ckpt != nullptr;
  const double t1d = a.t1v ? a.t1v[j] : a.t1;
  const float t1 = (float)t1d;
  const float rtol = (float)a.rtol, atol = (float)a.atol;
  F32Counters c;
  c.t = (float)a.t0;
  // the first step as the reference host computes it, (t1 - t0)/100 in float64, then rounded
  c.dt = (float)(a.dt0 > 0.0 ? a.dt0 : (t1d - a.t0) / 100.0);
  c.it = c.acc = c.rej = c.st = c.ck_cnt = c.ck_slot = 0;
  // this trajectory's slots of the current 4-step record chunk (rec_index, advanced)
  float* rp = rec_on ? rec + j * 4 : nullptr;
  const long long rstride = 4 * a.n;
  if (ck_on) store_ckpt_f32<D>(ckpt, a.n, j, 0, y, c.t);
  if constexpr (kMethod == 0) rhs_f1<F>(y, p, k1);
  while (c.it < a.max_steps && c.t < t1) {
    const float h = (t1 - c.t < c.dt) ? (t1 - c.t) : c.dt;
    if (kMethod == 1 && c.t + h == c.t) {  // the step no longer advances time
      c.st = 2;
      break;
    }
    ++c.it;
    float yn[D], kn[D], e[D];
    if constexpr (kMethod == 0) {
      using T = Tsit5;
      using R = typename F32Step<F>::R;
      R y1[D], p1[P], k11[D], yn1[D];
      to_f1<D>(y, y1);
      to_f1<P>(p, p1);
      to_f1<D>(k1, k11);
      Stages<F, R> S;
      tsit5_k2_to_k6<F>(y1, p1, k11, R(h), S);
      tsit5_y5<F>(y1, k11, S, R(h), yn1);
      from_f1<D>(yn1, yn);
      rhs_f1<F>(yn, p, kn);
#pragma unroll
      for (int i = 0; i < D; ++i)
        e[i] = h * (float(T::E1) * k1[i] + float(T::E2) * fval(S.k2[i]) +
                    float(T::E3) * fval(S.k3[i]) + float(T::E4) * fval(S.k4[i]) +
                    float(T::E5) * fval(S.k5[i]) + float(T::E6) * fval(S.k6[i]) +
                    float(T::E7) * kn[i]);
    } else {
      RosCore<F, float> rc;
      ros23_core<F>(y, p, h, rc, yn);
      float fy[D], r3[D], k3[D];
      F::rhs(yn, p, fy);
#pragma unroll
      for (int i = 0; i < D; ++i)
        r3[i] = fy[i] - float(Ros23::E32) * (rc.k2[i] - rc.F1[i]) - 2.0f * (rc.k1[i] - rc.F0[i]);
      lu_solve(rc.W, r3, k3);
#pragma unroll
      for (int i = 0; i < D; ++i) e[i] = (h / 6.0f) * (rc.k1[i] - 2.0f * rc.k2[i] + k3[i]);
    }
    const float S = sumsq_f32<D>(e, y, yn, rtol, atol);
    if (!(S == S)) {
      c.st = 1;
      break;
    }
    if (S <= a.ctrlf.accept_sum) {  // sqrtf(S / D) <= 1
      if ((rec_on || ck_on) && c.acc >= a.cap) {
        c.st = 3;
        break;
      }
      c.t = c.t + h;
      if (rec_on) {
        rp[c.acc & 3] = h;
        if ((c.acc & 3) == 3) rp += rstride;
      }
      ++c.acc;
#pragma unroll
      for (int i = 0; i < D; ++i) {
        y[i] = yn[i];
        if constexpr (kMethod == 0) k1[i] = kn[i];
      }
      if (ck_on && ++c.ck_cnt == a.ck_every) {
        c.ck_cnt = 0;
        if (++c.ck_slot < a.ck_slots) store_ckpt_f32<D>(ckpt, a.n, j, c.ck_slot, y, c.t);
      }
    } else {
      ++c.rej;
    }
    c.dt = step_from_sum_f32(S, h, a.ctrlf);
  }
  if (c.st == 0 && !(c.t >= t1)) c.st = 1;
  if (rec_on) {  // zero-pad the last chunk (identity steps)
    for (int s = c.acc; (s & 3) != 0; ++s) rp[s & 3] = 0.0f;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) a.yf[j * D + i] = (double)y[i];
  a.n_acc[j] = c.acc;
  a.n_rej[j] = c.rej;
  a.status[j] = c.st;
}

template <class F, int kMethod>
__device__ __forceinline__ void f32_step(float* y, const float* p, float dt) {
  if constexpr (kMethod == 0)
    tsit5_step_f1<F>(y, p, dt);
  else
    ros23_replay_step<F>(y, p, dt);
}

template <class F, int kMethod>
__global__ void __launch_bounds__(128) f32_replay_kernel(const ReplayArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  float y[D], p[P];
#pragma unroll
  for (int i = 0; i < D; ++i) y[i] = (float)a.y0[j * D + i];
#pragma unroll
  for (int i = 0; i < P; ++i) p[i] = (float)a.p[j * P + i];
  const float* rec = reinterpret_cast<const float*>(a.rec);
  float* ckpt = reinterpret_cast<float*>(a.ckpt);
  const int na = steps_in_record(a.n_acc, j, a.cap);
  float t = (float)a.t0;
  const bool ck_on = ckpt != nullptr;
  if (ck_on) store_ckpt_f32<D>(ckpt, a.n, j, 0, y, t);
  int ck_cnt = 0, ck_slot = 0;
  for (int s = 0; s < na; ++s) {
    const float dt = load_rec_f32(rec, a.n, j, s);
    f32_step<F, kMethod>(y, p, dt);
    t = t + dt;
    if (ck_on && ++ck_cnt == a.ck_every) {
      ck_cnt = 0;
      if (++ck_slot < a.ck_slots) store_ckpt_f32<D>(ckpt, a.n, j, ck_slot, y, t);
    }
  }
#pragma unroll
  for (int i = 0; i < D; ++i) a.yf[j * D + i] = (double)y[i];
}

// Per-thread float segment states in dynamic shared memory (element e of thread t at
// e * blockDim + t), K states of D floats.
extern __shared__ float gs_seg_smem_f32[];

template <class F, int kMethod>
__global__ void __launch_bounds__(128) f32_adjoint_kernel(const AdjointArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const long long j = lane_traj(a, t);
  if (j < 0) return;
  float p[P], lam[D], gp[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    p[i] = (float)a.p[j * P + i];
    gp[i] = 0.0f;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] = (float)a.ybar[j * D + i];
  const float* rec = reinterpret_cast<const float*>(a.rec);
  const float* ckpt = reinterpret_cast<const float*>(a.ckpt);
  float* st = gs_seg_smem_f32 + threadIdx.x;
  const int stride = blockDim.x;
  const int na = steps_in_record(a.n_acc, j, a.cap);
  const int K = a.ck_every;
  const int nseg = (na + K - 1) / K;
  const int top = warp_top_segments(nseg);
  for (int sg = top - 1; sg >= 0; --sg) {
    if (sg >= nseg) continue;  // in step with the warp's longest trajectory
    float y[D];
    load_ckpt_f32<D>(ckpt, a.n, j, sg, y);
    const int start = sg * K;
    for (int q = 0; q < K; ++q) {  // the segment's states, y_start .. y_start+K-1
#pragma unroll
      for (int i = 0; i < D; ++i) st[(q * D + i) * stride] = y[i];
      const int s = start + q;
      if (q + 1 < K && s < na) f32_step<F, kMethod>(y, p, load_rec_f32(rec, a.n, j, s));
    }
    for (int q = K - 1; q >= 0; --q) {
      const int s = start + q;
      if (s >= na) continue;
      const float dt = load_rec_f32(rec, a.n, j, s);
      if (dt == 0.0f) continue;
      float ys[D];
#pragma unroll
      for (int i = 0; i < D; ++i) ys[i] = st[(q * D + i) * stride];
      if constexpr (kMethod == 0)
        tsit5_step_vjp_f1<F>(ys, p, dt, lam, gp);
      else
        ros23_step_vjp<F>(ys, p, dt, lam, gp);
    }
  }
  if (a.gy0) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.gy0[j * D + i] = (double)lam[i];
  }
  if (a.gp) {
#pragma unroll
    for (int i = 0; i < P; ++i) a.gp[j * P + i] = (double)gp[i];
  }
}

// --- the float32 reverse pass, two trajectories per thread ---------------------------------
// Thread u sweeps lanes 2u and 2u + 1 (trajectories lane_traj(2u), lane_traj(2u + 1): with the
// lanes ordered by step count, neighbours with similar records) through f32_adjoint_kernel's
// segments, both halves in one F2 (gs_pack.cuh), so every float operation of the replay and
// the step VJPs is issued once for the pair.  The pair runs the longer of its two records: the
// shorter half takes dt = 0 steps past its own end from a zero state (a dt = 0 step is an
// exact identity in value and gradient), so its cotangent and gradient are left as its own
// record made them.  A half without a trajectory (odd n, or an order entry outside [0, n))
// runs as an empty record and writes nothing.

__device__ __forceinline__ F2 pair_dt(const float* rec, long long n, long long j0, long long j1,
                                      int na0, int na1, int s) {
  return F2(s < na0 ? load_rec_f32(rec, n, j0, s) : 0.0f,
            s < na1 ? load_rec_f32(rec, n, j1, s) : 0.0f);
}

template <class F>
__global__ void __launch_bounds__(128) f32_adjoint_pairs_kernel(const AdjointArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (2 * u >= a.n) return;
  const long long j0 = lane_traj(a, 2 * u);
  const long long j1 = 2 * u + 1 < a.n ? lane_traj(a, 2 * u + 1) : -1;
  F2 p[P], lam[D], gp[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    p[i] = F2(j0 >= 0 ? (float)a.p[j0 * P + i] : 0.0f, j1 >= 0 ? (float)a.p[j1 * P + i] : 0.0f);
    gp[i] = F2(0.0);
  }
#pragma unroll
  for (int i = 0; i < D; ++i)
    lam[i] = F2(j0 >= 0 ? (float)a.ybar[j0 * D + i] : 0.0f,
                j1 >= 0 ? (float)a.ybar[j1 * D + i] : 0.0f);
  const float* rec = reinterpret_cast<const float*>(a.rec);
  const float* ckpt = reinterpret_cast<const float*>(a.ckpt);
  // element e of thread t at e * blockDim + t, one F2 (8 bytes) per element
  F2* st = reinterpret_cast<F2*>(gs_seg_smem_f32) + threadIdx.x;
  const int stride = blockDim.x;
  const int na0 = j0 >= 0 ? steps_in_record(a.n_acc, j0, a.cap) : 0;
  const int na1 = j1 >= 0 ? steps_in_record(a.n_acc, j1, a.cap) : 0;
  const int K = a.ck_every;
  const int ns0 = (na0 + K - 1) / K, ns1 = (na1 + K - 1) / K;
  const int nseg = ns0 > ns1 ? ns0 : ns1;
  const int top = warp_top_segments(nseg);
  for (int sg = top - 1; sg >= 0; --sg) {
    if (sg >= nseg) continue;  // in step with the warp's longest trajectory
    float ya[D], yb[D];
    if (sg < ns0) {
      load_ckpt_f32<D>(ckpt, a.n, j0, sg, ya);
    } else {
#pragma unroll
      for (int i = 0; i < D; ++i) ya[i] = 0.0f;
    }
    if (sg < ns1) {
      load_ckpt_f32<D>(ckpt, a.n, j1, sg, yb);
    } else {
#pragma unroll
      for (int i = 0; i < D; ++i) yb[i] = 0.0f;
    }
    F2 y[D];
#pragma unroll
    for (int i = 0; i < D; ++i) y[i] = F2(ya[i], yb[i]);
    const int start = sg * K;
    for (int q = 0; q < K; ++q) {  // the segment's states, y_start .. y_start+K-1
#pragma unroll
      for (int i = 0; i < D; ++i) st[(q * D + i) * stride] = y[i];
      const int s = start + q;
      if (q + 1 < K && (s < na0 || s < na1))
        tsit5_replay_step<F>(y, p, pair_dt(rec, a.n, j0, j1, na0, na1, s));
    }
    for (int q = K - 1; q >= 0; --q) {
      const int s = start + q;
      const F2 dt = pair_dt(rec, a.n, j0, j1, na0, na1, s);
      if (dt.v.x == 0.0f && dt.v.y == 0.0f) continue;
      F2 ys[D];
#pragma unroll
      for (int i = 0; i < D; ++i) ys[i] = st[(q * D + i) * stride];
      tsit5_step_vjp<F>(ys, p, dt, lam, gp);
    }
  }
  if (a.gy0) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      if (j0 >= 0) a.gy0[j0 * D + i] = (double)lam[i].v.x;
      if (j1 >= 0) a.gy0[j1 * D + i] = (double)lam[i].v.y;
    }
  }
  if (a.gp) {
#pragma unroll
    for (int i = 0; i < P; ++i) {
      if (j0 >= 0) a.gp[j0 * P + i] = (double)gp[i].v.x;
      if (j1 >= 0) a.gp[j1 * P + i] = (double)gp[i].v.y;
    }
  }
}

// --- dense output (saveat) on the float32 route --------------------------------------------
// The semantics of replay_saveat_kernel / adjoint_saveat_kernel (gs_saveat.cuh,
// gradsolve/solvers/dense.py:106-163) in float: the reference's f32 closure casts the
// requested times to float32 with the rest (gradsolve/warp/warp_replay.py:213-217), so the
// times, the accumulated step times, the bracket tests and the re-step sizes ts_k - t are all
// float32 here.  The checkpoint rows carry each segment start's time (float32), from which the
// adjoint rebuilds the step times with the replay's own additions.
template <int D>
__device__ __forceinline__ void store_row_f32(double* dst, const float* v) {
#pragma unroll
  for (int i = 0; i < D; ++i) dst[i] = (double)v[i];
}

template <int D>
__device__ __forceinline__ float load_ckpt_time_f32(const float* ckpt, long long n, long long j,
                                                    int slot) {
  constexpr int CW = (D + 4) & ~3;
  return __ldg(ckpt + ((size_t)slot * (size_t)n + (size_t)j) * CW + D);
}

template <class F, int kMethod>
__global__ void __launch_bounds__(128) f32_replay_saveat_kernel(const SaveatArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  float y[D], p[P];
#pragma unroll
  for (int i = 0; i < D; ++i) y[i] = (float)a.y0[j * D + i];
#pragma unroll
  for (int i = 0; i < P; ++i) p[i] = (float)a.p[j * P + i];
  const float* rec = reinterpret_cast<const float*>(a.rec);
  float* ckpt = reinterpret_cast<float*>(a.ckpt);
  const double* ts = a.ts + j * a.ts_ld;
  double* ys = a.ys + j * (long long)a.K * D;
  const int na = steps_in_record(a.n_acc, j, a.cap);
  float t = (float)a.t0;
  int kk = 0;
  while (kk < a.K && (float)ts[kk] <= t) {  // never bracketed: y0
    store_row_f32<D>(ys + (long long)kk * D, y);
    ++kk;
  }
  const bool ck_on = ckpt != nullptr;
  if (ck_on) store_ckpt_f32<D>(ckpt, a.n, j, 0, y, t);
  int ck_cnt = 0, ck_slot = 0;
  for (int s = 0; s < na; ++s) {
    const float dt = load_rec_f32(rec, a.n, j, s);
    if (dt > 0.0f) {
      const float tn = t + dt;
      while (kk < a.K && (float)ts[kk] <= tn) {  // bracketed by this step: re-step to ts
        float yk[D];
#pragma unroll
        for (int i = 0; i < D; ++i) yk[i] = y[i];
        f32_step<F, kMethod>(yk, p, (float)ts[kk] - t);
        store_row_f32<D>(ys + (long long)kk * D, yk);
        ++kk;
      }
      f32_step<F, kMethod>(y, p, dt);
      t = tn;
    }
    if (ck_on && ++ck_cnt == a.ck_every) {
      ck_cnt = 0;
      if (++ck_slot < a.ck_slots) store_ckpt_f32<D>(ckpt, a.n, j, ck_slot, y, t);
    }
  }
  // times at or past the final accumulated time take y_final itself
  for (int k = a.K - 1; k >= 0 && (float)ts[k] >= t; --k) store_row_f32<D>(ys + (long long)k * D, y);
  for (int k = kk; k < a.K; ++k) store_row_f32<D>(ys + (long long)k * D, y);
  store_row_f32<D>(a.yf + j * D, y);
}

// Segment buffer in dynamic shared memory: K rows of D + 1 floats (state, step start time)
// per thread, element e of thread t at e * blockDim + t.
template <class F, int kMethod>
__global__ void __launch_bounds__(128) f32_adjoint_saveat_kernel(const SaveatArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  float p[P], lam[D], gp[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    p[i] = (float)a.p[j * P + i];
    gp[i] = 0.0f;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] = a.ybar ? (float)a.ybar[j * D + i] : 0.0f;
  const float* rec = reinterpret_cast<const float*>(a.rec);
  const float* ckpt = reinterpret_cast<const float*>(a.ckpt);
  const double* ts = a.ts + j * a.ts_ld;
  const double* ysb = a.ysbar + j * (long long)a.K * D;
  float* st = gs_seg_smem_f32 + threadIdx.x;
  const int stride = blockDim.x;
  const int na = steps_in_record(a.n_acc, j, a.cap);
  const int K = a.ck_every;
  const int nseg = (na + K - 1) / K;
  int kk = a.K;  // times [0, kk) not yet assigned to a step
  float tlast = kk > 0 ? (float)ts[kk - 1] : -CUDART_INF_F;
  auto pop = [&]() {
    --kk;
    tlast = kk > 0 ? (float)ts[kk - 1] : -CUDART_INF_F;
  };
  auto add_row = [&](float* acc, int k) {
#pragma unroll
    for (int i = 0; i < D; ++i) acc[i] += (float)ysb[(long long)k * D + i];
  };
  if (nseg == 0) {
    const float tfin = (float)a.t0;
    while (tlast >= tfin) {
      add_row(lam, kk - 1);
      pop();
    }
  }
  bool fin_done = false;  // cotangents of times >= t_fin joined lam
  const int top = warp_top_segments(nseg);
  for (int sg = top - 1; sg >= 0; --sg) {
    if (sg >= nseg) continue;  // in step with the warp's longest trajectory
    float y[D];
    load_ckpt_f32<D>(ckpt, a.n, j, sg, y);
    float t = load_ckpt_time_f32<D>(ckpt, a.n, j, sg);
    const int start = sg * K;
    for (int q = 0; q < K; ++q) {  // states y_{start+q} with their times; t ends at the segment end
#pragma unroll
      for (int i = 0; i < D; ++i) st[(q * (D + 1) + i) * stride] = y[i];
      st[(q * (D + 1) + D) * stride] = t;
      const int s = start + q;
      const float dt = s < na ? load_rec_f32(rec, a.n, j, s) : 0.0f;
      if (dt > 0.0f) {
        if (q + 1 < K) f32_step<F, kMethod>(y, p, dt);
        t = t + dt;
      }
    }
    if (!fin_done) {  // first processed segment: t is t_fin
      fin_done = true;
      while (tlast >= t) {
        add_row(lam, kk - 1);
        pop();
      }
    }
    for (int q = K - 1; q >= 0; --q) {
      const int s = start + q;
      const float dt = s < na ? load_rec_f32(rec, a.n, j, s) : 0.0f;
      if (!(dt > 0.0f)) continue;
      float ys[D], add[D];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        ys[i] = st[(q * (D + 1) + i) * stride];
        add[i] = 0.0f;
      }
      const float ts0 = st[(q * (D + 1) + D) * stride];
      while (tlast > ts0) {  // re-steps bracketed by this step
        const float tk = tlast;
        float w[D];
#pragma unroll
        for (int i = 0; i < D; ++i) w[i] = (float)ysb[(long long)(kk - 1) * D + i];
        pop();
        if constexpr (kMethod == 0)
          tsit5_step_vjp_f1<F>(ys, p, tk - ts0, w, gp);
        else
          ros23_step_vjp<F>(ys, p, tk - ts0, w, gp);
#pragma unroll
        for (int i = 0; i < D; ++i) add[i] += w[i];
      }
      if constexpr (kMethod == 0)
        tsit5_step_vjp_f1<F>(ys, p, dt, lam, gp);
      else
        ros23_step_vjp<F>(ys, p, dt, lam, gp);
#pragma unroll
      for (int i = 0; i < D; ++i) lam[i] += add[i];
    }
  }
  // remaining times were never bracketed (ts <= t0): their value is y0
  for (int k = 0; k < kk; ++k) add_row(lam, k);
  if (a.gy0) {
#pragma unroll
    for (int i = 0; i < D; ++i) a.gy0[j * D + i] = (double)lam[i];
  }
  if (a.gp) {
#pragma unroll
    for (int i = 0; i < P; ++i) a.gp[j * P + i] = (double)gp[i];
  }
}

}  // namespace gs
