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
// err <= 1, dt = h * clip(0.9 * max(err, 1e-10)^(-1/q), 0.2, 5) after accept and reject.
#pragma once

#include <math_constants.h>

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

// sum of squares (e_i / sc_i)^2, in component order
template <int D>
__device__ __forceinline__ float sumsq_f32(const float* e, const float* y, const float* yn,
                                           float rtol, float atol) {
  float acc = 0.0f;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    const float sc = atol + rtol * fmaxf(fabsf(y[i]), fabsf(yn[i]));
    const float q = e[i] / sc;
    acc += q * q;
  }
  return acc;
}

// The controller on err = sqrt(S / D) with exponent -1/q (q = 5 Tsit5, 3 Rosenbrock23).
__device__ __forceinline__ float step_f32(float err, float h, float expo) {
  float fac = 0.9f * powf(fmaxf(err, 1e-10f), expo);
  fac = fac > 0.2f ? fac : 0.2f;
  fac = 5.0f < fac ? 5.0f : fac;
  return h * fac;
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
  if (ck_on) store_ckpt_f32<D>(ckpt, a.n, j, 0, y, c.t);
  if constexpr (kMethod == 0) F::rhs(y, p, k1);
  const float expo = kMethod == 0 ? -0.2f : -1.0f / 3.0f;
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
      Stages<F, float> S;
      tsit5_k2_to_k6<F>(y, p, k1, h, S);
      tsit5_y5<F>(y, k1, S, h, yn);
      F::rhs(yn, p, kn);
#pragma unroll
      for (int i = 0; i < D; ++i)
        e[i] = h * (float(T::E1) * k1[i] + float(T::E2) * S.k2[i] + float(T::E3) * S.k3[i] +
                    float(T::E4) * S.k4[i] + float(T::E5) * S.k5[i] + float(T::E6) * S.k6[i] +
                    float(T::E7) * kn[i]);
    } else {
      RosCore<F, float> rc;
      ros23_core<F>(y, p, h, rc, yn);
      float F2[D], r3[D], k3[D];
      F::rhs(yn, p, F2);
#pragma unroll
      for (int i = 0; i < D; ++i)
        r3[i] = F2[i] - float(Ros23::E32) * (rc.k2[i] - rc.F1[i]) - 2.0f * (rc.k1[i] - rc.F0[i]);
      lu_solve(rc.W, r3, k3);
#pragma unroll
      for (int i = 0; i < D; ++i) e[i] = (h / 6.0f) * (rc.k1[i] - 2.0f * rc.k2[i] + k3[i]);
    }
    const float err = sqrtf(sumsq_f32<D>(e, y, yn, rtol, atol) / (float)D);
    if (!(err == err)) {
      c.st = 1;
      break;
    }
    if (err <= 1.0f) {
      if ((rec_on || ck_on) && c.acc >= a.cap) {
        c.st = 3;
        break;
      }
      c.t = c.t + h;
      if (rec_on) rec[rec_index(j, c.acc, a.n)] = h;
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
    c.dt = step_f32(err, h, expo);
  }
  if (c.st == 0 && !(c.t >= t1)) c.st = 1;
  if (rec_on) {  // zero-pad the last sector (identity steps)
    for (int s = c.acc; (s & 3) != 0; ++s) rec[rec_index(j, s, a.n)] = 0.0f;
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
    tsit5_replay_step<F>(y, p, dt);
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
        tsit5_step_vjp<F>(ys, p, dt, lam, gp);
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
          tsit5_step_vjp<F>(ys, p, tk - ts0, w, gp);
        else
          ros23_step_vjp<F>(ys, p, tk - ts0, w, gp);
#pragma unroll
        for (int i = 0; i < D; ++i) add[i] += w[i];
      }
      if constexpr (kMethod == 0)
        tsit5_step_vjp<F>(ys, p, dt, lam, gp);
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
