// gs_saveat.cuh -- dense output ("saveat") on the frozen-mesh replay, and its adjoint.
//
// Semantics of gradsolve/solvers/dense.py:106-163 (scan_saveat_one), per trajectory:
//   * a requested time ts_k is bracketed by the step [t, t+dt] with dt > 0, t < ts_k <= t+dt;
//     its value is ONE genuine step of the lane's own method of size ts_k - t from the
//     state at the start of that step (bracket-and-re-step, not an interpolant);
//   * times no step brackets (ts_k <= t0) take y0;
//   * times at or past the final accumulated time t_fin = t0 + sum(dt) take y_final itself,
//     bitwise (which makes y_saved[:, -1] == y_final when ts[-1] = t1).
// Requested times are sorted and validated on the host (dense.py:81-103).  Each trajectory
// may have its own row of times (row stride ts_ld) or share one row (ts_ld = 0), and its own
// end time (the record carries it).
//
// The adjoint adds, for every bracketed time, the VJP of its re-step at the bracketing step's
// start state to the cotangent of that state; cotangents of times >= t_fin join the final
// cotangent and those of times <= t0 go to dL/dy0 directly.  Times t_s of the steps are
// rebuilt from the checkpoints (which store t) with the replay's own additions, so the bracket
// decisions are bitwise those of the forward.
#pragma once
#include <math_constants.h>

#include "gs_mixed.cuh"
#include "gs_ros23.cuh"
#include "gs_tsit5.cuh"

namespace gs {

// Step policies: the lane's own step and step-VJP.  c is the compensated-sum carry of the
// float32-stage mode; pf the float parameters (both unused by the float64 methods).
struct Tsit5F64Step {
  template <class F>
  static __device__ __forceinline__ void step(double* y, double*, const double* p, const float*,
                                              double dt) {
    tsit5_replay_step<F>(y, p, dt);
  }
  template <class F>
  static __device__ __forceinline__ void vjp(const double* y, const double* p, const float*,
                                             double dt, double* lam, double* gp) {
    tsit5_step_vjp<F>(y, p, dt, lam, gp);
  }
};

struct Tsit5MixedStep {
  template <class F>
  static __device__ __forceinline__ void step(double* y, double* c, const double* p,
                                              const float* pf, double dt) {
    mixed_replay_step<F>(y, c, p, pf, dt);
  }
  template <class F>
  static __device__ __forceinline__ void vjp(const double* y, const double* p, const float* pf,
                                             double dt, double* lam, double* gp) {
    double acc[F::D];
#pragma unroll
    for (int i = 0; i < F::D; ++i) acc[i] = lam[i];
    mixed_step_vjp<F>(y, p, pf, dt, acc, gp);
#pragma unroll
    for (int i = 0; i < F::D; ++i) lam[i] = acc[i];
  }
};

struct Ros23Step {
  template <class F>
  static __device__ __forceinline__ void step(double* y, double*, const double* p, const float*,
                                              double dt) {
    ros23_replay_step<F>(y, p, dt);
  }
  template <class F>
  static __device__ __forceinline__ void vjp(const double* y, const double* p, const float*,
                                             double dt, double* lam, double* gp) {
    ros23_step_vjp<F>(y, p, dt, lam, gp);
  }
};

struct SaveatArgs {
  long long n;
  const double* y0;
  const double* p;
  double t0;
  const double* rec;
  const int* n_acc;
  int ck_every, ck_slots;
  double* ckpt;          // written by the replay, read by the adjoint
  const double* ts;      // requested times, row j at ts + j * ts_ld
  long long ts_ld;
  int K;                 // times per trajectory
  double* ys;            // (n, K, D) saved states (replay)
  double* yf;            // (n, D) final states (replay)
  const double* ysbar;   // (n, K, D) cotangents of ys (adjoint)
  const double* ybar;    // (n, D) cotangent of y_final or null (adjoint)
  double* gy0;
  double* gp;
  int cap;               // record capacity: step counts are clamped to [0, cap]
};

template <int D>
__device__ __forceinline__ void store_row(double* dst, const double* v) {
#pragma unroll
  for (int i = 0; i < D; ++i) dst[i] = v[i];
}

template <class F, class M>
__global__ void __launch_bounds__(128) replay_saveat_kernel(const SaveatArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  double y[D], c[D], p[P];
  float pf[P];
#pragma unroll
  for (int i = 0; i < D; ++i) { y[i] = a.y0[j * D + i]; c[i] = 0.0; }
#pragma unroll
  for (int i = 0; i < P; ++i) { p[i] = a.p[j * P + i]; pf[i] = (float)p[i]; }
  const double* ts = a.ts + j * a.ts_ld;
  double* ys = a.ys + j * (long long)a.K * D;
  const int na = steps_in_record(a.n_acc, j, a.cap);
  double t = a.t0;
  int kk = 0;
  while (kk < a.K && ts[kk] <= t) {  // never bracketed: y0
    store_row<D>(ys + (long long)kk * D, y);
    ++kk;
  }
  const bool ck_on = a.ckpt != nullptr;
  if (ck_on) store_ckpt<D>(a.ckpt, a.n, j, 0, y, t);
  int ck_cnt = 0, ck_slot = 0;
  for (int s = 0; s < na; ++s) {
    const double dt = load_rec(a.rec, a.n, j, s);
    if (dt > 0.0) {
      const double tn = t + dt;
      while (kk < a.K && ts[kk] <= tn) {  // bracketed by this step: re-step to ts
        double yk[D], ck[D];
#pragma unroll
        for (int i = 0; i < D; ++i) { yk[i] = y[i]; ck[i] = 0.0; }
        M::template step<F>(yk, ck, p, pf, ts[kk] - t);
        store_row<D>(ys + (long long)kk * D, yk);
        ++kk;
      }
      M::template step<F>(y, c, p, pf, dt);
      t = tn;
    }
    if (ck_on && ++ck_cnt == a.ck_every) {
      ck_cnt = 0;
      if (++ck_slot < a.ck_slots) store_ckpt<D>(a.ckpt, a.n, j, ck_slot, y, t);
    }
  }
  // times at or past the final accumulated time take y_final itself
  for (int k = a.K - 1; k >= 0 && ts[k] >= t; --k) store_row<D>(ys + (long long)k * D, y);
  for (int k = kk; k < a.K; ++k) store_row<D>(ys + (long long)k * D, y);
  store_row<D>(a.yf + j * D, y);
}

template <class F, class M>
__global__ void __launch_bounds__(128) adjoint_saveat_kernel(const SaveatArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  double p[P], lam[D], gp[P];
  float pf[P];
#pragma unroll
  for (int i = 0; i < P; ++i) { p[i] = a.p[j * P + i]; pf[i] = (float)p[i]; gp[i] = 0.0; }
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] = a.ybar ? a.ybar[j * D + i] : 0.0;
  const double* ts = a.ts + j * a.ts_ld;
  const double* ysb = a.ysbar + j * (long long)a.K * D;
  const int na = steps_in_record(a.n_acc, j, a.cap);
  const int K = a.ck_every;
  const int nseg = (na + K - 1) / K;
  // segment buffer (states with their step start time at index D) and cp.async prefetch of
  // the next segment's checkpoint and dts, as in tsit5_adjoint_kernel
  AdjBuf<D, D + 1> buf(K);
  int b = 0;
  int kk = a.K;  // times [0, kk) not yet assigned to a step
  // ts[kk - 1] held in a register (-inf once every time is assigned)
  double tlast = kk > 0 ? ts[kk - 1] : -CUDART_INF;
  auto pop = [&]() {
    --kk;
    tlast = kk > 0 ? ts[kk - 1] : -CUDART_INF;
  };
  if (nseg == 0) {
    const double tfin = a.t0;
    while (tlast >= tfin) {
#pragma unroll
      for (int i = 0; i < D; ++i) lam[i] += ysb[(long long)(kk - 1) * D + i];
      pop();
    }
  } else {
    prefetch_segment<D>(buf, b, a.ckpt, a.rec, a.n, j, nseg - 1, K, na);
  }
  bool fin_done = false;  // cotangents of times >= t_fin joined lam
  const int top = warp_top_segments(nseg);
  for (int sg = top - 1; sg >= 0; --sg) {
    if (sg >= nseg) continue;  // in step with the warp's longest trajectory
    cp_async_wait_all();
    double y[D], c[D];
#pragma unroll
    for (int i = 0; i < D; ++i) { y[i] = buf.ck(b, i); c[i] = 0.0; }
    double t = buf.ck(b, D);
    if (sg > 0) prefetch_segment<D>(buf, b ^ 1, a.ckpt, a.rec, a.n, j, sg - 1, K, na);
#pragma unroll
    for (int i = 0; i < D; ++i) buf.st(0, i) = y[i];
    buf.st(0, D) = t;
    for (int q = 1; q <= K; ++q) {  // states y_{start+q} and times (q = K: segment end)
      const double dt = buf.dt(b, q - 1);
      if (dt > 0.0) {
        if (q < K) M::template step<F>(y, c, p, pf, dt);
        t = t + dt;
      }
      if (q < K) {
#pragma unroll
        for (int i = 0; i < D; ++i) buf.st(q, i) = y[i];
        buf.st(q, D) = t;
      }
    }
    if (!fin_done) {  // first processed segment: t is t_fin
      fin_done = true;
      while (tlast >= t) {
#pragma unroll
        for (int i = 0; i < D; ++i) lam[i] += ysb[(long long)(kk - 1) * D + i];
        pop();
      }
    }
    for (int q = K - 1; q >= 0; --q) {
      const double dt = buf.dt(b, q);
      if (dt > 0.0) {
        double ys[D], add[D];
#pragma unroll
        for (int i = 0; i < D; ++i) { ys[i] = buf.st(q, i); add[i] = 0.0; }
        const double ts0 = buf.st(q, D);
        while (tlast > ts0) {  // re-steps bracketed by this step
          const double tk = tlast;
          double w[D];
#pragma unroll
          for (int i = 0; i < D; ++i) w[i] = ysb[(long long)(kk - 1) * D + i];
          pop();
          M::template vjp<F>(ys, p, pf, tk - ts0, w, gp);
#pragma unroll
          for (int i = 0; i < D; ++i) add[i] += w[i];
        }
        M::template vjp<F>(ys, p, pf, dt, lam, gp);
#pragma unroll
        for (int i = 0; i < D; ++i) lam[i] += add[i];
      }
    }
    b ^= 1;
  }
  // remaining times were never bracketed (ts <= t0): their value is y0
  for (int k = 0; k < kk; ++k) {
#pragma unroll
    for (int i = 0; i < D; ++i) lam[i] += ysb[(long long)k * D + i];
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

}  // namespace gs
