// gs_persistent.cuh -- persistent, work-stealing forward and reverse kernels.
//
// The grid holds one wave of resident blocks.  Every lane (thread) takes a trajectory index
// from a global counter (atomicAdd), integrates it, writes its outputs, and takes the next
// one, until the counter passes n.  Each loop iteration is one attempt (forward) or one whole
// segment (reverse) for every active lane, so the lanes of a warp execute the same code every
// iteration: a lane whose trajectory finishes refills itself with a fresh trajectory instead
// of idling until its warp's slowest trajectory ends.  This removes both the last partial
// wave of a one-thread-per-trajectory launch and the idle lanes of warps whose trajectories
// take very different numbers of steps (the uneven-batch workload: 4 to 7841 steps).
//
// The counter lives in a 256-byte control block after the checkpoint slots of the caller's
// checkpoint buffer (gs_ckpt_bytes includes it) and is zeroed on the stream before each
// launch.  Without a counter (a forward solve with neither record nor checkpoints) lanes take
// trajectories j, j + G, j + 2G, ... (G = resident threads) instead.
//
// Per-trajectory arithmetic is exactly that of gs_tsit5.cuh / gs_mixed.cuh / gs_ros23.cuh:
// results do not depend on which lane integrates which trajectory.
#pragma once
#include <math_constants.h>

#include "gs_mixed.cuh"
#include "gs_ros23.cuh"
#include "gs_saveat.cuh"
#include "gs_tsit5.cuh"

namespace gs {

constexpr int kCtrlBytes = 256;
constexpr int kCtrlFwd = 0;  // counter slots (unsigned long long) in the control block
constexpr int kCtrlAdj = 1;

struct Fetch {
  unsigned long long* counter;  // null: static striding
  long long next;
  long long stride;
  __device__ __forceinline__ Fetch(unsigned long long* c) : counter(c) {
    next = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    stride = (long long)gridDim.x * blockDim.x;
  }
  __device__ __forceinline__ long long get() {
    if (counter) return (long long)atomicAdd(counter, 1ull);
    const long long j = next;
    next += stride;
    return j;
  }
};

// ---- forward method policies: per-lane state carried between attempts -----------------
template <class F>
struct LaneTsit5F64 {
  static constexpr int D = F::D, QK = 10;
  using Step = Tsit5F64Step;  // the replay step (saveat re-steps)
  double k1[D], k7[D];
  __device__ __forceinline__ void start(const double* y, const double* p, const float*) {
    F::rhs(y, p, k1);
  }
  // candidate y5 for step h; returns the sum of squares of the scaled error
  __device__ __forceinline__ double trial(const double* y, const double* p, const float*, double h,
                                          double rtol, double atol, double* y5) {
    using T = Tsit5;
    Stages<F> S;
    double e[D];
    tsit5_k2_to_k6<F>(y, p, k1, h, S);
    tsit5_y5<F>(y, k1, S, h, y5);
    F::rhs(y5, p, k7);
#pragma unroll
    for (int i = 0; i < D; ++i)
      e[i] = h * (T::E1 * k1[i] + T::E2 * S.k2[i] + T::E3 * S.k3[i] + T::E4 * S.k4[i] +
                  T::E5 * S.k5[i] + T::E6 * S.k6[i] + T::E7 * k7[i]);
    return wrms_sumsq<D>(e, y, y5, rtol, atol);
  }
  __device__ __forceinline__ void commit() {
#pragma unroll
    for (int i = 0; i < D; ++i) k1[i] = k7[i];
  }
  __device__ __forceinline__ bool degenerate(double, double) const { return false; }
};

template <class F>
struct LaneTsit5Mixed {
  static constexpr int D = F::D, QK = 10;
  using Step = Tsit5MixedStep;
  double k1[D], k7[D], c[D], c5[D];
  __device__ __forceinline__ void start(const double* y, const double* p, const float*) {
    F::rhs(y, p, k1);
#pragma unroll
    for (int i = 0; i < D; ++i) c[i] = 0.0;
  }
  __device__ __forceinline__ double trial(const double* y, const double* p, const float* pf,
                                          double h, double rtol, double atol, double* y5) {
    using T = Tsit5f;
    const float hf = (float)h;
    float yf[D], k1f[D];
    double inc[D], ed[D];
    to_float<F>(y, yf);
    to_float<F>(k1, k1f);
    MixedStages<F> S;
    mixed_dk2_to_dk6<F>(yf, pf, k1f, hf, S);
    mixed_increment<F>(k1, S, h, hf, inc);
#pragma unroll
    for (int i = 0; i < D; ++i) { y5[i] = y[i]; c5[i] = c[i]; }
    kahan_add<D>(y5, c5, inc);
    F::rhs(y5, p, k7);
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const float dk7 = (float)(k7[i] - k1[i]);
      ed[i] = (double)(hf * (T::E2 * S.dk2[i] + T::E3 * S.dk3[i] + T::E4 * S.dk4[i] +
                             T::E5 * S.dk5[i] + T::E6 * S.dk6[i] + T::E7 * dk7));
    }
    return wrms_sumsq<D>(ed, y, y5, rtol, atol);
  }
  __device__ __forceinline__ void commit() {
#pragma unroll
    for (int i = 0; i < D; ++i) { k1[i] = k7[i]; c[i] = c5[i]; }
  }
  __device__ __forceinline__ bool degenerate(double, double) const { return false; }
};

template <class F>
struct LaneRos23 {
  static constexpr int D = F::D, QK = 6;
  using Step = Ros23Step;
  __device__ __forceinline__ void start(const double*, const double*, const float*) {}
  __device__ __forceinline__ double trial(const double* y, const double* p, const float*, double h,
                                          double rtol, double atol, double* ynew) {
    RosCore<F> c;
    ros23_core<F>(y, p, h, c, ynew);
    double F2[D], r3[D], k3[D], ev[D];
    F::rhs(ynew, p, F2);
#pragma unroll
    for (int i = 0; i < D; ++i)
      r3[i] = F2[i] - Ros23::E32 * (c.k2[i] - c.F1[i]) - 2.0 * (c.k1[i] - c.F0[i]);
    lu_solve<D>(c.W, r3, k3);
#pragma unroll
    for (int i = 0; i < D; ++i) ev[i] = (h / 6.0) * (c.k1[i] - 2.0 * c.k2[i] + k3[i]);
    return wrms_sumsq<D>(ev, y, ynew, rtol, atol);
  }
  __device__ __forceinline__ void commit() {}
  // the step no longer advances time: status 2 (gradsolve/solvers/record_jax.py:109)
  __device__ __forceinline__ bool degenerate(double t, double h) const { return t + h == t; }
};

// ---- one thread per trajectory: forward with record and saved states ------------------------
// The per-attempt code of record_persistent_kernel (the same lane policies, accept logic and
// saveat re-steps) without the refill machinery: every thread integrates one trajectory.  On
// Rosenbrock23 the refill state costs registers (VdP: 82 vs 61) and with them resident warps,
// which this latency-bound method needs -- at full occupancy the one-thread-per-trajectory
// forward ran 30% faster.  Uneven batches balance here when their rows come sorted by length
// (the planned tiers of a RecordSet do), since neighbouring threads then take similar numbers
// of attempts.
// A saveat re-step, out of line: re-steps are rare (a few per trajectory against thousands of
// attempts), and inlined, the step's temporaries would raise the register count of the whole
// attempt loop.  Arguments and result travel by value (no address of a register array).
template <int N>
struct DVec {
  double v[N];
};
template <int N>
struct FVec {
  float v[N];
};
template <class F, class L>
__device__ __noinline__ DVec<F::D> restep_out_of_line(DVec<F::D> y, DVec<F::P> p,
                                                      FVec<F::P> pf, double dt) {
  double c[F::D];
#pragma unroll
  for (int i = 0; i < F::D; ++i) c[i] = 0.0;
  L::Step::template step<F>(y.v, c, p.v, pf.v, dt);
  return y;
}

template <class F, class L>
__global__ void __launch_bounds__(128) record_static_kernel(const RecordArgs a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  const bool rec_on = a.rec != nullptr;
  const bool ck_on = a.ckpt != nullptr;
  const bool sv_on = a.ys != nullptr;
  double y[D], ynew[D], p[P];
  float pf[P];
#pragma unroll
  for (int i = 0; i < D; ++i) y[i] = a.y0[j * D + i];
#pragma unroll
  for (int i = 0; i < P; ++i) { p[i] = a.p[j * P + i]; pf[i] = (float)p[i]; }
  double t = a.t0;
  const double t1 = a.t1v ? a.t1v[j] : a.t1;
  double dt = a.dt0 > 0.0 ? a.dt0 : (t1 - a.t0) / 100.0;
  if (ck_on) store_ckpt<D>(a.ckpt, a.n, j, 0, y, t);
  L lane;
  lane.start(y, p, pf);
  const double* tsr = sv_on ? a.ts + j * a.ts_ld : nullptr;
  double* ysr = sv_on ? a.ys + j * (long long)a.K * D : nullptr;
  int kk = 0;
  double tnext = CUDART_INF;  // the next requested time (infinity once all are assigned)
  if (sv_on) {
    while (kk < a.K && tsr[kk] <= t) {  // never bracketed: y0
      store_row<D>(ysr + (long long)kk * D, y);
      ++kk;
    }
    tnext = kk < a.K ? tsr[kk] : CUDART_INF;
  }
  double* rp = rec_on ? a.rec + j * 4 : nullptr;  // this trajectory's slots of the sector
  const long long rstride = 4 * a.n;
  int acc = 0, rej = 0, st = 0, ck_cnt = 0, ck_slot = 0;
  for (int it = 0; it < a.max_steps; ++it) {
    if (t >= t1) break;
    const double h = (t1 - t < dt) ? (t1 - t) : dt;
    if (lane.degenerate(t, h)) {
      st = 2;
      break;
    }
    const double m = lane.trial(y, p, pf, h, a.rtol, a.atol, ynew);
    if (!(m == m)) {
      st = 1;
      break;
    }
    if (m <= a.ctrl.accept_sum) {
      if ((rec_on || ck_on) && acc >= a.cap) {
        st = 3;
        break;
      }
      if (sv_on) {
        const double tn = t + h;
        while (tnext <= tn) {  // bracketed by this step: re-step to ts
          DVec<D> yv;
          DVec<P> pv;
          FVec<P> pfv;
#pragma unroll
          for (int i = 0; i < D; ++i) yv.v[i] = y[i];
#pragma unroll
          for (int i = 0; i < P; ++i) { pv.v[i] = p[i]; pfv.v[i] = pf[i]; }
          const DVec<D> yk = restep_out_of_line<F, L>(yv, pv, pfv, tnext - t);
          store_row<D>(ysr + (long long)kk * D, yk.v);
          ++kk;
          tnext = kk < a.K ? tsr[kk] : CUDART_INF;
        }
      }
      t = t + h;
#pragma unroll
      for (int i = 0; i < D; ++i) y[i] = ynew[i];
      lane.commit();
      if (rec_on) {
        rp[acc & 3] = h;
        if ((acc & 3) == 3) rp += rstride;
      }
      ++acc;
      if (ck_on && ++ck_cnt == a.ck_every) {
        ck_cnt = 0;
        if (++ck_slot < a.ck_slots) store_ckpt<D>(a.ckpt, a.n, j, ck_slot, y, t);
      }
    } else {
      ++rej;
    }
    dt = step_from_sum<L::QK>(m, h, a.ctrl);
  }
  if (st == 0 && !(t >= t1)) st = 1;
  if (rec_on) {  // zero-pad the last sector (identity steps)
    for (int s = acc; (s & 3) != 0; ++s) rp[s & 3] = 0.0;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) a.yf[j * D + i] = y[i];
  if (sv_on) {  // times at or past the final accumulated time take y_final itself
    for (int k = a.K - 1; k >= 0 && tsr[k] >= t; --k) store_row<D>(ysr + (long long)k * D, y);
    for (int k = kk; k < a.K; ++k) store_row<D>(ysr + (long long)k * D, y);
  }
  a.n_acc[j] = acc;
  a.n_rej[j] = rej;
  a.status[j] = st;
}

// ---- persistent forward with record ---------------------------------------------------------
template <class F, class L>
__global__ void __launch_bounds__(128) record_persistent_kernel(const RecordArgs a,
                                                                unsigned long long* counter) {
  constexpr int D = F::D, P = F::P;
  Fetch fetch(counter);
  const bool rec_on = a.rec != nullptr;
  const bool ck_on = a.ckpt != nullptr;
  long long j = fetch.get();
  double y[D], ynew[D], p[P], t = 0.0, t1 = 0.0, dt = 0.0;
  float pf[P];
  int acc = 0, rej = 0, it = 0, ck_cnt = 0, ck_slot = 0;
  // dense output: the saveat rules of replay_saveat_kernel (gs_saveat.cuh) applied while the
  // trajectory is integrated -- a time bracketed by an accepted step [t, t+h] gets one
  // replay step of size ts - t from that step's start state
  const bool sv_on = a.ys != nullptr;
  const double* tsr = nullptr;
  double* ysr = nullptr;
  int kk = 0;
  // the next requested time, held in a register: the bracket test of every accepted step
  // then waits on no load (infinity once every time is assigned)
  double tnext = CUDART_INF;
  L lane;
  auto begin = [&](long long jj) {
#pragma unroll
    for (int i = 0; i < D; ++i) y[i] = a.y0[jj * D + i];
#pragma unroll
    for (int i = 0; i < P; ++i) { p[i] = a.p[jj * P + i]; pf[i] = (float)p[i]; }
    t = a.t0;
    t1 = a.t1v ? a.t1v[jj] : a.t1;
    dt = a.dt0 > 0.0 ? a.dt0 : (t1 - a.t0) / 100.0;
    acc = rej = it = ck_cnt = ck_slot = 0;
    if (ck_on) store_ckpt<D>(a.ckpt, a.n, jj, 0, y, t);
    lane.start(y, p, pf);
    if (sv_on) {
      tsr = a.ts + jj * a.ts_ld;
      ysr = a.ys + jj * (long long)a.K * D;
      kk = 0;
      while (kk < a.K && tsr[kk] <= t) {  // never bracketed: y0
        store_row<D>(ysr + (long long)kk * D, y);
        ++kk;
      }
      tnext = kk < a.K ? tsr[kk] : CUDART_INF;
    }
  };
  if (j < a.n) begin(j);
  while (j < a.n) {
    int st = -1;  // stays -1 while the trajectory is running
    if (t >= t1) {
      st = 0;
    } else if (it >= a.max_steps) {
      st = 1;
    } else {
      const double h = (t1 - t < dt) ? (t1 - t) : dt;
      if (lane.degenerate(t, h)) {
        st = 2;
      } else {
        const double m = lane.trial(y, p, pf, h, a.rtol, a.atol, ynew);
        ++it;
        if (!(m == m)) {
          st = 1;
        } else if (m <= a.ctrl.accept_sum) {
          if ((rec_on || ck_on) && acc >= a.cap) {
            st = 3;
          } else {
            if (sv_on) {
              const double tn = t + h;
              while (tnext <= tn) {  // bracketed by this step: re-step to ts
                DVec<D> yv;
                DVec<P> pv;
                FVec<P> pfv;
#pragma unroll
                for (int i = 0; i < D; ++i) yv.v[i] = y[i];
#pragma unroll
                for (int i = 0; i < P; ++i) { pv.v[i] = p[i]; pfv.v[i] = pf[i]; }
                const DVec<D> yk = restep_out_of_line<F, L>(yv, pv, pfv, tnext - t);
                store_row<D>(ysr + (long long)kk * D, yk.v);
                ++kk;
                tnext = kk < a.K ? tsr[kk] : CUDART_INF;
              }
            }
            t = t + h;
#pragma unroll
            for (int i = 0; i < D; ++i) y[i] = ynew[i];
            lane.commit();
            if (rec_on) a.rec[rec_index(j, acc, a.n)] = h;
            ++acc;
            if (ck_on && ++ck_cnt == a.ck_every) {
              ck_cnt = 0;
              if (++ck_slot < a.ck_slots) store_ckpt<D>(a.ckpt, a.n, j, ck_slot, y, t);
            }
          }
        } else {
          ++rej;
        }
        if (st < 0) dt = step_from_sum<L::QK>(m, h, a.ctrl);
      }
    }
    if (st >= 0) {  // finished: write this trajectory's outputs, take the next one
      if (rec_on) {  // zero-pad the last sector (identity steps)
        for (int s = acc; (s & 3) != 0; ++s) a.rec[rec_index(j, s, a.n)] = 0.0;
      }
#pragma unroll
      for (int i = 0; i < D; ++i) a.yf[j * D + i] = y[i];
      if (sv_on) {  // times at or past the final accumulated time take y_final itself
        for (int k = a.K - 1; k >= 0 && tsr[k] >= t; --k) store_row<D>(ysr + (long long)k * D, y);
        for (int k = kk; k < a.K; ++k) store_row<D>(ysr + (long long)k * D, y);
      }
      a.n_acc[j] = acc;
      a.n_rej[j] = rej;
      a.status[j] = st;
      j = fetch.get();
      if (j < a.n) begin(j);
    }
  }
}

// ---- persistent reverse pass (one segment of K steps per iteration) --------------------------
// The shared-memory segment buffer is that of the one-thread-per-trajectory reverse passes
// (AdjBuf: the K states, and double-buffered the dts and checkpoint of a segment): while a
// segment is replayed and differentiated, the copies of the trajectory's previous segment are
// in flight (cp.async), so a lane waits on DRAM once per trajectory instead of once per step.
template <class F, class M>
__global__ void __launch_bounds__(128) adjoint_persistent_kernel(const AdjointArgs a,
                                                                 unsigned long long* counter) {
  constexpr int D = F::D, P = F::P;
  Fetch fetch(counter);
  const int K = a.ck_every;
  AdjBuf<D> buf(K);
  double p[P], lam[D], gp[P];
  float pf[P];
  int na = 0, sg = -1, b = 0;
  long long j;
  // take trajectories until one has work (n_acc = 0 ones finish at once: gy0 = ybar), and
  // start the copies of its last segment into buffer b
  auto take = [&]() {
    for (;;) {
      j = fetch.get();
      if (j >= a.n) return;
#pragma unroll
      for (int i = 0; i < P; ++i) { p[i] = a.p[j * P + i]; pf[i] = (float)p[i]; gp[i] = 0.0; }
#pragma unroll
      for (int i = 0; i < D; ++i) lam[i] = a.ybar[j * D + i];
      na = steps_in_record(a.n_acc, j, a.cap);
      sg = (na + K - 1) / K - 1;
      if (sg >= 0) {
        prefetch_segment<D>(buf, b, a.ckpt, a.rec, a.n, j, sg, K, na);
        return;
      }
      if (a.gy0) {
#pragma unroll
        for (int i = 0; i < D; ++i) a.gy0[j * D + i] = lam[i];
      }
      if (a.gp) {
#pragma unroll
        for (int i = 0; i < P; ++i) a.gp[j * P + i] = 0.0;
      }
    }
  };
  take();
  while (j < a.n) {
    cp_async_wait_all();  // this segment's checkpoint and dts have landed
    double y[D], c[D];
#pragma unroll
    for (int i = 0; i < D; ++i) { y[i] = buf.ck(b, i); c[i] = 0.0; }
    if (sg > 0) prefetch_segment<D>(buf, b ^ 1, a.ckpt, a.rec, a.n, j, sg - 1, K, na);
#pragma unroll
    for (int i = 0; i < D; ++i) buf.st(0, i) = y[i];
    for (int q = 1; q < K; ++q) {
      const double dt = buf.dt(b, q - 1);
      if (dt != 0.0) M::template step<F>(y, c, p, pf, dt);
#pragma unroll
      for (int i = 0; i < D; ++i) buf.st(q, i) = y[i];
    }
    for (int q = K - 1; q >= 0; --q) {
      const double dt = buf.dt(b, q);
      if (dt != 0.0) {
        double ys[D];
#pragma unroll
        for (int i = 0; i < D; ++i) ys[i] = buf.st(q, i);
        M::template vjp<F>(ys, p, pf, dt, lam, gp);
      }
    }
    b ^= 1;
    if (--sg < 0) {
      if (a.gy0) {
#pragma unroll
        for (int i = 0; i < D; ++i) a.gy0[j * D + i] = lam[i];
      }
      if (a.gp) {
#pragma unroll
        for (int i = 0; i < P; ++i) a.gp[j * P + i] = gp[i];
      }
      take();
    }
  }
}

// ---- persistent saveat reverse pass (one segment per iteration) -------------------------------
// Per trajectory the arithmetic of adjoint_saveat_kernel (gs_saveat.cuh); the lane carries the
// trajectory's cursor (segment, saveat times not yet assigned, whether the final cotangents
// have joined) between iterations and refills itself when the trajectory is done.  Segments
// are prefetched as in adjoint_persistent_kernel (the buffer's states carry their step start
// time at index D), and the latest time not yet assigned is held in a register.
template <class F, class M>
__global__ void __launch_bounds__(128) adjoint_saveat_persistent_kernel(
    const SaveatArgs a, unsigned long long* counter) {
  constexpr int D = F::D, P = F::P;
  Fetch fetch(counter);
  const int K = a.ck_every;
  AdjBuf<D, D + 1> buf(K);
  double p[P], lam[D], gp[P];
  float pf[P];
  const double* ts = nullptr;
  const double* ysb = nullptr;
  int na = 0, sg = -1, kk = 0, b = 0;
  double tlast = -CUDART_INF;  // ts[kk - 1], or -inf once every time is assigned
  bool fin_done = false;
  long long j;
  auto pop = [&]() {  // time kk - 1 is assigned (the caller has taken its cotangent)
    --kk;
    tlast = kk > 0 ? ts[kk - 1] : -CUDART_INF;
  };
  auto finish = [&]() {  // times never bracketed (ts <= t0) take y0: their cotangent joins lam
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
  };
  auto take = [&]() {
    for (;;) {
      j = fetch.get();
      if (j >= a.n) return;
#pragma unroll
      for (int i = 0; i < P; ++i) { p[i] = a.p[j * P + i]; pf[i] = (float)p[i]; gp[i] = 0.0; }
#pragma unroll
      for (int i = 0; i < D; ++i) lam[i] = a.ybar ? a.ybar[j * D + i] : 0.0;
      ts = a.ts + j * a.ts_ld;
      ysb = a.ysbar + j * (long long)a.K * D;
      na = steps_in_record(a.n_acc, j, a.cap);
      sg = (na + K - 1) / K - 1;
      kk = a.K;
      tlast = kk > 0 ? ts[kk - 1] : -CUDART_INF;
      fin_done = false;
      if (sg >= 0) {
        prefetch_segment<D>(buf, b, a.ckpt, a.rec, a.n, j, sg, K, na);
        return;
      }
      const double tfin = a.t0;  // no steps: every time >= t0 is y_final = y0
      while (tlast >= tfin) {
#pragma unroll
        for (int i = 0; i < D; ++i) lam[i] += ysb[(long long)(kk - 1) * D + i];
        pop();
      }
      finish();
    }
  };
  take();
  while (j < a.n) {
    cp_async_wait_all();  // this segment's checkpoint (state and time) and dts have landed
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
    if (!fin_done) {  // the trajectory's last segment comes first: t is t_fin
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
    if (--sg < 0) {
      finish();
      take();
    }
  }
}

}  // namespace gs
