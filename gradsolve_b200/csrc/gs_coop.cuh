// gs_coop.cuh -- Tsit5 forward, replay and reverse pass for states of more than 8
// components: a group of G lanes of one warp integrates one trajectory.
//
// Lane l of a group holds the contiguous block of C = D / G components [l*C, l*C + C) of the
// state and of every stage in registers (G from coop_group: C <= 4 where D allows), so a
// 32-component Lorenz-96 trajectory runs on 8 lanes with 4 components each instead of one
// thread spilling 300 doubles.  The right-hand side reads a few components of the
// neighbouring blocks (the field's cyclic stencil, RHS_LO below and RHS_HI above the block):
// they come from the neighbouring lanes by warp shuffles, with the group's lane mask, so the
// rest of the warp may be elsewhere.  Lane<F, G> presents the lane's block as a field of
// dimension C, so the stage arithmetic, the replay step and the step VJP of gs_tsit5.cuh are
// used unchanged; what differs is
//   * the error norm: each lane sums the squares (e_i / sc_i)^2 of its block in component
//     order, then the group adds its lanes' sums by a butterfly (xor shuffles 1, 2, 4, ...),
//     which leaves the same total in every lane bit for bit (each addition pairs the same two
//     operands), so accept, reject and the next step size are uniform across the group and
//     the group stays converged; the order of additions differs from numpy's pairwise sum at
//     the rounding level only;
//   * the record: lane 0 stores the accepted dts; each lane stores its block of a checkpoint
//     (16-byte stores for even C), the last lane also the time, in the one-thread layout;
//   * the reverse pass: each lane keeps its block of the segment states in the thread-strided
//     shared-memory buffer and prefetches its block of the checkpoint and (redundantly, from
//     L1) the segment's dts; the parameter gradient is summed over the group at the end.
// Trajectory j is served by threads [j*G, j*G + G); G divides 32, so a group never straddles
// a warp and a whole group leaves together when j >= n.
#pragma once

#include "gs_tsit5.cuh"

namespace gs {

template <class F, int G>
struct Lane {
  static_assert(G >= 2 && G <= 32 && (G & (G - 1)) == 0, "group of 2..32 lanes");
  static_assert(F::D % G == 0, "the lanes hold equal blocks");
  static constexpr int C = F::D / G;
  static constexpr int D = C;  // what the shared step code works on: this lane's block
  static constexpr int P = F::P;
  static_assert(C >= F::RHS_LO && C >= F::RHS_HI && C >= F::VJP_YLO && C >= F::VJP_YHI &&
                    C >= F::VJP_WLO && C >= F::VJP_WHI,
                "a stencil reaches into the neighbouring block only");

  __device__ __forceinline__ static int lane() { return (int)(threadIdx.x & (unsigned)(G - 1)); }
  __device__ __forceinline__ static unsigned mask() {
    if constexpr (G == 32) {
      return 0xffffffffu;
    } else {
      return ((1u << G) - 1u) << (threadIdx.x & 31u & ~(unsigned)(G - 1));
    }
  }
  // vb = LO components below the block (from the previous lane, cyclically), the block, HI
  // components above it (from the next lane)
  template <int LO, int HI, class R>
  __device__ __forceinline__ static void halo(const R* v, R* vb) {
    const unsigned m = mask();
    const int base = (int)(threadIdx.x & 31u) & ~(G - 1), l = lane();
    const int prev = base + ((l + G - 1) & (G - 1)), next = base + ((l + 1) & (G - 1));
#pragma unroll
    for (int k = 0; k < LO; ++k) vb[k] = __shfl_sync(m, v[C - LO + k], prev);
#pragma unroll
    for (int k = 0; k < C; ++k) vb[LO + k] = v[k];
#pragma unroll
    for (int k = 0; k < HI; ++k) vb[LO + C + k] = __shfl_sync(m, v[k], next);
  }
  template <class R>
  __device__ __forceinline__ static void rhs(const R* y, const R* p, R* dy) {
    R yb[F::RHS_LO + C + F::RHS_HI];
    halo<F::RHS_LO, F::RHS_HI>(y, yb);
    F::template rhs_block<C>(yb, p, dy);
  }
  template <class R>
  __device__ __forceinline__ static void vjp(const R* y, const R* p, const R* w, R* gy, R* gp) {
    R yb[F::VJP_YLO + C + F::VJP_YHI], wb[F::VJP_WLO + C + F::VJP_WHI];
    halo<F::VJP_YLO, F::VJP_YHI>(y, yb);
    halo<F::VJP_WLO, F::VJP_WHI>(w, wb);
    F::template vjp_block<C>(yb, wb, p, gy, gp);
  }
  // the group's total, identical in every lane (see the file comment)
  __device__ __forceinline__ static double sum(double v) {
    const unsigned m = mask();
#pragma unroll
    for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(m, v, o);
    return v;
  }
};

// This lane's block of checkpoint slot `slot` of trajectory j (and, from the last lane, the
// time and the row's padding): the one-thread layout, row (slot*n + j)*CW, CW = D+1 rounded
// up to even.
template <class F, int G>
__device__ __forceinline__ void coop_store_ckpt(double* ckpt, long long n, long long j, int slot,
                                                const double* y, double t) {
  using L = Lane<F, G>;
  constexpr int C = L::C, D = F::D, CW = (D + 2) & ~1;
  double* row = ckpt + ((size_t)slot * (size_t)n + (size_t)j) * CW;
  const int l = L::lane();
  double* dst = row + l * C;
  if constexpr (C % 2 == 0) {  // l*C even: the block starts on a 16-byte boundary
#pragma unroll
    for (int u = 0; u < C / 2; ++u)
      reinterpret_cast<double2*>(dst)[u] = make_double2(y[2 * u], y[2 * u + 1]);
  } else {
#pragma unroll
    for (int k = 0; k < C; ++k) dst[k] = y[k];
  }
  if (l == G - 1) {
    row[D] = t;
    if constexpr (CW > D + 1) row[D + 1] = 0.0;
  }
}

// One attempt of the group from the state (y, k1) into (yo, ko): tsit5_attempt with the error
// norm summed over the group, the record written by lane 0 (rec_here) and block checkpoints.
template <class F, int G>
__device__ __forceinline__ bool tsit5_coop_attempt(const RecordArgs& a, long long j,
                                                   const double* p, double t1, bool rec_on,
                                                   bool rec_here, bool ck_on, long long rstride,
                                                   FwdCounters& c, const double* y,
                                                   const double* k1, double* yo, double* ko) {
  using L = Lane<F, G>;
  constexpr int C = L::C;
  using T = Tsit5;
  if (c.it >= a.max_steps || c.t >= t1) return false;
  ++c.it;
  const double h = (t1 - c.t < c.dt) ? (t1 - c.t) : c.dt;
  Stages<L> S;
  tsit5_k2_to_k6<L>(y, p, k1, h, S);
  tsit5_y5<L>(y, k1, S, h, yo);
  L::rhs(yo, p, ko);
  double part = 0.0;
#pragma unroll
  for (int i = 0; i < C; ++i) {
    const double e = h * (T::E1 * k1[i] + T::E2 * S.k2[i] + T::E3 * S.k3[i] + T::E4 * S.k4[i] +
                          T::E5 * S.k5[i] + T::E6 * S.k6[i] + T::E7 * ko[i]);
    const double sc = a.atol + a.rtol * fmax(fabs(y[i]), fabs(yo[i]));
    const double q = e / sc;
    part += q * q;
  }
  const double m = L::sum(part);
  if (!(m == m)) {  // NaN error: dt would turn NaN and the loop could never finish
    c.st = 1;
    return false;
  }
  if (m <= a.ctrl.accept_sum) {
    if ((rec_on || ck_on) && c.acc >= a.cap) {
      c.st = 3;
      return false;
    }
    c.t = c.t + h;
    if (rec_here) {
      c.rp[c.acc & 3] = h;
      if ((c.acc & 3) == 3) c.rp += rstride;
    }
    ++c.acc;
    if (ck_on && ++c.ck_cnt == a.ck_every) {
      c.ck_cnt = 0;
      if (++c.ck_slot < a.ck_slots) coop_store_ckpt<F, G>(a.ckpt, a.n, j, c.ck_slot, yo, c.t);
    }
  } else {
    ++c.rej;
#pragma unroll
    for (int i = 0; i < C; ++i) {
      yo[i] = y[i];
      ko[i] = k1[i];
    }
  }
  c.dt = step_from_sum<10>(m, h, a.ctrl);
  return true;
}

// Adaptive forward with record (kStore) or the forward-only solve (!kStore).
template <class F, int G, bool kStore>
__global__ void __launch_bounds__(128) tsit5_coop_record_kernel(const RecordArgs a) {
  using L = Lane<F, G>;
  constexpr int C = L::C, D = F::D, P = F::P;
  const long long j = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  if (j >= a.n) return;
  const int l = L::lane();
  double ya[C], ka[C], yb[C], kb[C], p[P];
#pragma unroll
  for (int k = 0; k < C; ++k) ya[k] = a.y0[j * D + l * C + k];
#pragma unroll
  for (int i = 0; i < P; ++i) p[i] = a.p[j * P + i];
  const double t1 = a.t1v ? a.t1v[j] : a.t1;
  const bool rec_on = kStore && a.rec != nullptr;
  const bool ck_on = kStore && a.ckpt != nullptr;
  const bool rec_here = rec_on && l == 0;
  const long long rstride = 4 * a.n;
  FwdCounters c;
  c.t = a.t0;
  c.dt = a.dt0 > 0.0 ? a.dt0 : (t1 - a.t0) / 100.0;
  c.it = c.acc = c.rej = c.st = c.ck_cnt = c.ck_slot = 0;
  c.rp = rec_here ? a.rec + j * 4 : nullptr;
  if (ck_on) coop_store_ckpt<F, G>(a.ckpt, a.n, j, 0, ya, c.t);
  L::rhs(ya, p, ka);
  bool in_b = false;
  for (;;) {
    if (!tsit5_coop_attempt<F, G>(a, j, p, t1, rec_on, rec_here, ck_on, rstride, c, ya, ka, yb,
                                  kb))
      break;
    if (!tsit5_coop_attempt<F, G>(a, j, p, t1, rec_on, rec_here, ck_on, rstride, c, yb, kb, ya,
                                  ka)) {
      in_b = true;
      break;
    }
  }
  if (c.st == 0 && !(c.t >= t1)) c.st = 1;
  if (rec_here) {  // zero-pad the last sector (identity steps)
    for (int s = c.acc; (s & 3) != 0; ++s) c.rp[s & 3] = 0.0;
  }
#pragma unroll
  for (int k = 0; k < C; ++k) a.yf[j * D + l * C + k] = in_b ? yb[k] : ya[k];
  if (l == 0) {
    a.n_acc[j] = c.acc;
    a.n_rej[j] = c.rej;
    a.status[j] = c.st;
  }
}

// Frozen-mesh replay, optionally writing checkpoints.
template <class F, int G>
__global__ void __launch_bounds__(128) tsit5_coop_replay_kernel(const ReplayArgs a) {
  using L = Lane<F, G>;
  constexpr int C = L::C, D = F::D, P = F::P;
  const long long j = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  if (j >= a.n) return;
  const int l = L::lane();
  double y[C], p[P];
#pragma unroll
  for (int k = 0; k < C; ++k) y[k] = a.y0[j * D + l * C + k];
#pragma unroll
  for (int i = 0; i < P; ++i) p[i] = a.p[j * P + i];
  const int na = steps_in_record(a.n_acc, j, a.cap);
  double t = a.t0;
  const bool ck_on = a.ckpt != nullptr;
  if (ck_on) coop_store_ckpt<F, G>(a.ckpt, a.n, j, 0, y, t);
  int ck_cnt = 0, ck_slot = 0;
  for (int s = 0; s < na; ++s) {
    const double dt = load_rec(a.rec, a.n, j, s);
    tsit5_replay_step<L>(y, p, dt);
    t = t + dt;
    if (ck_on && ++ck_cnt == a.ck_every) {
      ck_cnt = 0;
      if (++ck_slot < a.ck_slots) coop_store_ckpt<F, G>(a.ckpt, a.n, j, ck_slot, y, t);
    }
  }
#pragma unroll
  for (int k = 0; k < C; ++k) a.yf[j * D + l * C + k] = y[k];
}

// Start the copies of this lane's block of segment sg's checkpoint and of the segment's dts
// into buffer b.
template <class F, int G, class Buf>
__device__ __forceinline__ void coop_prefetch(Buf& buf, int b, const double* ckpt,
                                              const double* rec, long long n, long long j,
                                              int sg, int K, int na) {
  using L = Lane<F, G>;
  constexpr int C = L::C, CW = (F::D + 2) & ~1;
  SegIO<C>& io = buf.io;
  const double* src = ckpt + ((size_t)sg * (size_t)n + (size_t)j) * CW + L::lane() * C;
  if constexpr (C % 2 == 0) {
#pragma unroll
    for (int u = 0; u < C / 2; ++u) cp_async16(io.unit(b, io.KU + u), src + 2 * u);
  } else {
#pragma unroll
    for (int i = 0; i < C; ++i) cp_async8(&io.ck(b, i), src + i);
  }
  prefetch_dts<C>(io, b, rec, n, j, sg, K, na);
  cp_async_commit();
}

// Reverse-replay adjoint: each segment's states are recomputed from its checkpoint into the
// shared-memory buffer (this lane's block of each), then the step VJPs run backwards.
template <class F, int G>
__global__ void __launch_bounds__(128) tsit5_coop_adjoint_kernel(const AdjointArgs a) {
  using L = Lane<F, G>;
  constexpr int C = L::C, D = F::D, P = F::P;
  const long long g = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  if (g >= a.n) return;
  const long long j = lane_traj(a, g);  // the group's trajectory (one entry for all G lanes)
  if (j < 0) return;
  const int l = L::lane();
  double p[P], lam[C], gp[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    p[i] = a.p[j * P + i];
    gp[i] = 0.0;
  }
#pragma unroll
  for (int k = 0; k < C; ++k) lam[k] = a.ybar[j * D + l * C + k];
  const int na = steps_in_record(a.n_acc, j, a.cap);
  const int K = a.ck_every;
  const int nseg = (na + K - 1) / K;
  AdjBuf<C> buf(K);
  int b = 0;
  if (nseg > 0) coop_prefetch<F, G>(buf, b, a.ckpt, a.rec, a.n, j, nseg - 1, K, na);
  const int top = warp_top_segments(nseg);
  for (int sg = top - 1; sg >= 0; --sg) {
    if (sg >= nseg) continue;  // in step with the warp's longest trajectory
    cp_async_wait_all();  // this segment's checkpoint block and dts have landed
    double y[C];
#pragma unroll
    for (int k = 0; k < C; ++k) y[k] = buf.ck(b, k);
    if (sg > 0) coop_prefetch<F, G>(buf, b ^ 1, a.ckpt, a.rec, a.n, j, sg - 1, K, na);
#pragma unroll
    for (int k = 0; k < C; ++k) buf.st(0, k) = y[k];
    for (int q = 1; q < K; ++q) {
      const double dt = buf.dt(b, q - 1);  // the same in every lane of the group
      if (dt != 0.0) tsit5_replay_step<L>(y, p, dt);
#pragma unroll
      for (int k = 0; k < C; ++k) buf.st(q, k) = y[k];
    }
    for (int q = K - 1; q >= 0; --q) {
      const double dt = buf.dt(b, q);
      if (dt != 0.0) {
        double ys[C];
#pragma unroll
        for (int k = 0; k < C; ++k) ys[k] = buf.st(q, k);
        tsit5_step_vjp<L>(ys, p, dt, lam, gp);
      }
    }
    b ^= 1;
  }
  if (a.gy0) {
#pragma unroll
    for (int k = 0; k < C; ++k) a.gy0[j * D + l * C + k] = lam[k];
  }
#pragma unroll
  for (int i = 0; i < P; ++i) gp[i] = L::sum(gp[i]);
  if (a.gp && l == 0) {
#pragma unroll
    for (int i = 0; i < P; ++i) a.gp[j * P + i] = gp[i];
  }
}

}  // namespace gs
