// gs_ros23.cuh -- adaptive Rosenbrock23 (ode23s, autonomous) forward with dt record, its
// frozen-mesh replay and the hand-written reverse-replay adjoint (float64).
//
// Forward: the fused kernel of gradsolve/warp/_warp_rosenbrock.py:383-452, specified by
// tests/_oracles/gradsolve_g2_spike_oracle.py:138-184:
//   W = I - d*h*J(y);  k1 = W\f(y);  k2 = W\(f(y + h/2 k1) - k1) + k1;  ynew = y + h k2;
//   k3 = W\(f(ynew) - e32 (k2 - F1) - 2 (k1 - F0));  err_vec = h/6 (k1 - 2 k2 + k3);
//   WRMS norm, accept iff err <= 1, dt = h*clip(0.9*max(err,1e-10)^(-1/3), 0.2, 5) after both
//   outcomes.  W is factored once per attempt (partial pivoting) and the three solves reuse
//   the factors: the same elimination, in the same order, as the
//   reference kernel's three fresh eliminations (_gauss_solve, :346-381), because a row swap
//   moves the stored multipliers with the row.  The 3x3 LU stays in registers.  The
//   multipliers and the back substitutions multiply by the pivot's reciprocal, computed once
//   per column, where the reference divides by the pivot in each (within an ulp of the
//   division each time; it takes the dependent divisions off each attempt's critical path:
//   D divisions per factorisation instead of D (D + 1) / 2 + D per solve).  Float64 fields of
//   up to 3 components (Robertson, VdP) hold W as its explicit inverse instead (kInverseW
//   below): one division per attempt and matrix-vector products for the solves.
// Replay: gradsolve/solvers/rosenbrock23_step.py:47-66 (no k3) with the analytic Jacobian.
// Adjoint: reverse of that step, including the second-order term through W = I - d dt J(y,p):
//   Wbar = -(W^-T k2bar) k2'^T - (W^-T k1bar) k1^T,  then  d<-d dt Wbar, J(y,p)>/d(y,p).
// Record, checkpoint and segment scheme: as the Tsit5 kernels (gs_tsit5.cuh).
#pragma once
#include <type_traits>

#include "gs_fields.cuh"
#include "gs_tableau.cuh"
#include "gs_tsit5.cuh"

namespace gs {

// For float64 fields of up to 3 components W is held as its explicit inverse (cofactors over
// the determinant): the cofactors are independent products, so the factorisation has one
// reciprocal on its dependent chain instead of one pivot search and reciprocal per column,
// and each solve is a matrix-vector product instead of two substitution sweeps -- the
// Rosenbrock23 kernels are latency-bound, and this shortens every attempt's critical path.
// Against the partial-pivoting elimination the numbers agree to rounding (on the reference's
// Robertson goldens: the same accepted and rejected counts, dts within 1e-8 relative).  Larger
// fields and the float32 route keep the pivoted LU.
template <int D, class R>
constexpr bool kInverseW = D <= 3 && std::is_same<R, double>::value;

template <int D, class R = double>
struct LU {
  R a[D * D];  // L (unit, below diagonal) and U (on/above), row-swapped; or W^-1 (kInverseW)
  R inv[D];         // 1 / U's diagonal (LU only)
  int piv[D];       // (LU only)
};

template <int D, class R>
__device__ __forceinline__ void inverse_factor(LU<D, R>& f) {
  R* a = f.a;
  if constexpr (D == 1) {
    a[0] = R(1.0) / a[0];
  } else if constexpr (D == 2) {
    const R r = R(1.0) / (a[0] * a[3] - a[1] * a[2]);
    const R a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3];
    a[0] = a3 * r;
    a[1] = -a1 * r;
    a[2] = -a2 * r;
    a[3] = a0 * r;
  } else {
    // cofactors c_ij of W; W^-1 = adj(W) / det = (c_ji) / det
    const R c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8],
            c02 = a[3] * a[7] - a[4] * a[6];
    const R c10 = a[2] * a[7] - a[1] * a[8], c11 = a[0] * a[8] - a[2] * a[6],
            c12 = a[1] * a[6] - a[0] * a[7];
    const R c20 = a[1] * a[5] - a[2] * a[4], c21 = a[2] * a[3] - a[0] * a[5],
            c22 = a[0] * a[4] - a[1] * a[3];
    const R r = R(1.0) / (a[0] * c00 + a[1] * c01 + a[2] * c02);
    a[0] = c00 * r;
    a[1] = c10 * r;
    a[2] = c20 * r;
    a[3] = c01 * r;
    a[4] = c11 * r;
    a[5] = c21 * r;
    a[6] = c02 * r;
    a[7] = c12 * r;
    a[8] = c22 * r;
  }
}

template <int D, class R>
__device__ __forceinline__ void lu_factor(LU<D, R>& f) {
  if constexpr (kInverseW<D, R>) {
    inverse_factor(f);
    return;
  }
#pragma unroll
  for (int col = 0; col < D; ++col) {
    int pv = col;
    R big = fabs(f.a[col * D + col]);
#pragma unroll
    for (int r = col + 1; r < D; ++r) {
      const R v = fabs(f.a[r * D + col]);
      if (v > big) {
        big = v;
        pv = r;
      }
    }
    f.piv[col] = pv;
    if (pv != col) {
#pragma unroll
      for (int c = 0; c < D; ++c) {
        // select-based swap keeps the matrix in registers (no dynamic indexing)
#pragma unroll
        for (int r = col + 1; r < D; ++r) {
          const bool sw = r == pv;
          const R u = f.a[col * D + c], v = f.a[r * D + c];
          f.a[col * D + c] = sw ? v : u;
          f.a[r * D + c] = sw ? u : v;
        }
      }
    }
    // one reciprocal of the pivot serves the column's multipliers and the back substitutions
    f.inv[col] = R(1.0) / f.a[col * D + col];
#pragma unroll
    for (int r = col + 1; r < D; ++r) {
      const R factor = f.a[r * D + col] * f.inv[col];
      f.a[r * D + col] = factor;
#pragma unroll
      for (int c = col + 1; c < D; ++c) f.a[r * D + c] = f.a[r * D + c] - factor * f.a[col * D + c];
    }
  }
}

// x = W^-1 b.  lu_factor exchanges whole rows, the multipliers of earlier columns included,
// so L is stored in the final row order (W = P^T L U with P = P_{D-1} ... P_0): all row
// exchanges are applied to b first, then L and U are solved.  (Interleaving each exchange with
// its column's elimination would pair the multipliers, permuted by later pivots, with rows in
// the wrong order whenever a pivot is taken after the first column.)
template <int D, class R>
__device__ __forceinline__ void lu_solve(const LU<D, R>& f, const R* b, R* x) {
  if constexpr (kInverseW<D, R>) {  // x = W^-1 b
#pragma unroll
    for (int i = 0; i < D; ++i) {
      R s = f.a[i * D] * b[0];
#pragma unroll
      for (int c = 1; c < D; ++c) s = s + f.a[i * D + c] * b[c];
      x[i] = s;
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) x[i] = b[i];
#pragma unroll
  for (int k = 0; k < D; ++k) {
#pragma unroll
    for (int r = k + 1; r < D; ++r) {
      // selects, not a branch: written as an if, the compiler turns the swap into an
      // indexed access x[piv[k]] and moves x to local memory (a stack frame, L1/L2 traffic
      // every solve); as selects x stays in registers
      const bool sw = r == f.piv[k];
      const R xk = x[k], xr = x[r];
      x[k] = sw ? xr : xk;
      x[r] = sw ? xk : xr;
    }
  }
#pragma unroll
  for (int k = 0; k < D; ++k) {
#pragma unroll
    for (int r = k + 1; r < D; ++r) x[r] = x[r] - f.a[r * D + k] * x[k];
  }
#pragma unroll
  for (int ii = 0; ii < D; ++ii) {
    const int i = D - 1 - ii;
    R s = x[i];
#pragma unroll
    for (int c = i + 1; c < D; ++c) s = s - f.a[i * D + c] * x[c];
    x[i] = s * f.inv[i];
  }
}

// x = W^-T b   (W = P^T L U  =>  W^T = U^T L^T P)
template <int D, class R>
__device__ __forceinline__ void lu_solve_t(const LU<D, R>& f, const R* b, R* x) {
  if constexpr (kInverseW<D, R>) {  // x = W^-T b
#pragma unroll
    for (int i = 0; i < D; ++i) {
      R s = f.a[i] * b[0];
#pragma unroll
      for (int r = 1; r < D; ++r) s = s + f.a[r * D + i] * b[r];
      x[i] = s;
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) {
    R s = b[i];
#pragma unroll
    for (int jj = 0; jj < i; ++jj) s = s - f.a[jj * D + i] * x[jj];
    x[i] = s * f.inv[i];
  }
#pragma unroll
  for (int ii = 0; ii < D; ++ii) {
    const int i = D - 1 - ii;
    R s = x[i];
#pragma unroll
    for (int r = i + 1; r < D; ++r) s = s - f.a[r * D + i] * x[r];
    x[i] = s;
  }
#pragma unroll
  for (int kk = 0; kk < D; ++kk) {
    const int k = D - 1 - kk;
#pragma unroll
    for (int r = k + 1; r < D; ++r) {
      // selects, not a branch: written as an if, the compiler turns the swap into an
      // indexed access x[piv[k]] and moves x to local memory (a stack frame, L1/L2 traffic
      // every solve); as selects x stays in registers
      const bool sw = r == f.piv[k];
      const R xk = x[k], xr = x[r];
      x[k] = sw ? xr : xk;
      x[r] = sw ? xk : xr;
    }
  }
}

template <class F, class R = double>
__device__ __forceinline__ void ros23_build_w(const R* y, const R* p, R h, LU<F::D, R>& W) {
  constexpr int D = F::D;
  R J[D * D];
  F::jac(y, p, J);
#pragma unroll
  for (int i = 0; i < D; ++i) {
#pragma unroll
    for (int c = 0; c < D; ++c) W.a[i * D + c] = -R(Ros23::D) * h * J[i * D + c];
    W.a[i * D + i] = W.a[i * D + i] + R(1.0);
  }
  lu_factor(W);
}

// Shared part of the attempt and of the replay step: W factored, F0, k1, F1, k2, ynew.
template <class F, class R = double>
struct RosCore {
  static constexpr int D = F::D;
  LU<D, R> W;
  R F0[D], k1[D], F1[D], k2p[D], k2[D];  // k2 = k2p + k1
};

template <class F, class R = double>
__device__ __forceinline__ void ros23_core(const R* y, const R* p, R h, RosCore<F, R>& c,
                                           R* ynew) {
  constexpr int D = F::D;
  R s[D];
  ros23_build_w<F>(y, p, h, c.W);
  F::rhs(y, p, c.F0);
  lu_solve(c.W, c.F0, c.k1);
#pragma unroll
  for (int i = 0; i < D; ++i) s[i] = y[i] + R(0.5) * h * c.k1[i];
  F::rhs(s, p, c.F1);
#pragma unroll
  for (int i = 0; i < D; ++i) s[i] = c.F1[i] - c.k1[i];
  lu_solve(c.W, s, c.k2p);
#pragma unroll
  for (int i = 0; i < D; ++i) c.k2[i] = c.k2p[i] + c.k1[i];
#pragma unroll
  for (int i = 0; i < D; ++i) ynew[i] = y[i] + h * c.k2[i];
}

template <class F, class R = double>
__device__ __forceinline__ void ros23_replay_step(R* y, const R* p, R dt) {
  constexpr int D = F::D;
  RosCore<F, R> c;
  R yn[D];
  ros23_core<F>(y, p, dt, c, yn);
#pragma unroll
  for (int i = 0; i < D; ++i) y[i] = yn[i];
}

// Reverse of one replay step from the step's forward quantities: the factors of W, k1, the
// stage state s1 = y + dt/2 k1 and k2' = W \ (f(s1) - k1).
template <class F, class R = double>
__device__ __forceinline__ void ros23_vjp_core(const R* y, const R* p, R dt, const LU<F::D, R>& W,
                                               const R* k1, const R* s1, const R* k2p, R* lam,
                                               R* gp) {
  constexpr int D = F::D;
  R yb[D], k2b[D], k1b[D], r2b[D], s1b[D], r1b[D], G[D * D];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    yb[i] = lam[i];
    k2b[i] = dt * lam[i];
    k1b[i] = k2b[i];
    s1b[i] = R(0.0);
  }
  lu_solve_t(W, k2b, r2b);
  const R scale = R(Ros23::D) * dt;  // G = -d dt Wbar, Wbar = -(r2b k2p^T + r1b k1^T)
#pragma unroll
  for (int i = 0; i < D; ++i) {
#pragma unroll
    for (int c = 0; c < D; ++c) G[i * D + c] = scale * (r2b[i] * k2p[c]);
    k1b[i] -= r2b[i];
  }
  F::vjp(s1, p, r2b, s1b, gp);
#pragma unroll
  for (int i = 0; i < D; ++i) {
    yb[i] += s1b[i];
    k1b[i] += R(0.5) * dt * s1b[i];
  }
  lu_solve_t(W, k1b, r1b);
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int c = 0; c < D; ++c) G[i * D + c] += scale * (r1b[i] * k1[c]);
  F::vjp(y, p, r1b, yb, gp);
  F::jac_contract_grad(y, p, G, yb, gp);
#pragma unroll
  for (int i = 0; i < D; ++i) lam[i] = yb[i];
}

// Reverse of one replay step at (y, dt), recomputing its forward quantities (the expressions
// of ros23_core).
template <class F, class R = double>
__device__ __forceinline__ void ros23_step_vjp(const R* y, const R* p, R dt, R* lam, R* gp) {
  constexpr int D = F::D;
  RosCore<F, R> c;
  R yn[D], s1[D];
  ros23_core<F>(y, p, dt, c, yn);
#pragma unroll
  for (int i = 0; i < D; ++i) s1[i] = y[i] + R(0.5) * dt * c.k1[i];
  ros23_vjp_core<F>(y, p, dt, c.W, c.k1, s1, c.k2p, lam, gp);
}

// One attempt from the state y; the candidate is computed into yo.  Returns true when the
// integration goes on from yo (a copy of y after a rejection) and false when it stops with
// its state in y -- the register-set alternation of tsit5_attempt.
template <class F>
__device__ __forceinline__ bool ros23_attempt(const RecordArgs& a, long long j, const double* p,
                                              double t1, bool rec_on, bool ck_on,
                                              long long rstride, FwdCounters& c,
                                              const double* y, double* yo) {
  constexpr int D = F::D;
  if (c.it >= a.max_steps || c.t >= t1) return false;
  const double h = (t1 - c.t < c.dt) ? (t1 - c.t) : c.dt;
  if (c.t + h == c.t) {  // the step no longer advances time
    c.st = 2;
    return false;
  }
  ++c.it;
  RosCore<F> rc;
  ros23_core<F>(y, p, h, rc, yo);
  double F2[D], r3[D], k3[D], ev[D];
  F::rhs(yo, p, F2);
#pragma unroll
  for (int i = 0; i < D; ++i)
    r3[i] = F2[i] - Ros23::E32 * (rc.k2[i] - rc.F1[i]) - 2.0 * (rc.k1[i] - rc.F0[i]);
  lu_solve<D>(rc.W, r3, k3);
#pragma unroll
  for (int i = 0; i < D; ++i) ev[i] = (h / 6.0) * (rc.k1[i] - 2.0 * rc.k2[i] + k3[i]);
  const double m = wrms_sumsq<D>(ev, y, yo, a.rtol, a.atol);
  if (!(m == m)) {
    c.st = 1;
    return false;
  }
  if (m <= a.ctrl.accept_sum) {
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
    for (int i = 0; i < D; ++i) yo[i] = y[i];
  }
  c.dt = step_from_sum<6>(m, h, a.ctrl);
  return true;
}

// kStore = false: the forward-only solve (no record, no checkpoints), stores compiled out.
template <class F, bool kStore>
__device__ __forceinline__ void ros23_record_body(const RecordArgs& a) {
  constexpr int D = F::D, P = F::P;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.n) return;
  double ya[D], yb[D], p[P];
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
  bool in_b = false;  // where the state is when the loop stops
  for (;;) {
    if (!ros23_attempt<F>(a, j, p, t1, rec_on, ck_on, rstride, c, ya, yb)) break;
    if (!ros23_attempt<F>(a, j, p, t1, rec_on, ck_on, rstride, c, yb, ya)) {
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

template <class F, bool kStore = true>
__global__ void __launch_bounds__(128) ros23_record_kernel(const RecordArgs a) {
  ros23_record_body<F, kStore>(a);
}

// The recording forward with its registers bounded for kMinB resident blocks of 128 per SM
// (the instances the occupancy autotuner chooses among; same arithmetic, bit for bit).
template <class F, int kMinB>
__global__ void __launch_bounds__(128, kMinB) ros23_record_occ_kernel(const RecordArgs a) {
  ros23_record_body<F, true>(a);
}

template <class F>
__global__ void __launch_bounds__(128) ros23_replay_kernel(const ReplayArgs a) {
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
    ros23_replay_step<F>(y, p, dt);
    t = t + dt;
    if (ck_on && ++ck_cnt == a.ck_every) {
      ck_cnt = 0;
      if (++ck_slot < a.ck_slots) store_ckpt<D>(a.ckpt, a.n, j, ck_slot, y, t);
    }
  }
#pragma unroll
  for (int i = 0; i < D; ++i) a.yf[j * D + i] = y[i];
}

// Reverse pass.  As tsit5_adjoint_stages_kernel: the next segment's checkpoint and dts are
// prefetched (cp.async) into the shared-memory segment buffer, and the segment's replay keeps
// what the step VJPs need -- the factors of W (D^2 + 2D values), k1, s1 and k2' -- for the
// K-1 steps it takes, so only the segment's last step recomputes its forward quantities.
// kKeep = false (where the kept quantities would not fit shared memory): every step's VJP
// recomputes them, and the buffer holds only the states, dts and checkpoints.
template <int D, bool kKeep>
GS_HD int ros23_adjoint_smem_doubles(int K) {
  return K * D + (kKeep ? (K - 1) * (D * D + 5 * D) : 0) + seg_io_doubles<D>(K);
}

template <int D, bool kKeep>
struct AdjRosBuf {
  static constexpr int R = kKeep ? D * D + 5 * D : 0;  // kept values per step
  double* base;
  int stride, K;
  SegIO<D> io;
  __device__ __forceinline__ AdjRosBuf(int k)
      : base(gs_seg_smem + threadIdx.x), stride(blockDim.x), K(k), io(k * D + (k - 1) * R, k) {}
  __device__ __forceinline__ double& st(int q, int i) { return base[(q * D + i) * stride]; }
  __device__ __forceinline__ double& kept(int q, int v) {
    return base[(K * D + q * R + v) * stride];
  }
  __device__ __forceinline__ double& dt(int b, int q) { return io.dt(b, q); }
  __device__ __forceinline__ double& ck(int b, int i) { return io.ck(b, i); }
  // layout of a kept step: W.a, W.inv, W.piv (as doubles), k1, s1, k2' (kKeep only)
  __device__ __forceinline__ void keep(int q, const LU<D>& W, const double* k1, const double* s1,
                                       const double* k2p) {
#pragma unroll
    for (int v = 0; v < D * D; ++v) kept(q, v) = W.a[v];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      kept(q, D * D + i) = W.inv[i];
      kept(q, D * D + D + i) = (double)W.piv[i];
      kept(q, D * D + 2 * D + i) = k1[i];
      kept(q, D * D + 3 * D + i) = s1[i];
      kept(q, D * D + 4 * D + i) = k2p[i];
    }
  }
  __device__ __forceinline__ void restore(int q, LU<D>& W, double* k1, double* s1, double* k2p) {
#pragma unroll
    for (int v = 0; v < D * D; ++v) W.a[v] = kept(q, v);
#pragma unroll
    for (int i = 0; i < D; ++i) {
      W.inv[i] = kept(q, D * D + i);
      W.piv[i] = (int)kept(q, D * D + D + i);
      k1[i] = kept(q, D * D + 2 * D + i);
      s1[i] = kept(q, D * D + 3 * D + i);
      k2p[i] = kept(q, D * D + 4 * D + i);
    }
  }
};

// KC > 0: the segment length fixed at compile time (as tsit5_adjoint_stages_body).
template <class F, bool kKeep, int KC>
__device__ __forceinline__ void ros23_adjoint_body(const AdjointArgs& a) {
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
  AdjRosBuf<D, kKeep> buf(K);
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
    for (int q = 1; q < K; ++q) {  // replay steps 0..K-2, keeping their forward quantities
      const double dt = buf.dt(b, q - 1);
      if (dt != 0.0) {
        RosCore<F> c;
        double yn[D], s1[D];
        ros23_core<F>(y, p, dt, c, yn);
        if constexpr (kKeep) {
#pragma unroll
          for (int i = 0; i < D; ++i) s1[i] = y[i] + 0.5 * dt * c.k1[i];
          buf.keep(q - 1, c.W, c.k1, s1, c.k2p);
        }
#pragma unroll
        for (int i = 0; i < D; ++i) y[i] = yn[i];
      }
#pragma unroll
      for (int i = 0; i < D; ++i) buf.st(q, i) = y[i];
    }
    for (int q = K - 1; q >= 0; --q) {
      const double dt = buf.dt(b, q);
      if (dt != 0.0) {
        double ys[D];
#pragma unroll
        for (int i = 0; i < D; ++i) ys[i] = buf.st(q, i);
        // one VJP call site: the forward quantities come from the replay's kept copy, or
        // (the segment's last step, or nothing kept) are recomputed here
        RosCore<F> c;
        double s1[D];
        if (kKeep && q < K - 1) {
          buf.restore(q, c.W, c.k1, s1, c.k2p);
        } else {
          double yn[D];
          ros23_core<F>(ys, p, dt, c, yn);
#pragma unroll
          for (int i = 0; i < D; ++i) s1[i] = ys[i] + 0.5 * dt * c.k1[i];
        }
        ros23_vjp_core<F>(ys, p, dt, c.W, c.k1, s1, c.k2p, lam, gp);
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

template <class F, bool kKeep>
__global__ void __launch_bounds__(128) ros23_adjoint_kernel(const AdjointArgs a) {
  ros23_adjoint_body<F, kKeep, 0>(a);
}

// K = 2 with the kept factors, unrolled; bounded to 4 blocks of 128 per SM (kMinB = 0), or
// for kMinB blocks (the occupancy instances; same arithmetic, bit for bit)
template <class F, int kMinB = 0>
__global__ void __launch_bounds__(128, (kMinB > 0 ? kMinB : 4)) ros23_adjoint_k2_kernel(const AdjointArgs a) {
  ros23_adjoint_body<F, true, 2>(a);
}

}  // namespace gs
