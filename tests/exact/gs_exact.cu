// gs_exact.cu -- test-only: an exact-association instance of the Tsit5 forward with dt record.
//
// Built with -fmad=false (tests/exact/build.py), so every float64 multiply and add rounds on
// its own, as numpy's do.  The stage arithmetic is the product's own: tsit5_k2_to_k6 and
// tsit5_y5 from gs_tsit5.cuh and the fields' rhs from gs_fields.cuh, unchanged.  What differs
// from the tuned tsit5_record_kernel is the error norm and the controller, which follow
// tsit5_adaptive (gradsolve/solvers/tsit5_replay.py:107-122) literally:
//   e   = h * (E1*k1 + ... + E7*k7)
//   err = sqrt(mean((e / sc)^2)),  sc = atol + rtol * max(|y|, |y5|)
//         (one division per component; the mean summed in numpy's add.reduce order:
//          sequential below 8 terms, 8 accumulators combined pairwise from 8 to 128)
//   dt  = h * min(max(0.9 * max(err, 1e-10)^-0.2, 0.2), 5)
// where the tuned kernel uses a shared reciprocal, the sum S against a threshold and a
// series root.
//
// The one operation that cannot match by construction is the power: the reference's is the
// host libm's pow (Python float **), which is not correctly rounded (nor is CUDA's pow), and
// the two differ in the last bit for some arguments.  So the power can be supplied: with
// pow_table (n, A) given, attempt `it` of trajectory j uses pow_table[j*A + it] -- the host
// libm's value of max(err, 1e-10)^-0.2 for that attempt's err (NaN: not known; CUDA's pow is
// used) -- and err_log (n, 2A) receives each attempt's floored err and the power it used.
// The test feeds
// the log back through the host's pow until the table is a fixed point; with it the recorded
// dts and y_final of the reference's own goldens are reproduced bit for bit
// (tests/test_gpu_exact.py), which pins the product's stage arithmetic and fields to the
// reference's association.  The tuned kernel's measured distance from this instance is the
// dt tolerance its own tests use.
//
// Output layout: dts row-major (n, cap), zero past n_acc[j] (the reference's padded form).

#include <cuda_runtime.h>

#include "../../gradsolve_b200/csrc/gs_fields.cuh"
#include "../../gradsolve_b200/csrc/gs_tsit5.cuh"

namespace gx {

// numpy's float64 add.reduce order for a short contiguous array (pairwise_sum below 128)
template <int D>
__device__ __forceinline__ double numpy_sum(const double* a) {
  if constexpr (D < 8) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) s += a[i];
    return s;
  } else {
    static_assert(D <= 128, "numpy switches to recursive halving above 128 terms");
    double r[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = a[j];
    int i = 8;
#pragma unroll
    for (; i < D - (D % 8); i += 8) {
#pragma unroll
      for (int j = 0; j < 8; ++j) r[j] += a[i + j];
    }
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
#pragma unroll
    for (; i < D; ++i) res += a[i];
    return res;
  }
}

template <class F>
__global__ void exact_tsit5_record_kernel(long long n, const double* y0, const double* p,
                                          double t0, double t1, double rtol, double atol,
                                          double dt0, int max_steps, int cap, double* dts,
                                          double* yf, int* n_acc, int* n_rej, int* status,
                                          const double* pow_table, double* err_log, int A) {
  constexpr int D = F::D, P = F::P;
  using T = gs::Tsit5;
  using C = gs::Ctrl;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double y[D], k1[D], pp[P];
  for (int i = 0; i < D; ++i) y[i] = y0[j * D + i];
  for (int i = 0; i < P; ++i) pp[i] = p[j * P + i];
  double t = t0, dt = dt0 > 0.0 ? dt0 : (t1 - t0) / 100.0;
  F::rhs(y, pp, k1);
  int acc = 0, rej = 0, st = 0;
  for (int it = 0; it < max_steps; ++it) {
    if (t >= t1) break;
    const double h = dt <= t1 - t ? dt : t1 - t;  // Python's min(dt, t1 - t)
    gs::Stages<F> S;
    gs::tsit5_k2_to_k6<F>(y, pp, k1, h, S);
    double y5[D], k7[D], q[D];
    gs::tsit5_y5<F>(y, k1, S, h, y5);
    F::rhs(y5, pp, k7);
    for (int i = 0; i < D; ++i) {
      const double e = h * (T::E1 * k1[i] + T::E2 * S.k2[i] + T::E3 * S.k3[i] +
                            T::E4 * S.k4[i] + T::E5 * S.k5[i] + T::E6 * S.k6[i] +
                            T::E7 * k7[i]);
      const double ay = fabs(y[i]), an = fabs(y5[i]);
      const double sc = atol + rtol * (ay >= an ? ay : an);
      const double c = e / sc;
      q[i] = c * c;
    }
    const double err = sqrt(numpy_sum<D>(q) / (double)D);
    if (err <= 1.0) {
      if (acc >= cap) {
        st = 3;
        break;
      }
      t = t + h;
      for (int i = 0; i < D; ++i) {
        y[i] = y5[i];
        k1[i] = k7[i];
      }
      dts[j * cap + acc] = h;
      ++acc;
    } else {
      ++rej;
    }
    const double e = err > C::ERR_FLOOR ? err : C::ERR_FLOOR;
    double pw = pow(e, T::ORDER_EXP);
    if (pow_table && it < A) {  // the host libm's power, where the table has it (not NaN)
      const double v = pow_table[j * A + it];
      if (v == v) pw = v;
    }
    if (err_log && it < A) {
      err_log[(j * A + it) * 2] = e;
      err_log[(j * A + it) * 2 + 1] = pw;
    }
    const double fac = C::SAFETY * pw;
    const double lo = fac > C::FAC_MIN ? fac : C::FAC_MIN;
    dt = h * (C::FAC_MAX < lo ? C::FAC_MAX : lo);
  }
  if (st == 0 && !(t >= t1)) st = 1;
  for (int s = acc; s < cap; ++s) dts[j * cap + s] = 0.0;
  for (int i = 0; i < D; ++i) yf[j * D + i] = y[i];
  n_acc[j] = acc;
  n_rej[j] = rej;
  status[j] = st;
}

template <class F>
int launch(long long n, const double* y0, const double* p, double t0, double t1, double rtol,
           double atol, double dt0, int max_steps, int cap, double* dts, double* yf, int* n_acc,
           int* n_rej, int* status, const double* pow_table, double* err_log, int A,
           cudaStream_t s) {
  const unsigned block = 64;
  exact_tsit5_record_kernel<F><<<(unsigned)((n + block - 1) / block), block, 0, s>>>(
      n, y0, p, t0, t1, rtol, atol, dt0, max_steps, cap, dts, yf, n_acc, n_rej, status,
      pow_table, err_log, A);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace gx

// Field codes: those of include/gsolve.h; Linear<D> = 4000 + D and Lorenz96<D> = 5000 + D
// for the sizes the goldens hold.  pow_table and err_log may be null (A is then ignored).
// Returns 0, -1 (bad argument), -2 (field not built here) or -3 (launch failed).
extern "C" int gx_tsit5_record(int field, long long n, const double* y0, const double* p,
                               double t0, double t1, double rtol, double atol, double dt0,
                               int max_steps, int cap, double* dts, double* yf, int* n_acc,
                               int* n_rej, int* status, const double* pow_table,
                               double* err_log, int A, void* stream) {
  if (n < 0 || cap < 1 || max_steps < 1 || !y0 || !p || !dts || !yf || !n_acc || !n_rej ||
      !status || ((pow_table || err_log) && A < 1))
    return -1;
  if (n == 0) return 0;
  cudaStream_t s = (cudaStream_t)stream;
#define GX_CASE(code, Fld)                                                                 \
  case code:                                                                               \
    return gx::launch<Fld>(n, y0, p, t0, t1, rtol, atol, dt0, max_steps, cap, dts, yf,     \
                           n_acc, n_rej, status, pow_table, err_log, A, s);
  switch (field) {
    GX_CASE(gs::FIELD_LORENZ, gs::Lorenz)
    GX_CASE(gs::FIELD_VDP, gs::VdP)
    GX_CASE(gs::FIELD_LOTKA_VOLTERRA, gs::LotkaVolterra)
    GX_CASE(gs::FIELD_LORENZ3, gs::Lorenz3)
    GX_CASE(4003, gs::Linear<3>)
    GX_CASE(4010, gs::Linear<10>)
    GX_CASE(4032, gs::Linear<32>)
    GX_CASE(5005, gs::Lorenz96<5>)
    GX_CASE(5008, gs::Lorenz96<8>)
    GX_CASE(5032, gs::Lorenz96<32>)
  }
#undef GX_CASE
  return -2;
}
