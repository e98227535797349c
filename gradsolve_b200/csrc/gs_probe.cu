// gs_probe.cu -- CUDA-core FMA throughput probes (libgsprobe.so), used by bench.py to measure
// the float64 / float32 pipe peak that the solver kernels are compared against.  Each
// thread runs 8 independent multiply-add chains; flops = 2 * 8 * iters * threads.
#include <cuda_runtime.h>

template <class R>
__global__ void __launch_bounds__(256) fma_probe(R* out, int iters, R a, R b) {
  R x0 = (R)threadIdx.x * (R)1e-3, x1 = x0 + (R)1, x2 = x0 + (R)2, x3 = x0 + (R)3;
  R x4 = x0 + (R)4, x5 = x0 + (R)5, x6 = x0 + (R)6, x7 = x0 + (R)7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const R s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == (R)-1.2345) out[0] = s;  // keeps the chains live; never true for these inputs
}

extern "C" {
// flops per launch = 2 * 32 * iters * blocks * 256
int gs_probe_fp64(double* out, int blocks, int iters, void* stream) {
  fma_probe<double><<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters, 0.999999, 1e-7);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
int gs_probe_fp32(float* out, int blocks, int iters, void* stream) {
  fma_probe<float><<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters, 0.999999f, 1e-7f);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
}

// ---- controller check: the solver's pow-free step factor vs CUDA's pow --------------------
#include "gs_tsit5.cuh"

__global__ void step_factor_probe(const double* S, long long n, int order, int D,
                                  gs::CtrlConsts c, double* fast, double* ref, int* accept_fast,
                                  int* accept_ref) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = S[i];  // the solver's sum of squares; the reference's mean is fl(x / D)
  fast[i] = order == 5 ? gs::step_from_sum<10>(x, 1.0, c) : gs::step_from_sum<6>(x, 1.0, c);
  const double err = sqrt(x / (double)D);
  const double e = err > 1e-10 ? err : 1e-10;
  double fac = 0.9 * pow(e, order == 5 ? -0.2 : -1.0 / 3.0);
  fac = fac > 0.2 ? fac : 0.2;
  fac = 5.0 < fac ? 5.0 : fac;
  ref[i] = fac;
  accept_fast[i] = x <= c.accept_sum;
  accept_ref[i] = err <= 1.0;
}

// The solver's controller (accept test and step factor from the sum of squares, for state
// dimension D) against sqrt and pow of the mean, for n sums of squares S.
extern "C" int gs_probe_step_factor(const double* S, long long n, int order, int D, double* fast,
                                    double* ref, int* accept_fast, int* accept_ref,
                                    void* stream) {
  if (n <= 0) return 0;
  if (D < 1 || (order != 5 && order != 3)) return -1;
  const gs::CtrlConsts c = gs::make_ctrl_consts(D, order == 5 ? 10 : 6);
  step_factor_probe<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      S, n, order, D, c, fast, ref, accept_fast, accept_ref);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
