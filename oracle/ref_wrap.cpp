// ref_wrap.cpp -- batch entry point around the reference's own hand-CUDA forward, compiled
// for the host.  TEST INFRASTRUCTURE ONLY (a result to compare against and a CPU baseline,
// never the product).
//
// REF_SOURCE names a template from gradsolve/cuda/kernels/*.cu.in filled by
// oracle/build_ref.py exactly as gradsolve/cuda/_codegen.py:42-55 fills it; that file is
// generated into oracle/_ref/ (not committed) and included here unchanged.  Built with
// -ffp-contract=off as gradsolve/cuda/_build.py:56 builds its host target.
#include REF_SOURCE

#include <atomic>
#include <thread>
#include <vector>

namespace {
template <class Fn>
void parallel_rows(long n, int nthreads, Fn fn) {
  std::atomic<long> next{0};
  auto work = [&] {
    for (;;) {
      long j0 = next.fetch_add(16);
      if (j0 >= n) break;
      long j1 = j0 + 16 < n ? j0 + 16 : n;
      for (long j = j0; j < j1; ++j) fn(j);
    }
  };
  if (nthreads <= 1) { work(); return; }
  std::vector<std::thread> th;
  for (int i = 0; i < nthreads - 1; ++i) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
}
}  // namespace

extern "C" int ref_dim(void) { return DIM; }

#ifdef REF_TSIT5
// y0 (n, DIM) row-major, rho (n,), t0 = 0 (the template's convention, :82)
extern "C" int ref_fwd(long n, const double* y0, const double* rho, double t1, double rtol,
                       double atol, int max_steps, double* yf, int* nsteps, int nthreads) {
  parallel_rows(n, nthreads, [&](long j) {
    tsit5_fwd_one(y0 + j * DIM, rho[j], t1, rtol, atol, max_steps, yf + j * DIM, nsteps + j);
  });
  return 0;
}
#endif

#ifdef REF_ROS23
// y0 (n, DIM), p (n, NPARAM) row-major
extern "C" int ref_fwd(long n, const double* y0, const double* p, double t1, double rtol,
                       double atol, int max_steps, double* yf, int* nsteps, int nthreads) {
  parallel_rows(n, nthreads, [&](long j) {
    rosenbrock23_fwd_one(y0 + j * DIM, p + j * NPARAM, t1, rtol, atol, max_steps,
                         yf + j * DIM, nsteps + j);
  });
  return 0;
}
#endif
