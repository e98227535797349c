// gs_xla_ffi.cc -- typed XLA FFI handlers over the C ABI of libgsolve.so, so JAX programs call
// the B200 kernels as custom calls (jax.ffi.ffi_call) under jax.custom_vjp.
//
// The reference binds its hand-CUDA forward the same way (gradsolve/cuda/kernels/
// tsit5_template.cu.in:161-212, registered by gradsolve/cuda/_ffi_bridge.py:51-105); these
// handlers cover the record-and-replay path: forward with record, forward-only solve, replay,
// adjoint (Tsit5 and Rosenbrock23), and the replay gradient without workspace buffers.
// Every handler runs on the stream XLA gives it, allocates nothing (XLA owns every buffer:
// the dt record and the checkpoints are results of the forward and arguments of the later
// calls, sized on the Python side with gs_record_bytes / gs_ckpt_bytes), and is stateless and
// re-entrant, as XLA requires.  A failed call returns ffi::Error with gs_last_error()'s text;
// per-trajectory outcomes stay data in the status result (gradsolve/warp/warp_ode.py:319).
//
// Layouts are the C ABI's: y0, y_final, cotangents (n, D) row-major; params (n, P); dts
// (n, S) row-major for the static-scratch gradient; rec and ckpt flat float64 buffers.
//
// Built by gradsolve_b200/csrc/build.py into libgsolve_xla.so only where
// jax.ffi.include_dir() exists (JAX is not installed in this image); tests/test_xla_ffi.py
// compiles this file against a compile-only stand-in of the FFI header to check that every
// binding matches its handler and every call matches include/gsolve.h.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "xla/ffi/api/ffi.h"
#include "../../include/gsolve.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error status_of(int rc) {
  if (rc == GS_OK) return ffi::Error::Success();
  const std::string msg = std::string("libgsolve: ") + gs_last_error();
  return rc == GS_ERR_ARG ? ffi::Error::InvalidArgument(msg) : ffi::Error::Internal(msg);
}

// Trajectory count of an (n, ...) buffer.
template <class B>
long long rows(const B& b) {
  auto d = b.dimensions();
  return d.size() == 0 ? 0 : (long long)d[0];
}

using FwdFn = int (*)(int, int, long long, const double*, const double*, double, const double*,
                      double, double, double, double, int, int, int, double*, double*, double*,
                      int*, int*, int*, void*);
using ReplayFn = int (*)(int, int, long long, const double*, const double*, double,
                         const double*, const int*, int, int, double*, double*, void*);
using AdjointFn = int (*)(int, int, long long, const double*, const double*, const int*, int,
                          const double*, int, const double*, double*, double*, void*);

// Adaptive forward with record: rec and ckpt are results (capacity cap, interval ckpt_every).
ffi::Error fwd_record(FwdFn fn, cudaStream_t s, ffi::Buffer<ffi::F64> y0, ffi::Buffer<ffi::F64> p,
                      ffi::ResultBuffer<ffi::F64> yf, ffi::ResultBuffer<ffi::S32> n_acc,
                      ffi::ResultBuffer<ffi::S32> n_rej, ffi::ResultBuffer<ffi::S32> status,
                      ffi::ResultBuffer<ffi::F64> rec, ffi::ResultBuffer<ffi::F64> ckpt,
                      int64_t field, int64_t precision, double t0, double t1, double rtol,
                      double atol, double dt0, int64_t max_steps, int64_t cap,
                      int64_t ckpt_every) {
  return status_of(fn((int)field, (int)precision, rows(y0), y0.typed_data(), p.typed_data(), t0,
                      nullptr, t1, rtol, atol, dt0, (int)max_steps, (int)cap, (int)ckpt_every,
                      rec->typed_data(), ckpt->typed_data(), yf->typed_data(),
                      n_acc->typed_data(), n_rej->typed_data(), status->typed_data(), s));
}

ffi::Error tsit5_fwd(cudaStream_t s, ffi::Buffer<ffi::F64> y0, ffi::Buffer<ffi::F64> p,
                     ffi::ResultBuffer<ffi::F64> yf, ffi::ResultBuffer<ffi::S32> n_acc,
                     ffi::ResultBuffer<ffi::S32> n_rej, ffi::ResultBuffer<ffi::S32> status,
                     ffi::ResultBuffer<ffi::F64> rec, ffi::ResultBuffer<ffi::F64> ckpt,
                     int64_t field, int64_t precision, double t0, double t1, double rtol,
                     double atol, double dt0, int64_t max_steps, int64_t cap, int64_t ckpt_every) {
  return fwd_record(gs_tsit5_fwd_record, s, y0, p, yf, n_acc, n_rej, status, rec, ckpt, field,
                    precision, t0, t1, rtol, atol, dt0, max_steps, cap, ckpt_every);
}

ffi::Error ros23_fwd(cudaStream_t s, ffi::Buffer<ffi::F64> y0, ffi::Buffer<ffi::F64> p,
                     ffi::ResultBuffer<ffi::F64> yf, ffi::ResultBuffer<ffi::S32> n_acc,
                     ffi::ResultBuffer<ffi::S32> n_rej, ffi::ResultBuffer<ffi::S32> status,
                     ffi::ResultBuffer<ffi::F64> rec, ffi::ResultBuffer<ffi::F64> ckpt,
                     int64_t field, int64_t precision, double t0, double t1, double rtol,
                     double atol, double dt0, int64_t max_steps, int64_t cap, int64_t ckpt_every) {
  return fwd_record(gs_ros23_fwd_record, s, y0, p, yf, n_acc, n_rej, status, rec, ckpt, field,
                    precision, t0, t1, rtol, atol, dt0, max_steps, cap, ckpt_every);
}

// Forward-only solve (the reference's cuda_tsit5 lane): no record, no checkpoints.
ffi::Error tsit5_solve(cudaStream_t s, ffi::Buffer<ffi::F64> y0, ffi::Buffer<ffi::F64> p,
                       ffi::ResultBuffer<ffi::F64> yf, ffi::ResultBuffer<ffi::S32> n_acc,
                       ffi::ResultBuffer<ffi::S32> n_rej, ffi::ResultBuffer<ffi::S32> status,
                       int64_t field, int64_t precision, double t0, double t1, double rtol,
                       double atol, double dt0, int64_t max_steps) {
  return status_of(gs_tsit5_fwd_record((int)field, (int)precision, rows(y0), y0.typed_data(),
                                       p.typed_data(), t0, nullptr, t1, rtol, atol, dt0,
                                       (int)max_steps, 0, 1, nullptr, nullptr, yf->typed_data(),
                                       n_acc->typed_data(), n_rej->typed_data(),
                                       status->typed_data(), s));
}

// Frozen-mesh replay at (y0, p); writes the checkpoints the adjoint of this point reads.
ffi::Error replay(ReplayFn fn, cudaStream_t s, ffi::Buffer<ffi::F64> y0, ffi::Buffer<ffi::F64> p,
                  ffi::Buffer<ffi::F64> rec, ffi::Buffer<ffi::S32> n_acc,
                  ffi::ResultBuffer<ffi::F64> yf, ffi::ResultBuffer<ffi::F64> ckpt, int64_t field,
                  int64_t precision, double t0, int64_t cap, int64_t ckpt_every) {
  return status_of(fn((int)field, (int)precision, rows(y0), y0.typed_data(), p.typed_data(), t0,
                      rec.typed_data(), n_acc.typed_data(), (int)cap, (int)ckpt_every,
                      ckpt->typed_data(), yf->typed_data(), s));
}

ffi::Error tsit5_replay(cudaStream_t s, ffi::Buffer<ffi::F64> y0, ffi::Buffer<ffi::F64> p,
                        ffi::Buffer<ffi::F64> rec, ffi::Buffer<ffi::S32> n_acc,
                        ffi::ResultBuffer<ffi::F64> yf, ffi::ResultBuffer<ffi::F64> ckpt,
                        int64_t field, int64_t precision, double t0, int64_t cap,
                        int64_t ckpt_every) {
  return replay(gs_tsit5_replay, s, y0, p, rec, n_acc, yf, ckpt, field, precision, t0, cap,
                ckpt_every);
}

ffi::Error ros23_replay(cudaStream_t s, ffi::Buffer<ffi::F64> y0, ffi::Buffer<ffi::F64> p,
                        ffi::Buffer<ffi::F64> rec, ffi::Buffer<ffi::S32> n_acc,
                        ffi::ResultBuffer<ffi::F64> yf, ffi::ResultBuffer<ffi::F64> ckpt,
                        int64_t field, int64_t precision, double t0, int64_t cap,
                        int64_t ckpt_every) {
  return replay(gs_ros23_replay, s, y0, p, rec, n_acc, yf, ckpt, field, precision, t0, cap,
                ckpt_every);
}

// Reverse pass: gy0 = dL/dy0 and gp = dL/dp for the cotangent ybar = dL/dy_final.
ffi::Error adjoint(AdjointFn fn, cudaStream_t s, ffi::Buffer<ffi::F64> p,
                   ffi::Buffer<ffi::F64> rec, ffi::Buffer<ffi::S32> n_acc,
                   ffi::Buffer<ffi::F64> ckpt, ffi::Buffer<ffi::F64> ybar,
                   ffi::ResultBuffer<ffi::F64> gy0, ffi::ResultBuffer<ffi::F64> gp,
                   int64_t field, int64_t precision, int64_t cap, int64_t ckpt_every) {
  return status_of(fn((int)field, (int)precision, rows(ybar), p.typed_data(), rec.typed_data(),
                      n_acc.typed_data(), (int)cap, ckpt.typed_data(), (int)ckpt_every,
                      ybar.typed_data(), gy0->typed_data(), gp->typed_data(), s));
}

ffi::Error tsit5_adjoint(cudaStream_t s, ffi::Buffer<ffi::F64> p, ffi::Buffer<ffi::F64> rec,
                         ffi::Buffer<ffi::S32> n_acc, ffi::Buffer<ffi::F64> ckpt,
                         ffi::Buffer<ffi::F64> ybar, ffi::ResultBuffer<ffi::F64> gy0,
                         ffi::ResultBuffer<ffi::F64> gp, int64_t field, int64_t precision,
                         int64_t cap, int64_t ckpt_every) {
  return adjoint(gs_tsit5_adjoint, s, p, rec, n_acc, ckpt, ybar, gy0, gp, field, precision, cap,
                 ckpt_every);
}

ffi::Error ros23_adjoint(cudaStream_t s, ffi::Buffer<ffi::F64> p, ffi::Buffer<ffi::F64> rec,
                         ffi::Buffer<ffi::S32> n_acc, ffi::Buffer<ffi::F64> ckpt,
                         ffi::Buffer<ffi::F64> ybar, ffi::ResultBuffer<ffi::F64> gy0,
                         ffi::ResultBuffer<ffi::F64> gp, int64_t field, int64_t precision,
                         int64_t cap, int64_t ckpt_every) {
  return adjoint(gs_ros23_adjoint, s, p, rec, n_acc, ckpt, ybar, gy0, gp, field, precision, cap,
                 ckpt_every);
}

// The replay gradient from the reference's padded (n, S) dts with no workspace buffers at
// all (gs_tsit5_vjp_static keeps its record and checkpoints in the library's own scratch):
// the custom call for a JAX program that hands over only the recorded dts.
ffi::Error tsit5_vjp_static(cudaStream_t s, ffi::Buffer<ffi::F64> y0, ffi::Buffer<ffi::F64> p,
                            ffi::Buffer<ffi::F64> dts, ffi::Buffer<ffi::F64> ybar,
                            ffi::ResultBuffer<ffi::F64> yf, ffi::ResultBuffer<ffi::F64> gy0,
                            ffi::ResultBuffer<ffi::F64> gp, int64_t field, double t0) {
  auto d = dts.dimensions();
  const long long S = d.size() < 2 ? 0 : (long long)d[1];
  return status_of(gs_tsit5_vjp_static((int)field, rows(y0), y0.typed_data(), p.typed_data(), t0,
                                       dts.typed_data(), S, S, ybar.typed_data(),
                                       yf->typed_data(), gy0->typed_data(), gp->typed_data(), s));
}

}  // namespace

#define GS_FWD_BINDING                                                                         \
  ffi::Ffi::Bind()                                                                             \
      .Ctx<ffi::PlatformStream<cudaStream_t>>()                                                \
      .Arg<ffi::Buffer<ffi::F64>>()                                                            \
      .Arg<ffi::Buffer<ffi::F64>>()                                                            \
      .Ret<ffi::Buffer<ffi::F64>>()                                                            \
      .Ret<ffi::Buffer<ffi::S32>>()                                                            \
      .Ret<ffi::Buffer<ffi::S32>>()                                                            \
      .Ret<ffi::Buffer<ffi::S32>>()                                                            \
      .Ret<ffi::Buffer<ffi::F64>>()                                                            \
      .Ret<ffi::Buffer<ffi::F64>>()                                                            \
      .Attr<int64_t>("field")                                                                  \
      .Attr<int64_t>("precision")                                                              \
      .Attr<double>("t0")                                                                      \
      .Attr<double>("t1")                                                                      \
      .Attr<double>("rtol")                                                                    \
      .Attr<double>("atol")                                                                    \
      .Attr<double>("dt0")                                                                     \
      .Attr<int64_t>("max_steps")                                                              \
      .Attr<int64_t>("cap")                                                                    \
      .Attr<int64_t>("ckpt_every")

#define GS_REPLAY_BINDING                                                                      \
  ffi::Ffi::Bind()                                                                             \
      .Ctx<ffi::PlatformStream<cudaStream_t>>()                                                \
      .Arg<ffi::Buffer<ffi::F64>>()                                                            \
      .Arg<ffi::Buffer<ffi::F64>>()                                                            \
      .Arg<ffi::Buffer<ffi::F64>>()                                                            \
      .Arg<ffi::Buffer<ffi::S32>>()                                                            \
      .Ret<ffi::Buffer<ffi::F64>>()                                                            \
      .Ret<ffi::Buffer<ffi::F64>>()                                                            \
      .Attr<int64_t>("field")                                                                  \
      .Attr<int64_t>("precision")                                                              \
      .Attr<double>("t0")                                                                      \
      .Attr<int64_t>("cap")                                                                    \
      .Attr<int64_t>("ckpt_every")

#define GS_ADJOINT_BINDING                                                                     \
  ffi::Ffi::Bind()                                                                             \
      .Ctx<ffi::PlatformStream<cudaStream_t>>()                                                \
      .Arg<ffi::Buffer<ffi::F64>>()                                                            \
      .Arg<ffi::Buffer<ffi::F64>>()                                                            \
      .Arg<ffi::Buffer<ffi::S32>>()                                                            \
      .Arg<ffi::Buffer<ffi::F64>>()                                                            \
      .Arg<ffi::Buffer<ffi::F64>>()                                                            \
      .Ret<ffi::Buffer<ffi::F64>>()                                                            \
      .Ret<ffi::Buffer<ffi::F64>>()                                                            \
      .Attr<int64_t>("field")                                                                  \
      .Attr<int64_t>("precision")                                                              \
      .Attr<int64_t>("cap")                                                                    \
      .Attr<int64_t>("ckpt_every")

XLA_FFI_DEFINE_HANDLER_SYMBOL(GsTsit5Fwd, tsit5_fwd, GS_FWD_BINDING);
XLA_FFI_DEFINE_HANDLER_SYMBOL(GsRos23Fwd, ros23_fwd, GS_FWD_BINDING);
XLA_FFI_DEFINE_HANDLER_SYMBOL(GsTsit5Replay, tsit5_replay, GS_REPLAY_BINDING);
XLA_FFI_DEFINE_HANDLER_SYMBOL(GsRos23Replay, ros23_replay, GS_REPLAY_BINDING);
XLA_FFI_DEFINE_HANDLER_SYMBOL(GsTsit5Adjoint, tsit5_adjoint, GS_ADJOINT_BINDING);
XLA_FFI_DEFINE_HANDLER_SYMBOL(GsRos23Adjoint, ros23_adjoint, GS_ADJOINT_BINDING);

XLA_FFI_DEFINE_HANDLER_SYMBOL(GsTsit5Solve, tsit5_solve,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::S32>>()
                                  .Ret<ffi::Buffer<ffi::S32>>()
                                  .Ret<ffi::Buffer<ffi::S32>>()
                                  .Attr<int64_t>("field")
                                  .Attr<int64_t>("precision")
                                  .Attr<double>("t0")
                                  .Attr<double>("t1")
                                  .Attr<double>("rtol")
                                  .Attr<double>("atol")
                                  .Attr<double>("dt0")
                                  .Attr<int64_t>("max_steps"));

XLA_FFI_DEFINE_HANDLER_SYMBOL(GsTsit5VjpStatic, tsit5_vjp_static,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Attr<int64_t>("field")
                                  .Attr<double>("t0"));
