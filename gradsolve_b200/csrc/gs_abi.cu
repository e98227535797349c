// gs_abi.cu -- the extern "C" entry points of libgsolve.so (declared in include/gsolve.h).
//
// Host-side argument checking, field dispatch to the templated kernels, and launch on the
// caller's stream.  The library allocates nothing and keeps no state besides the
// per-thread error message.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>
#include <type_traits>

#include "../../include/gsolve.h"
#include "gs_coop.cuh"
#include "gs_f32.cuh"
#include "gs_fields.cuh"
#include "gs_mixed.cuh"
#include "gs_ros23.cuh"
#include "gs_persistent.cuh"
#include "gs_saveat.cuh"
#include "gs_tableau.cuh"
#include "gs_tsit5.cuh"

#ifdef GS_USER_FIELD_HEADER
// A library built for one generated field (gradsolve_b200/fieldgen.py): the header defines
// gs::UserField, GS_USER_FIELD_CODE and GS_USER_STIFF, and only that field is dispatched.
#include GS_USER_FIELD_HEADER
#endif

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// Kernel launches this library has issued in the process (every launch is followed by a
// cuda_check, which counts it); read through gs_launch_count.
std::atomic<unsigned long long> g_launches{0};

int cuda_check(const char* what) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(GS_ERR_CUDA, std::string("CUDA: ") + what + ": " + cudaGetErrorString(e));
  return GS_OK;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }
bool aligned8(const void* p) { return ((uintptr_t)p & 7u) == 0; }

constexpr int kBlock = 128;

unsigned grid_for(long long n) { return (unsigned)((n + kBlock - 1) / kBlock); }

#ifdef GS_USER_FIELD_HEADER
int field_dims(int field, int* D, int* P) {
  if (field == GS_USER_FIELD_CODE) {
    *D = gs::UserField::D;
    *P = gs::UserField::P;
    return GS_OK;
  }
  return fail(GS_ERR_FIELD, "this library serves the generated field " +
                                std::to_string(GS_USER_FIELD_CODE) + " only; got " +
                                std::to_string(field));
}

#define GS_TSIT5_DISPATCH(field, FN, ...)                                                   \
  switch (field) {                                                                          \
    case GS_USER_FIELD_CODE: return FN<gs::UserField>(__VA_ARGS__);                        \
    default: return fail(GS_ERR_FIELD, "unknown field code " + std::to_string(field));      \
  }

#if GS_USER_STIFF
#define GS_ROS23_DISPATCH(field, FN, ...)                                                   \
  switch (field) {                                                                          \
    case GS_USER_FIELD_CODE: return FN<gs::UserField>(__VA_ARGS__);                        \
    default: return fail(GS_ERR_FIELD, "unknown field code " + std::to_string(field));      \
  }
#else
#define GS_ROS23_DISPATCH(field, FN, ...)                                                   \
  return fail(GS_ERR_FIELD, "field " + std::to_string(field) +                              \
                                " was registered without stiff=True (no Jacobian)");
#endif

#else
int field_dims(int field, int* D, int* P) {
  switch (field) {
    case gs::FIELD_LORENZ: *D = 3; *P = 1; return GS_OK;
    case gs::FIELD_VDP: *D = 2; *P = 1; return GS_OK;
    case gs::FIELD_LOTKA_VOLTERRA: *D = 2; *P = 4; return GS_OK;
    case gs::FIELD_ROBERTSON: *D = 3; *P = 3; return GS_OK;
    case gs::FIELD_LORENZ3: *D = 3; *P = 3; return GS_OK;
    case 4001: *D = 1; *P = 1; return GS_OK;
    case 4002: *D = 2; *P = 1; return GS_OK;
    case 4003: *D = 3; *P = 1; return GS_OK;
    case 4004: *D = 4; *P = 1; return GS_OK;
    case 4008: *D = 8; *P = 1; return GS_OK;
    case 4010: *D = 10; *P = 1; return GS_OK;
    case 4032: *D = 32; *P = 1; return GS_OK;
    case 5004: *D = 4; *P = 1; return GS_OK;
    case 5008: *D = 8; *P = 1; return GS_OK;
    case 5032: *D = 32; *P = 1; return GS_OK;
    case gs::FIELD_HIRES: *D = 8; *P = 1; return GS_OK;
  }
  return fail(GS_ERR_FIELD, "unknown field code " + std::to_string(field));
}

// Non-stiff fields usable by the Tsit5 kernels.
#define GS_TSIT5_DISPATCH(field, FN, ...)                                                   \
  switch (field) {                                                                          \
    case gs::FIELD_LORENZ: return FN<gs::Lorenz>(__VA_ARGS__);                              \
    case gs::FIELD_LORENZ3: return FN<gs::Lorenz3>(__VA_ARGS__);                            \
    case gs::FIELD_VDP: return FN<gs::VdP>(__VA_ARGS__);                                    \
    case gs::FIELD_LOTKA_VOLTERRA: return FN<gs::LotkaVolterra>(__VA_ARGS__);               \
    case gs::FIELD_ROBERTSON: return FN<gs::Robertson>(__VA_ARGS__);                        \
    case 4001: return FN<gs::Linear<1>>(__VA_ARGS__);                                       \
    case 4002: return FN<gs::Linear<2>>(__VA_ARGS__);                                       \
    case 4003: return FN<gs::Linear<3>>(__VA_ARGS__);                                       \
    case 4004: return FN<gs::Linear<4>>(__VA_ARGS__);                                       \
    case 4008: return FN<gs::Linear<8>>(__VA_ARGS__);                                       \
    case 4010: return FN<gs::Linear<10>>(__VA_ARGS__);                                      \
    case 4032: return FN<gs::Linear<32>>(__VA_ARGS__);                                      \
    case 5004: return FN<gs::Lorenz96<4>>(__VA_ARGS__);                                     \
    case 5008: return FN<gs::Lorenz96<8>>(__VA_ARGS__);                                     \
    case 5032: return FN<gs::Lorenz96<32>>(__VA_ARGS__);                                    \
    case gs::FIELD_HIRES: return FN<gs::Hires>(__VA_ARGS__);                                \
    default: return fail(GS_ERR_FIELD, "unknown field code " + std::to_string(field));      \
  }

// Fields with an analytic Jacobian, usable by the Rosenbrock23 kernels.
#define GS_ROS23_DISPATCH(field, FN, ...)                                                   \
  switch (field) {                                                                          \
    case gs::FIELD_ROBERTSON: return FN<gs::Robertson>(__VA_ARGS__);                        \
    case gs::FIELD_VDP: return FN<gs::VdP>(__VA_ARGS__);                                    \
    case 4001: return FN<gs::Linear<1>>(__VA_ARGS__);                                       \
    case 4002: return FN<gs::Linear<2>>(__VA_ARGS__);                                       \
    case 4003: return FN<gs::Linear<3>>(__VA_ARGS__);                                       \
    case 4004: return FN<gs::Linear<4>>(__VA_ARGS__);                                       \
    case 4008: return FN<gs::Linear<8>>(__VA_ARGS__);                                       \
    case gs::FIELD_HIRES: return FN<gs::Hires>(__VA_ARGS__);                                \
    default:                                                                                \
      return fail(GS_ERR_FIELD,                                                             \
                  "field " + std::to_string(field) + " has no analytic Jacobian for Rosenbrock23"); \
  }

#endif  // GS_USER_FIELD_HEADER

// Launch shape of the adjoint kernels: each thread keeps its segment of K states (W doubles
// each) in shared memory, so the block shrinks (by powers of two, at least one warp) until the
// block's buffer fits the per-block budget.
struct SegCfg {
  unsigned block;
  size_t smem;
  long long resident;  // threads per SM at this shape (occupancy_cfg)
};

constexpr size_t kSegBudget = 200u * 1024u;

SegCfg seg_cfg(int K, int W) {
  const size_t per_thread = (size_t)K * (size_t)W * sizeof(double);
  const size_t budget = kSegBudget;
  unsigned block = kBlock;
  while (block > 32 && per_thread * block > budget) block /= 2;
  return {block, per_thread * block, 0};
}

// The same shrinking rule for a per-thread size given in doubles.
SegCfg seg_cfg_doubles(int doubles_per_thread) { return seg_cfg(1, doubles_per_thread); }

template <class Kern>
int allow_smem(Kern kernel, size_t smem) {
  if (smem <= 48u * 1024u) return GS_OK;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess)
    return fail(GS_ERR_CUDA, std::string("CUDA: cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  return GS_OK;
}

unsigned grid_for_block(long long n, unsigned block) { return (unsigned)((n + block - 1) / block); }

// Block size (128, 64 or 32) that keeps the most threads resident per SM for a kernel whose
// threads each use doubles_per_thread of dynamic shared memory (registers and shared memory
// both limit residency; smaller blocks pack the shared memory more finely).  Ties keep the
// larger block.  Sets the kernel's dynamic shared memory limit for the chosen size.
// occupancy_probe leaves out->resident = 0 (and reports no error) when no block size fits.
template <class Kern>
int occupancy_probe(Kern kernel, int doubles_per_thread, SegCfg* out) {
  SegCfg best{0, 0, 0};
  for (unsigned block : {128u, 64u, 32u}) {
    const size_t smem = (size_t)doubles_per_thread * sizeof(double) * block;
    if (smem > kSegBudget) continue;
    int rc = allow_smem(kernel, smem);
    if (rc) return rc;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem);
    if (e != cudaSuccess)
      return fail(GS_ERR_CUDA, std::string("CUDA: occupancy query: ") + cudaGetErrorString(e));
    const long long res = (long long)per_sm * block;
    if (res > best.resident) best = {block, smem, res};
  }
  *out = best;
  return best.resident > 0 ? allow_smem(kernel, best.smem) : GS_OK;
}

template <class Kern>
int occupancy_cfg(Kern kernel, int doubles_per_thread, SegCfg* out) {
  int rc = occupancy_probe(kernel, doubles_per_thread, out);
  if (rc) return rc;
  if (out->resident <= 0)
    return fail(GS_ERR_ARG, "segment buffer does not fit shared memory (checkpoint interval "
                            "too large for this state dimension)");
  return GS_OK;
}

// The reverse passes that keep a segment's forward quantities (Tsit5 stage inputs,
// Rosenbrock23 factors) save the recomputation of K-1 of every K step forwards, but their
// buffer grows with K and costs resident threads.  They are taken while they keep at least
// 3/5 of the recomputing kernel's residency: measured on Lorenz (Tsit5) the keeping kernel
// still wins at K = 4 (residency 384 vs 640 threads/SM: 15.9 vs 16.9 ms), and on VdP
// (Rosenbrock23, K = 8: 192 vs 640) it lost by 1.6x.
bool keeping_pays(const SegCfg& keep, const SegCfg& recompute) {
  return keep.resident > 0 && keep.resident * 5 >= recompute.resident * 3;
}

// ---- scheduling ------------------------------------------------------------------------------
// GS_SCHED_* flags ride in the high bits of the precision argument.  AUTO: one thread per
// trajectory (hardware block scheduling) for a shared end time, lane refill with a work
// counter when trajectories have their own end times (uneven batches); the reverse pass runs
// one thread per trajectory unless the caller asks for refill.
int forward_schedule(int precision, const double* t1v, const double* ckpt) {
  int s = precision & GS_SCHED_MASK;
  if (s == GS_SCHED_AUTO) s = t1v ? GS_SCHED_REFILL : GS_SCHED_STATIC;
  if (s == GS_SCHED_REFILL && !ckpt) s = GS_SCHED_STRIDED;  // no control block to count in
  return s;
}

int adjoint_schedule(int precision) {
  const int s = precision & GS_SCHED_MASK;
  return s == GS_SCHED_AUTO ? GS_SCHED_STATIC : s;
}

// ---- persistent launches (gs_persistent.cuh) ------------------------------------------------
// One wave of resident blocks; the work counter lives in the control block that follows the
// checkpoint slots (gs_ckpt_bytes includes it) and is zeroed on the stream before the launch.
unsigned long long* ctrl_counter(double* ckpt, long long n, int slots, int D, int which) {
  if (!ckpt) return nullptr;
  double* end = ckpt + (size_t)slots * (size_t)n * (size_t)gs::ckpt_width(D);
  return reinterpret_cast<unsigned long long*>(end) + which;
}

template <class Kern>
int persistent_grid(Kern kernel, unsigned block, size_t smem, long long n, unsigned* grid) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem);
  if (e != cudaSuccess)
    return fail(GS_ERR_CUDA, std::string("CUDA: occupancy query: ") + cudaGetErrorString(e));
  const long long resident = (long long)sms * (per_sm > 0 ? per_sm : 1);
  const long long needed = (n + block - 1) / block;
  *grid = (unsigned)(needed < resident ? needed : resident);
  return GS_OK;
}

int zero_counter(unsigned long long* c, cudaStream_t s) {
  if (!c) return GS_OK;
  cudaError_t e = cudaMemsetAsync(c, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess)
    return fail(GS_ERR_CUDA, std::string("CUDA: cudaMemsetAsync: ") + cudaGetErrorString(e));
  return GS_OK;
}

template <class F, class L>
int launch_record_persistent(const gs::RecordArgs& a_in, cudaStream_t s, bool use_counter) {
  gs::RecordArgs a = a_in;
  a.ctrl = gs::make_ctrl_consts(F::D, L::QK);
  unsigned long long* counter =
      use_counter ? ctrl_counter(a.ckpt, a.n, a.ck_slots, F::D, gs::kCtrlFwd) : nullptr;
  unsigned grid = 0;
  int rc;
  if ((rc = persistent_grid(gs::record_persistent_kernel<F, L>, kBlock, 0, a.n, &grid))) return rc;
  if ((rc = zero_counter(counter, s))) return rc;
  gs::record_persistent_kernel<F, L><<<grid, kBlock, 0, s>>>(a, counter);
  return cuda_check("record_persistent_kernel");
}

template <class F, class M>
int launch_adjoint_persistent(const gs::AdjointArgs& a, int cap, cudaStream_t s,
                              bool use_counter) {
  const SegCfg c = seg_cfg_doubles(gs::adjoint_smem_doubles<F::D>(a.ck_every));
  unsigned long long* counter =
      use_counter ? ctrl_counter(const_cast<double*>(a.ckpt), a.n,
                                 gs_ckpt_slots(cap, a.ck_every), F::D, gs::kCtrlAdj)
                  : nullptr;
  unsigned grid = 0;
  int rc;
  if ((rc = allow_smem(gs::adjoint_persistent_kernel<F, M>, c.smem))) return rc;
  if ((rc = persistent_grid(gs::adjoint_persistent_kernel<F, M>, c.block, c.smem, a.n, &grid)))
    return rc;
  if ((rc = zero_counter(counter, s))) return rc;
  gs::adjoint_persistent_kernel<F, M><<<grid, c.block, c.smem, s>>>(a, counter);
  return cuda_check("adjoint_persistent_kernel");
}

// ---- fields integrated by a group of lanes per trajectory (gs_coop.cuh) ----------------------
// Their D > 8 states run one group of lanes per trajectory in float64, one trajectory per
// group (the schedule flags do not apply); the float32-stage mode, the dense output and the
// static-scratch entry point are not built for them and refuse with GS_ERR_PRECISION /
// GS_ERR_FIELD.
template <class F>
constexpr bool kCoop = gs::group_of<F>::value > 1;

template <class F>
int coop_refuse(const char* what) {
  return fail(GS_ERR_FIELD, std::string(what) + " is not built for fields of more than 8 "
                                "components (D = " + std::to_string(F::D) +
                                ", integrated by a group of lanes per trajectory)");
}

int coop_refuse_mixed() {
  return fail(GS_ERR_PRECISION, "the float32-stage mode is not built for fields of more than 8 "
                                "components");
}

// The group sizes built for F: the default, then half and twice it where built.
template <class F>
int lane_choices(int* out, int cap) {
  constexpr int G0 = gs::group_of<F>::value;
  int k = 0;
  if (cap > k) out[k] = G0;
  ++k;
  if constexpr (G0 > 1) {
    if constexpr (gs::group_built<F::D, G0 / 2>()) {
      if (cap > k) out[k] = G0 / 2;
      ++k;
    }
    if constexpr (gs::group_built<F::D, 2 * G0>()) {
      if (cap > k) out[k] = 2 * G0;
      ++k;
    }
  }
  return k;
}

// Occupancy instances (GS_OCC) for fields of up to 4 components.  Rosenbrock23: the
// recording forward (unbounded by default) also bounded for 4 and 6 blocks per SM, the K = 2
// kept-factor reverse pass (default 4 blocks) for 3 and 5.  Tsit5: the float64 recording
// forward, whose default instance is bounded for 6 blocks per SM, also has instances bounded
// for 4 and 5 (more registers: longer-range scheduling, no spills where the default spills),
// 7 and 8 (fewer registers, more resident warps); the float64 reverse pass's K = 2
// stage-keeping instance (default 5 blocks) has 3, 4 and 6, the float32-stage one (default
// 6) 4 and 5.  Larger fields keep the compiler's
// allocation alone.
template <class F>
int occ_choices(int pass, int* out, int cap) {
  int k = 0;
  if (cap > k) out[k] = 0;
  ++k;
  if constexpr (F::D <= 4) {
    const std::initializer_list<int> fwd = {4, 5, 7, 8}, rev = {3, 4, 6}, rfwd = {4, 6},
                                     rrev = {3, 5}, mrev = {4, 5};
    for (int b : (pass == GS_OCC_REVERSE ? rev : pass == GS_OCC_ROS23_FORWARD ? rfwd
                  : pass == GS_OCC_ROS23_REVERSE ? rrev
                  : pass == GS_OCC_MIXED_REVERSE ? mrev : fwd)) {
      if (cap > k) out[k] = b;
      ++k;
    }
  }
  return k;
}

template <class F>
int launch_adjoint_k2_occ(const gs::AdjointArgs& a, cudaStream_t s, int occ, bool mixed) {
  if constexpr (F::D <= 4) {
    const int sd = mixed ? gs::mixed_stages_smem_doubles<F::D>(2)
                         : gs::adjoint_stages_smem_doubles<F::D>(2);
    auto go = [&](auto kern) -> int {
      SegCfg c{0, 0, 0};
      int rc;
      if ((rc = occupancy_probe(kern, sd, &c))) return rc;
      if (c.resident <= 0)
        return fail(GS_ERR_ARG, "GS_OCC: the K = 2 segment buffer does not fit shared memory");
      if ((rc = allow_smem(kern, c.smem))) return rc;
      kern<<<grid_for_block(a.n, c.block), c.block, c.smem, s>>>(a);
      return cuda_check("tsit5_adjoint_stages_kernel");
    };
    if (mixed) {
      switch (occ) {
        case 4: return go(gs::tsit5_mixed_adjoint_stages_k2_kernel<F, 4>);
        case 5: return go(gs::tsit5_mixed_adjoint_stages_k2_kernel<F, 5>);
        default: break;
      }
    } else {
      switch (occ) {
        case 3: return go(gs::tsit5_adjoint_stages_k2_kernel<F, 3>);
        case 4: return go(gs::tsit5_adjoint_stages_k2_kernel<F, 4>);
        case 6: return go(gs::tsit5_adjoint_stages_k2_kernel<F, 6>);
        default: break;
      }
    }
  }
  return fail(GS_ERR_ARG, "GS_OCC: no reverse-pass instance bounded for " + std::to_string(occ) +
                              " blocks per SM is built for D = " + std::to_string(F::D) +
                              " (gs_occ_choices)");
}

template <class F>
int launch_record_occ(const gs::RecordArgs& a, cudaStream_t s, int occ) {
  if constexpr (F::D <= 4) {
    switch (occ) {
      case 4: gs::tsit5_record_kernel<F, true, 4><<<grid_for(a.n), kBlock, 0, s>>>(a);
        return cuda_check("tsit5_record_kernel");
      case 5: gs::tsit5_record_kernel<F, true, 5><<<grid_for(a.n), kBlock, 0, s>>>(a);
        return cuda_check("tsit5_record_kernel");
      case 7: gs::tsit5_record_kernel<F, true, 7><<<grid_for(a.n), kBlock, 0, s>>>(a);
        return cuda_check("tsit5_record_kernel");
      case 8: gs::tsit5_record_kernel<F, true, 8><<<grid_for(a.n), kBlock, 0, s>>>(a);
        return cuda_check("tsit5_record_kernel");
      default: break;
    }
  }
  return fail(GS_ERR_ARG, "GS_OCC: no recording-forward instance bounded for " +
                              std::to_string(occ) + " blocks per SM is built for D = " +
                              std::to_string(F::D) + " (gs_occ_choices)");
}

// Launch `go` with the group size the precision flags ask for (GS_LANES; 0: the default):
// go is called with an integral_constant of the size, so each kernel is instantiated only for
// the built sizes.
template <class F, class Go>
int with_lanes(int precision, Go go) {
  constexpr int G0 = gs::group_of<F>::value;
  const int k = (precision & GS_LANES_MASK) >> GS_LANES_SHIFT;
  const int G = k == 0 ? G0 : (1 << k);
  if (G == G0) return go(std::integral_constant<int, G0>{});
  if constexpr (gs::group_built<F::D, G0 / 2>()) {
    if (G == G0 / 2) return go(std::integral_constant<int, G0 / 2>{});
  }
  if constexpr (gs::group_built<F::D, 2 * G0>()) {
    if (G == 2 * G0) return go(std::integral_constant<int, 2 * G0>{});
  }
  return fail(GS_ERR_ARG, "a group of " + std::to_string(G) + " lanes per trajectory is not " +
                              "built for D = " + std::to_string(F::D) + " (gs_lane_choices)");
}

template <class F>
int launch_coop_record(const gs::RecordArgs& a_in, cudaStream_t s, bool mixed, int precision) {
  if (mixed) return coop_refuse_mixed();
  gs::RecordArgs a = a_in;
  a.ctrl = gs::make_ctrl_consts(F::D, 10);
  return with_lanes<F>(precision, [&](auto g) {
    constexpr int G = decltype(g)::value;
    const unsigned grid = grid_for(a.n * G);
    if (!a.rec && !a.ckpt)
      gs::tsit5_coop_record_kernel<F, G, false><<<grid, kBlock, 0, s>>>(a);
    else
      gs::tsit5_coop_record_kernel<F, G, true><<<grid, kBlock, 0, s>>>(a);
    return cuda_check("tsit5_coop_record_kernel");
  });
}

template <class F>
int launch_coop_replay(const gs::ReplayArgs& a, cudaStream_t s, bool mixed, int precision) {
  if (mixed) return coop_refuse_mixed();
  return with_lanes<F>(precision, [&](auto g) {
    constexpr int G = decltype(g)::value;
    gs::tsit5_coop_replay_kernel<F, G><<<grid_for(a.n * G), kBlock, 0, s>>>(a);
    return cuda_check("tsit5_coop_replay_kernel");
  });
}

template <class F>
int launch_coop_adjoint(const gs::AdjointArgs& a, cudaStream_t s, bool mixed, int precision) {
  if (mixed) return coop_refuse_mixed();
  return with_lanes<F>(precision, [&](auto g) {
    constexpr int G = decltype(g)::value;
    constexpr int C = F::D / G;
    SegCfg c;
    int rc;
    if ((rc = occupancy_cfg(gs::tsit5_coop_adjoint_kernel<F, G>,
                            gs::adjoint_smem_doubles<C>(a.ck_every), &c)))
      return rc;
    gs::tsit5_coop_adjoint_kernel<F, G>
        <<<grid_for_block(a.n * G, c.block), c.block, c.smem, s>>>(a);
    return cuda_check("tsit5_coop_adjoint_kernel");
  });
}

// mixed = float32 stages (GS_PREC_MIXED, gs_mixed.cuh), else float64 throughout.
template <class F>
int launch_tsit5_record(const gs::RecordArgs& a_in, cudaStream_t s, bool mixed, int sched,
                        int precision) {
  if constexpr (kCoop<F>) {
    (void)sched;
    if (precision & GS_OCC_MASK)
      return fail(GS_ERR_ARG, "GS_OCC: fields of more than 8 components have no occupancy "
                              "instances (gs_occ_choices)");
    return launch_coop_record<F>(a_in, s, mixed, precision);
  } else {
  if (precision & GS_LANES_MASK)
    return fail(GS_ERR_ARG, "lanes per trajectory apply to fields of more than 8 components only");
  gs::RecordArgs a = a_in;
  a.ctrl = gs::make_ctrl_consts(F::D, 10);  // Tsit5: err^(-1/5) = m^(-1/10)
  const int occ = (precision & GS_OCC_MASK) >> GS_OCC_SHIFT;
  if (occ && (mixed || sched != GS_SCHED_STATIC || (!a.rec && !a.ckpt)))
    return fail(GS_ERR_ARG, "GS_OCC applies to the float64 recording forward, one thread per "
                            "trajectory");
  if (sched == GS_SCHED_STATIC) {
    if (mixed) {
      gs::tsit5_mixed_record_kernel<F><<<grid_for(a.n), kBlock, 0, s>>>(a);
      return cuda_check("tsit5_mixed_record_kernel");
    }
    if (occ) return launch_record_occ<F>(a, s, occ);
    if (!a.rec && !a.ckpt)
      gs::tsit5_record_kernel<F, false><<<grid_for(a.n), kBlock, 0, s>>>(a);
    else
      gs::tsit5_record_kernel<F><<<grid_for(a.n), kBlock, 0, s>>>(a);
    return cuda_check("tsit5_record_kernel");
  }
  const bool counter = sched == GS_SCHED_REFILL;
  return mixed ? launch_record_persistent<F, gs::LaneTsit5Mixed<F>>(a, s, counter)
               : launch_record_persistent<F, gs::LaneTsit5F64<F>>(a, s, counter);
  }
}
template <class F>
int launch_tsit5_replay(const gs::ReplayArgs& a, cudaStream_t s, bool mixed, int precision) {
  if constexpr (kCoop<F>) {
    return launch_coop_replay<F>(a, s, mixed, precision);
  } else {
  if (precision & GS_LANES_MASK)
    return fail(GS_ERR_ARG, "lanes per trajectory apply to fields of more than 8 components only");
  if (mixed) {
    gs::tsit5_mixed_replay_kernel<F><<<grid_for(a.n), kBlock, 0, s>>>(a);
    return cuda_check("tsit5_mixed_replay_kernel");
  }
  gs::tsit5_replay_kernel<F><<<grid_for(a.n), kBlock, 0, s>>>(a);
  return cuda_check("tsit5_replay_kernel");
  }
}
template <class F>
int launch_tsit5_adjoint(const gs::AdjointArgs& a, int cap, cudaStream_t s, bool mixed,
                         int sched, int variant, int precision) {
  const int occ = (precision & GS_OCC_MASK) >> GS_OCC_SHIFT;
  if (occ && (kCoop<F> || sched != GS_SCHED_STATIC || variant == GS_ADJ_RECOMPUTE ||
              a.ck_every != 2))
    return fail(GS_ERR_ARG, "GS_OCC applies to the reverse pass's K = 2 stage-keeping "
                            "instance, one thread per trajectory");
  if constexpr (kCoop<F>) {
    (void)cap; (void)sched; (void)variant;
    return launch_coop_adjoint<F>(a, s, mixed, precision);
  } else {
  if (precision & GS_LANES_MASK)
    return fail(GS_ERR_ARG, "lanes per trajectory apply to fields of more than 8 components only");
  if (occ) return launch_adjoint_k2_occ<F>(a, s, occ, mixed);
  if (sched == GS_SCHED_STATIC) {
    int rc;
    if (!mixed) {
      // the stage-keeping variant needs 5*D more doubles per replayed step of the segment:
      // taken when asked for (while it fits) or, by default, while it keeps enough residency
      // K = 2 (the autotuned interval of the built-in fields) has an unrolled instance, taken
      // where it keeps as many threads resident as the general one
      auto stages = gs::tsit5_adjoint_stages_kernel<F>;
      SegCfg ck{0, 0, 0}, cr{0, 0, 0};
      const int sd = gs::adjoint_stages_smem_doubles<F::D>(a.ck_every);
      if (variant != GS_ADJ_RECOMPUTE) {
        if ((rc = occupancy_probe(stages, sd, &ck))) return rc;
        // (only small states: the instance's register bound would spill an 8-state field's)
        if constexpr (F::D <= 4) {
          if (a.ck_every == 2) {
            SegCfg c2{0, 0, 0};
            if ((rc = occupancy_probe(gs::tsit5_adjoint_stages_k2_kernel<F>, sd, &c2)))
              return rc;
            if (c2.resident > 0 && c2.resident >= ck.resident) {
              stages = gs::tsit5_adjoint_stages_k2_kernel<F>;
              ck = c2;
            }
          }
        }
      }
      if ((rc = occupancy_probe(gs::tsit5_adjoint_kernel<F>,
                                gs::adjoint_smem_doubles<F::D>(a.ck_every), &cr)))
        return rc;
      if (ck.resident > 0 && (variant == GS_ADJ_STAGES || keeping_pays(ck, cr))) {
        if ((rc = allow_smem(stages, ck.smem))) return rc;
        stages<<<grid_for_block(a.n, ck.block), ck.block, ck.smem, s>>>(a);
        return cuda_check("tsit5_adjoint_stages_kernel");
      }
      if (cr.resident <= 0)
        return fail(GS_ERR_ARG, "segment buffer does not fit shared memory (checkpoint "
                                "interval too large for this state dimension)");
      if ((rc = allow_smem(gs::tsit5_adjoint_kernel<F>, cr.smem))) return rc;
      gs::tsit5_adjoint_kernel<F><<<grid_for_block(a.n, cr.block), cr.block, cr.smem, s>>>(a);
      return cuda_check("tsit5_adjoint_kernel");
    }
    // float32 stages: the same choice between keeping the replayed steps' stage inputs (6*D
    // floats per step) and recomputing them, with the same K = 2 instance for small states
    auto mstages = gs::tsit5_mixed_adjoint_stages_kernel<F>;
    SegCfg ck{0, 0, 0}, cr{0, 0, 0};
    const int msd = gs::mixed_stages_smem_doubles<F::D>(a.ck_every);
    if (variant != GS_ADJ_RECOMPUTE) {
      if ((rc = occupancy_probe(mstages, msd, &ck))) return rc;
      if constexpr (F::D <= 4) {
        if (a.ck_every == 2) {
          SegCfg c2{0, 0, 0};
          if ((rc = occupancy_probe(gs::tsit5_mixed_adjoint_stages_k2_kernel<F>, msd, &c2)))
            return rc;
          if (c2.resident > 0 && c2.resident >= ck.resident) {
            mstages = gs::tsit5_mixed_adjoint_stages_k2_kernel<F>;
            ck = c2;
          }
        }
      }
    }
    if ((rc = occupancy_probe(gs::tsit5_mixed_adjoint_kernel<F>,
                              gs::adjoint_smem_doubles<F::D>(a.ck_every), &cr)))
      return rc;
    if (ck.resident > 0 && (variant == GS_ADJ_STAGES || keeping_pays(ck, cr))) {
      if ((rc = allow_smem(mstages, ck.smem))) return rc;
      mstages<<<grid_for_block(a.n, ck.block), ck.block, ck.smem, s>>>(a);
      return cuda_check("tsit5_mixed_adjoint_stages_kernel");
    }
    if (cr.resident <= 0)
      return fail(GS_ERR_ARG, "segment buffer does not fit shared memory (checkpoint "
                              "interval too large for this state dimension)");
    if ((rc = allow_smem(gs::tsit5_mixed_adjoint_kernel<F>, cr.smem))) return rc;
    gs::tsit5_mixed_adjoint_kernel<F><<<grid_for_block(a.n, cr.block), cr.block, cr.smem, s>>>(a);
    return cuda_check("tsit5_mixed_adjoint_kernel");
  }
  const bool counter = sched == GS_SCHED_REFILL;
  return mixed ? launch_adjoint_persistent<F, gs::Tsit5MixedStep>(a, cap, s, counter)
               : launch_adjoint_persistent<F, gs::Tsit5F64Step>(a, cap, s, counter);
  }
}
template <class F>
int launch_ros23_record(const gs::RecordArgs& a_in, cudaStream_t s, int sched, int occ) {
  gs::RecordArgs a = a_in;
  a.ctrl = gs::make_ctrl_consts(F::D, 6);  // Rosenbrock23: err^(-1/3) = m^(-1/6)
  if (occ && (sched != GS_SCHED_STATIC || (!a.rec && !a.ckpt)))
    return fail(GS_ERR_ARG, "GS_OCC applies to the float64 recording forward, one thread per "
                            "trajectory");
  if (occ) {
    if constexpr (F::D <= 4) {
      switch (occ) {
        case 4: gs::ros23_record_occ_kernel<F, 4><<<grid_for(a.n), kBlock, 0, s>>>(a);
          return cuda_check("ros23_record_occ_kernel");
        case 6: gs::ros23_record_occ_kernel<F, 6><<<grid_for(a.n), kBlock, 0, s>>>(a);
          return cuda_check("ros23_record_occ_kernel");
        default: break;
      }
    }
    return fail(GS_ERR_ARG, "GS_OCC: no Rosenbrock23 forward instance bounded for " +
                                std::to_string(occ) + " blocks per SM is built for D = " +
                                std::to_string(F::D) + " (gs_occ_choices)");
  }
  if (sched == GS_SCHED_STATIC) {
    if (!a.rec && !a.ckpt)
      gs::ros23_record_kernel<F, false><<<grid_for(a.n), kBlock, 0, s>>>(a);
    else
      gs::ros23_record_kernel<F><<<grid_for(a.n), kBlock, 0, s>>>(a);
    return cuda_check("ros23_record_kernel");
  }
  return launch_record_persistent<F, gs::LaneRos23<F>>(a, s, sched == GS_SCHED_REFILL);
}
template <class F>
int launch_ros23_replay(const gs::ReplayArgs& a, cudaStream_t s) {
  gs::ros23_replay_kernel<F><<<grid_for(a.n), kBlock, 0, s>>>(a);
  return cuda_check("ros23_replay_kernel");
}
template <class F>
int launch_ros23_adjoint(const gs::AdjointArgs& a, int cap, cudaStream_t s, int sched, int occ) {
  if (occ) {
    if (sched != GS_SCHED_STATIC || a.ck_every != 2)
      return fail(GS_ERR_ARG, "GS_OCC applies to the Rosenbrock23 reverse pass's K = 2 "
                              "kept-factor instance, one thread per trajectory");
    if constexpr (F::D <= 4) {
      auto go = [&](auto kern) -> int {
        SegCfg c{0, 0, 0};
        int rc;
        if ((rc = occupancy_probe(kern, gs::ros23_adjoint_smem_doubles<F::D, true>(2), &c)))
          return rc;
        if (c.resident <= 0)
          return fail(GS_ERR_ARG, "GS_OCC: the K = 2 segment buffer does not fit shared memory");
        if ((rc = allow_smem(kern, c.smem))) return rc;
        kern<<<grid_for_block(a.n, c.block), c.block, c.smem, s>>>(a);
        return cuda_check("ros23_adjoint_kernel");
      };
      switch (occ) {
        case 3: return go(gs::ros23_adjoint_k2_kernel<F, 3>);
        case 5: return go(gs::ros23_adjoint_k2_kernel<F, 5>);
        default: break;
      }
    }
    return fail(GS_ERR_ARG, "GS_OCC: no Rosenbrock23 reverse-pass instance bounded for " +
                                std::to_string(occ) + " blocks per SM is built for D = " +
                                std::to_string(F::D) + " (gs_occ_choices)");
  }
  if (sched == GS_SCHED_STATIC) {
    SegCfg ck{0, 0, 0}, cr{0, 0, 0};
    int rc;
    if ((rc = occupancy_probe(gs::ros23_adjoint_kernel<F, true>,
                              gs::ros23_adjoint_smem_doubles<F::D, true>(a.ck_every), &ck)))
      return rc;
    if ((rc = occupancy_probe(gs::ros23_adjoint_kernel<F, false>,
                              gs::ros23_adjoint_smem_doubles<F::D, false>(a.ck_every), &cr)))
      return rc;
    if (keeping_pays(ck, cr)) {
      auto keep = gs::ros23_adjoint_kernel<F, true>;
      // the unrolled instance, where it keeps the residency (small states only: its register
      // bound would spill an 8-state field's)
      if constexpr (F::D <= 4) {
        if (a.ck_every == 2) {
          SegCfg c2{0, 0, 0};
          if ((rc = occupancy_probe(gs::ros23_adjoint_k2_kernel<F>,
                                    gs::ros23_adjoint_smem_doubles<F::D, true>(2), &c2)))
            return rc;
          if (c2.resident > 0 && c2.resident >= ck.resident) {
            keep = gs::ros23_adjoint_k2_kernel<F>;
            ck = c2;
          }
        }
      }
      if ((rc = allow_smem(keep, ck.smem))) return rc;
      keep<<<grid_for_block(a.n, ck.block), ck.block, ck.smem, s>>>(a);
      return cuda_check("ros23_adjoint_kernel");
    }
    // large K: the kept factors would cost too many resident threads (or not fit); recompute
    if (cr.resident <= 0)
      return fail(GS_ERR_ARG, "segment buffer does not fit shared memory (checkpoint interval "
                              "too large for this state dimension)");
    if ((rc = allow_smem(gs::ros23_adjoint_kernel<F, false>, cr.smem))) return rc;
    gs::ros23_adjoint_kernel<F, false><<<grid_for_block(a.n, cr.block), cr.block, cr.smem, s>>>(a);
    return cuda_check("ros23_adjoint_kernel");
  }
  return launch_adjoint_persistent<F, gs::Ros23Step>(a, cap, s, sched == GS_SCHED_REFILL);
}

// ---- the float32 route (GS_PREC_F32, gs_f32.cuh) ----------------------------------------
// One thread per trajectory, fields of at most 8 components; kMethod 0 = Tsit5, 1 =
// Rosenbrock23.  AUTO is the static schedule here, per-trajectory end times included.
// pairs_ok: the caller is the Tsit5 reverse pass, which takes GS_ADJ_RECOMPUTE (one trajectory
// per thread) and GS_ADJ_PAIRS (two per thread, packed float32x2) besides AUTO.
int f32_schedule(int precision, const char* what, bool pairs_ok = false) {
  const int s = precision & GS_SCHED_MASK;
  if (s != GS_SCHED_AUTO && s != GS_SCHED_STATIC)
    return fail(GS_ERR_ARG, std::string(what) + ": the float32 route runs one thread per "
                                                "trajectory (GS_SCHED_STATIC or AUTO)");
  const int v = precision & GS_ADJ_MASK;
  if ((precision & GS_LANES_MASK) || v == GS_ADJ_STAGES ||
      (v != GS_ADJ_AUTO && !pairs_ok))
    return fail(GS_ERR_ARG, std::string(what) + ": lanes and this reverse-pass variant are "
                                                "not float32-route options");
  return GS_OK;
}

template <class F>
constexpr bool kF32Built = F::D <= 8;

int f32_refuse_dim() {
  return fail(GS_ERR_PRECISION, "the float32 route is built for fields of at most 8 components");
}

template <class F, int kMethod>
int launch_f32_record(const gs::RecordArgs& a, cudaStream_t s) {
  if constexpr (!kF32Built<F>) {
    (void)a; (void)s;
    return f32_refuse_dim();
  } else {
    gs::RecordArgs b = a;
    b.ctrlf = gs::make_ctrl_consts_f32(F::D, kMethod == 0 ? 10 : 6);  // err^(-1/q) = m^(-1/2q)
    if (!b.rec && !b.ckpt)
      gs::f32_record_kernel<F, kMethod, false><<<grid_for(b.n), kBlock, 0, s>>>(b);
    else
      gs::f32_record_kernel<F, kMethod, true><<<grid_for(b.n), kBlock, 0, s>>>(b);
    return cuda_check("f32_record_kernel");
  }
}
template <class F, int kMethod>
int launch_f32_replay(const gs::ReplayArgs& a, cudaStream_t s) {
  if constexpr (!kF32Built<F>) {
    (void)a; (void)s;
    return f32_refuse_dim();
  } else {
    gs::f32_replay_kernel<F, kMethod><<<grid_for(a.n), kBlock, 0, s>>>(a);
    return cuda_check("f32_replay_kernel");
  }
}
template <class F, int kMethod>
int launch_f32_adjoint(const gs::AdjointArgs& a, cudaStream_t s) {
  if constexpr (!kF32Built<F>) {
    (void)a; (void)s;
    return f32_refuse_dim();
  } else {
    // K states of D floats per thread, counted in doubles for the occupancy helpers
    SegCfg c;
    int rc = occupancy_cfg(gs::f32_adjoint_kernel<F, kMethod>, (a.ck_every * F::D + 1) / 2, &c);
    if (rc) return rc;
    gs::f32_adjoint_kernel<F, kMethod><<<grid_for_block(a.n, c.block), c.block, c.smem, s>>>(a);
    return cuda_check("f32_adjoint_kernel");
  }
}
template <class F>
int launch_f32_tsit5_record(const gs::RecordArgs& a, cudaStream_t s) {
  return launch_f32_record<F, 0>(a, s);
}
template <class F>
int launch_f32_ros23_record(const gs::RecordArgs& a, cudaStream_t s) {
  return launch_f32_record<F, 1>(a, s);
}
template <class F>
int launch_f32_tsit5_replay(const gs::ReplayArgs& a, cudaStream_t s) {
  return launch_f32_replay<F, 0>(a, s);
}
template <class F>
int launch_f32_ros23_replay(const gs::ReplayArgs& a, cudaStream_t s) {
  return launch_f32_replay<F, 1>(a, s);
}
// variant AUTO: two trajectories per thread where the field is built for it (gs::Packable),
// else one; GS_ADJ_RECOMPUTE: one; GS_ADJ_PAIRS: two, refused for other fields.
template <class F>
int launch_f32_tsit5_adjoint(const gs::AdjointArgs& a, cudaStream_t s, int variant) {
  if constexpr (!kF32Built<F> || !gs::Packable<F>::value) {
    if (variant == GS_ADJ_PAIRS)
      return fail(GS_ERR_ARG, "gs_tsit5_adjoint: GS_ADJ_PAIRS is built for the built-in "
                              "nonstiff fields only");
    return launch_f32_adjoint<F, 0>(a, s);
  } else {
    if (variant == GS_ADJ_RECOMPUTE) return launch_f32_adjoint<F, 0>(a, s);
    // K states of D float pairs (8 bytes each) per thread, counted in doubles
    SegCfg c;
    int rc = occupancy_cfg(gs::f32_adjoint_pairs_kernel<F>, a.ck_every * F::D, &c);
    if (rc) return rc;
    const long long threads = (a.n + 1) / 2;
    gs::f32_adjoint_pairs_kernel<F><<<grid_for_block(threads, c.block), c.block, c.smem, s>>>(a);
    return cuda_check("f32_adjoint_pairs_kernel");
  }
}
template <class F>
int launch_f32_ros23_adjoint(const gs::AdjointArgs& a, cudaStream_t s) {
  return launch_f32_adjoint<F, 1>(a, s);
}

__global__ void device_tableau_kernel(double* out) {
  using T = gs::Tsit5;
  using C = gs::Ctrl;
  using R = gs::Ros23;
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const double v[41] = {T::C2,  T::C3,  T::C4,  T::C5,  T::A21, T::A31, T::A32, T::A41, T::A42,
                        T::A43, T::A51, T::A52, T::A53, T::A54, T::A61, T::A62, T::A63, T::A64,
                        T::A65, T::B1,  T::B2,  T::B3,  T::B4,  T::B5,  T::B6,  T::B7,  T::E1,
                        T::E2,  T::E3,  T::E4,  T::E5,  T::E6,  T::E7,  C::SAFETY, C::ERR_FLOOR,
                        C::FAC_MIN, C::FAC_MAX, T::ORDER_EXP, R::D, R::E32, R::ORDER_EXP};
  for (int i = 0; i < 41; ++i) out[i] = v[i];
}

// One warp per trajectory: the lanes scan the padded row together (consecutive lanes read
// consecutive dts, so each pass over a row is one coalesced 256-byte read), agree on the
// last non-zero step with a warp maximum, then write the row's 4-step sectors, lane c taking
// sector c (32 contiguous bytes read, one whole 32-byte sector written).  The caller has
// checked S <= the record's capacity.
constexpr unsigned kRowsPerBlock = kBlock / 32;

__global__ void record_from_padded_kernel(long long n, long long S, const double* dts,
                                          long long ld, double* rec, int* n_steps) {
  const long long j = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= n) return;  // uniform across the warp: blockDim is a multiple of 32
  const double* row = dts + j * ld;
  long long last = 0;
  for (long long s = lane; s < S; s += 32)
    if (row[s] != 0.0) last = s + 1;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const long long v = __shfl_xor_sync(0xffffffffu, last, o);
    last = v > last ? v : last;
  }
  const long long nch = (last + 3) / 4;
  for (long long c = lane; c < nch; c += 32) {
    double v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long s = c * 4 + q;
      v[q] = s < last ? row[s] : 0.0;
    }
    gs::store_rec_chunk(rec, n, j, (int)c, v[0], v[1], v[2], v[3]);
  }
  if (lane == 0) n_steps[j] = (int)last;
}

unsigned grid_rows(long long n) { return (unsigned)((n + kRowsPerBlock - 1) / kRowsPerBlock); }

__global__ void record_to_padded_kernel(long long n, const double* rec, const int* n_acc,
                                        long long S, double* dts) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * S) return;
  const long long j = idx / S, s = idx % S;
  dts[idx] = s < n_acc[j] ? rec[gs::rec_index(j, s, n)] : 0.0;
}

// Rows of `width` elements of T: gather dst[r] = src[idx[r]] or scatter dst[idx[r]] = src[r].
// One thread per element, so the plain side is read or written contiguously and the indexed
// side a row at a time.  Indices outside [0, src_rows) (gather) or [0, dst_rows) (scatter) are
// skipped and counted in *bad (the host turns a count into an error).
template <class T, bool kScatter>
__global__ void move_rows_kernel(const T* src, const long long* idx, long long rows, int width,
                                 long long limit, T* dst, unsigned long long* bad) {
  const long long total = rows * (long long)width;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / width, c = i - r * width;
    const long long k = idx[r];
    if (k < 0 || k >= limit) {
      if (c == 0) atomicAdd(bad, 1ull);
      continue;
    }
    if (kScatter)
      dst[k * width + c] = src[i];
    else
      dst[i] = src[k * width + c];
  }
}

int check_record_args(const char* who, long long n, const double* y0, const double* p,
                      double rtol, double atol, int max_steps, int cap, int ckpt_every,
                      const double* rec, const double* ckpt, const double* yf, const int* n_acc,
                      const int* n_rej, const int* status) {
  const std::string w(who);
  if (n < 0) return fail(GS_ERR_ARG, w + ": n < 0");
  if (n == 0) return GS_OK;  // empty ensemble: nothing is read or written
  if (!y0 || !p || !yf || !n_acc || !n_rej || !status)
    return fail(GS_ERR_ARG, w + ": y0, p, y_final, n_acc, n_rej and status are required");
  if (!aligned8(y0) || !aligned8(p) || !aligned8(yf))
    return fail(GS_ERR_ARG, w + ": float64 arrays must be 8-byte aligned");
  if (!(rtol >= 0.0) || !(atol >= 0.0)) return fail(GS_ERR_ARG, w + ": rtol/atol must be >= 0");
  if (max_steps < 0) return fail(GS_ERR_ARG, w + ": max_steps < 0");
  if ((rec || ckpt) && cap < 1) return fail(GS_ERR_ARG, w + ": cap must be >= 1 with a record");
  if (rec && !aligned16(rec)) return fail(GS_ERR_ARG, w + ": rec must be 16-byte aligned");
  if (ckpt) {
    if (!aligned16(ckpt)) return fail(GS_ERR_ARG, w + ": ckpt must be 16-byte aligned");
    if (ckpt_every < 1 || ckpt_every > gs::KMAX)
      return fail(GS_ERR_ARG, w + ": ckpt_every must be in [1, " + std::to_string(gs::KMAX) + "]");
  }
  return GS_OK;
}

int check_adjoint_args(const char* who, long long n, const double* p, const double* rec,
                       const int* n_acc, int cap, const double* ckpt, int ckpt_every,
                       const double* ybar) {
  const std::string w(who);
  if (n < 0) return fail(GS_ERR_ARG, w + ": n < 0");
  if (n == 0) return GS_OK;
  if (!p || !rec || !n_acc || !ckpt || !ybar)
    return fail(GS_ERR_ARG, w + ": p, rec, n_acc, ckpt and ybar are required");
  if (cap < 1) return fail(GS_ERR_ARG, w + ": cap must be >= 1");
  if (!aligned16(rec) || !aligned16(ckpt))
    return fail(GS_ERR_ARG, w + ": rec and ckpt must be 16-byte aligned");
  if (ckpt_every < 1 || ckpt_every > gs::KMAX)
    return fail(GS_ERR_ARG, w + ": ckpt_every must be in [1, " + std::to_string(gs::KMAX) + "]");
  return GS_OK;
}

}  // namespace

extern "C" {

int gs_version(void) { return 100; }

unsigned long long gs_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char* gs_last_error(void) { return g_err.c_str(); }

int gs_field_dims(int field, int* D, int* P) {
  if (!D || !P) return fail(GS_ERR_ARG, "gs_field_dims: null output");
  return field_dims(field, D, P);
}

int gs_tableau(double* out, int len) {
  using T = gs::Tsit5;
  using C = gs::Ctrl;
  using R = gs::Ros23;
  if (!out || len < 41) return fail(GS_ERR_ARG, "gs_tableau: need 41 doubles");
  const double v[41] = {T::C2,  T::C3,  T::C4,  T::C5,  T::A21, T::A31, T::A32, T::A41, T::A42,
                        T::A43, T::A51, T::A52, T::A53, T::A54, T::A61, T::A62, T::A63, T::A64,
                        T::A65, T::B1,  T::B2,  T::B3,  T::B4,  T::B5,  T::B6,  T::B7,  T::E1,
                        T::E2,  T::E3,  T::E4,  T::E5,  T::E6,  T::E7,  C::SAFETY, C::ERR_FLOOR,
                        C::FAC_MIN, C::FAC_MAX, T::ORDER_EXP, R::D, R::E32, R::ORDER_EXP};
  for (int i = 0; i < 41; ++i) out[i] = v[i];
  return GS_OK;
}

int gs_device_tableau(double* out_dev, void* stream) {
  if (!out_dev) return fail(GS_ERR_ARG, "gs_device_tableau: null output");
  device_tableau_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(out_dev);
  return cuda_check("device_tableau_kernel");
}

size_t gs_record_bytes(long long n, int cap) {
  if (n <= 0 || cap <= 0) return 0;
  return (size_t)((cap + 3) / 4) * (size_t)n * 4u * sizeof(double);
}

int gs_ckpt_slots(int cap, int ckpt_every) {
  if (cap <= 0 || ckpt_every <= 0) return 0;
  return (cap + ckpt_every - 1) / ckpt_every + 1;
}

size_t gs_ckpt_bytes(int field, long long n, int cap, int ckpt_every) {
  int D, P;
  if (field_dims(field, &D, &P) != GS_OK || n <= 0) return 0;
  return (size_t)gs_ckpt_slots(cap, ckpt_every) * (size_t)n * (size_t)gs::ckpt_width(D) *
             sizeof(double) +
         gs::kCtrlBytes;  // control block of the persistent kernels (work counters)
}

size_t gs_record_bytes_prec(int precision, long long n, int cap) {
  if ((precision & GS_PREC_MASK) != GS_PREC_F32) return gs_record_bytes(n, cap);
  if (n <= 0 || cap <= 0) return 0;
  return (size_t)((cap + 3) / 4) * (size_t)n * 4u * sizeof(float);
}

size_t gs_ckpt_bytes_prec(int field, int precision, long long n, int cap, int ckpt_every) {
  if ((precision & GS_PREC_MASK) != GS_PREC_F32) return gs_ckpt_bytes(field, n, cap, ckpt_every);
  int D, P;
  if (field_dims(field, &D, &P) != GS_OK || n <= 0) return 0;
  return (size_t)gs_ckpt_slots(cap, ckpt_every) * (size_t)n * (size_t)gs::ckpt_width_f32(D) *
             sizeof(float) +
         gs::kCtrlBytes;
}

int gs_max_ckpt_every(void) { return gs::KMAX; }

int gs_tsit5_fwd_record(int field, int precision, long long n, const double* y0,
                        const double* p, double t0, const double* t1v, double t1, double rtol,
                        double atol, double dt0, int max_steps, int cap, int ckpt_every,
                        double* rec, double* ckpt, double* y_final, int* n_acc, int* n_rej,
                        int* status, void* stream) {
  const int prec = precision & GS_PREC_MASK;
  if (prec != GS_PREC_F64 && prec != GS_PREC_MIXED && prec != GS_PREC_F32)
    return fail(GS_ERR_PRECISION, "gs_tsit5_fwd_record: unknown precision mode " + std::to_string(prec));
  int rc = check_record_args("gs_tsit5_fwd_record", n, y0, p, rtol, atol, max_steps, cap,
                             ckpt_every, rec, ckpt, y_final, n_acc, n_rej, status);
  if (rc) return rc;
  int D, P;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  gs::RecordArgs a{n, y0, p, t0, t1, rtol, atol, dt0, t1v, max_steps, cap, ckpt_every,
                   gs_ckpt_slots(cap, ckpt_every), rec, ckpt, y_final, n_acc, n_rej, status};
  if (prec == GS_PREC_F32) {
    if (precision & GS_OCC_MASK)
      return fail(GS_ERR_ARG, "GS_OCC applies to the float64 recording forward only");
    if ((rc = f32_schedule(precision, "gs_tsit5_fwd_record"))) return rc;
    GS_TSIT5_DISPATCH(field, launch_f32_tsit5_record, a, (cudaStream_t)stream)
  }
  GS_TSIT5_DISPATCH(field, launch_tsit5_record, a, (cudaStream_t)stream,
                    prec == GS_PREC_MIXED, forward_schedule(precision, t1v, ckpt), precision)
}

int gs_tsit5_replay(int field, int precision, long long n, const double* y0, const double* p,
                    double t0, const double* rec, const int* n_acc, int cap, int ckpt_every,
                    double* ckpt, double* y_final, void* stream) {
  const int prec = precision & ~GS_LANES_MASK;
  if (prec != GS_PREC_F64 && prec != GS_PREC_MIXED && precision != GS_PREC_F32)
    return fail(GS_ERR_PRECISION, "gs_tsit5_replay: unknown precision mode " + std::to_string(precision));
  if (n < 0) return fail(GS_ERR_ARG, "gs_tsit5_replay: n < 0");
  if (n == 0) return GS_OK;
  if (!y0 || !p || !rec || !n_acc || !y_final)
    return fail(GS_ERR_ARG, "gs_tsit5_replay: y0, p, rec, n_acc and y_final are required");
  if (cap < 1 || !aligned16(rec)) return fail(GS_ERR_ARG, "gs_tsit5_replay: bad record");
  if (ckpt && (!aligned16(ckpt) || ckpt_every < 1 || ckpt_every > gs::KMAX))
    return fail(GS_ERR_ARG, "gs_tsit5_replay: bad checkpoint buffer or interval");
  int D, P, rc;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  gs::ReplayArgs a{n, y0, p, t0, rec, n_acc, ckpt_every, gs_ckpt_slots(cap, ckpt_every), ckpt,
                   y_final, cap};
  if (precision == GS_PREC_F32) {
    GS_TSIT5_DISPATCH(field, launch_f32_tsit5_replay, a, (cudaStream_t)stream)
  }
  GS_TSIT5_DISPATCH(field, launch_tsit5_replay, a, (cudaStream_t)stream,
                    prec == GS_PREC_MIXED, precision)
}

static int tsit5_adjoint_impl(int field, int precision, long long n, const double* p,
                              const double* rec, const int* n_acc, int cap, const double* ckpt,
                              int ckpt_every, const double* ybar, double* gy0, double* gp,
                              const long long* order, void* stream) {
  const int prec = precision & GS_PREC_MASK;
  if (prec != GS_PREC_F64 && prec != GS_PREC_MIXED && prec != GS_PREC_F32)
    return fail(GS_ERR_PRECISION, "gs_tsit5_adjoint: unknown precision mode " + std::to_string(prec));
  int rc = check_adjoint_args("gs_tsit5_adjoint", n, p, rec, n_acc, cap, ckpt, ckpt_every, ybar);
  if (rc) return rc;
  int D, P;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  gs::AdjointArgs a{n, p, rec, n_acc, ckpt, ckpt_every, ybar, gy0, gp, cap, order};
  if (prec == GS_PREC_F32) {
    if (precision & GS_OCC_MASK)
      return fail(GS_ERR_ARG, "GS_OCC applies to the float64 reverse pass only");
    if ((rc = f32_schedule(precision, "gs_tsit5_adjoint", true))) return rc;
    GS_TSIT5_DISPATCH(field, launch_f32_tsit5_adjoint, a, (cudaStream_t)stream,
                      precision & GS_ADJ_MASK)
  }
  GS_TSIT5_DISPATCH(field, launch_tsit5_adjoint, a, cap, (cudaStream_t)stream,
                    prec == GS_PREC_MIXED, adjoint_schedule(precision), precision & GS_ADJ_MASK,
                    precision)
}

int gs_tsit5_adjoint(int field, int precision, long long n, const double* p, const double* rec,
                     const int* n_acc, int cap, const double* ckpt, int ckpt_every,
                     const double* ybar, double* gy0, double* gp, void* stream) {
  return tsit5_adjoint_impl(field, precision, n, p, rec, n_acc, cap, ckpt, ckpt_every, ybar,
                            gy0, gp, nullptr, stream);
}

int gs_lane_choices(int field, int* out, int cap) {
  int D, P, rc;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (!out && cap > 0) return fail(GS_ERR_ARG, "gs_lane_choices: null output");
  GS_TSIT5_DISPATCH(field, lane_choices, out, cap)
}

int gs_occ_choices(int field, int pass, int* out, int cap) {
  int D, P, rc;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (!out && cap > 0) return fail(GS_ERR_ARG, "gs_occ_choices: null output");
  if (pass == GS_OCC_ROS23_FORWARD || pass == GS_OCC_ROS23_REVERSE) {
    GS_ROS23_DISPATCH(field, occ_choices, pass, out, cap)
  }
  if (pass != GS_OCC_FORWARD && pass != GS_OCC_REVERSE && pass != GS_OCC_MIXED_REVERSE)
    return fail(GS_ERR_ARG, "gs_occ_choices: unknown pass " + std::to_string(pass));
  GS_TSIT5_DISPATCH(field, occ_choices, pass, out, cap)
}

int gs_ros23_fwd_record(int field, int precision, long long n, const double* y0,
                        const double* p, double t0, const double* t1v, double t1, double rtol,
                        double atol, double dt0, int max_steps, int cap, int ckpt_every,
                        double* rec, double* ckpt, double* y_final, int* n_acc, int* n_rej,
                        int* status, void* stream) {
  const int prec = precision & GS_PREC_MASK;
  if (prec != GS_PREC_F64 && prec != GS_PREC_F32)
    return fail(GS_ERR_PRECISION, "gs_ros23_fwd_record: Rosenbrock23 runs in float64 or float32");
  if ((precision & GS_OCC_MASK) && prec != GS_PREC_F64)
    return fail(GS_ERR_ARG, "GS_OCC applies to the float64 recording forward only");
  int rc = check_record_args("gs_ros23_fwd_record", n, y0, p, rtol, atol, max_steps, cap,
                             ckpt_every, rec, ckpt, y_final, n_acc, n_rej, status);
  if (rc) return rc;
  int D, P;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  gs::RecordArgs a{n, y0, p, t0, t1, rtol, atol, dt0, t1v, max_steps, cap, ckpt_every,
                   gs_ckpt_slots(cap, ckpt_every), rec, ckpt, y_final, n_acc, n_rej, status};
  if (prec == GS_PREC_F32) {
    if ((rc = f32_schedule(precision, "gs_ros23_fwd_record"))) return rc;
    GS_ROS23_DISPATCH(field, launch_f32_ros23_record, a, (cudaStream_t)stream)
  }
  GS_ROS23_DISPATCH(field, launch_ros23_record, a, (cudaStream_t)stream,
                    forward_schedule(precision, t1v, ckpt),
                    (precision & GS_OCC_MASK) >> GS_OCC_SHIFT)
}

int gs_ros23_replay(int field, int precision, long long n, const double* y0, const double* p,
                    double t0, const double* rec, const int* n_acc, int cap, int ckpt_every,
                    double* ckpt, double* y_final, void* stream) {
  if (precision != GS_PREC_F64 && precision != GS_PREC_F32)
    return fail(GS_ERR_PRECISION, "gs_ros23_replay: precision mode not built");
  if (n < 0) return fail(GS_ERR_ARG, "gs_ros23_replay: n < 0");
  if (n == 0) return GS_OK;
  if (!y0 || !p || !rec || !n_acc || !y_final)
    return fail(GS_ERR_ARG, "gs_ros23_replay: y0, p, rec, n_acc and y_final are required");
  if (cap < 1 || !aligned16(rec)) return fail(GS_ERR_ARG, "gs_ros23_replay: bad record");
  if (ckpt && (!aligned16(ckpt) || ckpt_every < 1 || ckpt_every > gs::KMAX))
    return fail(GS_ERR_ARG, "gs_ros23_replay: bad checkpoint buffer or interval");
  int D, P, rc;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  gs::ReplayArgs a{n, y0, p, t0, rec, n_acc, ckpt_every, gs_ckpt_slots(cap, ckpt_every), ckpt,
                   y_final, cap};
  if (precision == GS_PREC_F32) {
    GS_ROS23_DISPATCH(field, launch_f32_ros23_replay, a, (cudaStream_t)stream)
  }
  GS_ROS23_DISPATCH(field, launch_ros23_replay, a, (cudaStream_t)stream)
}

static int ros23_adjoint_impl(int field, int precision, long long n, const double* p,
                              const double* rec, const int* n_acc, int cap, const double* ckpt,
                              int ckpt_every, const double* ybar, double* gy0, double* gp,
                              const long long* order, void* stream) {
  const int prec = precision & GS_PREC_MASK;
  if (prec != GS_PREC_F64 && prec != GS_PREC_F32)
    return fail(GS_ERR_PRECISION, "gs_ros23_adjoint: Rosenbrock23 runs in float64 or float32");
  if ((precision & GS_OCC_MASK) && prec != GS_PREC_F64)
    return fail(GS_ERR_ARG, "GS_OCC applies to the float64 reverse pass only");
  int rc = check_adjoint_args("gs_ros23_adjoint", n, p, rec, n_acc, cap, ckpt, ckpt_every, ybar);
  if (rc) return rc;
  int D, P;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  gs::AdjointArgs a{n, p, rec, n_acc, ckpt, ckpt_every, ybar, gy0, gp, cap, order};
  if (prec == GS_PREC_F32) {
    if ((rc = f32_schedule(precision, "gs_ros23_adjoint"))) return rc;
    GS_ROS23_DISPATCH(field, launch_f32_ros23_adjoint, a, (cudaStream_t)stream)
  }
  GS_ROS23_DISPATCH(field, launch_ros23_adjoint, a, cap, (cudaStream_t)stream,
                    adjoint_schedule(precision), (precision & GS_OCC_MASK) >> GS_OCC_SHIFT)
}

int gs_ros23_adjoint(int field, int precision, long long n, const double* p, const double* rec,
                     const int* n_acc, int cap, const double* ckpt, int ckpt_every,
                     const double* ybar, double* gy0, double* gp, void* stream) {
  return ros23_adjoint_impl(field, precision, n, p, rec, n_acc, cap, ckpt, ckpt_every, ybar, gy0,
                            gp, nullptr, stream);
}

int gs_adjoint_ordered(int method, int field, int precision, long long n, const double* p,
                       const double* rec, const int* n_acc, int cap, const double* ckpt,
                       int ckpt_every, const double* ybar, double* gy0, double* gp,
                       const long long* order, void* stream) {
  if (!order || !aligned8(order))
    return fail(GS_ERR_ARG, "gs_adjoint_ordered: order must be an 8-byte aligned device array");
  if (adjoint_schedule(precision) != GS_SCHED_STATIC)
    return fail(GS_ERR_ARG, "gs_adjoint_ordered: the lane order applies to one thread per "
                            "trajectory (GS_SCHED_STATIC or AUTO); persistent lanes balance "
                            "themselves");
  if (method == GS_METHOD_TSIT5)
    return tsit5_adjoint_impl(field, precision, n, p, rec, n_acc, cap, ckpt, ckpt_every, ybar,
                              gy0, gp, order, stream);
  if (method == GS_METHOD_ROS23)
    return ros23_adjoint_impl(field, precision, n, p, rec, n_acc, cap, ckpt, ckpt_every, ybar,
                              gy0, gp, order, stream);
  return fail(GS_ERR_ARG, "gs_adjoint_ordered: unknown method " + std::to_string(method));
}

int gs_record_from_padded(long long n, long long S, const double* dts, long long ld,
                          double* rec, int cap, int* n_steps, void* stream) {
  if (n < 0 || S < 0 || ld < S) return fail(GS_ERR_ARG, "gs_record_from_padded: bad sizes");
  if (S > cap) return fail(GS_ERR_ARG, "gs_record_from_padded: S exceeds the record capacity");
  if (!rec || !n_steps || (S > 0 && !dts))
    return fail(GS_ERR_ARG, "gs_record_from_padded: null buffer");
  if (!aligned16(rec)) return fail(GS_ERR_ARG, "gs_record_from_padded: rec must be 16-byte aligned");
  if (n == 0) return GS_OK;
  record_from_padded_kernel<<<grid_rows(n), kBlock, 0, (cudaStream_t)stream>>>(n, S, dts, ld, rec,
                                                                                n_steps);
  return cuda_check("record_from_padded_kernel");
}

int gs_move_rows(int scatter, int elem_bytes, const void* src, const long long* idx,
                 long long rows, int width, long long limit, void* dst,
                 unsigned long long* bad, void* stream) {
  if (rows < 0 || width < 1 || limit < 0 || (elem_bytes != 4 && elem_bytes != 8))
    return fail(GS_ERR_ARG, "gs_move_rows: bad sizes");
  if (rows == 0) return GS_OK;
  if (!src || !idx || !dst || !bad) return fail(GS_ERR_ARG, "gs_move_rows: null buffer");
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess)
    return fail(GS_ERR_CUDA, std::string("CUDA: device query: ") + cudaGetErrorString(e));
  const long long total = rows * (long long)width;
  const long long want = (total + 255) / 256, cap = 8LL * sms;  // a few waves of 256-thread blocks
  const unsigned grid = (unsigned)(want < cap ? want : cap);
  const cudaStream_t s = (cudaStream_t)stream;
  if (elem_bytes == 8) {
    if (scatter)
      move_rows_kernel<unsigned long long, true><<<grid, 256, 0, s>>>(
          (const unsigned long long*)src, idx, rows, width, limit, (unsigned long long*)dst, bad);
    else
      move_rows_kernel<unsigned long long, false><<<grid, 256, 0, s>>>(
          (const unsigned long long*)src, idx, rows, width, limit, (unsigned long long*)dst, bad);
  } else {
    if (scatter)
      move_rows_kernel<unsigned, true><<<grid, 256, 0, s>>>((const unsigned*)src, idx, rows,
                                                           width, limit, (unsigned*)dst, bad);
    else
      move_rows_kernel<unsigned, false><<<grid, 256, 0, s>>>((const unsigned*)src, idx, rows,
                                                            width, limit, (unsigned*)dst, bad);
  }
  return cuda_check("move_rows_kernel");
}

int gs_record_to_padded(long long n, int cap, const double* rec, const int* n_acc, long long S,
                        double* dts, void* stream) {
  if (n < 0 || S < 0 || S > cap) return fail(GS_ERR_ARG, "gs_record_to_padded: bad sizes");
  if (!rec || !n_acc || (n * S > 0 && !dts)) return fail(GS_ERR_ARG, "gs_record_to_padded: null buffer");
  if (n == 0 || S == 0) return GS_OK;
  const long long total = n * S;
  record_to_padded_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      n, rec, n_acc, S, dts);
  return cuda_check("record_to_padded_kernel");
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Replay gradient without device allocation (gs_tsit5_vjp_static).
//
// Some callers cannot call cudaMalloc: a custom call running inside JAX/XLA, where XLA has
// already reserved most of the device memory for its own pool and owns the rest, and
// latency-critical callers for which the device-wide synchronisation of cudaMalloc and
// cudaFree is not acceptable.  This entry point gives them the replay gradient of
// gs_tsit5_replay + gs_tsit5_adjoint using a scratch array that lives in the library
// itself: the dt record, the checkpoints and the per-trajectory step counts are placed in
// g_vjp_scratch, a file-scope __device__ array of GS_STATIC_SCRATCH_BYTES bytes that every
// GPU which loads the library holds until the process exits.
//
// The array's name is only a host-side stand-in in host code, so its device address is
// looked up with cudaGetSymbolAddress, once per device, by the first call made on that
// device (with that device current); that first call should therefore come before any
// stream capture.  Every call shares the one array and it keeps the contents of the last
// call; nothing in it has to start at zero, because every region a call reads is written
// earlier in the same call.  Calls that overlap on the GPU (on different streams of the
// same device) race on the array and must be serialised by the caller.  The looked-up
// address is kept for the life of the process: resetting a device (cudaDeviceReset) after
// the first call on it is not supported, since the array may move when the module reloads.
//
// Only libgsolve.so carries the array.  A generated field's library (compiled from this file
// with GS_USER_FIELD_HEADER) exports the entry point as a stub that returns GS_ERR_FIELD, so
// registering N fields does not hold N more arrays on every device.
// ---------------------------------------------------------------------------------------
#ifndef GS_USER_FIELD_HEADER
namespace {

__device__ __align__(256) unsigned char g_vjp_scratch[GS_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::atomic<void*> g_vjp_scratch_addr[kMaxDevices];

int vjp_scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return fail(GS_ERR_CUDA, std::string("CUDA: cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(GS_ERR_ARG, "gs_tsit5_vjp_static: device ordinal " + std::to_string(dev) +
                                " is beyond the supported " + std::to_string(kMaxDevices));
  void* p = g_vjp_scratch_addr[dev].load(std::memory_order_acquire);
  if (!p) {
    e = cudaGetSymbolAddress(&p, g_vjp_scratch);
    if (e != cudaSuccess)
      return fail(GS_ERR_CUDA, std::string("CUDA: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_vjp_scratch_addr[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return GS_OK;
}

size_t round256(size_t b) { return (b + 255u) & ~size_t(255); }

template <class F>
int launch_tsit5_vjp_static(long long n, long long S, long long ld, const double* y0,
                            const double* p, double t0, const double* dts, const double* ybar,
                            double* y_final, double* gy0, double* gp, unsigned char* base,
                            int cap, int K, size_t off_rec, size_t off_ckpt, cudaStream_t s) {
  if constexpr (kCoop<F>) {
    return coop_refuse<F>("gs_tsit5_vjp_static");
  } else {
  int* n_steps = reinterpret_cast<int*>(base);
  double* rec = reinterpret_cast<double*>(base + off_rec);
  double* ckpt = reinterpret_cast<double*>(base + off_ckpt);
  record_from_padded_kernel<<<grid_rows(n), kBlock, 0, s>>>(n, S, dts, ld, rec, n_steps);
  int rc = cuda_check("record_from_padded_kernel");
  if (rc) return rc;
  gs::ReplayArgs ra{n, y0, p, t0, rec, n_steps, K, gs_ckpt_slots(cap, K), ckpt, y_final, cap};
  gs::tsit5_replay_kernel<F><<<grid_for(n), kBlock, 0, s>>>(ra);
  if ((rc = cuda_check("tsit5_replay_kernel"))) return rc;
  gs::AdjointArgs aa{n, p, rec, n_steps, ckpt, K, ybar, gy0, gp, cap};
  // the reverse pass gs_tsit5_adjoint would run (stage-keeping or recomputing by residency,
  // the unrolled K = 2 instance where it applies)
  return launch_tsit5_adjoint<F>(aa, cap, s, false, GS_SCHED_STATIC, GS_ADJ_AUTO, GS_PREC_F64);
  }
}

}  // namespace

extern "C" int gs_tsit5_vjp_static(int field, long long n, const double* y0, const double* p,
                                   double t0, const double* dts, long long S, long long ld,
                                   const double* ybar, double* y_final, double* gy0,
                                   double* gp, void* stream) {
  if (n < 0 || S < 0 || ld < S) return fail(GS_ERR_ARG, "gs_tsit5_vjp_static: bad sizes");
  int D, P, rc;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  if (!y0 || !p || !ybar || !y_final || (S > 0 && !dts))
    return fail(GS_ERR_ARG, "gs_tsit5_vjp_static: y0, p, dts, ybar and y_final are required");
  if (!aligned8(y0) || !aligned8(p) || !aligned8(ybar) || !aligned8(y_final) ||
      (dts && !aligned8(dts)))
    return fail(GS_ERR_ARG, "gs_tsit5_vjp_static: float64 arrays must be 8-byte aligned");
  // refuse before any size product is formed, so none of them can wrap: the step counts
  // alone take 4 bytes per trajectory and the record 8 bytes per step slot
  constexpr long long kScratch = (long long)GS_STATIC_SCRATCH_BYTES;
  if (n > kScratch / 4 || S > kScratch / 8 || n * (S > 0 ? S : 1) > kScratch / 8)
    return fail(GS_ERR_ARG, "gs_tsit5_vjp_static: n=" + std::to_string(n) + ", S=" +
                                std::to_string(S) + " does not fit: the static scratch holds " +
                                std::to_string((size_t)GS_STATIC_SCRATCH_BYTES) +
                                " bytes (use gs_tsit5_replay + gs_tsit5_adjoint with "
                                "caller-allocated buffers for larger ensembles)");
  const int cap = S > 0 ? (int)S : 1;
  // the shortest segments that fit: K = 2 where it can (the interval the autotuner picks
  // for the built-in fields), longer ones as the checkpoints outgrow the scratch
  const size_t b_steps = round256((size_t)n * sizeof(int));
  const size_t b_rec = round256(gs_record_bytes(n, cap));
  int K = cap > 1 ? 2 : 1;
  size_t need = b_steps + b_rec + round256(gs_ckpt_bytes(field, n, cap, K));
  while (need > (size_t)GS_STATIC_SCRATCH_BYTES && K < gs::KMAX && K < cap) {
    ++K;
    need = b_steps + b_rec + round256(gs_ckpt_bytes(field, n, cap, K));
  }
  if (need > (size_t)GS_STATIC_SCRATCH_BYTES)
    return fail(GS_ERR_ARG, "gs_tsit5_vjp_static: n=" + std::to_string(n) + ", S=" +
                                std::to_string(S) + " needs " + std::to_string(need) +
                                " bytes of scratch; the static scratch holds " +
                                std::to_string((size_t)GS_STATIC_SCRATCH_BYTES) +
                                " bytes (use gs_tsit5_replay + gs_tsit5_adjoint with "
                                "caller-allocated buffers for larger ensembles)");
  void* base = nullptr;
  if ((rc = vjp_scratch_address(&base))) return rc;
  GS_TSIT5_DISPATCH(field, launch_tsit5_vjp_static, n, S, ld, y0, p, t0, dts, ybar, y_final,
                    gy0, gp, static_cast<unsigned char*>(base), cap, K, b_steps,
                    b_steps + b_rec, (cudaStream_t)stream)
}
#else   // a generated field's library: no static array, the entry point refuses
extern "C" int gs_tsit5_vjp_static(int field, long long, const double*, const double*, double,
                                   const double*, long long, long long, const double*, double*,
                                   double*, double*, void*) {
  return fail(GS_ERR_FIELD, "gs_tsit5_vjp_static: field " + std::to_string(field) +
                                " is a generated field; the static-scratch entry point is "
                                "served by libgsolve.so for its built-in fields only");
}
#endif  // GS_USER_FIELD_HEADER

// ---------------------------------------------------------------------------------------
// Dense output (saveat) on the replay, and its adjoint (gs_saveat.cuh).
// ---------------------------------------------------------------------------------------
namespace {

template <class F, class M>
int launch_saveat(const gs::SaveatArgs& a, cudaStream_t s, bool adjoint) {
  if (adjoint) {
    SegCfg c;
    int rc;
    if ((rc = occupancy_cfg(gs::adjoint_saveat_kernel<F, M>,
                            gs::adjoint_smem_doubles<F::D, F::D + 1>(a.ck_every), &c)))
      return rc;
    gs::adjoint_saveat_kernel<F, M><<<grid_for_block(a.n, c.block), c.block, c.smem, s>>>(a);
    return cuda_check("adjoint_saveat_kernel");
  }
  gs::replay_saveat_kernel<F, M><<<grid_for(a.n), kBlock, 0, s>>>(a);
  return cuda_check("replay_saveat_kernel");
}

// Persistent saveat reverse pass; the work counter sits in the control block after the
// checkpoint slots, like the other reverse passes'.
template <class F, class M>
int launch_adjoint_saveat_persistent(const gs::SaveatArgs& a, cudaStream_t s, bool use_counter) {
  const SegCfg c = seg_cfg_doubles(gs::adjoint_smem_doubles<F::D, F::D + 1>(a.ck_every));
  unsigned long long* counter =
      use_counter ? ctrl_counter(a.ckpt, a.n, a.ck_slots, F::D, gs::kCtrlAdj) : nullptr;
  unsigned grid = 0;
  int rc;
  if ((rc = allow_smem(gs::adjoint_saveat_persistent_kernel<F, M>, c.smem))) return rc;
  if ((rc = persistent_grid(gs::adjoint_saveat_persistent_kernel<F, M>, c.block, c.smem, a.n,
                            &grid)))
    return rc;
  if ((rc = zero_counter(counter, s))) return rc;
  gs::adjoint_saveat_persistent_kernel<F, M><<<grid, c.block, c.smem, s>>>(a, counter);
  return cuda_check("adjoint_saveat_persistent_kernel");
}

template <class F, class M>
int launch_saveat_sched(const gs::SaveatArgs& a, cudaStream_t s, bool adjoint, int sched) {
  if (adjoint && sched != GS_SCHED_STATIC)
    return launch_adjoint_saveat_persistent<F, M>(a, s, sched == GS_SCHED_REFILL);
  return launch_saveat<F, M>(a, s, adjoint);
}

template <class F>
int launch_saveat_tsit5(const gs::SaveatArgs& a, cudaStream_t s, bool adjoint, bool mixed,
                        int sched) {
  if constexpr (kCoop<F>) {
    return coop_refuse<F>("the dense output (saveat)");
  } else {
    return mixed ? launch_saveat_sched<F, gs::Tsit5MixedStep>(a, s, adjoint, sched)
                 : launch_saveat_sched<F, gs::Tsit5F64Step>(a, s, adjoint, sched);
  }
}

template <class F>
int launch_saveat_ros23(const gs::SaveatArgs& a, cudaStream_t s, bool adjoint, int sched) {
  return launch_saveat_sched<F, gs::Ros23Step>(a, s, adjoint, sched);
}

// precision carries GS_PREC_* and, for the reverse pass, GS_SCHED_* (AUTO = one thread per
// trajectory; REFILL / STRIDED = persistent lanes).  The forward replay runs one thread per
// trajectory.
// The float32 route's dense output: one thread per trajectory, fields of at most 8 components.
template <class F, int kMethod>
int launch_f32_saveat(const gs::SaveatArgs& a, cudaStream_t s, bool adjoint) {
  if constexpr (!kF32Built<F>) {
    (void)a; (void)s; (void)adjoint;
    return f32_refuse_dim();
  } else {
    if (!adjoint) {
      gs::f32_replay_saveat_kernel<F, kMethod><<<grid_for(a.n), kBlock, 0, s>>>(a);
      return cuda_check("f32_replay_saveat_kernel");
    }
    // K rows of D + 1 floats per thread, counted in doubles for the occupancy helpers
    SegCfg c;
    int rc = occupancy_cfg(gs::f32_adjoint_saveat_kernel<F, kMethod>,
                           (a.ck_every * (F::D + 1) + 1) / 2, &c);
    if (rc) return rc;
    gs::f32_adjoint_saveat_kernel<F, kMethod><<<grid_for_block(a.n, c.block), c.block, c.smem, s>>>(a);
    return cuda_check("f32_adjoint_saveat_kernel");
  }
}
template <class F>
int launch_f32_saveat_tsit5(const gs::SaveatArgs& a, cudaStream_t s, bool adjoint) {
  return launch_f32_saveat<F, 0>(a, s, adjoint);
}
template <class F>
int launch_f32_saveat_ros23(const gs::SaveatArgs& a, cudaStream_t s, bool adjoint) {
  return launch_f32_saveat<F, 1>(a, s, adjoint);
}

int saveat_dispatch(int method, int field, int precision, const gs::SaveatArgs& a, void* stream,
                    bool adjoint) {
  const cudaStream_t s = (cudaStream_t)stream;
  const int prec = precision & GS_PREC_MASK;
  const int sched = adjoint ? adjoint_schedule(precision) : GS_SCHED_STATIC;
  if (prec == GS_PREC_F32) {
    int rc = f32_schedule(precision, adjoint ? "gs_adjoint_saveat" : "gs_replay_saveat");
    if (rc) return rc;
    if (method == GS_METHOD_TSIT5) {
      GS_TSIT5_DISPATCH(field, launch_f32_saveat_tsit5, a, s, adjoint)
    }
    if (method == GS_METHOD_ROS23) {
      GS_ROS23_DISPATCH(field, launch_f32_saveat_ros23, a, s, adjoint)
    }
    return fail(GS_ERR_ARG, "saveat: unknown method " + std::to_string(method));
  }
  if (method == GS_METHOD_TSIT5) {
    if (prec != GS_PREC_F64 && prec != GS_PREC_MIXED)
      return fail(GS_ERR_PRECISION, "saveat: unknown precision mode " + std::to_string(prec));
    GS_TSIT5_DISPATCH(field, launch_saveat_tsit5, a, s, adjoint, prec == GS_PREC_MIXED, sched)
  }
  if (method == GS_METHOD_ROS23) {
    if (prec != GS_PREC_F64)
      return fail(GS_ERR_PRECISION, "saveat: Rosenbrock23 runs in float64 only");
    GS_ROS23_DISPATCH(field, launch_saveat_ros23, a, s, adjoint, sched)
  }
  return fail(GS_ERR_ARG, "saveat: unknown method " + std::to_string(method));
}

// Forward with record and dense output: one thread per trajectory (kStatic), or persistent
// lanes refilled from the work counter (kRefill) or strided (kStrided).
enum FwdLanes { kStatic, kRefill, kStrided };

template <class F, class L>
int launch_fwd_lanes(const gs::RecordArgs& a_in, cudaStream_t s, FwdLanes lanes) {
  if (lanes != kStatic) return launch_record_persistent<F, L>(a_in, s, lanes == kRefill);
  gs::RecordArgs a = a_in;
  a.ctrl = gs::make_ctrl_consts(F::D, L::QK);
  gs::record_static_kernel<F, L><<<grid_for(a.n), kBlock, 0, s>>>(a);
  return cuda_check("record_static_kernel");
}

template <class F>
int launch_fwd_saveat_tsit5(const gs::RecordArgs& a, cudaStream_t s, bool mixed, FwdLanes lanes) {
  if constexpr (kCoop<F>) {
    return coop_refuse<F>("the dense output (saveat)");
  } else {
    return mixed ? launch_fwd_lanes<F, gs::LaneTsit5Mixed<F>>(a, s, lanes)
                 : launch_fwd_lanes<F, gs::LaneTsit5F64<F>>(a, s, lanes);
  }
}

template <class F>
int launch_fwd_saveat_ros23(const gs::RecordArgs& a, cudaStream_t s, FwdLanes lanes) {
  return launch_fwd_lanes<F, gs::LaneRos23<F>>(a, s, lanes);
}

int check_saveat(const char* who, long long n, const double* p, const double* rec,
                 const int* n_acc, int cap, const double* ckpt, int ckpt_every,
                 const double* ts, long long ts_ld, int K) {
  const std::string w(who);
  if (n < 0 || K < 0 || ts_ld < 0) return fail(GS_ERR_ARG, w + ": bad sizes");
  if (n == 0) return GS_OK;
  if (!p || !rec || !n_acc || (K > 0 && !ts))
    return fail(GS_ERR_ARG, w + ": p, rec, n_acc and ts are required");
  if (ts_ld != 0 && ts_ld < K) return fail(GS_ERR_ARG, w + ": ts row stride < K");
  if (cap < 1 || !aligned16(rec)) return fail(GS_ERR_ARG, w + ": bad record");
  if (ckpt && (!aligned16(ckpt) || ckpt_every < 1 || ckpt_every > gs::KMAX))
    return fail(GS_ERR_ARG, w + ": bad checkpoint buffer or interval");
  return GS_OK;
}

}  // namespace

extern "C" int gs_replay_saveat(int method, int field, int precision, long long n,
                                const double* y0, const double* p, double t0, const double* rec,
                                const int* n_acc, int cap, int ckpt_every, double* ckpt,
                                const double* ts, long long ts_ld, int K, double* ys,
                                double* y_final, void* stream) {
  int rc = check_saveat("gs_replay_saveat", n, p, rec, n_acc, cap, ckpt, ckpt_every, ts, ts_ld, K);
  if (rc) return rc;
  int D, P;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  if (!y0 || !y_final || (K > 0 && !ys))
    return fail(GS_ERR_ARG, "gs_replay_saveat: y0, ys and y_final are required");
  gs::SaveatArgs a{n, y0, p, t0, rec, n_acc, ckpt_every, gs_ckpt_slots(cap, ckpt_every), ckpt,
                   ts, ts_ld, K, ys, y_final, nullptr, nullptr, nullptr, nullptr, cap};
  return saveat_dispatch(method, field, precision, a, stream, false);
}

extern "C" int gs_fwd_record_saveat(int method, int field, int precision, long long n,
                                    const double* y0, const double* p, double t0,
                                    const double* t1v, double t1, double rtol, double atol,
                                    double dt0, int max_steps, int cap, int ckpt_every,
                                    double* rec, double* ckpt, double* y_final, int* n_acc,
                                    int* n_rej, int* status, const double* ts, long long ts_ld,
                                    int K, double* ys, void* stream) {
  const char* who = "gs_fwd_record_saveat";
  int rc = check_record_args(who, n, y0, p, rtol, atol, max_steps, cap, ckpt_every, rec, ckpt,
                             y_final, n_acc, n_rej, status);
  if (rc) return rc;
  if (K < 0 || ts_ld < 0 || (ts_ld != 0 && ts_ld < K))
    return fail(GS_ERR_ARG, std::string(who) + ": bad saveat sizes");
  int D, P;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  if (K > 0 && (!ts || !ys)) return fail(GS_ERR_ARG, std::string(who) + ": ts and ys are required");
  const int prec = precision & GS_PREC_MASK;
  const int sched = precision & GS_SCHED_MASK;
  // AUTO: lanes refilled from a work counter for per-trajectory end times, else one thread per
  // trajectory; refill needs the counter in the checkpoint buffer's control block
  const bool want_refill =
      sched == GS_SCHED_REFILL || (sched == GS_SCHED_AUTO && t1v != nullptr);
  const FwdLanes lanes = (want_refill && ckpt != nullptr) ? kRefill
                         : (sched == GS_SCHED_STATIC || sched == GS_SCHED_AUTO) ? kStatic
                                                                                 : kStrided;
  gs::RecordArgs a{n, y0, p, t0, t1, rtol, atol, dt0, t1v, max_steps, cap, ckpt_every,
                   gs_ckpt_slots(cap, ckpt_every), rec, ckpt, y_final, n_acc, n_rej, status,
                   gs::CtrlConsts{}, ts, ts_ld, K, K > 0 ? ys : nullptr};
  const cudaStream_t s = (cudaStream_t)stream;
  if (prec == GS_PREC_F32)
    return fail(GS_ERR_PRECISION, std::string(who) + ": the float32 route records without dense "
                                                     "output; replay its record with "
                                                     "gs_replay_saveat");
  if (method == GS_METHOD_TSIT5) {
    if (prec != GS_PREC_F64 && prec != GS_PREC_MIXED)
      return fail(GS_ERR_PRECISION, std::string(who) + ": unknown precision mode " + std::to_string(prec));
    GS_TSIT5_DISPATCH(field, launch_fwd_saveat_tsit5, a, s, prec == GS_PREC_MIXED, lanes)
  }
  if (method == GS_METHOD_ROS23) {
    if (prec != GS_PREC_F64)
      return fail(GS_ERR_PRECISION, std::string(who) + ": Rosenbrock23 runs in float64 only");
    GS_ROS23_DISPATCH(field, launch_fwd_saveat_ros23, a, s, lanes)
  }
  return fail(GS_ERR_ARG, std::string(who) + ": unknown method " + std::to_string(method));
}

extern "C" int gs_adjoint_saveat(int method, int field, int precision, long long n,
                                 const double* p, const double* rec, const int* n_acc, int cap,
                                 const double* ckpt, int ckpt_every, const double* ts,
                                 long long ts_ld, int K, const double* ysbar, const double* ybar,
                                 double* gy0, double* gp, void* stream) {
  int rc = check_saveat("gs_adjoint_saveat", n, p, rec, n_acc, cap, ckpt, ckpt_every, ts, ts_ld, K);
  if (rc) return rc;
  int D, P;
  if ((rc = field_dims(field, &D, &P))) return rc;
  if (n == 0) return GS_OK;
  if (!ckpt || (K > 0 && !ysbar))
    return fail(GS_ERR_ARG, "gs_adjoint_saveat: ckpt and ysbar are required");
  gs::SaveatArgs a{n, nullptr, p, 0.0, rec, n_acc, ckpt_every, gs_ckpt_slots(cap, ckpt_every),
                   const_cast<double*>(ckpt), ts, ts_ld, K, nullptr, nullptr, ysbar, ybar, gy0,
                   gp, cap};
  return saveat_dispatch(method, field, precision, a, stream, true);
}
