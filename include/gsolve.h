/*
 * gsolve.h -- C ABI of libgsolve.so, the B200 (sm_100a) ensemble adaptive ODE solve and
 * record-and-replay discrete adjoint.
 *
 * Plain C: device pointers, sizes and a CUDA stream passed as void*.  No framework types.
 * Every entry point returns an int status (GS_OK or a negative GS_ERR_*); the message of the
 * last failure on the calling thread is available from gs_last_error().  Per-trajectory
 * outcomes (reached t1, max_steps exhausted, record full) are DATA in the status[] output,
 * not call errors, exactly as the reference's kernels report them
 * (gradsolve/warp/_warp_kernel.py:396-399, gradsolve/solvers/record_jax.py:71).
 *
 * All launches are asynchronous on `stream` (NULL = the legacy default stream).  Calls are
 * stateless and re-entrant; the library allocates no device memory: the caller owns every
 * buffer (the workspace size helpers below give the record and checkpoint sizes).
 *
 * Layouts (float64 unless stated):
 *   y0, y_final, ybar, gy0 : (n, D) row-major        p, gp : (n, P) row-major
 *   rec   : dt record, chunk-interleaved: step s of trajectory j at ((s/4)*n + j)*4 + s%4,
 *           cap steps per trajectory; 16-byte aligned.  gs_record_bytes() gives its size.
 *   ckpt  : checkpoints, slot c of trajectory j = (state after c*K accepted steps, time) at
 *           (c*n + j)*CW doubles, CW = D+1 rounded up to even; 16-byte aligned.
 *           gs_ckpt_bytes() gives its size for (field, n, cap, K).
 *   n_acc, n_rej, status : (n,) int32.
 * Field codes: GS_FIELD_LORENZ (D=3,P=1: rho), GS_FIELD_VDP (D=2,P=1: mu),
 *   GS_FIELD_LOTKA_VOLTERRA (D=2,P=4: alpha,beta,gamma,delta), GS_FIELD_LINEAR*1000 + D
 *   (D in 1,2,3,4,8,10,32; P=1, ignored; stiff-capable for D <= 8), GS_FIELD_LORENZ96*1000
 *   + D (D in 4,8,32; P=1: F), GS_FIELD_ROBERTSON (D=3,P=3: k1,k2,k3; stiff),
 *   GS_FIELD_LORENZ3 (D=3,P=3: sigma,beta,rho), GS_FIELD_HIRES (D=8,P=1 ignored; stiff).
 *   Other dimensions of the linear and lorenz96 families, and registered fields, are served
 *   by libraries of their own with this same ABI (gradsolve_b200/fieldgen.py).
 * State dimensions above 8 are integrated by a group of lanes per trajectory (float64; the
 *   float32-stage mode, the dense output and gs_tsit5_vjp_static refuse them); the fused
 *   lanes stop at D = 64, the reference's GPU limit (gradsolve/warp/warp_ode.py:75-81).
 */
#ifndef GSOLVE_H_
#define GSOLVE_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_OK 0
#define GS_ERR_ARG (-1)      /* invalid argument (null pointer, bad size, misalignment) */
#define GS_ERR_FIELD (-2)    /* unknown field code, or field not available for the method */
#define GS_ERR_CUDA (-3)     /* a CUDA launch or runtime call failed */
#define GS_ERR_PRECISION (-4)/* precision mode not available for this entry point */

#define GS_FIELD_LORENZ 1
#define GS_FIELD_VDP 2
#define GS_FIELD_LOTKA_VOLTERRA 3
#define GS_FIELD_LINEAR 4
#define GS_FIELD_LORENZ96 5
#define GS_FIELD_ROBERTSON 10
#define GS_FIELD_LORENZ3 11
#define GS_FIELD_HIRES 12

#define GS_PREC_F64 0   /* everything float64 */
#define GS_PREC_MIXED 1 /* float32 stages/RHS; float64 time, controller, error norm, state */
/* Everything float32 (state, stages, time, error norm, controller): the reference's
 * precision="float32" lane (gradsolve/api.py:253-274, gradsolve/warp/warp_replay.py:87-94, 140-160, 200-219).
 * rec and ckpt then hold float32 data -- size them with gs_record_bytes_prec /
 * gs_ckpt_bytes_prec (half the float64 record) -- while y0, p, y_final, cotangents and
 * gradients stay float64 arrays holding float32 values.  Tsit5 and Rosenbrock23, fields of
 * at most 8 components, one thread per trajectory (STATIC or AUTO schedule), no saveat. */
#define GS_PREC_F32 2
#define GS_PREC_MASK 0xff

/* Scheduling flags, OR-ed into the precision argument of the forward and adjoint entry
 * points.  STATIC: one thread per trajectory.  REFILL: a persistent grid whose lanes take
 * the next trajectory from a work counter when theirs finishes (uneven batches; the counter
 * lives in the checkpoint buffer's control block).  STRIDED: persistent lanes taking
 * trajectories j, j+G, ...  AUTO (0): STATIC, except REFILL for a forward with per-trajectory
 * end times. */
#define GS_SCHED_AUTO 0x000
#define GS_SCHED_STATIC 0x100
#define GS_SCHED_REFILL 0x200
#define GS_SCHED_STRIDED 0x300
#define GS_SCHED_MASK 0x300

/* Reverse-pass variant flags, OR-ed into the precision argument of gs_tsit5_adjoint (float64
 * and float32-stage modes, one thread per trajectory).  RECOMPUTE: the reverse sweep
 * re-evaluates each step's stages from the segment's states.  STAGES: the segment's replay
 * keeps the stage inputs of the steps it evaluates (5*D doubles per step of shared memory;
 * 6*D floats in the float32-stage mode), so only each segment's last step
 * evaluates its stages twice; falls back to RECOMPUTE where that buffer would not fit.  AUTO
 * (0): STAGES while its shared memory leaves it at least 3/5 of RECOMPUTE's resident threads
 * per SM (the autotuned K = 2 of the built-in fields: equal residency, 4-6% faster), else
 * RECOMPUTE.  gs_ros23_adjoint applies the same rule to keeping the factors of W. */
#define GS_ADJ_AUTO 0x000
#define GS_ADJ_RECOMPUTE 0x400
#define GS_ADJ_STAGES 0x800
/* The float32 route's Tsit5 reverse pass (GS_PREC_F32): PAIRS runs two trajectories per thread
 * (lanes 2u and 2u + 1, in packed float32x2 arithmetic: one instruction for both), built for
 * the built-in nonstiff fields and refused for others; RECOMPUTE runs one per thread; AUTO is
 * PAIRS where it is built, else RECOMPUTE.  The two agree to float rounding (the packed
 * expressions fuse their own choice of products).  STAGES is a float64 / float32-stage
 * option. */
#define GS_ADJ_PAIRS 0xC00
#define GS_ADJ_MASK 0xC00

/* Lanes per trajectory for the fields of more than 8 components (a group of G lanes
 * integrates one trajectory, gs_coop.cuh), OR-ed into the precision argument of
 * gs_tsit5_fwd_record, gs_tsit5_replay and gs_tsit5_adjoint: GS_LANES(k) asks for G = 2^k
 * lanes; 0 takes the field's default.  gs_lane_choices lists the group sizes built for a
 * field (the default first); any other is refused with GS_ERR_ARG.  Results do not depend
 * on G beyond rounding (the error norm's and the parameter gradient's sums are grouped by
 * lane). */
#define GS_LANES_SHIFT 12
#define GS_LANES_MASK 0x7000
#define GS_LANES(log2_lanes) ((log2_lanes) << GS_LANES_SHIFT)

/* Registers and occupancy, OR-ed into the precision argument of gs_tsit5_fwd_record /
 * gs_ros23_fwd_record (the float64 recording forward, one thread per trajectory) and of
 * gs_tsit5_adjoint / gs_ros23_adjoint / gs_adjoint_ordered (the reverse pass's K = 2
 * instance that keeps the replayed steps' stage inputs or factors, float64 or, for Tsit5,
 * float32-stage, one thread per trajectory): GS_OCC(b) runs the kernel instance whose registers are bounded for b resident
 * blocks of 128 threads per SM; 0 takes the default instance.  gs_occ_choices lists the
 * values built for a field and pass (0 first); any other value, and any nonzero value on
 * another path (the float32-stage forward, the float32 route, the forward without a record,
 * persistent schedules, another checkpoint interval or reverse-pass variant), is refused with
 * GS_ERR_ARG.  The instances run the same arithmetic: results are bit for bit those of the
 * default. */
#define GS_OCC_SHIFT 15
#define GS_OCC_MASK 0x78000
#define GS_OCC(blocks) ((blocks) << GS_OCC_SHIFT)
#define GS_OCC_FORWARD 0       /* Tsit5 recording forward */
#define GS_OCC_REVERSE 1       /* Tsit5 reverse pass at K = 2 */
#define GS_OCC_ROS23_FORWARD 2 /* Rosenbrock23 recording forward */
#define GS_OCC_ROS23_REVERSE 3 /* Rosenbrock23 reverse pass at K = 2 */
#define GS_OCC_MIXED_REVERSE 4 /* Tsit5 float32-stage reverse pass at K = 2 */

/* per-trajectory status values written to status[] */
#define GS_TRAJ_OK 0          /* reached t1 */
#define GS_TRAJ_MAX_STEPS 1   /* max_steps attempts exhausted (or non-finite error) */
#define GS_TRAJ_UNDERFLOW 2   /* step size underflow (Rosenbrock23 only) */
#define GS_TRAJ_RECORD_FULL 3 /* more than cap accepted steps; grow the record and retry */

/* Library version (major*10000 + minor*100 + patch). */
int gs_version(void);

/* Kernel launches this library has issued in the process so far (all entry points,
 * counted as they are made): a measurement aid, e.g. the launches inside a timed region. */
unsigned long long gs_launch_count(void);

/* Message of the last failed call on this thread ("" if none). */
const char* gs_last_error(void);

/* State dimension D and parameter count P of a field code.  Replaces the registry lookup
 * of gradsolve/warp/_warp_kernel.py:229-286 (_field_entry / field_dim). */
int gs_field_dims(int field, int* D, int* P);

/* Host copy of the method constants in this order: C2..C5 (4), A21..A65 (15), B1..B7 (7),
 * E1..E7 (7), SAFETY, ERR_FLOOR, FAC_MIN, FAC_MAX, TSIT5_EXP (5), ROS_D, ROS_E32, ROS_EXP (3):
 * 41 values.  The constants of gradsolve/solvers/tsit5_step.py:26-77 and
 * gradsolve/warp/_warp_rosenbrock.py:62-70.  len must be >= 41. */
int gs_tableau(double* out, int len);

/* The same 41 constants as compiled into device code, written by a kernel to a device
 * buffer of 41 doubles. */
int gs_device_tableau(double* out_dev, void* stream);

/* Bytes of a dt record for n trajectories of capacity cap. */
size_t gs_record_bytes(long long n, int cap);

/* Number of checkpoint slots for capacity cap and interval K (ceil(cap/K) + 1). */
int gs_ckpt_slots(int cap, int ckpt_every);

/* Bytes of the checkpoint buffer for (field, n, cap, K); 0 for an unknown field. */
size_t gs_ckpt_bytes(int field, long long n, int cap, int ckpt_every);

/* The two sizes above for a precision mode: GS_PREC_F32 records 4-byte steps (the record
 * is exactly half the float64 one) and 4-byte checkpoint rows of D+1 values rounded up to a
 * multiple of 4; any other mode gives the float64 sizes.  0 for an unknown field. */
size_t gs_record_bytes_prec(int precision, long long n, int cap);
size_t gs_ckpt_bytes_prec(int field, int precision, long long n, int cap, int ckpt_every);

/* Largest checkpoint interval K the adjoint kernels accept. */
int gs_max_ckpt_every(void);

/* Lanes per trajectory built for a field: writes up to cap group sizes to out (the default
 * first; 1 alone for fields integrated one thread per trajectory) and returns how many, or a
 * negative GS_ERR_* for an unknown field.  No counterpart in the reference, whose fused lane
 * is one thread per trajectory (gradsolve/warp/_warp_kernel.py:325-399); it serves the
 * autotuner that picks the group size. */
int gs_lane_choices(int field, int* out, int cap);

/* Occupancy choices built for a field, pass = GS_OCC_FORWARD (the float64 Tsit5 recording
 * forward; default instance bounded for 6 blocks per SM at up to 4 components, unbounded
 * above), GS_OCC_REVERSE (the float64 Tsit5 reverse pass at K = 2; default 5 blocks),
 * GS_OCC_ROS23_FORWARD (Rosenbrock23 forward; default unbounded) or GS_OCC_ROS23_REVERSE
 * (Rosenbrock23 reverse pass at K = 2; default 4 blocks) or GS_OCC_MIXED_REVERSE (the Tsit5
 * float32-stage reverse pass at K = 2; default 6 blocks): writes up to cap GS_OCC values to
 * out (0, the default instance, first) and returns how many, or a negative GS_ERR_* for an
 * unknown field or pass (or a field without a Jacobian for the Rosenbrock23 passes).  No counterpart in the
 * reference, whose kernels take the compiler's register allocation
 * (gradsolve/warp/_warp_kernel.py:325-399); it serves the autotuner that picks registers and
 * occupancy per field. */
int gs_occ_choices(int field, int pass, int* out, int cap);

/*
 * Adaptive Tsit5 forward solve that records the accepted step sizes.
 * Replaces gradsolve/warp/_warp_kernel.py:325-399 (_tsit5_adaptive_general, record == 1)
 * as launched by gradsolve/warp/warp_ode.py:215-327 (_launch), and the host recorder
 * gradsolve/solvers/tsit5_replay.py:62-124 (tsit5_adaptive) it is specified by.
 *   t1v  : per-trajectory end times (n,) or NULL for the scalar t1.
 *   dt0  : first step; <= 0 selects (t1_j - t0)/100 per trajectory (warp_replay.py:157).
 *   rec  : dt record of capacity cap, or NULL (no record).
 *   ckpt : checkpoints every ckpt_every accepted steps (1..gs_max_ckpt_every()), or NULL.
 *   A trajectory that would accept more than cap steps stops with status 3 when rec or ckpt
 *   is given.  y_final is the last reached state (rows with status != 0 are not NaN'd here;
 *   the reference's driver does that, gradsolve/warp/warp_ode.py:319).
 *   With rec and ckpt both NULL this is the forward-only solve (the reference's cuda_tsit5
 *   lane, gradsolve/cuda/kernels/tsit5_template.cu.in), run by a kernel instance with the
 *   store paths compiled out.
 */
int gs_tsit5_fwd_record(int field, int precision, long long n, const double* y0,
                        const double* p, double t0, const double* t1v, double t1, double rtol,
                        double atol, double dt0, int max_steps, int cap, int ckpt_every,
                        double* rec, double* ckpt, double* y_final, int* n_acc, int* n_rej,
                        int* status, void* stream);

/*
 * Frozen-mesh replay: re-integrate n_acc[j] recorded steps of trajectory j with fixed
 * steps.  Replaces gradsolve/warp/warp_replay.py:30-55 (replay_solve_jax) over
 * gradsolve/solvers/tsit5_step.py:80-102 (tsit5_step).  Optionally writes checkpoints
 * (ckpt != NULL), so a record that came from elsewhere (gs_record_from_padded) can feed
 * gs_tsit5_adjoint.
 */
int gs_tsit5_replay(int field, int precision, long long n, const double* y0, const double* p,
                    double t0, const double* rec, const int* n_acc, int cap, int ckpt_every,
                    double* ckpt, double* y_final, void* stream);

/*
 * Discrete adjoint of the frozen-mesh replay: given ybar = dL/dy_final, writes
 * gy0 = dL/dy0 and gp = dL/dp (either may be NULL) with the recorded dts held fixed -- the
 * gradient jax.grad takes through replay_solve_jax (gradsolve/warp/warp_replay.py:30-55,
 * closures :186-237; gradsolve/solvers/tsit5_replay.py:192-232).  Needs the checkpoints of
 * the forward (or of gs_tsit5_replay) with the same ckpt_every.
 */
int gs_tsit5_adjoint(int field, int precision, long long n, const double* p, const double* rec,
                     const int* n_acc, int cap, const double* ckpt, int ckpt_every,
                     const double* ybar, double* gy0, double* gp, void* stream);

/*
 * Adaptive Rosenbrock23 (ode23s, autonomous) forward with dt record.  Replaces
 * gradsolve/warp/_warp_rosenbrock.py:383-452 (_rosenbrock23_adaptive, record == 1) as
 * launched by gradsolve/warp/warp_rosenbrock.py:166-218 (_launch); specified by
 * tests/_oracles/gradsolve_g2_spike_oracle.py:138-184.  Same arguments and outputs as
 * gs_tsit5_fwd_record; fields need an analytic Jacobian (GS_FIELD_ROBERTSON, linear).
 * Additionally stops with status 2 when a step no longer advances time (t + h == t).
 */
int gs_ros23_fwd_record(int field, int precision, long long n, const double* y0,
                        const double* p, double t0, const double* t1v, double t1, double rtol,
                        double atol, double dt0, int max_steps, int cap, int ckpt_every,
                        double* rec, double* ckpt, double* y_final, int* n_acc, int* n_rej,
                        int* status, void* stream);

/* Frozen-mesh Rosenbrock23 replay.  Replaces gradsolve/warp/warp_replay.py:267-293
 * (replay_solve_rosenbrock_jax) over gradsolve/solvers/rosenbrock23_step.py:47-66. */
int gs_ros23_replay(int field, int precision, long long n, const double* y0, const double* p,
                    double t0, const double* rec, const int* n_acc, int cap, int ckpt_every,
                    double* ckpt, double* y_final, void* stream);

/* Discrete adjoint of the Rosenbrock23 replay (the gradient jax.grad takes through
 * gradsolve/warp/warp_replay.py:344-384), including the second-order term through
 * W = I - d*dt*J(y, p). */
int gs_ros23_adjoint(int field, int precision, long long n, const double* p, const double* rec,
                     const int* n_acc, int cap, const double* ckpt, int ckpt_every,
                     const double* ybar, double* gy0, double* gp, void* stream);

/* gs_tsit5_adjoint (method GS_METHOD_TSIT5) or gs_ros23_adjoint (GS_METHOD_ROS23) with the
 * lanes in a given order: lane t integrates trajectory order[t], a device array of n int64
 * forming a permutation of [0, n) (an entry outside [0, n) leaves its lane idle).  Every
 * input and output keeps the batch's own order; only the assignment of trajectories to
 * threads changes, so the results equal the unordered call's bit for bit.  Ordered by step
 * count (longest first), a warp's lanes take similar numbers of steps: the reverse pass of a
 * record whose step counts spread widely then wastes no lanes on finished trajectories.  One
 * thread per trajectory only (GS_SCHED_STATIC or AUTO).  No counterpart in the reference. */
int gs_adjoint_ordered(int method, int field, int precision, long long n, const double* p,
                       const double* rec, const int* n_acc, int cap, const double* ckpt,
                       int ckpt_every, const double* ybar, double* gy0, double* gp,
                       const long long* order, void* stream);

#define GS_METHOD_TSIT5 0
#define GS_METHOD_ROS23 1

/*
 * Dense output on the frozen-mesh replay: the states at requested times ts (sorted, within
 * [t0, t1_j]; row j at ts + j*ts_ld, ts_ld = 0 shares one row) by bracket-and-re-step:
 * one step of the method, of size ts_k - t, from the start of the step bracketing ts_k;
 * times <= t0 give y0 and times >= the final accumulated time give y_final bitwise.
 * Replaces gradsolve/warp/warp_replay.py:58-94 (replay_solve_saveat_jax and its Rosenbrock
 * twin) over gradsolve/solvers/dense.py:106-163,318-335 (scan_saveat_one / vmap_saveat);
 * per-trajectory rows of times are an extension (the reference shares one grid).
 * ys: (n, K, D).  Writes checkpoints for gs_adjoint_saveat when ckpt != NULL.
 * method: GS_METHOD_TSIT5 (float64 or mixed) or GS_METHOD_ROS23 (float64).
 */
int gs_replay_saveat(int method, int field, int precision, long long n, const double* y0,
                     const double* p, double t0, const double* rec, const int* n_acc, int cap,
                     int ckpt_every, double* ckpt, const double* ts, long long ts_ld, int K,
                     double* ys, double* y_final, void* stream);

/*
 * The adaptive forward with record (gs_tsit5_fwd_record / gs_ros23_fwd_record) that also
 * produces the dense output of gs_replay_saveat at the same time: each requested time is
 * re-stepped from the start of the accepted step that brackets it, as the trajectory is
 * integrated, so the recording point needs no separate replay pass.  ys equals what
 * gs_replay_saveat gives on the recorded mesh to rounding (the same step function, compiled
 * into another kernel).  Schedules: lanes refilled from a work counter (GS_SCHED_REFILL, or
 * AUTO when trajectories have their own end times; needs ckpt), persistent strided lanes
 * (GS_SCHED_STRIDED), one thread per trajectory otherwise (GS_SCHED_STATIC, or AUTO with a
 * shared end time).  No counterpart in the reference,
 * whose saveat always replays the recorded mesh (gradsolve/warp/warp_replay.py:58-84).
 * method: GS_METHOD_TSIT5 (float64 or mixed) or GS_METHOD_ROS23 (float64).
 */
int gs_fwd_record_saveat(int method, int field, int precision, long long n, const double* y0,
                         const double* p, double t0, const double* t1v, double t1, double rtol,
                         double atol, double dt0, int max_steps, int cap, int ckpt_every,
                         double* rec, double* ckpt, double* y_final, int* n_acc, int* n_rej,
                         int* status, const double* ts, long long ts_ld, int K, double* ys,
                         void* stream);

/*
 * Adjoint of gs_replay_saveat for a loss of the saved states (and optionally y_final):
 * ysbar (n, K, D) = dL/dys, ybar (n, D) = dL/dy_final or NULL -> gy0, gp (either may be
 * NULL).  The gradient jax.grad takes through replay_solve_saveat_jax
 * (gradsolve/warp/warp_replay.py:58-84, gradsolve/api.py:748-752).  precision may carry
 * GS_SCHED_REFILL / GS_SCHED_STRIDED (persistent lanes, for uneven batches); AUTO runs one
 * thread per trajectory.
 */
int gs_adjoint_saveat(int method, int field, int precision, long long n, const double* p,
                      const double* rec, const int* n_acc, int cap, const double* ckpt,
                      int ckpt_every, const double* ts, long long ts_ld, int K,
                      const double* ysbar, const double* ybar, double* gy0, double* gp,
                      void* stream);

/*
 * Record conversion between the reference's padded (n, S) layout (row j = trajectory j's
 * accepted dts, zero padded; gradsolve/warp/warp_replay.py:181-182) and the chunked record.
 * from_padded also writes n_steps[j] = index of the last non-zero dt + 1 (zero steps
 * before it are kept: they are identity steps).  dts row stride is ld (>= S).
 */
int gs_record_from_padded(long long n, long long S, const double* dts, long long ld,
                          double* rec, int cap, int* n_steps, void* stream);
int gs_record_to_padded(long long n, int cap, const double* rec, const int* n_acc, long long S,
                        double* dts, void* stream);

/*
 * Row moves for batches split into tiers or reordered (the host side's tier plan): rows of
 * `width` elements of elem_bytes (4 or 8) bytes.  scatter = 0: dst[r] = src[idx[r]] for r <
 * rows (idx into `limit` source rows); scatter = 1: dst[idx[r]] = src[r] (idx into `limit`
 * destination rows).  Indices outside [0, limit) are skipped and counted into *bad (a device
 * counter the caller zeroes and reads).  No counterpart in the reference, which re-solves the
 * whole batch instead of planning tiers (gradsolve/solvers/record_jax.py:192-199).
 */
int gs_move_rows(int scatter, int elem_bytes, const void* src, const long long* idx,
                 long long rows, int width, long long limit, void* dst,
                 unsigned long long* bad, void* stream);

/* Size of the library's own device scratch used by gs_tsit5_vjp_static: 64 MiB, held by
 * every GPU that loads libgsolve.so until the process exits.  Only libgsolve.so carries it:
 * the libraries built for generated fields (gradsolve_b200/fieldgen.py) export
 * gs_tsit5_vjp_static as a stub that returns GS_ERR_FIELD and hold no such array. */
#define GS_STATIC_SCRATCH_BYTES (64ull << 20)

/*
 * Replay gradient that allocates nothing.  No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc -- a custom call inside JAX/XLA, where XLA has already
 * reserved most of the device memory for its own pool, and latency-critical callers that
 * cannot accept the device-wide synchronisation of cudaMalloc/cudaFree.
 * Given the recorded dts in the reference's padded (n, S) layout (row stride ld >= S), it
 * replays them at (y0, p) into y_final and writes gy0 = dL/dy0 and gp = dL/dp (either may
 * be NULL) for the cotangent ybar = dL/dy_final: the result of gs_record_from_padded +
 * gs_tsit5_replay + gs_tsit5_adjoint, computed with the dt record, checkpoints and step
 * counts in a static device array inside the library instead of caller buffers.
 * Checkpoints every K steps, the shortest K >= 2 for which the record + checkpoints + counts
 * fit GS_STATIC_SCRATCH_BYTES, and the reverse pass gs_tsit5_adjoint would choose for it.
 * Limits: those must fit at K = 64 at least (roughly n * S <= 7.5e6 steps for the 3-state
 * fields); larger problems return GS_ERR_ARG with the numbers -- use the allocating entry
 * points for them.
 * The first call on each device looks up the array's device address (cudaGetSymbolAddress,
 * with that device current); make that first call before any stream capture.  The address
 * is kept until the process exits, so resetting the device (cudaDeviceReset) after that
 * first call is not supported.  All calls share the one array, which keeps the last call's
 * contents: calls that overlap on the GPU race and must be serialised by the caller.
 * Non-stiff (Tsit5) built-in fields only (GS_ERR_FIELD from a generated field's library).
 */
int gs_tsit5_vjp_static(int field, long long n, const double* y0, const double* p, double t0,
                        const double* dts, long long S, long long ld, const double* ybar,
                        double* y_final, double* gy0, double* gp, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GSOLVE_H_ */
