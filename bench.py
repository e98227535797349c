"""Benchmark: trajectory-gradients/s (adaptive forward with record + reverse-replay adjoint).

Workload ("differentiation at scale"): Lorenz (sigma=10, beta=8/3, per-trajectory rho),
n = 2^20 trajectories per GPU, y0 = [1,0,0] + N(0, 0.1^2) and rho ~ U(20, 30) from
numpy default_rng(seed) (seed 0 on rank 0, seed r on rank r), t in [0, 10], Tsit5 with
rtol = atol = 1e-8, float64, loss = mean(y_final^2), gradient w.r.t. rho, sqrt(N) segment
checkpointing.  A step = one adaptive forward solve that records the accepted dts and the
checkpoints + the cotangent of the loss + one reverse-replay adjoint, over the whole batch.

Usage:  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Multi-GPU: one process per GPU (torchrun); each rank solves its own 2^20 trajectories
(weak scaling, no data-path collective); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "trajectory grads/s (fwd+adjoint), FP64 vs mixed at <=1e-6 rel err; % FP peak"
UNIT = "trajectory-gradients/s"
T0, T1, RTOL, ATOL = 0.0, 10.0, 1e-8, 1e-8
N_DEFAULT = 1 << 20
L2_BYTES = 126 * 1024 * 1024


def make_inputs(n: int, seed: int):
    rng = np.random.default_rng(seed)
    y0 = np.array([1.0, 0.0, 0.0]) + rng.normal(0.0, 0.1, (n, 3))
    rho = rng.uniform(20.0, 30.0, (n, 1))
    return y0, rho


def shard_seed(rank: int) -> int:
    return rank


class LorenzProblem:
    name = "diffeqgpu_lorenz"
    dim = 3
    t0 = T0
    t1 = T1
    is_stiff = False


# ------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------
# peaks
# ------------------------------------------------------------------------------------
def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def probe_fp64_tflops(torch, stream) -> float:
    """FP64 FMA throughput of this GPU, measured now with libgsprobe (the denominator for
    the CUDA-core-bound solver kernels)."""
    import ctypes

    L = ctypes.CDLL(str(ROOT / "gradsolve_b200" / "libgsprobe.so"))
    L.gs_probe_fp64.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, iters = sms * 8, 4096
    for _ in range(2):
        L.gs_probe_fp64(out.data_ptr(), blocks, iters, stream.cuda_stream)
    best = 0.0
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        L.gs_probe_fp64(out.data_ptr(), blocks, iters, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = max(best, 2.0 * 32 * iters * blocks * 256 / (ms * 1e-3) / 1e12)
    return best


# ------------------------------------------------------------------------------------
# CPU baseline: the oracle port (record + replay adjoint) on the host cores
# ------------------------------------------------------------------------------------
def cpu_gradient_rate(target_s: float = 12.0, threads: int = 0) -> dict:
    from oracle import oracle as O

    O.build()
    cores = threads or os.cpu_count() or 1

    def run(m):
        y0, rho = make_inputs(m, 1000)
        t = time.perf_counter()
        r = O.record("tsit5", "lorenz", y0, rho, T0, T1, RTOL, ATOL, max_steps=100000,
                     cap=4096, nthreads=cores)
        ybar = 2.0 * r["y_final"] / r["y_final"].size
        O.replay_vjp("tsit5", "lorenz", y0, rho, r["dts"], ybar, nthreads=cores)
        return time.perf_counter() - t

    m = max(64, cores * 16)
    dt = run(m)
    m2 = int(min(1 << 20, max(m, m * target_s / max(dt, 1e-3))))
    dt2 = run(m2)
    return {"value": m2 / dt2, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{m2} trajectories of the same workload (seed 1000), C restatement of "
                      f"tsit5_adaptive record + replay adjoint, {cores} host threads, "
                      f"{dt2:.1f} s"}


def reference_forward_rate(m: int, cores: int) -> float | None:
    """The reference's own C++ forward (gradsolve/cuda/kernels/tsit5_template.cu.in,
    host build in oracle/_ref/) on m trajectories, trajectory-solves/s."""
    import ctypes

    so = ROOT / "oracle" / "_ref" / "libref_tsit5_lorenz.so"
    if not so.exists():
        return None
    L = ctypes.CDLL(str(so))
    dp = ctypes.POINTER(ctypes.c_double)
    L.ref_fwd.argtypes = [ctypes.c_long, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                          ctypes.c_int, dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    y0, rho = make_inputs(m, 1000)
    y0 = np.ascontiguousarray(y0)
    rho1 = np.ascontiguousarray(rho[:, 0])
    yf = np.zeros_like(y0)
    ns = np.zeros(m, np.int32)
    t = time.perf_counter()
    L.ref_fwd(m, y0.ctypes.data_as(dp), rho1.ctypes.data_as(dp), T1, RTOL, ATOL, 100000,
              yf.ctypes.data_as(dp), ns.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), cores)
    return m / (time.perf_counter() - t)


def run_reference(args) -> None:
    """--impl reference: the reference path's CPU implementation on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O

    O.build()
    cores = os.cpu_count() or 1
    # size one step to about 4 s of work
    cal = cpu_gradient_rate(target_s=2.0, threads=cores)
    m = int(max(cores * 8, min(1 << 16, cal["value"] * 4.0)))
    y0, rho = make_inputs(m, 1000)

    def step():
        r = O.record("tsit5", "lorenz", y0, rho, T0, T1, RTOL, ATOL, max_steps=100000,
                     cap=4096, nthreads=cores)
        ybar = 2.0 * r["y_final"] / r["y_final"].size
        O.replay_vjp("tsit5", "lorenz", y0, rho, r["dts"], ybar, nthreads=cores)

    for _ in range(args.warmup):
        step()
    t = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t
    value = m * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, numpy default_rng)",
        "config": {"workload": "lorenz n=2^20 t=[0,10] tsit5 rtol=atol=1e-8 grad wrt rho "
                               f"(bounded sample of {m} trajectories per step)",
                   "sample_trajectories": m},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{m} trajectories per step; the reference's gradient "
                                   "path needs JAX, absent here, so the record and replay "
                                   "adjoint run as the C restatement (oracle/gs_oracle.c)"},
        "reference_forward_solves_per_s": reference_forward_rate(min(m, 8192), cores),
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------
# the B200 arm
# ------------------------------------------------------------------------------------
def _time_steps(torch, step, steps, flush, stream):
    """Run `steps` timed steps (L2 flushed before each, outside the events); returns the
    per-step (forward, adjoint, whole) milliseconds and the last step's outputs."""
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(steps)]
    out = None
    for k in range(steps):
        flush.zero_()
        out = step(ev[k])
    torch.cuda.synchronize()
    fwd = [e[0].elapsed_time(e[1]) for e in ev]
    adj = [e[2].elapsed_time(e[3]) for e in ev]
    whole = [e[0].elapsed_time(e[3]) for e in ev]
    return fwd, adj, whole, out


def _grad_err(g, ref):
    """Per-trajectory relative error of gradient rows g vs ref (both (n, P) tensors)."""
    import torch
    num = (g - ref).abs().amax(dim=1)
    den = ref.abs().amax(dim=1).clamp_min(1e-300)
    q = (num / den).double()
    rel_l2 = float(((g - ref).norm() / ref.norm()).item())
    return {"max": float(q.max().item()), "median": float(q.median().item()),
            "p99": float(torch.quantile(q[: min(q.numel(), 1 << 24)], 0.99).item()),
            "rel_l2": rel_l2}


def run_b200(args) -> None:
    import torch
    import torch.distributed as dist

    from gradsolve_b200 import engine, flops
    from gradsolve_b200.fields import field_spec

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    n = args.n
    spec = field_spec("lorenz")
    y0_np, rho_np = make_inputs(n, shard_seed(rank))
    y0 = torch.tensor(y0_np, device=dev)
    rho = torch.tensor(rho_np, device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    inv = 1.0 / (n * 3 * world)

    def make_step(precision):
        ws = {"r": None}  # the record/checkpoint buffers are allocated once and reused

        def step(events=None):
            if events:
                events[0].record(stream)
            r = engine.forward_record("tsit5", spec, y0, rho, t0=T0, t1=T1, rtol=RTOL,
                                      atol=ATOL, max_steps=100000, cap0=args.cap,
                                      checkpoint=args.checkpoint, precision=precision,
                                      workspace=ws["r"], schedule=args.schedule)
            ws["r"] = r
            if events:
                events[1].record(stream)
            ybar = (2.0 * inv) * r.y_final
            if events:
                events[2].record(stream)
            _gy0, gp = engine.adjoint(r, rho, ybar, want_y0=False, precision=precision,
                                      schedule=args.schedule)
            if events:
                events[3].record(stream)
            return r, gp
        return step

    # clocks are sampled from the start of the warm-up to the end of the timed steps
    clocks = ClockSampler(local)
    clocks.start()
    step = make_step("float64")
    for _ in range(args.warmup):  # warm-up (also sizes the record so timed steps never regrow)
        r, gp = step()
    torch.cuda.synchronize()
    assert int((r.status != 0).sum().item()) == 0, "warm-up solve failed"
    att = int((r.n_acc.to(torch.int64) + r.n_rej.to(torch.int64)).sum().item())
    acc = int(r.n_acc.to(torch.int64).sum().item())
    S = int(r.n_acc.max().item())
    K = r.ckpt_every
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    fwd_ms, adj_ms, step_ms, (r, gp) = _time_steps(torch, step, args.steps, flush, stream)
    if world > 1:
        dist.barrier()
    ms_per_step = float(np.mean(step_ms))
    if world > 1:
        t = torch.tensor([ms_per_step], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_per_step = float(t.item())
    value = n * world / (ms_per_step * 1e-3)
    assert torch.isfinite(gp).all()

    # ---- the float32-stage variant on the same workload, and its accuracy ---------------
    mixed = None
    if not args.no_mixed:
        mstep = make_step("mixed")
        for _ in range(args.warmup):
            rm, gpm = mstep()
        m_fwd, m_adj, m_step, (rm, gpm) = _time_steps(torch, mstep, args.steps, flush, stream)
        m_ms = float(np.mean(m_step))
        if world > 1:
            t = torch.tensor([m_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            m_ms = float(t.item())
        # same mesh: the float64 record replayed and differentiated with float32 stages
        ybar64 = (2.0 * inv) * r.y_final
        yf_sm = engine.replay(r, y0, rho, write_ckpt=True, precision="mixed")
        _g, gp_sm = engine.adjoint(r, rho, ybar64, want_y0=False, precision="mixed")
        n_acc_diff = (rm.n_acc.to(torch.int64) - r.n_acc.to(torch.int64)).abs()
        yrel = ((yf_sm - r.y_final).abs() / r.y_final.abs().clamp_min(1e-300)).amax(dim=1)
        mixed = {"value": n * world / (m_ms * 1e-3), "ms_per_step": m_ms,
                 "fwd_ms": float(np.mean(m_fwd)), "adj_ms": float(np.mean(m_adj)),
                 "speedup_vs_f64": ms_per_step / m_ms,
                 "grad_rel_err_own_mesh": _grad_err(gpm, gp),
                 "grad_rel_err_same_mesh": _grad_err(gp_sm, gp),
                 "y_final_rel_err_same_mesh_max": float(yrel.max().item()),
                 "y_final_rel_err_same_mesh_median": float(yrel.median().item()),
                 "n_acc_diff_max": int(n_acc_diff.max().item()),
                 "meets_1e-6": _grad_err(gp_sm, gp)["max"] <= 1e-6}
    clk = clocks.stop()

    # ---- e2e through the public API, host buffers, H2D + D2H inside the timed region ----
    e2e = None
    if not args.no_e2e:
        import gradsolve_b200 as gsb
        y0_h = torch.tensor(y0_np).pin_memory()
        rho_h = torch.tensor(rho_np).pin_memory()
        grad_h = torch.empty_like(rho_h).pin_memory()
        prob = LorenzProblem()

        def e2e_step():
            clo = gsb.grad_closure(prob, y0_h, rho_h, rtol=RTOL, atol=ATOL,
                                   checkpoint=args.checkpoint, max_steps=100000, device=dev)
            p = clo.state.p_rec.clone().requires_grad_(True)
            yf = clo(p)
            loss = (yf * yf).sum() * inv
            loss.backward()
            grad_h.copy_(p.grad)
            return float(loss.item())

        for _ in range(max(1, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        ke = max(1, min(args.steps, 5))
        t0 = time.perf_counter()
        for _ in range(ke):
            e2e_step()
        torch.cuda.synchronize()
        el = (time.perf_counter() - t0) / ke
        if world > 1:
            t = torch.tensor([el], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        e2e = {"value": n * world / el, "unit": UNIT,
               "h2d_bytes_per_step": int(y0_h.numel() * 8 + rho_h.numel() * 8),
               "d2h_bytes_per_step": int(grad_h.numel() * 8 + 8),
               "ms_per_step": el * 1e3, "api": "gradsolve_b200.grad_closure + torch autograd"}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant kernel -------------------------------------------
    fp64_peak = probe_fp64_tflops(torch, stream)
    peaks = measured_peaks()
    f_fwd = flops.solve_flops("tsit5", "lorenz", att)
    f_adj = flops.adjoint_flops("tsit5", "lorenz", acc)
    fwd_avg, adj_avg = float(np.mean(fwd_ms)), float(np.mean(adj_ms))
    kernels = {
        "tsit5_record_kernel": {"ms": fwd_avg, "tflops": f_fwd / (fwd_avg * 1e-3) / 1e12},
        "tsit5_adjoint_kernel": {"ms": adj_avg, "tflops": f_adj / (adj_avg * 1e-3) / 1e12},
    }
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    nslots = math.ceil(S / K) + 1
    rec_bytes = acc * 8 * 2                     # dts written by the forward, read by the adjoint
    ck_bytes = n * nslots * 4 * 8 * 2          # checkpoints written + read
    io_bytes = n * (3 + 1) * 8 + n * (3 + 1 + 3) * 8
    achieved = kernels[dom]["tflops"]
    roofline = {
        "bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
        "frac": achieved / fp64_peak, "traffic": None, "kernel": dom,
        "peak_source": "measured in this run: libgsprobe FP64 FMA loop (8 chains/thread)",
        "per_kernel": kernels,
        "hbm": {"algorithmic_bytes_per_step": rec_bytes + ck_bytes + io_bytes,
                "achieved_gbs": (rec_bytes + ck_bytes + io_bytes) / (ms_per_step * 1e-3) / 1e9,
                "peak_gbs": peaks["hbm_gbs"], "peak_source": peaks["source"]},
        "flops_per_unit": {"F_att": flops.COUNTS[("tsit5", "lorenz")]["F_att"],
                           "F_step": flops.COUNTS[("tsit5", "lorenz")]["F_step"],
                           "F_vjp": flops.COUNTS[("tsit5", "lorenz")]["F_vjp"],
                           "attempts": att, "accepted": acc},
    }
    cpu = None
    if world == 1 and not args.no_cpu:
        cpu = cpu_gradient_rate(target_s=args.cpu_seconds)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy default_rng; seed = rank)",
        "config": {"workload": "lorenz n=2^20/GPU t=[0,10] tsit5 rtol=atol=1e-8 fp64, "
                               "grad of mean(y_final^2) wrt rho, segment checkpointing "
                               "(checkpoints every K accepted steps, segments recomputed "
                               "in the reverse pass)",
                   "checkpoint_policy": str(args.checkpoint),
                   "n_per_gpu": n, "record_len_max": S, "checkpoint_every": K,
                   "attempts": att, "accepted": acc, "parallelism": f"shard{world}",
                   "l2": "flushed between timed steps (record traffic also >> L2)"},
        "gpu_launches": 2 * args.steps,
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
        "fwd_ms": fwd_avg, "adj_ms": adj_avg, "mixed": mixed,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--cap", type=int, default=1024)
    ap.add_argument("--checkpoint", default="auto")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--schedule", default="auto", choices=["auto", "static", "refill", "strided"])
    args = ap.parse_args()
    if args.checkpoint not in ("sqrt", "all", "auto"):
        args.checkpoint = int(args.checkpoint)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
