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


# DRAM bytes per trajectory of each kernel on this workload, from ncu captures at n = 2^18
# (dram__bytes_read.sum + dram__bytes_write.sum per launch / 2^18), by checkpoint interval;
# profiles/tsit5_f64_lorenz_bench_n2e20_launches_n2e18_K2.md (the timed step's launches:
# lanes ordered by cost, segments swept in step with the warp's longest trajectory).
# Traffic grows with the trajectory count.
DRAM_BYTES_PER_TRAJ = {
    "tsit5_adjoint_stages_k2_kernel": {2: (4.266209e9 + 5.998e6) / 2**18},
    "tsit5_record_kernel": {2: (0.146856e9 + 4.304376e9) / 2**18},
}


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
class _NoGC:
    """Python's garbage collector paused around a timed loop, as timeit does: a collection
    that lands between a synchronising host call and the next launch would leave the GPU idle
    inside the events and be billed to the kernels."""

    def __enter__(self):
        import gc
        gc.collect()
        self.was = gc.isenabled()
        gc.disable()

    def __exit__(self, *exc):
        import gc
        if self.was:
            gc.enable()


def _time_steps(torch, step, steps, flush, stream):
    """Run `steps` timed steps (L2 flushed before each, outside the events); returns the
    per-step (forward, adjoint, whole) milliseconds and the last step's outputs."""
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(steps)]
    out = None
    with _NoGC():
        for k in range(steps):
            # the previous step's outputs are released first, as a training loop consumes a
            # gradient before the next step: holding them would make every other step allocate
            # fresh device memory (cudaMalloc) inside its events
            out = None
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


def headline_checks(torch, engine, spec, r, gp, y0_np, rho_np, inv, dev, m: int = 64) -> dict:
    """Checks of the timed run's own gradients on m trajectories drawn as the reference's
    finite-difference test draws them (numpy default_rng(1).choice(n, m)):
      * oracle: the C oracle's replay and reverse pass over the mesh the GPU recorded --
        y_final of the replay against the GPU forward's, gradients against the adjoint's;
      * fd: central differences of sum(y_final_j**2) w.r.t. rho_j, step 1e-6 * max(1, |rho_j|),
        through the frozen mesh (the GPU replay of the same dts, never re-recorded), against
        the adjoint's gradient of mean(y_final**2) rescaled to that loss; the error measure
        max |g - fd| / max(|fd|, 1e-8) of tests/test_adjoint_replay.py:109-123 in the
        reference."""
    from oracle import oracle as O
    O.build()
    idx = np.random.default_rng(1).choice(r.n, m)
    rows = torch.tensor(idx, device=dev)
    dts = r.dts_rows(rows).contiguous()
    dts_np = dts.cpu().numpy()
    g = gp[rows].cpu().numpy()                    # d mean(y_final^2) / d rho_j
    yf = r.y_final[rows].cpu().numpy()
    y0s, ps = y0_np[idx], rho_np[idx]
    yf_o = O.replay("tsit5", "lorenz", y0s, ps, dts_np)
    _gy, g_o = O.replay_vjp("tsit5", "lorenz", y0s, ps, dts_np, (2.0 * inv) * yf)
    rowrel = lambda a, b: np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-300)
    q_y, q_g = rowrel(yf, yf_o), rowrel(g, g_o)
    # frozen-mesh central differences with the GPU replay of the sampled rows
    sub = engine.record_from_padded("tsit5", spec, dts, T0, checkpoint=1)
    y0_t = torch.tensor(y0s, device=dev)
    h = 1e-6 * np.maximum(np.abs(ps), 1.0)
    y_mid = engine.replay(sub, y0_t, torch.tensor(ps, device=dev), write_ckpt=False)
    y_p = engine.replay(sub, y0_t, torch.tensor(ps + h, device=dev), write_ckpt=False)
    y_m = engine.replay(sub, y0_t, torch.tensor(ps - h, device=dev), write_ckpt=False)
    y_p, y_m = y_p.cpu().numpy(), y_m.cpu().numpy()
    fd = ((y_p ** 2).sum(axis=1) - (y_m ** 2).sum(axis=1))[:, None] / (2.0 * h)
    g_sum = g / inv                               # d sum(y_final_j^2) / d rho_j
    q_fd = np.abs(g_sum - fd).max(axis=1) / np.maximum(np.abs(fd).max(axis=1), 1e-8)
    return {
        "rows": m, "sampler": "numpy default_rng(1).choice(n, 64)",
        "oracle": {"grad_rowrel_max": float(q_g.max()), "grad_rowrel_median": float(np.median(q_g)),
                   "y_final_rowrel_max": float(q_y.max()),
                   "within_1e-9": bool(q_g.max() <= 1e-9), "y_final_within_1e-10": bool(q_y.max() <= 1e-10)},
        "fd": {"eps": "1e-6*max(1,|rho|)", "loss": "sum(y_final_j**2)", "mesh": "frozen (GPU replay)",
               "rel_err_max": float(q_fd.max()), "rel_err_median": float(np.median(q_fd)),
               "within_1e-6": bool(q_fd.max() <= 1e-6)},
        "replay_equals_forward": bool(torch.equal(y_mid, r.y_final[rows])),
    }


def mixed_precision_config(args, dev) -> dict:
    """The mixed-precision configuration: Lotka-Volterra and Lorenz, n = 2^22 each, t in
    [0, 20], rtol 1e-6 / atol 1e-8, float32 stages against plain float64 -- each workload's
    float64 step rate and FP64 fraction, the float32-stage speed-up, and the float32-stage
    gradient's error against float64 on the same mesh (`meets_1e-6` is the bar)."""
    import copy

    import torch
    sub = copy.copy(args)
    sub.steps, sub.warmup, sub.no_cpu, sub.no_mixed = 3, 2, True, False
    sub.checkpoint, sub.schedule, sub.adjoint_variant = "auto", "auto", "auto"
    out = {}
    for name in ("lv_2e22", "lorenz_2e22"):
        line = measure_workload(sub, name, WORKLOAD_N[name], dev)
        g = line["groups"][0]
        m = line["mixed"] or {}
        err = (m.get("grad_rel_err_same_mesh") or {}).get(g["group"], {})
        out[name] = {"n": g["n"], "f64_value": line["value"], "f64_ms_per_step": line["ms_per_step"],
                     "f64_frac_of_fp64_peak": g["frac_of_fp64_peak"],
                     "mixed_value": m.get("value"), "mixed_ms_per_step": m.get("ms_per_step"),
                     "speedup_vs_f64": m.get("speedup_vs_f64"),
                     "grad_rel_err_same_mesh": err, "meets_1e-6": m.get("meets_1e-6"),
                     "oracle_parity_sample": line["oracle_parity_sample"].get(g["group"])}
        torch.cuda.empty_cache()
    return out


def other_configs(args, dev) -> dict:
    """The other workloads at their bench sizes, float64, in the default run's line (one
    GPU): the stiff Robertson batch (Rosenbrock23, 2^18), the uneven VdP batch with dense
    output (2^20), and the two 32-component fields integrated by groups of lanes (2^18
    each) -- per group the step time, the FP64 fraction and the 32-row oracle parity sample
    (the full lines: `bench.py --workload <name>`)."""
    import copy

    import torch
    sub = copy.copy(args)
    sub.steps, sub.warmup, sub.no_cpu, sub.no_mixed = 3, 2, True, True
    sub.checkpoint, sub.schedule, sub.adjoint_variant = "auto", "auto", "auto"
    out = {}
    for name in ("robertson_2e18", "vdp_uneven_saveat", "lorenz96_32", "linear_32"):
        line = measure_workload(sub, name, WORKLOAD_N[name], dev)
        out[name] = {"value": line["value"], "unit": UNIT, "ms_per_step": line["ms_per_step"],
                     "groups": [{k: g[k] for k in ("group", "method", "n", "ms",
                                                   "frac_of_fp64_peak", "checkpoint_every",
                                                   "record_len_max")}
                                for g in line["groups"]],
                     "oracle_parity_sample": line["oracle_parity_sample"],
                     "gpu_launches": line["gpu_launches"]}
        torch.cuda.empty_cache()
    return out


def replay_graph_config(dev, calls: int = 50) -> dict:
    """The small plain-method Lorenz case (n = 1024, y0 = (1, 0, 0), rho = linspace(20, 30),
    t in [0, 1], rtol = atol = 1e-8): the frozen-mesh replay + cotangent + reverse pass at a
    new point, launched one by one (replay, adjoint) and as the captured CUDA graph
    (engine.ReplayGraph) -- mean ms per gradient evaluation over ``calls`` calls each: queued
    back to back (CUDA events around the loop: the device's rate) and one at a time with the
    result waited for (host clock: the latency an optimiser that reads each gradient sees);
    results bit for bit equal."""
    import torch

    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    n = 1024
    spec = field_spec("lorenz")
    y0 = torch.tensor(np.tile([1.0, 0.0, 0.0], (n, 1)), device=dev)
    p = torch.linspace(20.0, 30.0, n, dtype=torch.float64, device=dev).reshape(n, 1)
    r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=1.0, rtol=1e-8, atol=1e-8,
                              checkpoint=2)
    cot = lambda yf: 2.0 * yf  # noqa: E731
    pts = [p * (1.0 + 1e-3 * k) for k in range(4)]

    def eager(pk):
        yf = engine.replay(r, y0, pk, write_ckpt=True)
        return engine.adjoint(r, pk, cot(yf))

    g = engine.ReplayGraph(r, y0, p, cot)
    same = all(torch.equal(eager(pk)[1], g(None, pk)[2]) for pk in pts)
    out = {}
    for name, fn in (("eager", eager), ("graph", lambda pk: g(None, pk))):
        for pk in pts:
            fn(pk)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(calls):
            fn(pts[k % len(pts)])
        e1.record()
        e1.synchronize()
        out[f"{name}_queued_ms"] = e0.elapsed_time(e1) / calls
        t0 = time.perf_counter()
        for k in range(calls):
            fn(pts[k % len(pts)])
            torch.cuda.synchronize()
        out[f"{name}_latency_ms"] = (time.perf_counter() - t0) * 1e3 / calls
    return {"workload": "lorenz n=1024, y0=(1,0,0), rho=linspace(20,30), t in [0,1], "
                        "rtol=atol=1e-8: replay + cotangent + reverse pass at a new point",
            **out, "latency_speedup": out["eager_latency_ms"] / out["graph_latency_ms"],
            "bitwise_equal": bool(same)}


def float32_route_config(args, dev, n: int = 1 << 20) -> dict:
    """The float32 route on the reference's f32 nonstiff cell (tests/test_f32_replay.py:84-117:
    diffeqgpu_lorenz, y0 = [1, 0, 0] + 0.01 N(0, 1) seed 0, rho = 28, t in [0, 1], rtol 1e-6 /
    atol 1e-9, loss sum(y_final**2)) at n = 2^20: float64 and float32 gradient steps (record
    + reverse pass), the record bytes of each, and the float32 gradient against the float64
    reverse pass over the same float32-recorded mesh (rel-L2 <= 1e-3 and cosine >= 1 - 1e-6
    are the reference's bars)."""
    import torch

    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    spec = field_spec("lorenz")
    rng = np.random.default_rng(0)
    y0 = torch.tensor(np.tile([1.0, 0.0, 0.0], (n, 1)) + 0.01 * rng.standard_normal((n, 3)),
                      device=dev)
    rho = torch.full((n, 1), 28.0, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    out = {"workload": "lorenz f32 cell, n=2^20, t in [0, 1], rtol 1e-6, atol 1e-9"}
    recs = {}
    for prec in ("float64", "float32"):
        ws = {"r": None}

        def step(events=None, prec=prec, ws=ws):
            if events:
                events[0].record(stream)
            r = engine.forward_record("tsit5", spec, y0, rho, t0=0.0, t1=1.0, rtol=1e-6,
                                      atol=1e-9, max_steps=100000, checkpoint="auto",
                                      precision=prec, workspace=ws["r"])
            ws["r"] = r
            if events:
                events[1].record(stream)
            ybar = 2.0 * r.y_final
            if events:
                events[2].record(stream)
            _g, gp = engine.adjoint(r, rho, ybar, want_y0=False, precision=prec)
            if events:
                events[3].record(stream)
            return r, gp

        for _ in range(3):
            step()
        torch.cuda.synchronize()
        fwd, adj, whole, (r, gp) = _time_steps(torch, step, 5, flush, stream)
        ms = float(np.mean(whole))
        recs[prec] = (r, gp)
        out[prec] = {"value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                     "fwd_ms": float(np.mean(fwd)), "adj_ms": float(np.mean(adj)),
                     "record_bytes": int(r.record_bytes),
                     "accepted_steps": int(r.n_acc.to(torch.int64).sum().item())}
    out["speedup_vs_f64"] = out["float64"]["ms_per_step"] / out["float32"]["ms_per_step"]
    out["record_bytes_ratio"] = out["float32"]["record_bytes"] / out["float64"]["record_bytes"]
    # same mesh: the float32 record's dts replayed and differentiated in float64
    r32, g32 = recs["float32"]
    r64 = engine.record_from_padded("tsit5", spec, r32.padded_dts().double(), 0.0,
                                    checkpoint=r32.ckpt_every)
    y64 = engine.replay(r64, y0, rho, write_ckpt=True)
    _g, g64 = engine.adjoint(r64, rho, 2.0 * y64, want_y0=False)
    a, b = g32.double().flatten(), g64.flatten()
    err = _grad_err(g32.double(), g64)
    err["cosine"] = float((a @ b / (a.norm() * b.norm())).item())
    err["meets_reference_bars"] = bool(err["rel_l2"] <= 1e-3 and err["cosine"] >= 1 - 1e-6)
    out["grad_vs_f64_same_mesh"] = err
    recs = r64 = None
    torch.cuda.empty_cache()
    return out


def run_b200(args) -> None:
    import torch
    import torch.distributed as dist

    from gradsolve_b200 import engine, flops
    from gradsolve_b200.fields import field_spec
    from gradsolve_b200.sharding import max_over_ranks

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
    if args.occupancy != "auto":  # pinned instances (a profile of a known kernel)
        f_occ, r_occ = (int(x) for x in args.occupancy.split(","))
        engine.set_occupancy(spec, f_occ, "forward")
        engine.set_occupancy(spec, r_occ, "reverse")
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
                                      schedule=args.schedule, variant=args.adjoint_variant)
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
    r = gp = None  # the warm-up's outputs (the record stays alive as the step's workspace)
    # the timed steps follow the warm-up directly (the GPU does not idle between them); the
    # step statistics are read from the last timed step, which integrates the same batch
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    from gradsolve_b200 import _lib
    launches0 = _lib.launch_count()
    fwd_ms, adj_ms, step_ms, (r, gp) = _time_steps(torch, step, args.steps, flush, stream)
    gpu_launches = _lib.launch_count() - launches0  # this library's kernels in the timed steps
    if world > 1:
        dist.barrier()
    ms_per_step = float(np.mean(step_ms))
    ms_per_step = max_over_ranks(ms_per_step, dev)
    value = n * world / (ms_per_step * 1e-3)
    assert int((r.status != 0).sum().item()) == 0, "solve failed"
    assert torch.isfinite(gp).all()
    att = int((r.n_acc.to(torch.int64) + r.n_rej.to(torch.int64)).sum().item())
    acc = int(r.n_acc.to(torch.int64).sum().item())
    S = int(r.n_acc.max().item())
    K = r.ckpt_every
    # the occupancy instances the timed steps ran (GS_OCC blocks per SM; 0 = default: 6 for
    # the forward, 5 for the K = 2 reverse pass)
    occ_f = engine._OCC.get(("tsit5", spec.key), 0)
    occ_r = engine._OCC_REV.get(("tsit5", spec.key), 0) if K == 2 else None
    # the timed run's own gradients, checked on 64 sampled trajectories (oracle + FD)
    # (rank 0 alone: only its line is printed, and the checks run no collective)
    checks = None if (args.no_checks or rank != 0) else headline_checks(
        torch, engine, spec, r, gp, y0_np, rho_np, inv, dev)

    # ---- the float32-stage variant on the same workload, and its accuracy ---------------
    mixed = None
    if not args.no_mixed:
        mstep = make_step("mixed")
        for _ in range(args.warmup):
            rm, gpm = mstep()
        rm = gpm = None
        m_fwd, m_adj, m_step, (rm, gpm) = _time_steps(torch, mstep, args.steps, flush, stream)
        m_ms = float(np.mean(m_step))
        m_ms = max_over_ranks(m_ms, dev)
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
    # ---- forward-only solve lane (no record, no checkpoints): trajectory-solves/s ------
    solve = {}
    if not args.no_solve:
        for prec in ("float64",) + (() if args.no_mixed else ("mixed",)):
            def fwd_only():
                return engine.forward_record("tsit5", spec, y0, rho, t0=T0, t1=T1, rtol=RTOL,
                                             atol=ATOL, max_steps=100000, record=False,
                                             precision=prec, schedule=args.schedule)
            for _ in range(args.warmup):
                fwd_only()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
            rs = None
            with _NoGC():
                for e0, e1 in evs:
                    rs = None  # release the previous solve's outputs before the next allocates
                    flush.zero_()
                    e0.record(stream)
                    rs = fwd_only()
                    e1.record(stream)
                torch.cuda.synchronize()
            s_ms = float(np.mean([e0.elapsed_time(e1) for e0, e1 in evs]))
            s_ms = max_over_ranks(s_ms, dev)
            s_att = int((rs.n_acc.to(torch.int64) + rs.n_rej.to(torch.int64)).sum().item())
            solve[prec] = {"value": n * world / (s_ms * 1e-3), "unit": "trajectory-solves/s",
                           "ms_per_step": s_ms, "attempts": s_att,
                           "tflops": flops.solve_flops("tsit5", "lorenz", s_att) / (s_ms * 1e-3) / 1e12}
    clk = clocks.stop()

    # ---- e2e through the public API, host buffers, H2D + D2H inside the timed region ----
    # the step workspaces above are done with: give their memory back before the API path
    # allocates its own records (it holds one closure's record at a time)
    step = mstep = r = rm = gpm = yf_sm = gp_sm = None
    import gc
    gc.collect()
    torch.cuda.empty_cache()
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
        ke = max(1, min(args.steps, 10))
        with _NoGC():
            t0 = time.perf_counter()
            marks = [t0]
            for _ in range(ke):
                e2e_step()  # ends on the loss read-back: the step's work is done
                marks.append(time.perf_counter())
            torch.cuda.synchronize()
            el = (time.perf_counter() - t0) / ke
        el = max_over_ranks(el, dev)
        e2e = {"value": n * world / el, "unit": UNIT,
               "h2d_bytes_per_step": int(y0_h.numel() * 8 + rho_h.numel() * 8),
               "d2h_bytes_per_step": int(grad_h.numel() * 8 + 8),
               "ms_per_step": el * 1e3, "api": "gradsolve_b200.grad_closure + torch autograd",
               "ms_steps": [round((b - a) * 1e3, 3) for a, b in zip(marks, marks[1:])]}

    # ---- the mixed-precision configuration (LV and Lorenz, 2^22 each, t in [0, 20]) -----
    # float64 vs float32 stages, speed and gradient error, in the default run's line (one GPU)
    config3 = None
    if world == 1 and not args.no_config3:
        clo = y0_h = rho_h = grad_h = None
        gc.collect()
        torch.cuda.empty_cache()
        config3 = mixed_precision_config(args, dev)
    f32_route = None
    if world == 1 and not args.no_config3:
        f32_route = float32_route_config(args, dev)
    others = None
    if world == 1 and not args.no_config3:
        others = other_configs(args, dev)
    graph_cfg = None
    if world == 1 and not args.no_config3:
        graph_cfg = replay_graph_config(dev)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant kernel -------------------------------------------
    fp64_peak = probe_fp64_tflops(torch, stream)
    for v in solve.values():
        v["frac_of_fp64_peak"] = v["tflops"] / fp64_peak
    peaks = measured_peaks()
    f_fwd = flops.solve_flops("tsit5", "lorenz", att)
    f_adj = flops.adjoint_flops("tsit5", "lorenz", acc)
    fwd_avg, adj_avg = float(np.mean(fwd_ms)), float(np.mean(adj_ms))
    kernels = {
        "tsit5_record_kernel": {"ms": fwd_avg, "tflops": f_fwd / (fwd_avg * 1e-3) / 1e12},
        # the reverse pass the run used: stage-keeping by default (its unrolled instance at
        # K = 2, which keeps the general one's 90 registers on Lorenz), recompute on request
        ("tsit5_adjoint_kernel" if args.adjoint_variant == "recompute"
         else "tsit5_adjoint_stages_k2_kernel" if K == 2
         else "tsit5_adjoint_stages_kernel"): {"ms": adj_avg,
                                               "tflops": f_adj / (adj_avg * 1e-3) / 1e12},
    }
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    nslots = math.ceil(S / K) + 1
    rec_bytes = acc * 8 * 2                     # dts written by the forward, read by the adjoint
    ck_bytes = n * nslots * 4 * 8 * 2          # checkpoints written + read
    io_bytes = n * (3 + 1) * 8 + n * (3 + 1 + 3) * 8
    achieved = kernels[dom]["tflops"]
    roofline = {
        "bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
        "frac": achieved / fp64_peak,
        "traffic": (DRAM_BYTES_PER_TRAJ[dom][K] * n if K in DRAM_BYTES_PER_TRAJ.get(dom, {})
                    else None),
        "traffic_source": (f"ncu capture of {dom} at n=2^18, K={K} (occupancy instances "
                           f"GS_OCC 5 / 4), scaled to n={n} (bytes grow with the trajectory "
                           "count)"
                           if K in DRAM_BYTES_PER_TRAJ.get(dom, {}) else
                           f"no ncu capture at K={K}"),
        "kernel": dom,
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
                   "occupancy": {"forward_blocks_per_sm": occ_f, "reverse_blocks_per_sm": occ_r,
                                 "policy": args.occupancy},
                   "l2": "flushed between timed steps (record traffic also >> L2)"},
        "gpu_launches": gpu_launches,
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
        "parity_sample": checks, "config3_mixed": config3, "float32_route": f32_route,
        "other_configs": others, "replay_graph": graph_cfg,
        "fwd_ms": fwd_avg, "adj_ms": adj_avg, "mixed": mixed, "solve": solve or None,
        "fwd_ms_steps": [round(x, 3) for x in fwd_ms], "adj_ms_steps": [round(x, 3) for x in adj_ms],
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()

# ------------------------------------------------------------------------------------
# the other workloads of the path: one JSON line each (the default run is the headline)
# ------------------------------------------------------------------------------------
class Group:
    """One homogeneous sub-batch: a method, a field and its inputs (numpy, host)."""

    def __init__(self, name, method, field, y0, p, t1, rtol, atol, *, t1v=None, ts=None,
                 dt0=None, cap=1024, loss="mean_sq", pilot_p=None):
        self.name, self.method, self.field = name, method, field
        self.y0, self.p, self.t1, self.rtol, self.atol = y0, p, t1, rtol, atol
        self.t1v, self.ts, self.dt0, self.cap, self.loss = t1v, ts, dt0, cap, loss
        self.pilot_p = pilot_p  # saveat target: the float64 solution at these parameters


def workload_groups(name: str, n: int, seed_shift: int):
    """Seeded inputs of each workload (numpy default_rng; seed + seed_shift per rank)."""
    if name == "lv_2e22":
        rng = np.random.default_rng(2 + seed_shift)
        prm = rng.uniform(0.5, 1.5, (n, 4))            # [alpha, beta, gamma, delta]
        y0 = rng.uniform(0.5, 2.0, (n, 2))
        return [Group("lv", "tsit5", "lv", y0, prm, 20.0, 1e-6, 1e-8, cap=256)]
    if name == "lorenz_2e22":
        y0, rho = make_inputs(n, 3 + seed_shift)
        return [Group("lorenz", "tsit5", "lorenz", y0, rho, 20.0, 1e-6, 1e-8, cap=1024)]
    if name == "robertson_2e18":
        rng = np.random.default_rng(4 + seed_shift)
        k = np.array([0.04, 3e7, 1e4]) * 10.0 ** rng.uniform(-0.5, 0.5, (n, 3))
        y0 = np.tile(np.array([1.0, 0.0, 0.0]), (n, 1))
        return [Group("robertson", "rosenbrock23", "robertson", y0, k, 1e4, 1e-6, 1e-10,
                      dt0=100.0, cap=1024, loss="last")]
    if name == "vdp_uneven_saveat":
        rng = np.random.default_rng(5 + seed_shift)
        mu = 10.0 ** rng.uniform(-1.0, 2.0, n)
        t1 = 10.0 ** rng.uniform(-1.0, math.log10(20.0), n)
        y0 = rng.uniform(-2.0, 2.0, (n, 2))
        mu_t = mu * (1.0 + 0.05 * np.random.default_rng(6 + seed_shift).normal(0.0, 1.0, n))
        ts = t1[:, None] * np.linspace(0.0, 1.0, 64)[None, :]
        out = []
        for gname, method, sel in (("vdp_tsit5", "tsit5", mu < 10.0),
                                   ("vdp_ros23", "rosenbrock23", mu >= 10.0)):
            out.append(Group(gname, method, "vdp", y0[sel], mu[sel, None], float(t1[sel].max()),
                             1e-6, 1e-9, t1v=t1[sel], ts=ts[sel],
                             cap=1024 if method == "tsit5" else 8192, loss="mse",
                             pilot_p=mu_t[sel, None]))
        return out
    if name == "lorenz96_32":  # 32 components: eight lanes per trajectory
        rng = np.random.default_rng(13 + seed_shift)
        F = rng.uniform(7.5, 8.5, (n, 1))
        y0 = F + rng.normal(0.0, 0.5, (n, 32))
        return [Group("lorenz96_32", "tsit5", "lorenz96_32", y0, F, 2.0, 1e-8, 1e-8, cap=512)]
    if name == "linear_32":
        rng = np.random.default_rng(15 + seed_shift)
        y0 = rng.uniform(-2.0, 2.0, (n, 32))
        return [Group("linear_32", "tsit5", "linear_32", y0, np.zeros((n, 1)), 4.0, 1e-10,
                      1e-10, cap=128)]
    raise ValueError(f"unknown workload {name!r}")


WORKLOAD_N = {"lv_2e22": 1 << 22, "lorenz_2e22": 1 << 22, "robertson_2e18": 1 << 18,
              "vdp_uneven_saveat": 1 << 20, "lorenz96_32": 1 << 18, "linear_32": 1 << 18}


def run_workload(args) -> None:
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    n = args.n if args.n != N_DEFAULT else WORKLOAD_N[args.workload]
    line = measure_workload(args, args.workload, n, dev, world, rank)
    if line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def measure_workload(args, name: str, n: int, dev, world: int = 1, rank: int = 0):
    """One workload's JSON line (rank 0; None on the other ranks): the float64 step timed
    over all groups, per-group FLOP rates, a 32-row oracle parity sample, the float32-stage
    variant with its same-mesh and own-mesh gradient errors, and the CPU baseline."""
    import torch

    from gradsolve_b200 import engine, flops
    from gradsolve_b200.fields import field_spec
    from gradsolve_b200.sharding import max_over_ranks

    stream = torch.cuda.current_stream()
    groups = workload_groups(name, n, 1000 * rank)
    n_tot = n * world
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    D = field_spec(groups[0].field).dim
    for g in groups:
        g.spec = field_spec(g.field)
        g.y0_d = torch.tensor(g.y0, device=dev)
        g.p_d = torch.tensor(g.p, device=dev)
        g.t1v_d = None if g.t1v is None else torch.tensor(g.t1v, device=dev)
        g.ts_d = None if g.ts is None else torch.tensor(g.ts, device=dev)
        g.target = None
        if g.pilot_p is not None:  # the float64 solution at the perturbed parameters
            pt = torch.tensor(g.pilot_p, device=dev)
            r = engine.forward_record(g.method, g.spec, g.y0_d, pt, t0=0.0, t1=g.t1,
                                      t1v=g.t1v_d, rtol=g.rtol, atol=g.atol, dt0=g.dt0,
                                      cap0=g.cap, checkpoint=8, saveat_ts=g.ts_d)
            engine.raise_on_failed(r, 100000, g.t1)
            g.target = r.ys
            del r
            torch.cuda.empty_cache()
        g.ws = None

    def cotangent(g, r, prec, ys=None):
        if g.loss == "mean_sq":
            return (2.0 / (n_tot * D)) * r.y_final
        if g.loss == "last":
            yb = torch.zeros_like(r.y_final)
            yb[:, 2] = 1.0
            return yb
        return (2.0 / (n_tot * ys.shape[1] * D)) * (ys - g.target)

    def group_step(g, prec, r=None):
        """forward (record) + loss cotangent + reverse pass; with ``r`` given, the record is
        replayed instead (same mesh) in precision ``prec``."""
        if r is None:
            # the forward also produces the saved states (no replay at the recording point)
            r = engine.forward_record(g.method, g.spec, g.y0_d, g.p_d, t0=0.0, t1=g.t1,
                                      t1v=g.t1v_d, rtol=g.rtol, atol=g.atol, dt0=g.dt0,
                                      max_steps=100000, cap0=g.cap, checkpoint=args.checkpoint,
                                      precision=prec, workspace=g.ws, schedule=args.schedule,
                                      saveat_ts=g.ts_d)
            g.ws = r
            replay_ck = False
        else:
            replay_ck = True
        if g.ts_d is None:
            if replay_ck:
                engine.replay(r, g.y0_d, g.p_d, write_ckpt=True, precision=prec)
            gy0, gp = engine.adjoint(r, g.p_d, cotangent(g, r, prec), want_y0=False,
                                     precision=prec, schedule=args.schedule,
                                     variant=args.adjoint_variant)
        else:
            if replay_ck:
                _yf, ys = engine.replay_saveat(r, g.y0_d, g.p_d, g.ts_d, write_ckpt=True,
                                               precision=prec)
            else:
                ys = r.ys
            gy0, gp = engine.adjoint_saveat(r, g.p_d, g.ts_d, cotangent(g, r, prec, ys),
                                            want_y0=False, precision=prec,
                                            schedule=args.schedule)
        return r, gp

    def prec_of(g, variant):
        return "mixed" if (variant == "mixed" and g.method == "tsit5") else "float64"

    def time_variant(variant):
        for _ in range(args.warmup):
            for g in groups:
                group_step(g, prec_of(g, variant))
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(len(groups) + 1)]
               for _ in range(args.steps)]
        outs = None
        from gradsolve_b200 import _lib
        launches0 = _lib.launch_count()
        nogc = _NoGC()
        nogc.__enter__()
        for e in evs:
            flush.zero_()
            e[0].record(stream)
            outs = []
            for k, g in enumerate(groups):
                outs.append(group_step(g, prec_of(g, variant)))
                e[k + 1].record(stream)
        torch.cuda.synchronize()
        nogc.__exit__(None, None, None)
        time_variant.launches = _lib.launch_count() - launches0
        per_group = [float(np.mean([e[k].elapsed_time(e[k + 1]) for e in evs]))
                     for k in range(len(groups))]
        steps_ms = [e[0].elapsed_time(e[-1]) for e in evs]
        whole = max_over_ranks(float(np.mean(steps_ms)), dev)
        time_variant.steps_ms = [round(x, 3) for x in steps_ms]
        return whole, per_group, outs

    clocks = ClockSampler(dev.index if dev.index is not None else 0)
    clocks.start()
    ms, per_group, outs = time_variant("float64")
    steps_ms = time_variant.steps_ms
    gpu_launches = time_variant.launches
    infos = []
    for g, t_ms, (r, gp) in zip(groups, per_group, outs):
        assert int((r.status != 0).sum().item()) == 0, f"{g.name}: solve failed"
        att = int((r.n_acc.to(torch.int64) + r.n_rej.to(torch.int64)).sum().item())
        acc = int(r.n_acc.to(torch.int64).sum().item())
        fl = flops.gradient_flops(g.method, g.field, att, acc)
        resteps = 0  # requested times strictly inside (t0, t1): one re-step each
        if g.ts is not None:
            t1row = (np.full(g.ts.shape[0], g.t1) if g.t1v is None else g.t1v)[:, None]
            resteps = int(((g.ts > 0.0) & (g.ts < t1row)).sum())
        fl_sv = fl + flops.saveat_flops(g.method, g.field, resteps)
        infos.append({"group": g.name, "method": g.method, "field": g.field, "n": r.n,
                      "attempts": att, "accepted": acc, "record_len_max": int(r.n_acc.max()),
                      "checkpoint_every": r.ckpt_every, "ms": t_ms,
                      "tflops": fl / (t_ms * 1e-3) / 1e12,
                      "saveat_points": None if g.ts is None else int(g.ts.shape[1]),
                      "saveat_resteps": resteps,
                      "tflops_incl_saveat": fl_sv / (t_ms * 1e-3) / 1e12})
        g.gp64 = gp.clone()
        g.r64 = r

    # parity at scale: 32 sampled rows of each group against the oracle on the GPU's own mesh
    from oracle import oracle as O
    O.build()
    parity = {}
    for g, info in zip(groups, infos):
        r = g.r64
        m = min(32, r.n)
        idx = np.sort(np.random.default_rng(1).choice(r.n, m, replace=False))
        dts = r.dts_rows(torch.tensor(idx, device=dev)).cpu().numpy()
        y0s, ps = g.y0[idx], g.p[idx]
        if g.ts is None:
            ybar = cotangent(g, r, "float64")[torch.tensor(idx, device=dev)].cpu().numpy()
            _oy, op = O.replay_vjp(g.method, g.field, y0s, ps, dts, ybar)
        else:
            _yf, ys = engine.replay_saveat(r, g.y0_d, g.p_d, g.ts_d, write_ckpt=False)
            ysbar = cotangent(g, r, "float64", ys)[torch.tensor(idx, device=dev)].cpu().numpy()
            _oy, op = O.replay_saveat_vjp(g.method, g.field, y0s, ps, dts, g.ts[idx], ysbar)
        got = g.gp64[torch.tensor(idx, device=dev)].cpu().numpy()
        den = np.maximum(np.abs(op).max(axis=1), 1e-300)
        q = np.abs(got - op).max(axis=1) / den
        parity[g.name] = {"rows": m, "grad_rowrel_max": float(q.max()),
                          "within_1e-9": bool(q.max() <= 1e-9)}

    outs = r = gp = None  # the float64 records stay reachable through g.r64 only
    mixed = None
    # (the float32-stage mode is not built for the states integrated by a group of lanes)
    if not args.no_mixed and any(g.method == "tsit5" for g in groups) and D <= 8:
        same = {}
        for g in groups:
            if g.method != "tsit5":
                continue
            _r, gp_sm = group_step(g, "mixed", r=g.r64)
            same[g.name] = _grad_err(gp_sm, g.gp64)
        for g in groups:  # release the float64 record before the mixed one is allocated
            g.r64 = g.ws = None
        torch.cuda.empty_cache()
        m_ms, m_groups, m_outs = time_variant("mixed")
        own = {}
        for g, (r, gp) in zip(groups, m_outs):
            if g.method == "tsit5":
                own[g.name] = _grad_err(gp, g.gp64)
        mixed = {"value": n_tot / (m_ms * 1e-3), "ms_per_step": m_ms, "group_ms": m_groups,
                 "speedup_vs_f64": ms / m_ms, "grad_rel_err_same_mesh": same,
                 "grad_rel_err_own_mesh": own,
                 "meets_1e-6": all(e["max"] <= 1e-6 for e in same.values()),
                 "note": "float32 stage increments on the tsit5 groups; rosenbrock23 groups "
                         "stay float64"}
    clk = clocks.stop()
    if rank != 0:
        return None
    fp64_peak = probe_fp64_tflops(torch, stream)
    for info in infos:
        info["frac_of_fp64_peak"] = info["tflops"] / fp64_peak
        info["frac_of_fp64_peak_incl_saveat"] = info["tflops_incl_saveat"] / fp64_peak
    cpu = None
    if world == 1 and not args.no_cpu:
        cpu = cpu_workload_rate(groups, args.cpu_seconds)
    line = {
        "workload": name, "metric": "trajectory grads/s (fwd+adjoint)",
        "value": n_tot / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "dtype": "f64", "data": "synthetic (seeded numpy default_rng)", "groups": infos,
        "fp64_peak_tflops": fp64_peak, "oracle_parity_sample": parity, "mixed": mixed,
        "cpu_baseline": cpu, "clocks": clk, "ms_steps": steps_ms, "gpu_launches": gpu_launches,
        "config": {"n_per_gpu": n, "checkpoint_policy": str(args.checkpoint),
                   "schedule": args.schedule, "l2": "flushed between timed steps"},
    }
    return line


def cpu_workload_rate(groups, target_s: float) -> dict:
    """The oracle port's record + replay adjoint on a bounded sample of each group, all host
    cores (saveat re-steps are not included: a lower bound of the CPU cost there)."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    total_t, total_n = 0.0, 0
    for g in groups:
        def run(m):
            t = time.perf_counter()
            rr = O.record(g.method, g.field, g.y0[:m], g.p[:m], 0.0, g.t1, g.rtol, g.atol,
                          dt0=g.dt0, cap=16384, nthreads=cores,
                          t1v=None if g.t1v is None else g.t1v[:m])
            O.replay_vjp(g.method, g.field, g.y0[:m], g.p[:m], rr["dts"],
                         np.ones_like(rr["y_final"]), nthreads=cores)
            return time.perf_counter() - t
        m = min(len(g.y0), cores * 8)
        dt = run(m)
        share = target_s / len(groups)
        m2 = int(min(len(g.y0), max(m, m * share / max(dt, 1e-3))))
        total_t += run(m2)
        total_n += m2
    return {"value": total_n / total_t, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{total_n} trajectories (first rows of each group), C restatement of the "
                      f"record + replay adjoint, {cores} host threads, {total_t:.1f} s"}



# ------------------------------------------------------------------------------------
# the reference's own published configuration (H200 NVL numbers, benchmarks/*.ipynb outputs)
# ------------------------------------------------------------------------------------
H200_GRAD_MS = {1e-3: 1.056, 1e-4: 1.479, 1e-5: 2.306, 1e-6: 3.417, 1e-7: 5.331, 1e-8: 8.342}
H200_FWD_MS = {1e-3: 0.276, 1e-6: 0.657, 1e-8: 1.424}


def run_published(args) -> None:
    """Lorenz, rho = linspace(0, 21, n), y0 = (1, 0, 0), t in [0, 1], atol = rtol * 1e-3
    (benchmarks/reverse_mode_vs_diffrax.py:59-65, benchmarks/forward_vs_diffeqgpu.py:116):
    the gradient of sum(y_final^2) on a recorded mesh (replay + reverse pass, what
    jax.grad of the closure runs per call) at n = 32768, and the forward-only solve lane at
    n = 524288, beside the reference's published H200 NVL times."""
    import torch

    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec

    spec = field_spec("lorenz")
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream()
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    def inputs(n):
        y0 = torch.tensor(np.tile([1.0, 0.0, 0.0], (n, 1)), device=dev)
        rho = torch.tensor(np.linspace(0.0, 21.0, n)[:, None], device=dev)
        return y0, rho

    def timed(fn, reps):
        for _ in range(max(3, args.warmup)):
            fn()
        ms = []
        with _NoGC():
            for _ in range(reps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
        return float(np.median(ms)), float(np.min(ms))

    grad = {}
    y0, rho = inputs(32768)
    for rtol in sorted(H200_GRAD_MS, reverse=True):
        r = engine.forward_record("tsit5", spec, y0, rho, t0=0.0, t1=1.0, rtol=rtol,
                                  atol=rtol * 1e-3, checkpoint="auto")
        ybar = 2.0 * r.y_final

        def g():
            engine.replay(r, y0, rho, write_ckpt=True)
            engine.adjoint(r, rho, ybar, want_y0=False)

        def rec():
            engine.forward_record("tsit5", spec, y0, rho, t0=0.0, t1=1.0, rtol=rtol,
                                  atol=rtol * 1e-3, checkpoint="auto", workspace=r)
        med, best = timed(g, args.steps)
        rmed, _ = timed(rec, args.steps)
        grad[f"{rtol:g}"] = {"ms": med, "ms_best": best, "h200_warp_replay_ms": H200_GRAD_MS[rtol],
                             "ratio_h200_over_b200": H200_GRAD_MS[rtol] / best,
                             "record_ms": rmed, "accepted_max": int(r.n_acc.max())}
    fwd = {}
    y0, rho = inputs(524288)
    for rtol in sorted(H200_FWD_MS, reverse=True):
        def f():
            engine.forward_record("tsit5", spec, y0, rho, t0=0.0, t1=1.0, rtol=rtol,
                                  atol=rtol * 1e-3, record=False)
        med, best = timed(f, args.steps)
        fwd[f"{rtol:g}"] = {"ms": med, "ms_best": best, "h200_cuda_tsit5_ms": H200_FWD_MS[rtol],
                            "ratio_h200_over_b200": H200_FWD_MS[rtol] / best,
                            "solves_per_s": 524288 / (best * 1e-3)}
    print(json.dumps({
        "workload": "published_h200", "n_gpus": 1, "dtype": "f64",
        "data": "Lorenz, rho = linspace(0, 21, n), y0 = (1, 0, 0), t in [0, 1], atol = rtol*1e-3",
        "gradient_n32768": grad, "forward_only_n524288": fwd,
        "timing": "B200: CUDA events around the kernels (L2 flushed), median and best of "
                  f"{args.steps}; H200: the reference's notebooks, host wall clock of the "
                  "jitted call, best of 5",
    }), flush=True)


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
    ap.add_argument("--no-config3", action="store_true",
                    help="skip the mixed-precision configuration (LV and Lorenz at 2^22), "
                         "the float32-route leg (the reference's f32 Lorenz cell at 2^20) and "
                         "the other workloads' summaries")
    ap.add_argument("--no-checks", action="store_true",
                    help="skip the oracle/FD checks of 64 sampled trajectories (outside timing)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--schedule", default="auto", choices=["auto", "static", "refill", "strided"])
    ap.add_argument("--adjoint-variant", default="auto", choices=["auto", "stages", "recompute"])
    ap.add_argument("--occupancy", default="auto",
                    help="'auto' (autotuned per field) or 'F,R': the GS_OCC blocks per SM of "
                         "the Lorenz forward and K = 2 reverse-pass instances (0 = default)")
    ap.add_argument("--workload", default="lorenz_2e20",
                    choices=["lorenz_2e20", "published_h200"] + sorted(WORKLOAD_N))
    args = ap.parse_args()
    if args.checkpoint not in ("sqrt", "all", "auto"):
        args.checkpoint = int(args.checkpoint)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "published_h200":
        run_published(args)
    elif args.workload != "lorenz_2e20":
        run_workload(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
