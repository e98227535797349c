"""Device-level driver: owns the workspaces and calls the libgsolve entry points.

PyTorch is used only as the device allocator and stream provider (tensors on the current
CUDA device, the current stream); all arithmetic happens in libgsolve.so.  The functions
here work on device tensors and return device tensors; the public API (``api.py``) and the
autograd adapter (``torch_adapter.py``) sit on top.

Record capacity follows the reference's device recorder (gradsolve/solvers/record_jax.py:
171-213): start with a bounded capacity, and if any trajectory reports a full record
(status 3) double it (up to ``max_steps``) and run again.  Failures then raise with the
reference's messages ("exhausted max_steps", "underflow").
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from .fields import FieldSpec

METHOD_TSIT5 = "tsit5"
METHOD_ROS23 = "rosenbrock23"
_PREC = {"float64": _lib.GS_PREC_F64, "mixed": _lib.GS_PREC_MIXED}
# scheduling flags (include/gsolve.h GS_SCHED_*): one thread per trajectory, persistent lanes
# refilled from a work counter, or persistent lanes with strided assignment
_SCHED = {"auto": 0x000, "static": 0x100, "refill": 0x200, "strided": 0x300}

# default record capacity before growth (the reference's device recorder starts at 1024)
DEFAULT_CAP0 = 1024
CTRL_DOUBLES = 256 // 8  # control block after the checkpoint slots (work counters)


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def ckpt_width(dim: int) -> int:
    return (dim + 2) & ~1


def choose_ckpt_every(policy, dim: int, n: int, cap: int, budget_bytes: Optional[int],
                      tuned: Optional[int] = None) -> int:
    """Checkpoint interval K (the segment length of the reverse pass).

    ``policy``: an int K; ``"all"`` (K = 1, every state stored, no recomputation);
    ``"sqrt"`` (K = ceil(sqrt(cap)), the classic sqrt(N) segment scheme); ``"auto"``: the
    segment length the autotuner measured fastest for this (method, field, precision)
    (``tuned``; 8 before tuning), raised until the checkpoints fit ``budget_bytes``
    (default: a quarter of the free device memory)."""
    kmax = _lib.lib().gs_max_ckpt_every()
    if isinstance(policy, int):
        if not 1 <= policy <= kmax:
            raise ValueError(f"checkpoint interval must be in [1, {kmax}]; got {policy}")
        return policy
    sq = max(2, min(kmax, int(math.ceil(math.sqrt(max(cap, 1))))))
    if policy == "all":
        return 1
    if policy == "sqrt":
        return sq
    if policy != "auto":
        raise ValueError(f"checkpoint policy must be 'auto', 'all', 'sqrt' or an int; got {policy!r}")
    if budget_bytes is None:
        free, _total = torch.cuda.mem_get_info()
        budget_bytes = free // 4
    K = tuned or 8
    while K < kmax and (cap // K + 2) * n * ckpt_width(dim) * 8 > budget_bytes:
        K *= 2
    return min(K, kmax)


# ---- checkpoint-interval autotuner ---------------------------------------------------------
# The reverse pass keeps each thread's K segment states (and, for Tsit5 float64, their stage
# inputs) in shared memory, so K trades recomputation and checkpoint traffic (none and the
# most at K = 1) against occupancy (the buffer grows with K).
# The best K depends on the field, the method and the precision; it is measured once per
# process on a sample of the caller's own trajectories and cached.
_TUNED: dict = {}
TUNE_CANDIDATES = (2, 3, 4, 6, 8, 12, 16)


def tuned_ckpt_every(method: str, spec: FieldSpec, precision: str) -> Optional[int]:
    return _TUNED.get((method, spec.key, precision))


def autotune_ckpt_every(method: str, spec: FieldSpec, y0: torch.Tensor, p: torch.Tensor, *,
                        t0: float, t1: float, rtol: float, atol: float,
                        t1v: Optional[torch.Tensor] = None, max_steps: int = 100000,
                        precision: str = "float64", sample: int = 1 << 17,
                        candidates=TUNE_CANDIDATES) -> int:
    """Time forward + reverse pass for each candidate K on up to ``sample`` trajectories
    (about two waves of the GPU) and cache the fastest."""
    m = min(y0.shape[0], sample)
    ys, ps = y0[:m].contiguous(), p[:m].contiguous()
    tv = None if t1v is None else t1v[:m].contiguous()
    best, best_ms = None, float("inf")
    for K in candidates:
        kw = dict(t0=t0, t1=t1, t1v=tv, rtol=rtol, atol=atol, max_steps=max_steps,
                  checkpoint=K, precision=precision)
        r = forward_record(method, spec, ys, ps, **kw)
        ybar = torch.ones_like(r.y_final)
        adjoint(r, ps, ybar, precision=precision)  # warm
        # forward (checkpoint writes grow as K shrinks) + reverse pass, buffers reused
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = forward_record(method, spec, ys, ps, workspace=r, **kw)
        adjoint(r, ps, ybar, precision=precision)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        if ms < best_ms:
            best, best_ms = K, ms
    _TUNED[(method, spec.key, precision)] = best
    return best


@dataclass
class Record:
    """Everything the forward leaves on the device for the adjoint."""
    method: str
    spec: FieldSpec
    n: int
    t0: float
    cap: int
    ckpt_every: int
    rec: torch.Tensor        # chunked dt record (flat float64)
    ckpt: torch.Tensor       # checkpoints (flat float64)
    y_final: torch.Tensor    # (n, D)
    n_acc: torch.Tensor      # (n,) int32
    n_rej: torch.Tensor      # (n,) int32
    status: torch.Tensor     # (n,) int32
    uneven: bool = False     # per-trajectory end times: the reverse pass refills lanes

    def padded_dts(self, S: Optional[int] = None) -> torch.Tensor:
        """The record in the reference's (n, S) zero-padded layout."""
        if S is None:
            S = int(self.n_acc.max().item()) if self.n else 0
        out = torch.zeros((self.n, S), dtype=torch.float64, device=self.rec.device)
        _lib.check(_lib.lib().gs_record_to_padded(self.n, self.cap, _ptr(self.rec),
                                                  _ptr(self.n_acc), S, _ptr(out), _stream()),
                   "gs_record_to_padded")
        return out

    def dts_rows(self, rows: torch.Tensor, S: Optional[int] = None) -> torch.Tensor:
        """Padded dts of the selected trajectories only (a torch gather of the
        chunk-interleaved record: step s of trajectory j sits at ((s//4)*n + j)*4 + s%4)."""
        rows = rows.to(device=self.rec.device, dtype=torch.int64)
        na = self.n_acc[rows].to(torch.int64)
        if S is None:
            S = int(na.max().item()) if rows.numel() else 0
        s = torch.arange(S, device=rows.device, dtype=torch.int64)
        idx = ((s // 4)[None, :] * self.n + rows[:, None]) * 4 + (s % 4)[None, :]
        out = self.rec[idx.clamp_max(self.rec.numel() - 1)]
        return torch.where(s[None, :] < na[:, None], out, torch.zeros_like(out))


def _alloc_record(n: int, cap: int, dim: int, K: int, device) -> tuple:
    L = _lib.lib()
    rec_elems = L.gs_record_bytes(n, cap) // 8
    slots = L.gs_ckpt_slots(cap, K)
    rec = torch.empty(max(rec_elems, 2), dtype=torch.float64, device=device)
    # checkpoint slots + the persistent kernels' 256-byte control block (gs_ckpt_bytes)
    ckpt = torch.empty(slots * n * ckpt_width(dim) + CTRL_DOUBLES, dtype=torch.float64,
                       device=device)
    return rec, ckpt


def forward_record(method: str, spec: FieldSpec, y0: torch.Tensor, p: torch.Tensor, *,
                   t0: float, t1: float, rtol: float, atol: float, dt0: Optional[float] = None,
                   t1v: Optional[torch.Tensor] = None, max_steps: int = 100000,
                   cap0: int = DEFAULT_CAP0, checkpoint="auto",
                   budget_bytes: Optional[int] = None, precision: str = "float64",
                   record: bool = True, workspace: Optional[Record] = None,
                   schedule: str = "auto") -> Record:
    """Adaptive solve on the device; with ``record`` the dts and checkpoints are kept.

    ``y0`` (n, D) and ``p`` (n, P) float64 contiguous device tensors.  ``workspace``: a Record
    from an earlier call of the same shape whose buffers are reused (overwritten) instead of
    allocating new ones -- the steady-state pattern of a training loop."""
    n = y0.shape[0]
    device = y0.device
    L = _lib.lib()
    fn = L.gs_tsit5_fwd_record if method == METHOD_TSIT5 else L.gs_ros23_fwd_record
    ws = workspace if (workspace is not None and workspace.n == n and
                       workspace.spec.dim == spec.dim) else None
    yf = ws.y_final if ws is not None else torch.empty_like(y0)
    n_acc = ws.n_acc if ws is not None else torch.empty(n, dtype=torch.int32, device=device)
    n_rej = ws.n_rej if ws is not None else torch.empty(n, dtype=torch.int32, device=device)
    status = ws.status if ws is not None else torch.empty(n, dtype=torch.int32, device=device)
    dt0_arg = -1.0 if dt0 is None else float(dt0)
    mode = _PREC[precision] | _SCHED[schedule]
    if not record:
        _lib.check(fn(spec.code, mode, n, _ptr(y0), _ptr(p), float(t0), _ptr(t1v),
                      float(t1), float(rtol), float(atol), dt0_arg, int(max_steps), 0, 1, None,
                      None, _ptr(yf), _ptr(n_acc), _ptr(n_rej), _ptr(status), _stream()),
                   fn.__name__)
        empty = torch.empty(0, dtype=torch.float64, device=device)
        return Record(method, spec, n, float(t0), 0, 1, empty, empty, yf, n_acc, n_rej, status,
                      uneven=t1v is not None)
    cap = max(1, min(int(cap0), int(max_steps)))
    if ws is not None and ws.cap > cap:
        cap = ws.cap
    if checkpoint == "auto" and tuned_ckpt_every(method, spec, precision) is None and n >= 4096:
        autotune_ckpt_every(method, spec, y0, p, t0=t0, t1=t1, t1v=t1v, rtol=rtol, atol=atol,
                            max_steps=max_steps, precision=precision)
    while True:
        K = choose_ckpt_every(checkpoint, spec.dim, n, cap, budget_bytes,
                              tuned_ckpt_every(method, spec, precision))
        if ws is not None and ws.cap == cap and ws.ckpt_every == K and ws.rec.numel() > 2:
            rec, ckpt = ws.rec, ws.ckpt
        else:
            rec, ckpt = _alloc_record(n, cap, spec.dim, K, device)
        _lib.check(fn(spec.code, mode, n, _ptr(y0), _ptr(p), float(t0), _ptr(t1v),
                      float(t1), float(rtol), float(atol), dt0_arg, int(max_steps), cap, K,
                      _ptr(rec), _ptr(ckpt), _ptr(yf), _ptr(n_acc), _ptr(n_rej), _ptr(status),
                      _stream()), fn.__name__)
        if n == 0 or cap >= max_steps or not bool((status == 3).any().item()):
            break
        cap = min(2 * cap, int(max_steps))
    return Record(method, spec, n, float(t0), cap, K, rec, ckpt, yf, n_acc, n_rej, status,
                  uneven=t1v is not None)


def raise_on_failed(r: Record, max_steps: int, t1) -> None:
    """Refuse an incomplete mesh, with the reference's messages
    (gradsolve/warp/warp_replay.py:167-173, gradsolve/solvers/record_jax.py:201-211)."""
    if r.n == 0:
        return
    bad = torch.nonzero(r.status != 0).flatten()
    if bad.numel() == 0:
        return
    i = int(bad[0].item())
    st = int(r.status[i].item())
    if st == 2:
        raise RuntimeError(
            f"record: trajectory {i} reached the step-size underflow floor before t1={t1} — a "
            "singular or non-finite field (check the RHS; loosen the tol or shorten the "
            "horizon); the recorded dt sequence is degenerate and a frozen replay of it would "
            "be silently wrong.")
    raise RuntimeError(
        f"record: {bad.numel()} trajectories (rows {bad[:8].tolist()}...) exhausted "
        f"max_steps={max_steps} before t1 — the recorded dt sequence is incomplete and a "
        "frozen replay of it would be silently wrong. Increase max_steps, loosen the tol, "
        "or shorten the horizon.")


def replay(r: Record, y0: torch.Tensor, p: torch.Tensor, *, write_ckpt: bool = True,
           precision: str = "float64") -> torch.Tensor:
    """Frozen-mesh replay at (y0, p); refreshes the checkpoints for a following adjoint."""
    L = _lib.lib()
    fn = L.gs_tsit5_replay if r.method == METHOD_TSIT5 else L.gs_ros23_replay
    yf = torch.empty_like(y0)
    _lib.check(fn(r.spec.code, _PREC[precision], r.n, _ptr(y0), _ptr(p), float(r.t0), _ptr(r.rec),
                  _ptr(r.n_acc), max(r.cap, 1), r.ckpt_every,
                  _ptr(r.ckpt) if write_ckpt else None, _ptr(yf), _stream()), fn.__name__)
    return yf


_ADJ = {"auto": 0x000, "recompute": 0x400, "stages": 0x800}


def adjoint(r: Record, p: torch.Tensor, ybar: torch.Tensor, *, want_y0: bool = True,
            want_p: bool = True, precision: str = "float64", schedule: str = "auto",
            variant: str = "auto"):
    """(dL/dy0, dL/dp) for cotangent ybar = dL/dy_final, using the record's checkpoints.
    ``schedule="auto"`` refills lanes from a work counter when the record came from an
    uneven batch (per-trajectory end times), else runs one thread per trajectory.
    ``variant`` (Tsit5, float64, one thread per trajectory): "stages" keeps each step's stage
    inputs from the segment's forward pass, "recompute" re-evaluates them in the reverse
    sweep; "auto" is "recompute" (the larger stage buffer costs more occupancy than the
    saved stage evaluations gain for the built-in fields)."""
    L = _lib.lib()
    fn = L.gs_tsit5_adjoint if r.method == METHOD_TSIT5 else L.gs_ros23_adjoint
    gy0 = torch.empty((r.n, r.spec.dim), dtype=torch.float64, device=p.device) if want_y0 else None
    gp = torch.empty((r.n, p.shape[1]), dtype=torch.float64, device=p.device) if want_p else None
    ybar = ybar.contiguous()
    if schedule == "auto" and r.uneven:
        schedule = "refill"
    flags = _PREC[precision] | _SCHED[schedule] | (_ADJ[variant] if fn is L.gs_tsit5_adjoint else 0)
    _lib.check(fn(r.spec.code, flags, r.n, _ptr(p), _ptr(r.rec),
                  _ptr(r.n_acc),
                  max(r.cap, 1), _ptr(r.ckpt), r.ckpt_every, _ptr(ybar), _ptr(gy0), _ptr(gp),
                  _stream()), fn.__name__)
    return gy0, gp


def record_from_padded(method: str, spec: FieldSpec, dts: torch.Tensor, t0: float,
                       checkpoint="auto", budget_bytes: Optional[int] = None) -> Record:
    """A Record built from a padded (n, S) dt array (e.g. the reference's own record).
    Checkpoints are filled by the next ``replay``."""
    dts = dts.contiguous()
    n, S = dts.shape
    cap = max(S, 1)
    K = choose_ckpt_every(checkpoint, spec.dim, n, cap, budget_bytes)
    rec, ckpt = _alloc_record(n, cap, spec.dim, K, dts.device)
    n_steps = torch.empty(n, dtype=torch.int32, device=dts.device)
    _lib.check(_lib.lib().gs_record_from_padded(n, S, _ptr(dts), S, _ptr(rec), cap,
                                                _ptr(n_steps), _stream()),
               "gs_record_from_padded")
    zeros = torch.zeros(n, dtype=torch.int32, device=dts.device)
    yf = torch.empty((n, spec.dim), dtype=torch.float64, device=dts.device)
    return Record(method, spec, n, float(t0), cap, K, rec, ckpt, yf, n_steps, zeros,
                  zeros.clone())


_METHOD_CODE = {METHOD_TSIT5: 0, METHOD_ROS23: 1}


def _ts_arg(ts: torch.Tensor, n: int):
    ts = ts.to(dtype=torch.float64).contiguous()
    if ts.ndim == 1:
        return ts, 0, ts.shape[0]
    if ts.ndim != 2 or ts.shape[0] != n:
        raise ValueError(f"saveat times must be (K,) or (n, K); got {tuple(ts.shape)}")
    return ts, ts.shape[1], ts.shape[1]


def replay_saveat(r: Record, y0: torch.Tensor, p: torch.Tensor, ts: torch.Tensor, *,
                  write_ckpt: bool = True, precision: str = "float64"):
    """Frozen-mesh replay with dense output at ``ts`` ((K,) shared or (n, K) per trajectory).
    Returns (y_final (n, D), ys (n, K, D)); refreshes the checkpoints for the adjoint."""
    ts, ld, K = _ts_arg(ts, r.n)
    yf = torch.empty_like(y0)
    ys = torch.empty((r.n, K, r.spec.dim), dtype=torch.float64, device=y0.device)
    _lib.check(_lib.lib().gs_replay_saveat(
        _METHOD_CODE[r.method], r.spec.code, _PREC[precision], r.n, _ptr(y0), _ptr(p),
        float(r.t0), _ptr(r.rec), _ptr(r.n_acc), max(r.cap, 1), r.ckpt_every,
        _ptr(r.ckpt) if write_ckpt else None, _ptr(ts), ld, K, _ptr(ys), _ptr(yf), _stream()),
        "gs_replay_saveat")
    return yf, ys


def adjoint_saveat(r: Record, p: torch.Tensor, ts: torch.Tensor, ysbar: torch.Tensor,
                   ybar: Optional[torch.Tensor] = None, *, want_y0: bool = True,
                   want_p: bool = True, precision: str = "float64"):
    """(dL/dy0, dL/dp) for cotangents ysbar = dL/dys (n, K, D) and ybar = dL/dy_final."""
    ts, ld, K = _ts_arg(ts, r.n)
    gy0 = torch.empty((r.n, r.spec.dim), dtype=torch.float64, device=p.device) if want_y0 else None
    gp = torch.empty((r.n, p.shape[1]), dtype=torch.float64, device=p.device) if want_p else None
    ysbar = ysbar.to(torch.float64).contiguous()
    ybar = None if ybar is None else ybar.to(torch.float64).contiguous()
    _lib.check(_lib.lib().gs_adjoint_saveat(
        _METHOD_CODE[r.method], r.spec.code, _PREC[precision], r.n, _ptr(p), _ptr(r.rec),
        _ptr(r.n_acc), max(r.cap, 1), _ptr(r.ckpt), r.ckpt_every, _ptr(ts), ld, K, _ptr(ysbar),
        _ptr(ybar), _ptr(gy0), _ptr(gp), _stream()), "gs_adjoint_saveat")
    return gy0, gp
