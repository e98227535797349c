"""Device-level driver: owns the workspaces and calls the libgsolve entry points.

PyTorch is used only as the device allocator and stream provider (tensors on the current
CUDA device, the current stream); all arithmetic happens in libgsolve.so.  The functions
here work on device tensors and return device tensors; the public API (``api.py``) and the
autograd adapter (``torch_adapter.py``) sit on top.

Record capacity starts bounded, as in the reference's device recorder
(gradsolve/solvers/record_jax.py:171-213).  Where the reference doubles the capacity and
re-solves the whole batch when any trajectory reports a full record (status 3), the rows that
overflowed are re-solved alone with a larger capacity, in further tiers (``RecordSet``), so
memory follows the step-count distribution of ragged batches.  Failures then raise with the
reference's messages ("exhausted max_steps", "underflow").
"""
from __future__ import annotations

import ctypes

import math
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from .fields import FieldSpec

METHOD_TSIT5 = "tsit5"
METHOD_ROS23 = "rosenbrock23"
_PREC = {"float64": _lib.GS_PREC_F64, "mixed": _lib.GS_PREC_MIXED,
         "float32": _lib.GS_PREC_F32}
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


def ckpt_width_f32(dim: int) -> int:
    """Floats per checkpoint row of the float32 route: the state and the time, rounded up
    to 16 bytes."""
    return (dim + 4) & ~3


def record_dtype(precision: str) -> torch.dtype:
    """Element type of the dt record and the checkpoints: float32 on the float32 route (the
    reference's f32 lane records float32 dts, gradsolve/warp/warp_replay.py:87-94), float64
    otherwise (the mixed mode keeps float64 time and state)."""
    return torch.float32 if precision == "float32" else torch.float64


# The checkpoint budget, a quarter of the memory free for the checkpoints (the device's free
# memory plus what the caching allocator holds unused).  cudaMemGetInfo took 0.1-1 ms per
# call on B200, inside every solve; the answer is kept while the allocator's reservation is
# unchanged (the steady state of a training loop) and for at most BUDGET_TTL seconds, so a
# solve re-queries after its own process allocated or released device memory.
BUDGET_TTL = 5.0
_BUDGET: dict = {}


def _checkpoint_budget() -> int:
    import time
    dev = torch.cuda.current_device()
    reserved = torch.cuda.memory_reserved()
    hit = _BUDGET.get(dev)
    now = time.monotonic()
    if hit is not None and hit[1] == reserved and now - hit[2] < BUDGET_TTL:
        return hit[0]
    free, _total = torch.cuda.mem_get_info()
    cached = reserved - torch.cuda.memory_allocated()
    budget = (free + max(cached, 0)) // 4
    _BUDGET[dev] = (budget, reserved, now)
    return budget


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
        budget_bytes = _checkpoint_budget()
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
_IN_TUNER = [0]  # nonzero while an autotuner runs its own forwards (no nested tuning)


def _tuner(fn):
    """Mark the autotuner's own forwards, so they start no other autotuner."""
    def run(*args, **kwargs):
        _IN_TUNER[0] += 1
        try:
            return fn(*args, **kwargs)
        finally:
            _IN_TUNER[0] -= 1
    run.__name__, run.__doc__, run.__wrapped__ = fn.__name__, fn.__doc__, fn
    return run
# On the float32 route a checkpoint row is 16 bytes for D <= 3 (against 32 in float64), and
# storing every state (K = 1) can win: the Lorenz f32 cell at 2^20 measured 1.37 ms per
# gradient step at K = 1 against 1.43 at K = 2 and 1.45 at K = 4.
TUNE_CANDIDATES_F32 = (1,) + TUNE_CANDIDATES


def tuned_ckpt_every(method: str, spec: FieldSpec, precision: str) -> Optional[int]:
    return _TUNED.get((method, spec.key, precision))


@_tuner
def autotune_ckpt_every(method: str, spec: FieldSpec, y0: torch.Tensor, p: torch.Tensor, *,
                        t0: float, t1: float, rtol: float, atol: float,
                        t1v: Optional[torch.Tensor] = None, max_steps: int = 100000,
                        precision: str = "float64", sample: int = 1 << 21,
                        candidates=None, reps: int = 3) -> int:
    """Time forward + reverse pass for each candidate K on up to ``sample`` trajectories and
    cache the fastest (best of ``reps`` timings).  The sample spans many waves of the GPU:
    the candidates' reverse passes hold different numbers of blocks per SM (their shared
    memory grows with K), and on a few waves the partial last wave, not the kernel, decides
    (a 2^19-row sample of a 2^22 Lotka-Volterra batch chose K = 4, where the full batch runs
    5% faster at K = 2)."""
    m = min(y0.shape[0], sample)
    ys, ps = y0[:m].contiguous(), p[:m].contiguous()
    tv = None if t1v is None else t1v[:m].contiguous()
    if candidates is None:
        candidates = TUNE_CANDIDATES_F32 if precision == "float32" else TUNE_CANDIDATES
    budget = _checkpoint_budget()
    row = 4 * ckpt_width_f32(spec.dim) if precision == "float32" else 8 * ckpt_width(spec.dim)
    best, best_ms = None, float("inf")
    for K in candidates:
        if (DEFAULT_CAP0 // K + 2) * m * row > budget and K != candidates[-1]:
            continue  # this interval's checkpoints would not fit beside the caller's data
        kw = dict(t0=t0, t1=t1, t1v=tv, rtol=rtol, atol=atol, max_steps=max_steps,
                  checkpoint=K, precision=precision)
        r = forward_record(method, spec, ys, ps, **kw)
        ybar = torch.ones_like(r.y_final)
        adjoint(r, ps, ybar, precision=precision)  # warm
        for _ in range(2):  # the steady state of a reused workspace (lanes ordered by cost,
            # the allocator's blocks cycling between two steps' outputs): no cudaMalloc timed
            r = forward_record(method, spec, ys, ps, workspace=r, **kw)
            adjoint(r, ps, ybar, precision=precision)
        # forward (checkpoint writes grow as K shrinks) + reverse pass, buffers reused
        ms = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = forward_record(method, spec, ys, ps, workspace=r, **kw)
            adjoint(r, ps, ybar, precision=precision)
            e1.record()
            e1.synchronize()
            ms = min(ms, e0.elapsed_time(e1))
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
    rec: torch.Tensor        # chunked dt record (flat; float32 on the float32 route)
    ckpt: torch.Tensor       # checkpoints (flat; float32 on the float32 route)
    y_final: torch.Tensor    # (n, D)
    n_acc: torch.Tensor      # (n,) int32
    n_rej: torch.Tensor      # (n,) int32
    status: torch.Tensor     # (n,) int32
    uneven: bool = False     # per-trajectory end times: the reverse pass refills lanes
    ys: Optional[torch.Tensor] = None  # (n, K, D) dense output of the forward, if asked for
    lane_order: Optional[torch.Tensor] = None  # the reverse pass's lane order, if prepared
    status_max: Optional[int] = None  # largest status code, once a check has read it

    @property
    def record_bytes(self) -> int:
        """Bytes of the dt record buffer (float32 on the float32 route)."""
        return self.rec.numel() * self.rec.element_size()

    def padded_dts(self, S: Optional[int] = None) -> torch.Tensor:
        """The record in the reference's (n, S) zero-padded layout, in the record's type."""
        if S is None:
            S = int(self.n_acc.max().item()) if self.n else 0
        if self.rec.dtype != torch.float64:
            return self.dts_rows(torch.arange(self.n, device=self.rec.device), S)
        out = torch.zeros((self.n, S), dtype=torch.float64, device=self.rec.device)
        L = _lib.lib_for(self.spec)
        _lib.check(L.gs_record_to_padded(self.n, self.cap, _ptr(self.rec), _ptr(self.n_acc), S,
                                         _ptr(out), _stream()), "gs_record_to_padded", L)
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


# capacity factor between the tiers of a RecordSet
TIER_GROWTH = 4


@dataclass
class RecordSet:
    """A record kept in tiers, for batches whose step counts differ widely.

    The first tier holds every trajectory at the first capacity.  Trajectories whose record
    overflowed it (status 3) are solved again, alone, with TIER_GROWTH times the capacity,
    and so on up to ``max_steps`` -- the reference's device recorder doubles the capacity and
    re-solves the whole batch instead (gradsolve/solvers/record_jax.py:192-199).  Memory then
    follows the step-count distribution (the sum over tiers of rows x capacity) rather than
    n x the longest trajectory, and each tier's launch holds trajectories of similar length.

    ``parts`` lists (rows, Record): rows None for a tier covering every trajectory, else the
    batch indices the tier covers, in the tier's order; a later tier's results replace the
    earlier ones for its rows.  Per-trajectory results are those of a single record (trajectories are
    independent and every tier runs the same kernel).

    A RecordSet passed back as the ``workspace`` of the next solve of the same batch is a
    plan: each trajectory goes straight to the tier that held it last time, every tier is
    launched at once on its own stream (the long-trajectory tier overlaps the bulk instead of
    following it), and only trajectories that outgrow their tier are re-solved.  The replay
    and reverse passes also run the tiers concurrently, on the same streams."""
    method: str
    spec: FieldSpec
    n: int
    t0: float
    parts: list
    sub: object               # the nested result of the overflowed rows (workspace reuse)
    y_final: torch.Tensor
    n_acc: torch.Tensor
    n_rej: torch.Tensor
    status: torch.Tensor
    uneven: bool = False
    ys: Optional[torch.Tensor] = None
    streams: Optional[list] = None  # per part: None (the caller's stream) or a side stream
    status_max: Optional[int] = None  # largest status code, once a check has read it

    @property
    def cap(self) -> int:
        return max(r.cap for _, r in self.parts)

    @property
    def ckpt_every(self) -> int:
        return self.parts[0][1].ckpt_every

    @property
    def nbytes(self) -> int:
        return sum(r.rec.numel() * r.rec.element_size() + r.ckpt.numel() * r.ckpt.element_size()
                   for _, r in self.parts)

    def plan_rows(self) -> list:
        """For each part, the rows whose final tier it is, longest first (by this record's
        step counts): lanes refilled from a work counter then take the long trajectories
        first, and the short ones fill in around them instead of the long ones ending last."""
        if len(self.parts) == 1 and self.parts[0][0] is None:  # one tier: no host sync
            cost = (self.n_acc + self.n_rej).to(torch.int64)
            return [torch.argsort(cost, descending=True, stable=True)]
        owner = torch.zeros(self.n, dtype=torch.int64, device=self.y_final.device)
        for k, (rows, _r) in enumerate(self.parts):
            if rows is None:
                owner.fill_(k)
            else:
                owner.index_fill_(0, rows, k)
        out = []
        for k in range(len(self.parts)):
            rows = torch.nonzero(owner == k).squeeze(1)
            if rows.numel() > 1:
                cost = (self.n_acc + self.n_rej).index_select(0, rows).to(torch.int64)
                rows = rows.index_select(0, torch.argsort(cost, descending=True, stable=True))
            out.append(rows)
        return out

    @property
    def record_bytes(self) -> int:
        return sum(r.record_bytes for _, r in self.parts)

    @property
    def rec_dtype(self) -> torch.dtype:
        return self.parts[0][1].rec.dtype

    def padded_dts(self, S: Optional[int] = None) -> torch.Tensor:
        if S is None:
            S = int(self.n_acc.max().item()) if self.n else 0
        out = torch.zeros((self.n, S), dtype=self.rec_dtype, device=self.y_final.device)
        for rows, r in self.parts:
            w = min(S, r.cap)  # a tier holds at most its capacity
            part = r.padded_dts(w)
            if rows is None:
                out[:, :w].copy_(part)
            else:
                out[:, :w].index_copy_(0, rows, part)
                out[rows, w:] = 0.0
        return out

    def dts_rows(self, rows: torch.Tensor, S: Optional[int] = None) -> torch.Tensor:
        rows = rows.to(device=self.y_final.device, dtype=torch.int64)
        if S is None:
            S = int(self.n_acc[rows].max().item()) if rows.numel() else 0
        out = torch.zeros((rows.numel(), S), dtype=self.rec_dtype, device=rows.device)
        for prow, r in self.parts:
            if prow is None:
                out.copy_(r.dts_rows(rows, S))
                continue
            if prow.numel() == 0:
                continue
            pos = _positions(prow, rows, self.n)
            hit = pos >= 0
            if bool(hit.any()):
                sel = torch.nonzero(hit).squeeze(1)
                out.index_copy_(0, sel, r.dts_rows(pos[sel], S))
        return out


def _positions(part_rows: torch.Tensor, rows: torch.Tensor, n: int) -> torch.Tensor:
    """For each of ``rows``, its position in ``part_rows`` (any order), or -1."""
    inv = torch.full((n,), -1, dtype=torch.int64, device=part_rows.device)
    inv.index_copy_(0, part_rows, torch.arange(part_rows.numel(), device=part_rows.device))
    return inv[rows]


def _parts(r):
    return r.parts if isinstance(r, RecordSet) else [(None, r)]


# Row moves of the tier plan (gather into a tier's order, scatter back) run in libgsolve's
# gs_move_rows: one thread per element, the contiguous side streamed.  (torch's index_select
# took 2.2 ms for the 4M parameter rows of a 2^22 Lotka-Volterra batch; this kernel is
# HBM-bound.)  Out-of-range indices are skipped and counted in a per-device counter, which
# the forward reads with its status codes in its one synchronisation (_status_max).
_ELEM_BYTES = {torch.float64: 8, torch.int64: 8, torch.float32: 4, torch.int32: 4}
_BAD_MOVES: dict = {}


def _bad_counter(device) -> torch.Tensor:
    key = device.index
    if key not in _BAD_MOVES:
        _BAD_MOVES[key] = torch.zeros(1, dtype=torch.int64, device=device)
    return _BAD_MOVES[key]


def _raise_bad_moves(c: torch.Tensor, n: int) -> None:
    c.zero_()
    raise RuntimeError(f"gs_move_rows skipped {n} out-of-range row indices (a tier plan "
                       "referenced rows outside its batch)")


def _check_moves(device) -> None:
    c = _BAD_MOVES.get(device.index)
    if c is not None:
        n = int(c.item())
        if n != 0:
            _raise_bad_moves(c, n)


def _status_max(status: torch.Tensor, device) -> int:
    """The largest status code of a forward's trajectories (0 ok, 1 not finished, 2 step-size
    underflow, 3 record full), read together with the row-move counter in one device-to-host
    copy: the forward's one synchronisation when nothing went wrong."""
    c = _BAD_MOVES.get(device.index)
    smax = status.max().to(torch.int64).reshape(1)
    vals = (torch.cat([smax, c]) if c is not None else smax).tolist()
    if c is not None and vals[1] != 0:
        _raise_bad_moves(c, int(vals[1]))
    return int(vals[0])


def _movable(t: torch.Tensor) -> bool:
    return t.is_cuda and t.dtype in _ELEM_BYTES and t.is_contiguous() and t.ndim >= 1


def _move_rows(src: torch.Tensor, idx: torch.Tensor, dst: torch.Tensor, scatter: bool) -> None:
    width = 1
    for d in src.shape[1:]:
        width *= int(d)
    if idx.numel() == 0 or width == 0:
        return
    idx = idx.to(device=src.device, dtype=torch.int64).contiguous()
    L = _lib.lib()
    _lib.check(L.gs_move_rows(int(scatter), _ELEM_BYTES[src.dtype], _ptr(src), _ptr(idx),
                              idx.numel(), width, dst.shape[0] if scatter else src.shape[0],
                              _ptr(dst), _ptr(_bad_counter(src.device)), _stream()),
               "gs_move_rows", L)


def _put_rows(dst: torch.Tensor, rows: torch.Tensor, src: torch.Tensor) -> None:
    """dst[rows] = src along the leading dimension, on the current stream."""
    if _movable(dst) and _movable(src) and src.dtype == dst.dtype:
        _move_rows(src, rows, dst, scatter=True)
    else:
        dst.index_copy_(0, rows, src)


def _take(t: Optional[torch.Tensor], rows: Optional[torch.Tensor]):
    """Rows of t on the current stream (t stays alive until this stream has read it)."""
    if t is None or rows is None:
        return t
    if t.is_cuda:
        t.record_stream(torch.cuda.current_stream())
    if _movable(t):
        out = torch.empty((rows.numel(),) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
        _move_rows(t, rows, out, scatter=False)
        return out
    return t.index_select(0, rows).contiguous()


def _take_ts(ts: Optional[torch.Tensor], rows: Optional[torch.Tensor]):
    return ts if (ts is None or ts.ndim == 1) else _take(ts, rows)


def _side_stream(device):
    """A stream for a tier that should overlap the others (None off the GPU: tiers then run
    one after another on the current stream).  Side streams carry the longer tiers, whose
    few, long trajectories set the end of the launch: they get the higher priority, so their
    blocks are placed first whenever the bulk tier and they compete for SMs."""
    if device.type != "cuda":
        return None
    return torch.cuda.Stream(device=device, priority=-1)


def _over_parts(r, fn) -> list:
    """fn(record, rows) -> tuple of tensors (or None), for every part of r.  The first part
    runs on the caller's stream; the others on their own streams, launched first so that
    they overlap it.  Returns [(rows, outputs)], all ready for use on the caller's stream."""
    parts = _parts(r)
    streams = getattr(r, "streams", None) or [None] * len(parts)
    if all(st is None for st in streams):
        return [(rows, fn(rr, rows)) for rows, rr in parts]
    main = torch.cuda.current_stream()
    out = [None] * len(parts)
    order = [k for k in range(len(parts)) if streams[k] is not None] + \
            [k for k in range(len(parts)) if streams[k] is None]
    for k in order:
        st = streams[k]
        if st is None:
            out[k] = fn(parts[k][1], parts[k][0])
            continue
        st.wait_stream(main)
        with torch.cuda.stream(st):
            out[k] = fn(parts[k][1], parts[k][0])
    for k in range(len(parts)):
        if streams[k] is not None:
            main.wait_stream(streams[k])
            for t in out[k]:
                if t is not None:
                    t.record_stream(main)
    return [(parts[k][0], out[k]) for k in range(len(parts))]


def _alloc_record(n: int, cap: int, dim: int, K: int, device,
                  precision: str = "float64") -> tuple:
    L = _lib.lib()
    slots = L.gs_ckpt_slots(cap, K)
    if precision == "float32":
        # half the float64 record (gs_record_bytes_prec); float32 checkpoint rows + the
        # 256-byte control block
        rec = torch.empty(max(L.gs_record_bytes_prec(_lib.GS_PREC_F32, n, cap) // 4, 4),
                          dtype=torch.float32, device=device)
        ckpt = torch.empty(slots * n * ckpt_width_f32(dim) + 2 * CTRL_DOUBLES,
                           dtype=torch.float32, device=device)
        return rec, ckpt
    rec_elems = L.gs_record_bytes(n, cap) // 8
    rec = torch.empty(max(rec_elems, 2), dtype=torch.float64, device=device)
    # checkpoint slots + the persistent kernels' 256-byte control block (gs_ckpt_bytes)
    ckpt = torch.empty(slots * n * ckpt_width(dim) + CTRL_DOUBLES, dtype=torch.float64,
                       device=device)
    return rec, ckpt


# ---- lanes per trajectory (fields of more than 8 components) -------------------------------
# A group of G lanes integrates one trajectory of a field with D > 8 (gs_coop.cuh).  The
# library builds the default G and, where the blocks stay 2..8 components, half and twice it
# (gs_lane_choices); fewer lanes hold more of the state each (more registers, fewer resident
# trajectories' worth of shuffles), more lanes fewer.  The autotuner times forward + reverse
# pass for each on a sample of the caller's trajectories and keeps the fastest per field.
_LANES: dict = {}  # field key -> lanes per trajectory chosen for it


def lane_choices(spec: FieldSpec) -> list:
    """Group sizes built for the field, the default first (one entry: [1] for the fields that
    run one thread per trajectory)."""
    L = _lib.lib_for(spec)
    buf = (ctypes.c_int * 8)()
    k = L.gs_lane_choices(spec.code, buf, 8)
    if k < 0:
        _lib.check(k, "gs_lane_choices", L)
    return list(buf[: min(k, 8)])


def set_lanes(spec: FieldSpec, lanes: Optional[int]) -> None:
    """Pin the lanes per trajectory of a field (None: back to the default / autotuning)."""
    if lanes is None:
        _LANES.pop(spec.key, None)
        return
    if lanes not in lane_choices(spec):
        raise ValueError(f"{lanes} lanes per trajectory are not built for {spec.key!r}; "
                         f"built: {lane_choices(spec)}")
    _LANES[spec.key] = int(lanes)


def _lanes_flag(method: str, spec: FieldSpec) -> int:
    G = _LANES.get(spec.key) if method == METHOD_TSIT5 else None
    return 0 if not G or G == 1 else int(G).bit_length() - 1 << 12


# ---- registers and occupancy of the float64 forward and reverse pass ---------------------
# For each field of up to 4 components the library builds the Tsit5 recording forward with its
# registers bounded for 6 resident blocks of 128 threads per SM (the default) and for 4, 5, 7
# and 8, the Tsit5 K = 2 stage-keeping reverse pass for 5 (the default), 3, 4 and 6, the
# Rosenbrock23 forward unbounded (the default) and for 4 and 6, and its K = 2 kept-factor
# reverse pass for 4 (the default), 3 and 5 (gs_occ_choices): more registers (longer-range
# scheduling, no spills) against more resident warps to hide the FP64 pipe's latency.  The
# instances compute the same values bit for bit; which runs fastest depends on the method and
# the field and is measured once per process on a sample of the caller's trajectories.
_OCC: dict = {}      # (method, field key) -> GS_OCC blocks per SM of the forward (0: default)
_OCC_REV: dict = {}  # (method, field key) -> the same for the reverse pass at K = 2
OCC_MARGIN = 0.01    # another instance replaces the default only when faster by more than 1%
MIXED = "tsit5/mixed"  # the tables' method key of the Tsit5 float32-stage reverse pass
_OCC_PASS = {(METHOD_TSIT5, "forward"): 0, (METHOD_TSIT5, "reverse"): 1,
             (METHOD_ROS23, "forward"): 2, (METHOD_ROS23, "reverse"): 3,
             (MIXED, "reverse"): 4}


def occ_choices(spec: FieldSpec, pass_: str = "forward", method: str = METHOD_TSIT5) -> list:
    """GS_OCC values built for the field's float64 recording forward ("forward") or K = 2
    reverse pass ("reverse") of ``method``, 0 (the default instance) first."""
    L = _lib.lib_for(spec)
    buf = (ctypes.c_int * 8)()
    k = L.gs_occ_choices(spec.code, _OCC_PASS[(method, pass_)], buf, 8)
    if k < 0:
        _lib.check(k, "gs_occ_choices", L)
    return list(buf[: min(k, 8)])


def set_occupancy(spec: FieldSpec, blocks: Optional[int], pass_: str = "forward",
                  method: str = METHOD_TSIT5) -> None:
    """Pin the occupancy instance of a field's forward or reverse pass (None: back to
    autotuning)."""
    table = _OCC if pass_ == "forward" else _OCC_REV
    if blocks is None:
        table.pop((method, spec.key), None)
        return
    if blocks not in occ_choices(spec, pass_, method):
        raise ValueError(f"no {pass_} instance for {blocks} blocks per SM is built for "
                         f"{spec.key!r} ({method}); built: {occ_choices(spec, pass_, method)}")
    table[(method, spec.key)] = int(blocks)


def _occ_applies(method, precision, schedule, t1v, saveat_ts) -> bool:
    """The recording forward that GS_OCC selects among: float64, one thread per trajectory
    (the static schedule, which "auto" is without per-trajectory end times)."""
    return (precision == "float64" and saveat_ts is None and
            (schedule == "static" or (schedule == "auto" and t1v is None)))


def _occ_flag(method, spec, precision, schedule, t1v, saveat_ts) -> int:
    if not _occ_applies(method, precision, schedule, t1v, saveat_ts):
        return 0
    return int(_OCC.get((method, spec.key)) or 0) << 15


def _occ_rev_flag(r, precision: str, schedule: str, variant: str) -> int:
    """The reverse pass's GS_OCC: at K = 2, the instance that keeps the replayed steps' stage
    inputs (Tsit5, float64 or float32-stage) or factors (Rosenbrock23, float64), one thread
    per trajectory."""
    if (r.ckpt_every != 2 or schedule not in ("auto", "static") or
            (r.method == METHOD_TSIT5 and variant == "recompute")):
        return 0
    if precision == "float64":
        key = (r.method, r.spec.key)
    elif precision == "mixed" and r.method == METHOD_TSIT5:
        key = (MIXED, r.spec.key)
    else:
        return 0
    return int(_OCC_REV.get(key) or 0) << 15


def _time_ms(fn, reps: int) -> float:
    best = float("inf")
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def _pick(times: dict) -> int:
    best = min(times, key=times.get)
    return 0 if times[best] > times[0] * (1.0 - OCC_MARGIN) else best


@_tuner
def autotune_occupancy(spec: FieldSpec, y0: torch.Tensor, p: torch.Tensor, *, t0: float,
                       t1: float, rtol: float, atol: float, max_steps: int = 100000,
                       checkpoint="auto", sample: int = 1 << 20, reps: int = 3,
                       method: str = METHOD_TSIT5, t1v: Optional[torch.Tensor] = None,
                       dt0: Optional[float] = None) -> tuple:
    """Time the float64 recording forward of each built occupancy instance on up to
    ``sample`` of the caller's trajectories (buffers reused, lanes ordered by cost as in a
    training loop's steady state; best of ``reps``), then, where the record's checkpoint
    interval is 2, the reverse pass's instances on that record; keep the fastest of each per
    field (the default unless another is faster by more than ``OCC_MARGIN``).  Returns
    (forward, reverse) GS_OCC values."""
    key = (method, spec.key)
    fwd, rev = occ_choices(spec, "forward", method), occ_choices(spec, "reverse", method)
    _OCC[key] = 0
    _OCC_REV[key] = 0
    if len(fwd) < 2:
        return 0, 0
    m = min(y0.shape[0], sample)
    ys, ps = y0[:m].contiguous(), p[:m].contiguous()
    tv = None if t1v is None else t1v[:m].contiguous()
    kw = dict(t0=t0, t1=t1, t1v=tv, dt0=dt0, rtol=rtol, atol=atol, max_steps=max_steps,
              checkpoint=checkpoint)
    box = {"r": None}

    def fwd_once():
        box["r"] = forward_record(method, spec, ys, ps, workspace=box["r"], **kw)

    times = {}
    for b in fwd:
        _OCC[key] = b
        for _ in range(2):  # warm: the record sized, the lanes ordered by cost
            fwd_once()
        times[b] = _time_ms(fwd_once, reps)
    _OCC[key] = _pick(times)
    r = box["r"]
    parts = [rr for _rows, rr in _parts(r)]
    if all(rr.ckpt_every == 2 for rr in parts) and len(rev) > 1:
        ybar = torch.ones_like(r.y_final)
        times = {}
        for b in rev:
            _OCC_REV[key] = b
            adjoint(r, ps, ybar)  # warm
            times[b] = _time_ms(lambda: adjoint(r, ps, ybar), reps)
        _OCC_REV[key] = _pick(times)
    return _OCC[key], _OCC_REV[key]


@_tuner
def autotune_mixed_reverse(spec: FieldSpec, y0: torch.Tensor, p: torch.Tensor, *, t0: float,
                           t1: float, rtol: float, atol: float, max_steps: int = 100000,
                           checkpoint="auto", sample: int = 1 << 20, reps: int = 3) -> int:
    """The float32-stage Tsit5 reverse pass's occupancy instance at K = 2, timed like
    ``autotune_occupancy``'s reverse half on a float32-stage record of up to ``sample`` of
    the caller's trajectories (0 where the record's interval is not 2)."""
    key = (MIXED, spec.key)
    choices = occ_choices(spec, "reverse", MIXED)
    _OCC_REV[key] = 0
    m = min(y0.shape[0], sample)
    ys, ps = y0[:m].contiguous(), p[:m].contiguous()
    r = forward_record(METHOD_TSIT5, spec, ys, ps, t0=t0, t1=t1, rtol=rtol, atol=atol,
                       max_steps=max_steps, checkpoint=checkpoint, precision="mixed")
    if len(choices) < 2 or any(rr.ckpt_every != 2 for _rows, rr in _parts(r)):
        return 0
    ybar = torch.ones_like(r.y_final)
    times = {}
    for b in choices:
        _OCC_REV[key] = b
        adjoint(r, ps, ybar, precision="mixed")  # warm
        times[b] = _time_ms(lambda: adjoint(r, ps, ybar, precision="mixed"), reps)
    _OCC_REV[key] = _pick(times)
    return _OCC_REV[key]


@_tuner
def autotune_lanes(spec: FieldSpec, y0: torch.Tensor, p: torch.Tensor, *, t0: float,
                   t1: float, rtol: float, atol: float, t1v: Optional[torch.Tensor] = None,
                   max_steps: int = 100000, sample: int = 1 << 16, reps: int = 2) -> int:
    """Time forward + reverse pass for each built group size on up to ``sample`` of the
    caller's trajectories; keep (and return) the fastest."""
    choices = lane_choices(spec)
    if len(choices) < 2:
        _LANES[spec.key] = choices[0]
        return choices[0]
    m = min(y0.shape[0], sample)
    ys, ps = y0[:m].contiguous(), p[:m].contiguous()
    tv = None if t1v is None else t1v[:m].contiguous()
    best, best_ms = choices[0], float("inf")
    for G in choices:
        _LANES[spec.key] = G
        kw = dict(t0=t0, t1=t1, t1v=tv, rtol=rtol, atol=atol, max_steps=max_steps, checkpoint=4)
        r = forward_record(METHOD_TSIT5, spec, ys, ps, **kw)
        ybar = torch.ones_like(r.y_final)
        adjoint(r, ps, ybar)
        ms = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = forward_record(METHOD_TSIT5, spec, ys, ps, workspace=r, **kw)
            adjoint(r, ps, ybar)
            e1.record()
            e1.synchronize()
            ms = min(ms, e0.elapsed_time(e1))
        if ms < best_ms:
            best, best_ms = G, ms
    _LANES[spec.key] = best
    return best


def forward_record(method: str, spec: FieldSpec, y0: torch.Tensor, p: torch.Tensor, *,
                   t0: float, t1: float, rtol: float, atol: float, dt0: Optional[float] = None,
                   t1v: Optional[torch.Tensor] = None, max_steps: int = 100000,
                   cap0: int = DEFAULT_CAP0, checkpoint="auto",
                   budget_bytes: Optional[int] = None, precision: str = "float64",
                   record: bool = True, workspace=None,
                   schedule: str = "auto", saveat_ts: Optional[torch.Tensor] = None):
    """Adaptive solve on the device; with ``record`` the dts and checkpoints are kept.

    ``y0`` (n, D) and ``p`` (n, P) float64 contiguous device tensors.  ``workspace``: the
    Record (or RecordSet) of an earlier call on the same batch, whose buffers are reused
    (overwritten) instead of allocating new ones -- the steady-state pattern of a training
    loop; a RecordSet also plans the tiers.  ``saveat_ts`` ((K,) shared or (n, K) per
    trajectory, sorted): the forward also produces the dense output ``r.ys`` (n, K, D) --
    what ``replay_saveat`` gives on the recorded mesh -- so the recording point needs no
    replay pass.  Returns a Record, or a RecordSet when trajectories needed more than ``cap0``
    steps."""
    n = y0.shape[0]
    device = y0.device
    ws = workspace if (workspace is not None and workspace.n == n and
                       workspace.spec.dim == spec.dim and workspace.method == method) else None
    kw = dict(t0=t0, t1=t1, rtol=rtol, atol=atol, dt0=dt0, max_steps=max_steps,
              checkpoint=checkpoint, budget_bytes=budget_bytes, precision=precision,
              schedule=schedule)
    if not record:
        L = _lib.lib_for(spec)
        fn = L.gs_tsit5_fwd_record if method == METHOD_TSIT5 else L.gs_ros23_fwd_record
        wsr = ws if isinstance(ws, Record) else None
        yf = wsr.y_final if wsr is not None else torch.empty_like(y0)
        n_acc, n_rej, status = (
            (wsr.n_acc, wsr.n_rej, wsr.status) if wsr is not None else
            tuple(torch.empty(n, dtype=torch.int32, device=device) for _ in range(3)))
        _lib.check(fn(spec.code, _PREC[precision] | _SCHED[schedule] | _lanes_flag(method, spec),
                      n, _ptr(y0), _ptr(p),
                      float(t0), _ptr(t1v), float(t1), float(rtol), float(atol),
                      -1.0 if dt0 is None else float(dt0), int(max_steps), 0, 1, None, None,
                      _ptr(yf), _ptr(n_acc), _ptr(n_rej), _ptr(status), _stream()),
                   fn.__name__, L)
        empty = torch.empty(0, dtype=torch.float64, device=device)
        return Record(method, spec, n, float(t0), 0, 1, empty, empty, yf, n_acc, n_rej, status,
                      uneven=t1v is not None)
    if (method == METHOD_TSIT5 and spec.dim > 8 and spec.key not in _LANES and n >= 4096 and
            precision == "float64"):
        autotune_lanes(spec, y0, p, t0=t0, t1=t1, t1v=t1v, rtol=rtol, atol=atol,
                       max_steps=max_steps)
    if checkpoint == "auto" and tuned_ckpt_every(method, spec, precision) is None and n >= 4096:
        autotune_ckpt_every(method, spec, y0, p, t0=t0, t1=t1, t1v=t1v, rtol=rtol, atol=atol,
                            max_steps=max_steps, precision=precision)
    occ_sched = "static" if method == METHOD_ROS23 and schedule == "auto" and isinstance(
        ws, RecordSet) else schedule  # (planned Rosenbrock23 tiers run one thread per row)
    if (precision == "mixed" and method == METHOD_TSIT5 and (MIXED, spec.key) not in _OCC_REV
            and not _IN_TUNER[0] and n >= 4096 and
            _occ_applies(method, "float64", occ_sched, t1v, saveat_ts)):
        autotune_mixed_reverse(spec, y0, p, t0=t0, t1=t1, rtol=rtol, atol=atol,
                               max_steps=max_steps, checkpoint=checkpoint)
    if ((method, spec.key) not in _OCC and not _IN_TUNER[0] and n >= 4096 and
            _occ_applies(method, precision, occ_sched, t1v, saveat_ts)):
        autotune_occupancy(spec, y0, p, t0=t0, t1=t1, rtol=rtol, atol=atol,
                           max_steps=max_steps, checkpoint=checkpoint, method=method,
                           t1v=t1v, dt0=dt0)
    if isinstance(ws, RecordSet):
        return _forward_planned(method, spec, y0, p, t1v, saveat_ts, ws, kw)
    if isinstance(ws, Record) and n > 32 and ws.rec.numel() > 2:
        # a record of the same batch: its step counts order the lanes (one tier, trajectories
        # sorted by last time's attempts, so a warp's lanes take similar numbers of steps and
        # none idles while the longest finishes)
        plan = RecordSet(method, spec, n, ws.t0, [(None, ws)], None, ws.y_final, ws.n_acc,
                         ws.n_rej, ws.status, uneven=ws.uneven, ys=ws.ys, streams=[None])
        return _forward_planned(method, spec, y0, p, t1v, saveat_ts, plan, kw)
    cap = max(1, min(int(cap0), int(max_steps)))
    r0 = _forward_one(method, spec, y0, p, t1v, saveat_ts, cap, ws, kw)
    return _grow(method, spec, y0, p, t1v, saveat_ts, r0, None, kw)


def _forward_one(method, spec, y0, p, t1v, saveat_ts, cap, ws, kw) -> Record:
    """One record of capacity ``cap`` for all rows of y0 (buffers reused from ws if they
    match), on the current stream."""
    n = y0.shape[0]
    device = y0.device
    L = _lib.lib_for(spec)
    precision = kw["precision"]
    ok = ws is not None and ws.n == n
    if kw["checkpoint"] == "auto" and ok and ws.cap == cap and ws.rec.numel() > 2:
        K = ws.ckpt_every  # sticky: the workspace's interval, so its buffers are reused
    else:
        K = choose_ckpt_every(kw["checkpoint"], spec.dim, n, cap, kw["budget_bytes"],
                              tuned_ckpt_every(method, spec, precision))
    yf = ws.y_final if ok else torch.empty_like(y0)
    n_acc, n_rej, status = ((ws.n_acc, ws.n_rej, ws.status) if ok else
                            tuple(torch.empty(n, dtype=torch.int32, device=device)
                                  for _ in range(3)))
    if (ok and ws.cap == cap and ws.ckpt_every == K and ws.rec.numel() > 2 and
            ws.rec.dtype == record_dtype(precision)):
        rec, ckpt = ws.rec, ws.ckpt
    else:
        rec, ckpt = _alloc_record(n, cap, spec.dim, K, device, precision)
    mode = (_PREC[precision] | _SCHED[kw["schedule"]] | _lanes_flag(method, spec) |
            _occ_flag(method, spec, precision, kw["schedule"], t1v, saveat_ts))
    dt0_arg = -1.0 if kw["dt0"] is None else float(kw["dt0"])
    args = (float(kw["t0"]), _ptr(t1v), float(kw["t1"]), float(kw["rtol"]), float(kw["atol"]),
            dt0_arg, int(kw["max_steps"]), cap, K, _ptr(rec), _ptr(ckpt), _ptr(yf),
            _ptr(n_acc), _ptr(n_rej), _ptr(status))
    ys = None
    if n == 0:
        pass
    elif saveat_ts is None:
        fn = L.gs_tsit5_fwd_record if method == METHOD_TSIT5 else L.gs_ros23_fwd_record
        _lib.check(fn(spec.code, mode, n, _ptr(y0), _ptr(p), *args, _stream()), fn.__name__, L)
    else:
        ts, ld, Kt = _ts_arg(saveat_ts, n)
        ys = (ws.ys if ok and ws.ys is not None and ws.ys.shape == (n, Kt, spec.dim)
              else torch.empty((n, Kt, spec.dim), dtype=torch.float64, device=device))
        _lib.check(L.gs_fwd_record_saveat(_METHOD_CODE[method], spec.code, mode, n, _ptr(y0),
                                          _ptr(p), *args, _ptr(ts), ld, Kt, _ptr(ys),
                                          _stream()), "gs_fwd_record_saveat", L)
    if n == 0 and saveat_ts is not None:
        ys = torch.empty((0, _ts_arg(saveat_ts, 0)[2] if saveat_ts.ndim == 1 else
                          saveat_ts.shape[1], spec.dim), dtype=torch.float64, device=device)
    return Record(method, spec, n, float(kw["t0"]), cap, K, rec, ckpt, yf, n_acc, n_rej,
                  status, uneven=t1v is not None, ys=ys)


def _assemble(method, spec, n, device, parts, t1v, saveat_ts, streams, sub=None):
    """Batch-order results of the parts (later parts win for shared rows)."""
    D = spec.dim
    yf = torch.empty((n, D), dtype=torch.float64, device=device)
    n_acc, n_rej, status = (torch.empty(n, dtype=torch.int32, device=device) for _ in range(3))
    ys = None
    for rows, rr in parts:
        if rows is None:
            yf.copy_(rr.y_final), n_acc.copy_(rr.n_acc), n_rej.copy_(rr.n_rej)
            status.copy_(rr.status)
        else:
            _put_rows(yf, rows, rr.y_final)
            _put_rows(n_acc, rows, rr.n_acc)
            _put_rows(n_rej, rows, rr.n_rej)
            _put_rows(status, rows, rr.status)
        if rr.ys is not None:
            if ys is None:
                ys = torch.empty((n,) + tuple(rr.ys.shape[1:]), dtype=torch.float64,
                                 device=device)
            if rows is None:
                ys.copy_(rr.ys)
            else:
                _put_rows(ys, rows, rr.ys)
    return RecordSet(method, spec, n, float(parts[0][1].t0), parts, sub, yf, n_acc, n_rej,
                     status, uneven=t1v is not None, ys=ys, streams=streams)


def _grow(method, spec, y0, p, t1v, saveat_ts, r0, streams, kw):
    """Re-solve the rows of r0 (a Record over all of y0's rows) that overflowed it, in further
    tiers; r0 alone when nothing overflowed."""
    n = y0.shape[0]
    max_steps = int(kw["max_steps"])
    if n == 0 or r0.cap >= max_steps:
        return r0
    r0.status_max = _status_max(r0.status, y0.device)
    if r0.status_max < 3:  # no row overflowed the record
        return r0
    rows = torch.nonzero(r0.status == 3).squeeze(1)
    sub = forward_record(method, spec, _take(y0, rows), _take(p, rows), t1v=_take(t1v, rows),
                         cap0=min(TIER_GROWTH * r0.cap, max_steps),
                         saveat_ts=_take_ts(saveat_ts, rows), **kw)
    parts = [(None, r0)]
    for srows, rr in _parts(sub):
        parts.append((rows if srows is None else rows.index_select(0, srows), rr))
    out = _assemble(method, spec, n, y0.device, parts, t1v, saveat_ts,
                    [None] + [_side_stream(y0.device) for _ in parts[1:]], sub)
    # in the first tier the overflowed rows become empty (0 steps), so its replay and reverse
    # passes skip them instead of integrating a truncated record whose result is replaced
    r0.n_acc.index_fill_(0, rows, 0)
    return out


def _forward_planned(method, spec, y0, p, t1v, saveat_ts, ws: RecordSet, kw):
    """The tiers of ws, re-solved directly: every trajectory in the tier that held it last
    time, all tiers at once (side streams), overflowing rows re-solved afterwards."""
    n = y0.shape[0]
    rows_by_part = ws.plan_rows()
    keep = [k for k in range(len(ws.parts)) if rows_by_part[k].numel() > 0]
    old = [ws.streams[k] if ws.streams is not None else None for k in keep]
    streams = [None] + [old[i] if old[i] is not None else _side_stream(y0.device)
                        for i in range(1, len(keep))]
    plan = [(rows_by_part[k], ws.parts[k][1]) for k in keep]
    # A planned tier's rows come sorted by their previous cost, so neighbouring threads take
    # similar numbers of attempts and one thread per trajectory stays balanced.  Rosenbrock23
    # then runs that way: it is latency-bound, and the one-thread kernel holds more warps
    # than the refilled lanes (uneven VdP: its group 36.6 -> 35.5 ms); Tsit5 keeps the
    # refilled lanes (its group measured 11.44 ms refilled, 11.54 one thread per trajectory).
    kwp = kw
    if method == METHOD_ROS23 and kw["schedule"] == "auto":
        kwp = dict(kw, schedule="static")
    launch = lambda rows, wsr: _forward_one(  # noqa: E731
        method, spec, _take(y0, rows), _take(p, rows), _take(t1v, rows),
        _take_ts(saveat_ts, rows), wsr.cap, wsr, kwp)
    out = [None] * len(plan)
    if all(st is None for st in streams):
        out = [(rows, launch(rows, wsr)) for rows, wsr in plan]
    else:
        main = torch.cuda.current_stream()
        for i in list(range(1, len(plan))) + [0]:  # the side tiers first, to overlap tier 0
            rows, wsr = plan[i]
            st = streams[i]
            if st is not None:
                st.wait_stream(main)
            with torch.cuda.stream(st if st is not None else main):
                out[i] = (rows, launch(rows, wsr))
        for i in range(1, len(plan)):
            main.wait_stream(streams[i])
            rr = out[i][1]
            for t in (rr.y_final, rr.n_acc, rr.n_rej, rr.status, rr.ys):
                if t is not None:
                    t.record_stream(main)
    res = _assemble(method, spec, n, y0.device, out, t1v, saveat_ts, streams)
    # trajectories that outgrew their planned tier: solved again with more capacity
    res.status_max = _status_max(res.status, y0.device)
    if res.status_max < 3:
        return res
    over = torch.nonzero(res.status == 3).squeeze(1)
    cap_of_row = torch.zeros(n, dtype=torch.int64, device=y0.device)
    for rows, rr in out:
        cap_of_row.index_fill_(0, rows, rr.cap)
    grown = min(TIER_GROWTH * int(cap_of_row[over].max().item()), int(kw["max_steps"]))
    sub = forward_record(method, spec, _take(y0, over), _take(p, over), t1v=_take(t1v, over),
                         cap0=grown, saveat_ts=_take_ts(saveat_ts, over), **kw)
    parts = list(out)
    for rows, rr in out:  # empty the overflowed rows in the tiers that held them
        pos = _positions(rows, over, n)
        hit = pos >= 0
        if bool(hit.any()):
            rr.n_acc.index_fill_(0, pos[hit], 0)
    for srows, rr in _parts(sub):
        parts.append((over if srows is None else over.index_select(0, srows), rr))
    return _assemble(method, spec, n, y0.device, parts, t1v, saveat_ts,
                     streams + [_side_stream(y0.device) for _ in parts[len(out):]],
                     sub)


def raise_on_failed(r: Record, max_steps: int, t1) -> None:
    """Refuse an incomplete mesh, with the reference's messages
    (gradsolve/warp/warp_replay.py:167-173, gradsolve/solvers/record_jax.py:201-211)."""
    if r.n == 0 or r.status_max == 0:  # (the forward's own check read every status)
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


def replay(r, y0: torch.Tensor, p: torch.Tensor, *, write_ckpt: bool = True,
           precision: str = "float64") -> torch.Tensor:
    """Frozen-mesh replay at (y0, p); refreshes the checkpoints for a following adjoint."""
    res = _over_parts(r, lambda rr, rows: (_replay_one(
        rr, _take(y0, rows), _take(p, rows), write_ckpt=write_ckpt, precision=precision),))
    return _scatter(r, res, 0)


def _scatter(r, res, i):
    """Output i of every part, in batch order (later parts win for shared rows)."""
    first = res[0][1][i]
    if len(res) == 1 and res[0][0] is None:
        return first
    if first is None:
        return None
    out = torch.empty((r.n,) + tuple(first.shape[1:]), dtype=first.dtype, device=first.device)
    for rows, outs in res:
        if rows is None:
            out.copy_(outs[i])
        else:
            _put_rows(out, rows, outs[i])
    return out


def _replay_one(r: Record, y0: torch.Tensor, p: torch.Tensor, *, write_ckpt: bool,
                precision: str) -> torch.Tensor:
    L = _lib.lib_for(r.spec)
    fn = L.gs_tsit5_replay if r.method == METHOD_TSIT5 else L.gs_ros23_replay
    yf = torch.empty_like(y0)
    _lib.check(fn(r.spec.code, _PREC[precision] | _lanes_flag(r.method, r.spec), r.n,
                  _ptr(y0), _ptr(p), float(r.t0),
                  _ptr(r.rec), _ptr(r.n_acc), max(r.cap, 1), r.ckpt_every,
                  _ptr(r.ckpt) if write_ckpt else None, _ptr(yf), _stream()), fn.__name__, L)
    return yf


_ADJ = {"auto": 0x000, "recompute": 0x400, "stages": 0x800, "pairs": 0xC00}


def adjoint(r, p: torch.Tensor, ybar: torch.Tensor, *, want_y0: bool = True,
            want_p: bool = True, precision: str = "float64", schedule: str = "auto",
            variant: str = "auto"):
    """(dL/dy0, dL/dp) for cotangent ybar = dL/dy_final, using the record's checkpoints.
    ``schedule="auto"`` refills lanes from a work counter when the record came from an
    uneven batch (per-trajectory end times), else runs one thread per trajectory.
    ``variant`` (Tsit5, float64, one thread per trajectory): "stages" keeps the stage inputs
    the segment's replay evaluates, "recompute" re-evaluates every step's stages in the
    reverse sweep; "auto" is "stages" while its buffer leaves it at least 3/5 of the
    recomputing kernel's resident threads, else "recompute".  On the float32 route (Tsit5)
    "pairs" runs two trajectories per thread in packed float32x2 arithmetic (built-in
    nonstiff fields), "recompute" one per thread, and "auto" is "pairs" where it is built."""
    if schedule == "auto" and r.uneven and precision != "float32":
        schedule = "refill"  # (the float32 route runs one thread per trajectory)
    res = _over_parts(r, lambda rr, rows: _adjoint_one(
        rr, _take(p, rows), _take(ybar, rows), want_y0=want_y0, want_p=want_p,
        precision=precision, schedule=schedule, variant=variant, in_batch_order=rows is None))
    return _scatter(r, res, 0), _scatter(r, res, 1)


def prepare_lane_order(r) -> Optional[torch.Tensor]:
    """Queue the sort that orders a batch-order record's reverse lanes by step count (longest
    first) on the current stream, so it runs while the host prepares the cotangent; the
    reverse pass picks it up.  Planned records (already ordered by cost) need none."""
    if isinstance(r, Record) and r.n >= ORDER_LANES_MIN:
        r.lane_order = torch.argsort(r.n_acc, descending=True, stable=True)
        return r.lane_order
    return None


# A record in batch order (a fresh forward; a planned tier is already ordered by cost) runs its
# reverse pass with the lanes ordered by step count, longest first, from this many
# trajectories up (the sort costs ~0.1 ms at 2^20 and saves the idle lanes of warps whose
# trajectories' step counts differ).
ORDER_LANES_MIN = 1 << 12


def _adjoint_one(r: Record, p: torch.Tensor, ybar: torch.Tensor, *, want_y0: bool,
                 want_p: bool, precision: str, schedule: str, variant: str,
                 in_batch_order: bool = False):
    L = _lib.lib_for(r.spec)
    fn = L.gs_tsit5_adjoint if r.method == METHOD_TSIT5 else L.gs_ros23_adjoint
    gy0 = torch.empty((r.n, r.spec.dim), dtype=torch.float64, device=p.device) if want_y0 else None
    gp = torch.empty((r.n, p.shape[1]), dtype=torch.float64, device=p.device) if want_p else None
    ybar = ybar.contiguous()
    if schedule == "auto" and r.uneven and precision != "float32":
        schedule = "refill"
    flags = (_PREC[precision] | _SCHED[schedule] | _lanes_flag(r.method, r.spec) |
             (_ADJ[variant] if r.method == METHOD_TSIT5 else 0) |
             _occ_rev_flag(r, precision, schedule, variant))
    if in_batch_order and r.n >= ORDER_LANES_MIN and schedule in ("auto", "static"):
        order = r.lane_order if r.lane_order is not None else prepare_lane_order(r)
        _lib.check(L.gs_adjoint_ordered(_METHOD_CODE[r.method], r.spec.code, flags, r.n, _ptr(p),
                                        _ptr(r.rec), _ptr(r.n_acc), max(r.cap, 1), _ptr(r.ckpt),
                                        r.ckpt_every, _ptr(ybar), _ptr(gy0), _ptr(gp),
                                        _ptr(order), _stream()), "gs_adjoint_ordered", L)
        return gy0, gp
    _lib.check(fn(r.spec.code, flags, r.n, _ptr(p), _ptr(r.rec), _ptr(r.n_acc),
                  max(r.cap, 1), _ptr(r.ckpt), r.ckpt_every, _ptr(ybar), _ptr(gy0), _ptr(gp),
                  _stream()), fn.__name__, L)
    return gy0, gp


class ReplayGraph:
    """The frozen-mesh replay, a cotangent and the reverse pass, captured once as a CUDA
    graph and re-launched as one unit (gradsolve/warp/warp_replay.py:30-55 and 186-237, the
    replay and its gradient, which the reference runs as one jitted computation).

    For loops that evaluate the same recorded mesh at many points -- an optimiser stepping
    the parameters of a fixed mesh, a finite-difference or Newton iteration -- the per-call
    host work (argument checks, the reverse pass's occupancy queries, the launches) is paid
    once at capture.  ``cotangent(y_final) -> ybar`` is the loss's derivative written with
    torch operations; it is captured with the kernels.  ``graph(y0, p)`` copies the point
    into the graph's input buffers, re-launches, and returns (y_final, gy0, gp): the graph's
    own output buffers, overwritten by the next call (clone what must be kept).  Results are
    bit for bit those of ``replay`` + ``adjoint`` called one by one.

    Float64, one Record (a RecordSet's tiers run on side streams and are not captured); the
    record's buffers must stay alive and unmodified while the graph is used (a new forward
    into the same record changes the mesh the graph replays)."""

    def __init__(self, r, y0: torch.Tensor, p: torch.Tensor, cotangent, *,
                 want_y0: bool = True, want_p: bool = True):
        if not isinstance(r, Record):
            raise TypeError("ReplayGraph captures a single Record (not the tiers of a RecordSet)")
        if r.rec.dtype != torch.float64:
            raise TypeError("ReplayGraph captures the float64 replay only")
        self.r = r
        self.y0 = y0.detach().clone().contiguous()
        self.p = p.detach().clone().contiguous()
        self.cotangent = cotangent
        self.want_y0, self.want_p = want_y0, want_p
        prepare_lane_order(r)  # the sort stays outside the graph
        main = torch.cuda.current_stream()
        side = torch.cuda.Stream(device=self.y0.device)
        side.wait_stream(main)
        with torch.cuda.stream(side):  # one eager pass first: kernel attributes set, caches warm
            self._run()
        main.wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.out = self._run()

    def _run(self):
        yf = replay(self.r, self.y0, self.p, write_ckpt=True)
        gy0, gp = adjoint(self.r, self.p, self.cotangent(yf), want_y0=self.want_y0,
                          want_p=self.want_p)
        return yf, gy0, gp

    def __call__(self, y0: Optional[torch.Tensor] = None, p: Optional[torch.Tensor] = None):
        if y0 is not None:
            self.y0.copy_(y0)
        if p is not None:
            self.p.copy_(p)
        self.graph.replay()
        return self.out


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
    L = _lib.lib_for(spec)
    _lib.check(L.gs_record_from_padded(n, S, _ptr(dts), S, _ptr(rec), cap, _ptr(n_steps),
                                       _stream()), "gs_record_from_padded", L)
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


def replay_saveat(r, y0: torch.Tensor, p: torch.Tensor, ts: torch.Tensor, *,
                  write_ckpt: bool = True, precision: str = "float64"):
    """Frozen-mesh replay with dense output at ``ts`` ((K,) shared or (n, K) per trajectory).
    Returns (y_final (n, D), ys (n, K, D)); refreshes the checkpoints for the adjoint."""
    res = _over_parts(r, lambda rr, rows: _replay_saveat_one(
        rr, _take(y0, rows), _take(p, rows), _take_ts(ts, rows), write_ckpt=write_ckpt,
        precision=precision))
    return _scatter(r, res, 0), _scatter(r, res, 1)


def _replay_saveat_one(r: Record, y0: torch.Tensor, p: torch.Tensor, ts: torch.Tensor, *,
                       write_ckpt: bool, precision: str):
    ts, ld, K = _ts_arg(ts, r.n)
    yf = torch.empty_like(y0)
    ys = torch.empty((r.n, K, r.spec.dim), dtype=torch.float64, device=y0.device)
    L = _lib.lib_for(r.spec)
    _lib.check(L.gs_replay_saveat(
        _METHOD_CODE[r.method], r.spec.code, _PREC[precision], r.n, _ptr(y0), _ptr(p),
        float(r.t0), _ptr(r.rec), _ptr(r.n_acc), max(r.cap, 1), r.ckpt_every,
        _ptr(r.ckpt) if write_ckpt else None, _ptr(ts), ld, K, _ptr(ys), _ptr(yf), _stream()),
        "gs_replay_saveat", L)
    return yf, ys


def adjoint_saveat(r, p: torch.Tensor, ts: torch.Tensor, ysbar: torch.Tensor,
                   ybar: Optional[torch.Tensor] = None, *, want_y0: bool = True,
                   want_p: bool = True, precision: str = "float64", schedule: str = "auto"):
    """(dL/dy0, dL/dp) for cotangents ysbar = dL/dys (n, K, D) and ybar = dL/dy_final.
    ``schedule="auto"`` refills lanes from a work counter for an uneven batch (per-trajectory
    end times), else runs one thread per trajectory."""
    if schedule == "auto" and r.uneven and precision != "float32":
        schedule = "refill"  # (the float32 route runs one thread per trajectory)
    res = _over_parts(r, lambda rr, rows: _adjoint_saveat_one(
        rr, _take(p, rows), _take_ts(ts, rows), _take(ysbar, rows), _take(ybar, rows),
        want_y0=want_y0, want_p=want_p, precision=precision, schedule=schedule))
    return _scatter(r, res, 0), _scatter(r, res, 1)


def _adjoint_saveat_one(r: Record, p: torch.Tensor, ts: torch.Tensor, ysbar: torch.Tensor,
                        ybar: Optional[torch.Tensor], *, want_y0: bool, want_p: bool,
                        precision: str, schedule: str):
    ts, ld, K = _ts_arg(ts, r.n)
    gy0 = torch.empty((r.n, r.spec.dim), dtype=torch.float64, device=p.device) if want_y0 else None
    gp = torch.empty((r.n, p.shape[1]), dtype=torch.float64, device=p.device) if want_p else None
    ysbar = ysbar.to(torch.float64).contiguous()
    ybar = None if ybar is None else ybar.to(torch.float64).contiguous()
    L = _lib.lib_for(r.spec)
    _lib.check(L.gs_adjoint_saveat(
        _METHOD_CODE[r.method], r.spec.code, _PREC[precision] | _SCHED[schedule], r.n, _ptr(p),
        _ptr(r.rec), _ptr(r.n_acc), max(r.cap, 1), _ptr(r.ckpt), r.ckpt_every, _ptr(ts), ld, K, _ptr(ysbar),
        _ptr(ybar), _ptr(gy0), _ptr(gp), _stream()), "gs_adjoint_saveat", L)
    return gy0, gp
