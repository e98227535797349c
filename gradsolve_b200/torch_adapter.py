"""``torch.autograd.Function`` around the frozen-mesh replay and its hand-written adjoint.

This is the PyTorch face of the reference's closure contract
(gradsolve/warp/warp_replay.py:186-237, gradsolve/solvers/tsit5_replay.py:192-232): the
mesh is recorded ONCE at (y0, params0); the closure's forward re-integrates that frozen
mesh at the (y0, params) it is given (the replay value, ``warp_replay.py:30-55``), and its
backward is the discrete adjoint of that replay with the dts held fixed -- computed by the
reverse-replay kernel instead of by ``jax.grad``.

When the closure is called at exactly the recording point (same y0 and params, bitwise),
the recording pass already produced the replay's value, its saved states (saveat) and its
checkpoints (the adaptive forward and the replay evaluate the same expressions in the same
order), so no second forward is launched.
"""
from __future__ import annotations

import torch

from . import engine


def _point(y0: torch.Tensor, pk: torch.Tensor) -> tuple:
    """A replay point: the tensors and their version counters at capture."""
    return (y0, pk, y0._version, pk._version)


def _same(a: torch.Tensor, b: torch.Tensor) -> bool:
    """a equals b elementwise.  The same view of the same storage answers without a device
    synchronisation (the caller has checked b's version counter, which a shares)."""
    if (a.data_ptr() == b.data_ptr() and a.shape == b.shape and a.stride() == b.stride()
            and a.dtype == b.dtype and a.device == b.device):
        return True
    return torch.equal(a, b)


def _at_point(y0: torch.Tensor, pk: torch.Tensor, point) -> bool:
    """(y0, pk) is the stored point, and the point's tensors were not modified in place since
    it was taken."""
    if point is None:
        return False
    y0r, pr, v0, v1 = point
    if y0r._version != v0 or pr._version != v1:
        return False
    return _same(y0, y0r) and _same(pk, pr)


class ReplayState:
    """The frozen record plus bookkeeping shared by every call of one closure."""

    def __init__(self, record, y0_rec: torch.Tensor, p_rec: torch.Tensor,
                 nparam: int, precision: str = "float64", reuse_recording: bool = True,
                 ts_rec=None):
        self.record = record
        self.y0_rec = y0_rec
        self.p_rec = p_rec
        self.nparam = nparam
        self.precision = precision
        self.version = 0           # bumps whenever the checkpoints are rewritten
        self.ckpt_point = _point(y0_rec, p_rec) if reuse_recording else None
        self.ts_rec = ts_rec       # the saveat times the recording pass also saved at

    def at_recording(self, y0: torch.Tensor, pk: torch.Tensor) -> bool:
        """The checkpoints are the recording pass's own and (y0, pk) is its point."""
        return self.version == 0 and _at_point(y0, pk, self.ckpt_point)

    def kernel_p(self, p: torch.Tensor) -> torch.Tensor:
        if p.shape[1] < self.nparam:  # only fields that ignore their parameter get here
            p = torch.nn.functional.pad(p, (0, self.nparam - p.shape[1]))
        return p[:, : self.nparam].contiguous()

    def run_forward(self, y0: torch.Tensor, p: torch.Tensor) -> torch.Tensor:
        pk = self.kernel_p(p)
        if _at_point(y0, pk, self.ckpt_point):
            return self.record.y_final.clone()
        yf = engine.replay(self.record, y0.contiguous(), pk, write_ckpt=True,
                           precision=self.precision)
        self.ckpt_point = _point(y0.detach().clone(), pk.detach().clone())
        self.version += 1
        return yf


class _ReplayFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y0, p, state):
        y0 = y0.contiguous()
        p = p.contiguous()
        yf = state.run_forward(y0, p)
        ctx.state = state
        ctx.version = state.version
        ctx.save_for_backward(y0, p)
        return yf

    @staticmethod
    def backward(ctx, ybar):
        state: ReplayState = ctx.state
        y0, p = ctx.saved_tensors
        pk = state.kernel_p(p)
        # the checkpoints are this forward's while no other forward of the closure ran since
        # (autograd refuses saved tensors modified in place)
        if state.version != ctx.version:
            # another forward of the same closure rewrote the checkpoints: rebuild ours
            engine.replay(state.record, y0, pk, write_ckpt=True, precision=state.precision)
            state.ckpt_point = _point(y0.detach().clone(), pk.detach().clone())
            state.version += 1
        need_y0, need_p = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        gy0, gpk = engine.adjoint(state.record, pk, ybar.to(torch.float64),
                                  want_y0=need_y0, want_p=need_p, precision=state.precision)
        gp = None
        if need_p:
            if p.shape[1] == state.nparam:
                gp = gpk
            else:
                gp = torch.zeros_like(p)
                gp[:, : state.nparam] = gpk
        return gy0, gp, None


def replay_apply(state: ReplayState, y0: torch.Tensor, p: torch.Tensor) -> torch.Tensor:
    return _ReplayFn.apply(y0, p, state)


class _SaveatFn(torch.autograd.Function):
    """Dense-output closure: (y0, p) -> ys (n, K, D) on the frozen mesh
    (gradsolve/warp/warp_replay.py:58-84); backward = the saveat adjoint kernel."""

    @staticmethod
    def forward(ctx, y0, p, state, ts):
        y0 = y0.contiguous()
        p = p.contiguous()
        pk = state.kernel_p(p)
        rec = state.record
        if (rec.ys is not None and state.ts_rec is not None and state.at_recording(y0, pk)
                and torch.equal(ts, state.ts_rec)):
            ys = rec.ys.clone()  # the recording pass saved these states itself
        else:
            _yf, ys = engine.replay_saveat(rec, y0, pk, ts, write_ckpt=True,
                                           precision=state.precision)
            state.ckpt_point = _point(y0.detach().clone(), pk.detach().clone())
            state.version += 1
        ctx.state, ctx.ts, ctx.version = state, ts, state.version
        ctx.save_for_backward(y0, p)
        return ys

    @staticmethod
    def backward(ctx, ysbar):
        state: ReplayState = ctx.state
        y0, p = ctx.saved_tensors
        pk = state.kernel_p(p)
        if state.version != ctx.version:
            engine.replay_saveat(state.record, y0, pk, ctx.ts, write_ckpt=True,
                                 precision=state.precision)
            state.ckpt_point = _point(y0.detach().clone(), pk.detach().clone())
            state.version += 1
        need_y0, need_p = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        gy0, gpk = engine.adjoint_saveat(state.record, pk, ctx.ts, ysbar, None,
                                         want_y0=need_y0, want_p=need_p,
                                         precision=state.precision)
        gp = None
        if need_p:
            gp = gpk if p.shape[1] == state.nparam else torch.zeros_like(p)
            if p.shape[1] != state.nparam:
                gp[:, : state.nparam] = gpk
        return gy0, gp, None, None


def saveat_apply(state: ReplayState, y0: torch.Tensor, p: torch.Tensor,
                 ts: torch.Tensor) -> torch.Tensor:
    return _SaveatFn.apply(y0, p, state, ts)
