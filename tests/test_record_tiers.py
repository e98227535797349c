"""Host logic of the tiered record (engine.RecordSet), on the CPU.

The library's entry points are replaced by a stand-in that works on host tensors through
their pointers: trajectory j needs ``steps[j]`` accepted steps (taken from its first
parameter), overflows a record of capacity ``cap`` with status 3 (n_acc = cap), and its
"adjoint" returns values that identify which record served it.  The test checks that the
overflowed rows are re-solved alone with a larger capacity, that later tiers' results
replace the first tier's for their rows, and that replay/adjoint/padded dts are scattered
back to the caller's order.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from gradsolve_b200 import engine
from gradsolve_b200.fields import field_spec


def _arr(ptr, count, ctype=ctypes.c_double):
    return np.ctypeslib.as_array((ctype * count).from_address(ptr)) if count else np.zeros(0)


class FakeLib:
    """Stand-in for libgsolve on host memory (one call = one 'launch')."""

    def __init__(self):
        self.launches = []  # (n, cap) of every forward with a record

    def gs_max_ckpt_every(self):
        return 64

    def gs_record_bytes(self, n, cap):
        return ((cap + 3) // 4) * 4 * n * 8

    def gs_ckpt_slots(self, cap, K):
        return cap // K + 2

    def gs_tsit5_fwd_record(self, field, mode, n, y0, p, t0, t1v, t1, rtol, atol, dt0,
                            max_steps, cap, K, rec, ckpt, yf, n_acc, n_rej, status, stream):
        D, P = 3, 1
        y0a, pa = _arr(y0, n * D).reshape(n, D), _arr(p, n * P).reshape(n, P)
        yfa = _arr(yf, n * D).reshape(n, D)
        na = _arr(n_acc, n, ctypes.c_int)
        nr = _arr(n_rej, n, ctypes.c_int)
        st = _arr(status, n, ctypes.c_int)
        reca = _arr(rec, ((cap + 3) // 4) * 4 * n) if rec else None
        if rec:
            self.launches.append((n, cap))
        for j in range(n):
            steps = int(pa[j, 0])
            if rec and steps > cap:
                na[j], st[j] = cap, 3
            else:
                na[j], st[j] = steps, 0
            nr[j] = 0
            yfa[j] = y0a[j] + (steps if st[j] == 0 else -1.0)
            if reca is not None:
                for s in range(na[j]):
                    reca[((s // 4) * n + j) * 4 + s % 4] = 1.0 / steps
        return 0

    def gs_tsit5_replay(self, field, mode, n, y0, p, t0, rec, n_acc, cap, K, ckpt, yf, stream):
        D = 3
        y0a, yfa = _arr(y0, n * D).reshape(n, D), _arr(yf, n * D).reshape(n, D)
        na = _arr(n_acc, n, ctypes.c_int)
        yfa[:] = y0a + na[:, None] + 1000.0 * cap  # tags the record capacity used
        return 0

    def gs_tsit5_adjoint(self, field, mode, n, p, rec, n_acc, cap, ckpt, K, ybar, gy0, gp,
                         stream):
        D, P = 3, 1
        na = _arr(n_acc, n, ctypes.c_int)
        yb = _arr(ybar, n * D).reshape(n, D)
        if gy0:
            _arr(gy0, n * D).reshape(n, D)[:] = yb * 2.0
        if gp:
            _arr(gp, n * P).reshape(n, P)[:, 0] = na + 1e6 * cap
        return 0

    def gs_replay_saveat(self, method, field, mode, n, y0, p, t0, rec, n_acc, cap, K, ckpt, ts,
                         ts_ld, Kt, ys, yf, stream):
        D = 3
        tsa = _arr(ts, (n if ts_ld else 1) * Kt).reshape(-1, Kt)
        na = _arr(n_acc, n, ctypes.c_int)
        ysa = _arr(ys, n * Kt * D).reshape(n, Kt, D)
        ysa[:] = (tsa[:, :, None] if ts_ld else tsa[None, :, :, None][0]) + 1000.0 * cap
        _arr(yf, n * D).reshape(n, D)[:] = na[:, None]
        return 0

    def gs_adjoint_saveat(self, method, field, mode, n, p, rec, n_acc, cap, ckpt, K, ts, ts_ld,
                          Kt, ysbar, ybar, gy0, gp, stream):
        D = 3
        ysb = _arr(ysbar, n * Kt * D).reshape(n, Kt, D)
        if gp:
            _arr(gp, n).reshape(n, 1)[:, 0] = ysb.sum(axis=(1, 2)) + 1e6 * cap
        if gy0:
            _arr(gy0, n * D).reshape(n, D)[:] = 0.0
        return 0

    def gs_last_error(self):
        return b"stand-in error"

    def gs_record_to_padded(self, n, cap, rec, n_acc, S, dts, stream):
        if S > cap:  # the library refuses it too
            return -1
        reca = _arr(rec, ((cap + 3) // 4) * 4 * n)
        na = _arr(n_acc, n, ctypes.c_int)
        out = _arr(dts, n * S).reshape(n, S)
        for j in range(n):
            for s in range(min(na[j], S)):
                out[j, s] = reca[((s // 4) * n + j) * 4 + s % 4]
        return 0


@pytest.fixture
def fake(monkeypatch):
    f = FakeLib()
    monkeypatch.setattr(engine._lib, "lib", lambda: f)
    monkeypatch.setattr(engine, "_stream", lambda: 0)
    return f


def test_overflowed_rows_are_resolved_in_larger_tiers(fake):
    spec = field_spec("lorenz")
    steps = np.array([5, 3, 40, 7, 300, 2, 17, 1000], dtype=np.float64)
    n = steps.size
    y0 = torch.zeros((n, 3), dtype=torch.float64)
    p = torch.tensor(steps[:, None])
    r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=1.0, rtol=1e-6, atol=1e-6,
                              max_steps=5000, cap0=8, checkpoint=4, budget_bytes=1 << 40)
    assert isinstance(r, engine.RecordSet)
    # tier capacities 8, 32, 128, 512, 2048: each re-solves only the rows that overflowed
    assert fake.launches == [(8, 8), (4, 32), (3, 128), (2, 512), (1, 2048)]
    np.testing.assert_array_equal(r.n_acc.numpy(), steps.astype(np.int32))
    assert np.all(r.status.numpy() == 0)
    np.testing.assert_array_equal(r.y_final.numpy(), np.repeat(steps[:, None], 3, axis=1))
    caps = {int(rr.cap): (None if rows is None else rows.tolist()) for rows, rr in r.parts}
    # a tier's own counts leave out the rows a later tier re-solved
    tier0 = r.parts[0][1]
    assert tier0.n_acc.tolist() == [5, 3, 0, 7, 0, 2, 0, 0]
    assert caps == {8: None, 32: [2, 4, 6, 7], 128: [2, 4, 7], 512: [4, 7], 2048: [7]}
    # the trajectory's final tier serves its replay and its gradient
    final_cap = np.array([8, 8, 128, 8, 512, 8, 32, 2048])
    yf = engine.replay(r, y0, p)
    np.testing.assert_array_equal(yf[:, 0].numpy(), steps + 1000.0 * final_cap)
    ybar = torch.arange(n * 3, dtype=torch.float64).reshape(n, 3)
    gy0, gp = engine.adjoint(r, p, ybar)
    np.testing.assert_array_equal(gy0.numpy(), 2.0 * ybar.numpy())
    np.testing.assert_array_equal(gp[:, 0].numpy(), steps + 1e6 * final_cap)
    # the padded record in the caller's order, and a row subset
    d = r.padded_dts()
    assert d.shape == (n, 1000)
    for j in range(n):
        k = int(steps[j])
        assert np.all(d[j, :k].numpy() == 1.0 / steps[j]) and np.all(d[j, k:].numpy() == 0)
    sub = r.dts_rows(torch.tensor([7, 0, 4]))
    np.testing.assert_array_equal(sub.numpy(), d[[7, 0, 4]].numpy())


def test_single_tier_when_everything_fits(fake):
    spec = field_spec("lorenz")
    p = torch.tensor([[3.0], [8.0]], dtype=torch.float64)
    r = engine.forward_record("tsit5", spec, torch.zeros((2, 3), dtype=torch.float64), p,
                              t0=0.0, t1=1.0, rtol=1e-6, atol=1e-6, cap0=8, checkpoint=4,
                              budget_bytes=1 << 40)
    assert isinstance(r, engine.Record)
    assert fake.launches == [(2, 8)]


def test_max_steps_bounds_the_last_tier(fake):
    spec = field_spec("lorenz")
    p = torch.tensor([[3.0], [100.0]], dtype=torch.float64)
    r = engine.forward_record("tsit5", spec, torch.zeros((2, 3), dtype=torch.float64), p,
                              t0=0.0, t1=1.0, rtol=1e-6, atol=1e-6, cap0=8, max_steps=50,
                              checkpoint=4, budget_bytes=1 << 40)
    assert fake.launches == [(2, 8), (1, 32), (1, 50)]
    assert r.status.tolist() == [0, 3]  # the stand-in never exhausts max_steps itself


def test_saveat_on_tiers_uses_each_rows_times(fake):
    spec = field_spec("lorenz")
    steps = np.array([5, 40, 3, 100], dtype=np.float64)
    n = steps.size
    p = torch.tensor(steps[:, None])
    y0 = torch.zeros((n, 3), dtype=torch.float64)
    r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=1.0, rtol=1e-6, atol=1e-6,
                              cap0=8, checkpoint=4, budget_bytes=1 << 40)
    assert isinstance(r, engine.RecordSet)
    final_cap = np.array([8, 128, 8, 128])
    ts = torch.arange(n * 2, dtype=torch.float64).reshape(n, 2)
    yf, ys = engine.replay_saveat(r, y0, p, ts)
    np.testing.assert_array_equal(ys[:, :, 0].numpy(), ts.numpy() + 1000.0 * final_cap[:, None])
    np.testing.assert_array_equal(yf[:, 0].numpy(), steps)
    ysbar = torch.ones((n, 2, 3), dtype=torch.float64) * torch.arange(n)[:, None, None]
    _gy0, gp = engine.adjoint_saveat(r, p, ts, ysbar)
    np.testing.assert_array_equal(gp[:, 0].numpy(), 6.0 * np.arange(n) + 1e6 * final_cap)


def test_planned_tiers_from_the_workspace(fake):
    """With the previous RecordSet as workspace, every trajectory goes straight to the tier
    that held it (the side tiers are launched first), nothing is re-solved, and the results
    are those of the first solve."""
    spec = field_spec("lorenz")
    steps = np.array([5, 3, 40, 7, 300, 2, 17, 1000], dtype=np.float64)
    n = steps.size
    y0 = torch.zeros((n, 3), dtype=torch.float64)
    p = torch.tensor(steps[:, None])
    kw = dict(t0=0.0, t1=1.0, rtol=1e-6, atol=1e-6, max_steps=5000, cap0=8, checkpoint=4,
              budget_bytes=1 << 40)
    r1 = engine.forward_record("tsit5", spec, y0, p, **kw)
    fake.launches.clear()
    r2 = engine.forward_record("tsit5", spec, y0, p, workspace=r1, **kw)
    # (off the GPU the tiers run one after another; on it, side tiers first, concurrently)
    assert sorted(fake.launches) == [(1, 32), (1, 128), (1, 512), (1, 2048), (4, 8)]
    assert isinstance(r2, engine.RecordSet)
    np.testing.assert_array_equal(r2.n_acc.numpy(), steps.astype(np.int32))
    np.testing.assert_array_equal(r2.y_final.numpy(), r1.y_final.numpy())
    np.testing.assert_array_equal(r2.padded_dts().numpy(), r1.padded_dts().numpy())
    ybar = torch.arange(n * 3, dtype=torch.float64).reshape(n, 3)
    a1, b1 = engine.adjoint(r1, p, ybar)
    a2, b2 = engine.adjoint(r2, p, ybar)
    np.testing.assert_array_equal(a1.numpy(), a2.numpy())
    np.testing.assert_array_equal(b1.numpy(), b2.numpy())
    # a third solve reuses the planned tiers' own buffers
    fake.launches.clear()
    r3 = engine.forward_record("tsit5", spec, y0, p, workspace=r2, **kw)
    assert sorted(fake.launches) == [(1, 32), (1, 128), (1, 512), (1, 2048), (4, 8)]
    assert r3.parts[0][1].rec.data_ptr() == r2.parts[0][1].rec.data_ptr()


def test_planned_tier_outgrown(fake):
    spec = field_spec("lorenz")
    steps = np.array([5, 3, 40], dtype=np.float64)
    y0 = torch.zeros((3, 3), dtype=torch.float64)
    kw = dict(t0=0.0, t1=1.0, rtol=1e-6, atol=1e-6, max_steps=5000, cap0=8, checkpoint=4,
              budget_bytes=1 << 40)
    r1 = engine.forward_record("tsit5", spec, y0, torch.tensor(steps[:, None]), **kw)
    steps2 = np.array([5, 20, 40], dtype=np.float64)  # row 1 now needs more than its tier
    fake.launches.clear()
    r2 = engine.forward_record("tsit5", spec, y0, torch.tensor(steps2[:, None]), workspace=r1,
                               **kw)
    # planned tiers (cap 8: rows 0, 1; cap 128: row 2), then row 1 again with 4 x 8
    assert sorted(fake.launches[:2]) == [(1, 128), (2, 8)] and fake.launches[2:] == [(1, 32)]
    np.testing.assert_array_equal(r2.n_acc.numpy(), steps2.astype(np.int32))
    assert np.all(r2.status.numpy() == 0)
    yf = engine.replay(r2, y0, torch.tensor(steps2[:, None]))
    np.testing.assert_array_equal(yf[:, 0].numpy(), steps2 + 1000.0 * np.array([8, 32, 128]))


def test_reused_single_record_orders_lanes_by_cost(fake):
    """A record reused as the next solve's workspace becomes a one-tier plan whose rows run
    longest first (by the previous record's attempts); its results come back in batch order."""
    spec = field_spec("lorenz")
    rng = np.random.default_rng(3)
    steps = rng.integers(1, 8, 40).astype(np.float64)
    p = torch.tensor(steps[:, None])
    y0 = torch.zeros((40, 3), dtype=torch.float64)
    kw = dict(t0=0.0, t1=1.0, rtol=1e-6, atol=1e-6, cap0=8, checkpoint=4, budget_bytes=1 << 40)
    r1 = engine.forward_record("tsit5", spec, y0, p, **kw)
    assert isinstance(r1, engine.Record)
    r2 = engine.forward_record("tsit5", spec, y0, p, workspace=r1, **kw)
    assert isinstance(r2, engine.RecordSet) and len(r2.parts) == 1
    rows = r2.parts[0][0].numpy()
    assert np.all(np.diff(steps[rows]) <= 0)           # longest first
    np.testing.assert_array_equal(r2.n_acc.numpy(), steps.astype(np.int32))
    np.testing.assert_array_equal(r2.y_final.numpy(), y0.numpy() + steps[:, None])
    gy0, gp = engine.adjoint(r2, p, torch.ones((40, 3), dtype=torch.float64))
    np.testing.assert_array_equal(gp[:, 0].numpy(), steps + 1e6 * 8)
    d = r2.padded_dts().numpy()
    for j in range(40):
        np.testing.assert_array_equal(d[j, : int(steps[j])], 1.0 / steps[j])
