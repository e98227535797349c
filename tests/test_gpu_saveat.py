"""Dense output (saveat) on the replay and its adjoint, against the oracle's restatement of
gradsolve/solvers/dense.py:106-163 (bracket-and-re-step), including the reference's own
saveat contracts (tests/test_saveat.py:271-312: ys[:, -1] == y_final bitwise) and the
per-trajectory end times / time rows of the uneven-batch workload (an extension)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu


def rowrel(a, b):
    return float(np.max(np.abs(a - b).max(axis=-1) / np.maximum(np.abs(b).max(axis=-1), 1e-300)))


def _ref_record(cuda, method, field, g):
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    spec = field_spec(field)
    r = engine.record_from_padded(method, spec, torch.tensor(g["dts"], device=cuda), 0.0,
                                  checkpoint="sqrt")
    y0 = torch.tensor(g["y0"], device=cuda)
    p = torch.tensor(g["params"][:, : spec.nparam], device=cuda).contiguous()
    return spec, r, y0, p


CASES = [("tsit5", "vdp_batch", "vdp", [0.0, 0.0, 0.05, 0.3, 0.3, 0.7654321, 0.999, 1.0]),
         ("tsit5", "lorenz_small", "lorenz", [0.0, 0.1, 0.5, 0.95, 1.0]),
         ("tsit5", "lv_mixed", "lv", list(np.linspace(0.0, 20.0, 64))),
         ("rosenbrock23", "robertson_toy", "robertson", [0.0, 0.01, 0.2, 0.49, 0.5])]


@pytest.mark.parametrize("method,case,field,ts", CASES)
def test_saveat_values_and_gradients_vs_oracle(gslib, oracle, cuda, method, case, field, ts):
    from gradsolve_b200 import engine
    g = load_golden(case)
    spec, r, y0, p = _ref_record(cuda, method, field, g)
    ts_t = torch.tensor(ts, dtype=torch.float64, device=cuda)
    yf, ys = engine.replay_saveat(r, y0, p, ts_t)
    ryf, rys = oracle.replay_saveat(method, field, g["y0"], g["params"], g["dts"], np.array(ts))
    assert rowrel(ys.cpu().numpy(), rys) <= 1e-10
    assert rowrel(yf.cpu().numpy(), ryf) <= 1e-10
    # the reference's contracts: last saved state IS y_final, times at t0 ARE y0 (bitwise)
    assert torch.equal(ys[:, -1], yf)
    assert torch.equal(ys[:, 0], y0)
    rng = np.random.default_rng(7)
    ysbar = rng.normal(size=tuple(ys.shape))
    ybar = rng.normal(size=tuple(yf.shape))
    oy, op = oracle.replay_saveat_vjp(method, field, g["y0"], g["params"], g["dts"],
                                      np.array(ts), ysbar, ybar)
    outs = {}
    for sched in ("static", "refill", "strided"):  # one thread per trajectory / persistent lanes
        gy0, gp = engine.adjoint_saveat(r, p, ts_t, torch.tensor(ysbar, device=cuda),
                                        torch.tensor(ybar, device=cuda), schedule=sched)
        assert rowrel(gy0.cpu().numpy(), oy) <= 1e-9, sched
        assert rowrel(gp.cpu().numpy(), op[:, : spec.nparam]) <= 1e-9, sched
        outs[sched] = (gy0.cpu(), gp.cpu())
    if method == "tsit5":  # same expressions, same lane code: bitwise
        for sched in ("refill", "strided"):
            assert torch.equal(outs[sched][0], outs["static"][0])
            assert torch.equal(outs[sched][1], outs["static"][1])


def test_per_trajectory_end_times_and_rows(gslib, oracle, cuda):
    """Uneven batch: VdP, mu log-uniform, per-trajectory t1 and 64 saved times per row."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    rng = np.random.default_rng(5)
    n = 48
    mu = 10 ** rng.uniform(-1, np.log10(9.0), (n, 1))
    t1v = 10 ** rng.uniform(-1, np.log10(20.0), n)
    y0 = rng.uniform(-2, 2, (n, 2))
    ts = np.stack([np.linspace(0.0, t, 64) for t in t1v])
    spec = field_spec("vdp")
    r = engine.forward_record("tsit5", spec, torch.tensor(y0, device=cuda),
                              torch.tensor(mu, device=cuda), t0=0.0, t1=float(t1v.max()),
                              t1v=torch.tensor(t1v, device=cuda), rtol=1e-6, atol=1e-8,
                              checkpoint="sqrt")
    assert (r.status.cpu().numpy() == 0).all()
    dts = r.padded_dts().cpu().numpy()
    y0_t = torch.tensor(y0, device=cuda)
    mu_t = torch.tensor(mu, device=cuda)
    ts_t = torch.tensor(ts, device=cuda)
    yf, ys = engine.replay_saveat(r, y0_t, mu_t, ts_t)
    ryf, rys = oracle.replay_saveat("tsit5", "vdp", y0, mu, dts, ts)
    assert rowrel(ys.cpu().numpy(), rys) <= 1e-10
    assert torch.equal(ys[:, -1], yf)
    ysbar = rng.normal(size=tuple(ys.shape))
    gy0, gp = engine.adjoint_saveat(r, mu_t, ts_t, torch.tensor(ysbar, device=cuda))
    oy, op = oracle.replay_saveat_vjp("tsit5", "vdp", y0, mu, dts, ts, ysbar)
    assert rowrel(gy0.cpu().numpy(), oy) <= 1e-9
    assert rowrel(gp.cpu().numpy(), op) <= 1e-9


@pytest.mark.parametrize("method", ["tsit5", "rosenbrock23"])
def test_saveat_schedules_with_empty_trajectories(gslib, oracle, cuda, method):
    """Persistent saveat reverse passes (lanes refilled from a counter, strided lanes) against
    one thread per trajectory and the oracle, on a batch where every fifth trajectory has no
    steps (t1 = t0) and the others end at their own times, with a segment length that leaves
    partial last segments."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    rng = np.random.default_rng(11)
    n = 160
    mu = 10 ** rng.uniform(-1, 0.9, (n, 1)) if method == "tsit5" else \
        10 ** rng.uniform(1.0, 1.5, (n, 1))
    t1v = 10 ** rng.uniform(-1, np.log10(3.0), n)
    t1v[::5] = 0.0
    y0 = rng.uniform(-2, 2, (n, 2))
    ts = np.stack([np.linspace(0.0, t, 16) for t in t1v])
    spec = field_spec("vdp")
    r = engine.forward_record(method, spec, torch.tensor(y0, device=cuda),
                              torch.tensor(mu, device=cuda), t0=0.0, t1=float(t1v.max()),
                              t1v=torch.tensor(t1v, device=cuda), rtol=1e-6, atol=1e-9,
                              max_steps=50000, checkpoint=5)
    assert (r.status.cpu().numpy() == 0).all()
    assert (r.n_acc.cpu().numpy()[::5] == 0).all()
    dts = r.padded_dts().cpu().numpy()
    mu_t, ts_t = torch.tensor(mu, device=cuda), torch.tensor(ts, device=cuda)
    ysbar = rng.normal(size=(n, 16, 2))
    ybar = rng.normal(size=(n, 2))
    oy, op = oracle.replay_saveat_vjp(method, "vdp", y0, mu, dts, ts, ysbar, ybar)
    outs = {}
    for sched in ("static", "refill", "strided"):
        gy0, gp = engine.adjoint_saveat(r, mu_t, ts_t, torch.tensor(ysbar, device=cuda),
                                        torch.tensor(ybar, device=cuda), schedule=sched)
        assert rowrel(gy0.cpu().numpy(), oy) <= 1e-9, sched
        assert rowrel(gp.cpu().numpy(), op) <= 1e-9, sched
        outs[sched] = (gy0.cpu(), gp.cpu())
    # no steps: the gradient is the cotangent of y_final plus those of every saved time (= y0)
    e = outs["refill"][0].numpy()[::5]
    np.testing.assert_allclose(e, ybar[::5] + ysbar[::5].sum(axis=1), rtol=0, atol=1e-12)
    if method == "tsit5":  # same expressions, same lane code: bitwise
        for sched in ("refill", "strided"):
            assert torch.equal(outs[sched][0], outs["static"][0])
            assert torch.equal(outs[sched][1], outs["static"][1])


def test_stiff_vdp_saveat(gslib, oracle, cuda):
    """VdP at mu >= 10 through Rosenbrock23 (the stiff half of the uneven workload)."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    rng = np.random.default_rng(6)
    n = 16
    mu = 10 ** rng.uniform(1, 2, (n, 1))
    y0 = rng.uniform(-2, 2, (n, 2))
    ts = np.linspace(0.0, 3.0, 16)
    spec = field_spec("vdp")
    r = engine.forward_record("rosenbrock23", spec, torch.tensor(y0, device=cuda),
                              torch.tensor(mu, device=cuda), t0=0.0, t1=3.0, rtol=1e-6,
                              atol=1e-8, max_steps=50000, checkpoint="sqrt")
    assert (r.status.cpu().numpy() == 0).all()
    o = oracle.record("rosenbrock23", "vdp", y0, mu, 0.0, 3.0, 1e-6, 1e-8, max_steps=50000)
    np.testing.assert_array_equal(r.n_acc.cpu().numpy(), o["n_acc"])
    dts = r.padded_dts().cpu().numpy()
    mu_t = torch.tensor(mu, device=cuda)
    ts_t = torch.tensor(ts, device=cuda)
    yf, ys = engine.replay_saveat(r, torch.tensor(y0, device=cuda), mu_t, ts_t)
    ryf, rys = oracle.replay_saveat("rosenbrock23", "vdp", y0, mu, dts, ts)
    assert rowrel(ys.cpu().numpy(), rys) <= 1e-9
    ysbar = rng.normal(size=tuple(ys.shape))
    gy0, gp = engine.adjoint_saveat(r, mu_t, ts_t, torch.tensor(ysbar, device=cuda))
    oy, op = oracle.replay_saveat_vjp("rosenbrock23", "vdp", y0, mu, dts, ts, ysbar)
    assert rowrel(gy0.cpu().numpy(), oy) <= 1e-8
    assert rowrel(gp.cpu().numpy(), op) <= 1e-8


def test_api_solve_and_grad_closure_saveat(gslib, oracle, cuda):
    import gradsolve_b200 as gsb

    class VdP:
        name = "vdp"
        dim = 2
        t0 = 0.0
        t1 = 1.0
        is_stiff = False

    g = load_golden("vdp_batch")
    ts = np.array([0.0, 0.25, 0.5, 1.0])
    res = gsb.solve(VdP(), g["y0"], g["params"], saveat=ts)
    assert res.y_saved.shape == (3, 4, 2) and np.array_equal(res.ts_saved, ts)
    np.testing.assert_array_equal(res.y_saved[:, -1], res.y_final)
    clo = gsb.grad_closure(VdP(), g["y0"], g["params"], saveat=ts)
    p = torch.tensor(g["params"], device="cuda", requires_grad=True)
    ys = clo(p)
    assert ys.shape == (3, 4, 2)
    (ys ** 2).sum().backward()
    dts = clo.state.record.padded_dts().cpu().numpy()
    _, rys = oracle.replay_saveat("tsit5", "vdp", g["y0"], g["params"], dts, ts)
    _, op = oracle.replay_saveat_vjp("tsit5", "vdp", g["y0"], g["params"], dts, ts, 2 * rys)
    assert rowrel(p.grad.cpu().numpy(), op) <= 1e-9
    with pytest.raises(ValueError, match="sorted"):
        gsb.grad_closure(VdP(), g["y0"], g["params"], saveat=[0.5, 0.1])
    with pytest.raises(ValueError, match="within the problem domain"):
        gsb.solve(VdP(), g["y0"], g["params"], saveat=[0.0, 1.5])


def test_mixed_saveat_close_to_f64(gslib, cuda):
    from gradsolve_b200 import engine
    g = load_golden("lv_mixed")
    spec, r, y0, p = _ref_record(cuda, "tsit5", "lv", g)
    ts_t = torch.linspace(0.0, 20.0, 32, dtype=torch.float64, device=cuda)
    _, ys64 = engine.replay_saveat(r, y0, p, ts_t)
    _, ysm = engine.replay_saveat(r, y0, p, ts_t, precision="mixed")
    assert rowrel(ysm.cpu().numpy(), ys64.cpu().numpy()) <= 1e-5
    ysbar = torch.ones_like(ysm)
    g64 = engine.adjoint_saveat(r, p, ts_t, ysbar)[1]
    _, ysm = engine.replay_saveat(r, y0, p, ts_t, precision="mixed")
    gm = engine.adjoint_saveat(r, p, ts_t, ysbar, precision="mixed")[1]
    assert rowrel(gm.cpu().numpy(), g64.cpu().numpy()) <= 1e-3


@pytest.mark.parametrize("method,field,prec", [("tsit5", "vdp", "float64"),
                                               ("tsit5", "vdp", "mixed"),
                                               ("tsit5", "lorenz", "float64"),
                                               ("rosenbrock23", "vdp", "float64")])
def test_forward_dense_output_equals_replay(gslib, cuda, method, field, prec):
    """The forward that re-steps each bracketed time as it integrates gives the dense output
    of replay_saveat on the recorded mesh, with per-trajectory end times and time rows, and
    with records split in tiers (a small first capacity).  The re-step is the replay's own
    step function, but inlined into a different kernel the compiler may contract its
    multiply-adds differently, so saved states agree to rounding (each is one step from a
    bitwise-equal state); y0 and y_final rows are copies and equal bitwise."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    spec = field_spec(field)
    rng = np.random.default_rng(11)
    n = 700
    y0 = torch.tensor(rng.uniform(-2, 2, (n, spec.dim)), device=cuda)
    if field == "vdp":
        p = torch.tensor(10 ** rng.uniform(-1, 1.5, (n, 1)), device=cuda)
    else:
        p = torch.tensor(rng.uniform(20, 30, (n, 1)), device=cuda)
        y0 = y0 + torch.tensor([1.0, 0.0, 0.0], device=cuda)
    t1v = torch.tensor(10 ** rng.uniform(-1, 1, n), device=cuda)
    ts = t1v[:, None] * torch.linspace(0.0, 1.0, 16, dtype=torch.float64, device=cuda)[None, :]
    ts[:, 5] = ts[:, 4]  # a repeated time
    for cap0 in (1024, 16):  # one record, and tiers
        r = engine.forward_record(method, spec, y0, p, t0=0.0, t1=float(t1v.max()), t1v=t1v,
                                  rtol=1e-6, atol=1e-9, max_steps=200000, cap0=cap0,
                                  checkpoint=4, precision=prec, saveat_ts=ts)
        torch.cuda.synchronize()
        assert int((r.status != 0).sum()) == 0
        yf, ys = engine.replay_saveat(r, y0, p, ts, write_ckpt=False, precision=prec)
        torch.cuda.synchronize()
        assert r.ys.shape == ys.shape
        # float32 stage increments round at ~1e-7 of the step: the two kernels' contractions
        # differ at that level in the float32-stage mode
        tol = 1e-12 if prec == "float64" else 1e-6
        assert rowrel(r.ys.cpu().numpy(), ys.cpu().numpy()) <= tol, cap0
        assert rowrel(r.y_final.cpu().numpy(), yf.cpu().numpy()) <= tol, cap0
        assert torch.equal(r.ys[:, -1], r.y_final)  # ts[-1] = t1: y_final itself
        assert torch.equal(r.ys[:, 0], y0)          # ts[0] = t0: y0 itself
    # the tiered record as the workspace of the next solve: planned tiers on their own
    # streams, the same per-trajectory results, and the same gradient (Rosenbrock23's planned
    # tiers run one thread per trajectory instead of refilled lanes: the same expressions in
    # another kernel, equal to rounding, with the same step counts)
    assert isinstance(r, engine.RecordSet) and len(r.parts) > 1
    ysbar = torch.tensor(rng.normal(size=tuple(r.ys.shape)), device=cuda)
    g1 = engine.adjoint_saveat(r, p, ts, ysbar, precision=prec)
    r2 = engine.forward_record(method, spec, y0, p, t0=0.0, t1=float(t1v.max()), t1v=t1v,
                               rtol=1e-6, atol=1e-9, max_steps=200000, cap0=16, checkpoint=4,
                               precision=prec, saveat_ts=ts, workspace=r)
    g2 = engine.adjoint_saveat(r2, p, ts, ysbar, precision=prec)
    torch.cuda.synchronize()
    assert torch.equal(r.n_acc, r2.n_acc)
    for a, b in ((r.ys, r2.ys), (r.y_final, r2.y_final), (g1[0], g2[0]), (g1[1], g2[1])):
        if method == "tsit5":
            assert torch.equal(a, b)
        else:
            a, b = a.reshape(a.shape[0], -1).cpu().numpy(), b.reshape(b.shape[0], -1).cpu().numpy()
            assert rowrel(a, b) <= 1e-10


@pytest.mark.parametrize("method,prec", [("tsit5", "float64"), ("tsit5", "mixed"),
                                         ("rosenbrock23", "float64")])
def test_forward_dense_output_schedules(gslib, cuda, method, prec):
    """The forward with saved states on its three schedules -- one thread per trajectory,
    lanes refilled from a work counter, strided lanes -- and with a shared end time (the
    automatic choice is then one thread per trajectory): the same counts and dts, the same
    saved states (Tsit5 bitwise: one lane policy; Rosenbrock23 to rounding, the compiler
    contracting multiply-adds differently in the two kernels)."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    spec = field_spec("vdp")
    rng = np.random.default_rng(13)
    n = 500
    y0 = torch.tensor(rng.uniform(-2, 2, (n, 2)), device=cuda)
    lo, hi = (-1.0, 0.9) if method == "tsit5" else (1.0, 1.6)
    p = torch.tensor(10 ** rng.uniform(lo, hi, (n, 1)), device=cuda)
    for shared in (False, True):
        t1v = None if shared else torch.tensor(10 ** rng.uniform(-1, 0.7, n), device=cuda)
        t1 = 3.0 if shared else float(t1v.max())
        row = torch.linspace(0.0, 1.0, 12, dtype=torch.float64, device=cuda)
        ts = t1 * row if shared else t1v[:, None] * row[None, :]
        outs = {}
        for sched in ("static", "refill", "strided", "auto"):
            r = engine.forward_record(method, spec, y0, p, t0=0.0, t1=t1, t1v=t1v, rtol=1e-6,
                                      atol=1e-9, max_steps=50000, cap0=4096, checkpoint=4,
                                      precision=prec, saveat_ts=ts, schedule=sched)
            torch.cuda.synchronize()
            assert int((r.status != 0).sum()) == 0, sched
            outs[sched] = (r.n_acc.cpu(), r.padded_dts().cpu().numpy(), r.ys.cpu().numpy(),
                           r.y_final.cpu().numpy())
        ref = outs["static"]
        for sched in ("refill", "strided", "auto"):
            got = outs[sched]
            assert torch.equal(got[0], ref[0]), (shared, sched)
            if method == "tsit5":
                for a, b in zip(got[1:], ref[1:]):
                    np.testing.assert_array_equal(a, b)
            else:
                assert rowrel(got[2].reshape(n, -1), ref[2].reshape(n, -1)) <= 1e-10
                assert rowrel(got[3], ref[3]) <= 1e-10
