"""The float32 route (precision="float32", GS_PREC_F32): record, replay and reverse pass all
in float32, on the reference's own f32 test cells (tests/test_f32_replay.py:1-31, 84-93).

  * nonstiff: diffeqgpu_lorenz, n = 2048, t in [0, 1], rtol 1e-6 / atol 1e-9;
  * stiff:    robertson, n = 256, t in [0, 1e4], rtol 1e-5 / atol 1e-8;
  * loss sum(y_final**2).

Correctness isolates the arithmetic from the mesh, as the reference does: the float32
gradient is compared with the float64 oracle's reverse pass over the SAME float32-recorded
mesh (gradient rel-L2 <= 1e-3 and direction cosine >= 1 - 1e-6), and the float32 primal with a
tight float64 solve (<= 1e-4 relative, Lorenz; <= 1e-3 absolute, Robertson).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LORENZ_CELL = dict(n=2048, rtol=1e-6, atol=1e-9)
ROBERTSON_CELL = dict(n=256, rtol=1e-5, atol=1e-8)
GRAD_REL_L2_TOL = 1e-3
GRAD_COSINE_TOL = 1e-6
PRIMAL_TOL_LORENZ = 1e-4
PRIMAL_TOL_ROBERTSON = 1e-3


class Lorenz:
    name = "diffeqgpu_lorenz"
    dim = 3
    t0 = 0.0
    t1 = 1.0
    is_stiff = False


class Robertson:
    name = "robertson"
    dim = 3
    t0 = 0.0
    t1 = 1.0e4
    is_stiff = True


def lorenz_batch(n=LORENZ_CELL["n"]):
    rng = np.random.default_rng(0)
    y0 = np.tile(np.array([1.0, 0.0, 0.0]), (n, 1)) + 0.01 * rng.standard_normal((n, 3))
    return y0, np.full((n, 1), 28.0)


def robertson_batch(n=ROBERTSON_CELL["n"]):
    return (np.tile(np.array([1.0, 0.0, 0.0]), (n, 1)),
            np.tile(np.array([0.04, 3.0e7, 1.0e4]), (n, 1)))


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cosine(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))


def f32_grad(problem, y0, params, cell):
    """dL/dparams of L = sum(closure(params)**2) on the float32 route, with its mesh."""
    import gradsolve_b200 as gsb
    clo = gsb.grad_closure(problem, y0, params, precision="float32", rtol=cell["rtol"],
                           atol=cell["atol"])
    p = torch.tensor(params, dtype=torch.float32, device="cuda", requires_grad=True)
    out = clo(p)
    assert out.dtype == torch.float32
    (out.double() ** 2).sum().backward()
    assert p.grad.dtype == torch.float32
    dts = clo.state.record.padded_dts().cpu().numpy()
    return p.grad.cpu().numpy().astype(np.float64), dts, out.detach().cpu().numpy()


def test_record_and_closure_are_float32(gslib, cuda):
    import gradsolve_b200 as gsb
    y0, params = lorenz_batch(64)
    yf, n_acc, dts = gsb.record(Lorenz(), y0, params, rtol=1e-6, atol=1e-9,
                                precision="float32")
    assert dts.dtype == np.float32 and yf.dtype == np.float32
    assert dts.shape == (64, int(n_acc.max()))
    clo = gsb.grad_closure(Lorenz(), y0, params, engine="warp_replay", precision="float32",
                           rtol=1e-6, atol=1e-9)
    assert clo.route.actual == "b200_tsit5" and clo.route.reason == "served-by-b200_tsit5"
    y0s, ps = robertson_batch(8)
    _yf, _n, dts_s = gsb.record(Robertson(), y0s, ps, rtol=1e-5, atol=1e-8,
                                precision="float32")
    assert dts_s.dtype == np.float32
    clo_s = gsb.grad_closure(Robertson(), y0s, ps, engine="warp_rosenbrock",
                             precision="float32", rtol=1e-5, atol=1e-8)
    assert clo_s(torch.tensor(ps, dtype=torch.float32, device="cuda")).dtype == torch.float32


@pytest.mark.parametrize("problem,batch,kw", [
    (Lorenz(), lorenz_batch, dict(rtol=1e-6, atol=1e-9)),
    (Robertson(), robertson_batch, dict(rtol=1e-5, atol=1e-8))])
def test_record_buffer_halves_per_step(gslib, cuda, problem, batch, kw):
    """Per step the float32 record is exactly half (4 vs 8 bytes); its device buffer is
    exactly half the float64 one at the same capacity; the meshes' lengths differ by the few
    steps the float32 controller accepts differently (tests/test_f32_replay.py:194-247)."""
    import gradsolve_b200 as gsb
    from gradsolve_b200 import _lib
    n = 64 if problem.name != "robertson" else 8
    y0, params = batch(n)
    _y, n64, d64 = gsb.record(problem, y0, params, precision="float64", **kw)
    _y, n32, d32 = gsb.record(problem, y0, params, precision="float32", **kw)
    assert d64.dtype == np.float64 and d32.dtype == np.float32
    assert d32.itemsize * 2 == d64.itemsize
    assert 0.45 <= d32.nbytes / d64.nbytes <= 0.55
    L = _lib.lib()
    for cap in (1, 7, 1024, 4099):
        assert 2 * L.gs_record_bytes_prec(_lib.GS_PREC_F32, n, cap) == L.gs_record_bytes(n, cap)
    assert np.max(np.abs(n64.astype(np.int64) - n32.astype(np.int64))) <= 2


def test_float32_mesh_differs_slightly_from_float64(gslib, cuda):
    """A float32 controller, not float64 arithmetic on the float64 steps: some step counts
    differ, by at most a couple (tests/test_f32_replay.py:250-276)."""
    import gradsolve_b200 as gsb
    y0, params = lorenz_batch(64)
    _y, n64, _d = gsb.record(Lorenz(), y0, params, rtol=1e-6, atol=1e-9, precision="float64")
    _y, n32, _d = gsb.record(Lorenz(), y0, params, rtol=1e-6, atol=1e-9, precision="float32")
    assert np.any(n64 != n32)
    assert np.max(np.abs(n64.astype(np.int64) - n32.astype(np.int64))) <= 2


def test_gradient_matches_f64_oracle_on_the_same_mesh_lorenz(gslib, oracle, cuda):
    y0, params = lorenz_batch()
    g32, dts32, _ = f32_grad(Lorenz(), y0, params, LORENZ_CELL)
    dts = dts32.astype(np.float64)
    y64 = oracle.replay("tsit5", "lorenz", y0, params, dts, nthreads=8)
    _gy, g64 = oracle.replay_vjp("tsit5", "lorenz", y0, params, dts, 2.0 * y64, nthreads=8)
    rel, cos = rel_l2(g32, g64), cosine(g32, g64)
    print(f"lorenz f32: grad rel-L2 {rel:.3e}, cosine 1 - {1 - cos:.2e}")
    assert rel <= GRAD_REL_L2_TOL
    assert cos >= 1 - GRAD_COSINE_TOL


def test_gradient_matches_f64_oracle_on_the_same_mesh_robertson(gslib, oracle, cuda):
    y0, params = robertson_batch()
    import gradsolve_b200 as gsb
    clo = gsb.grad_closure(Robertson(), y0, params, precision="float32",
                           rtol=ROBERTSON_CELL["rtol"], atol=ROBERTSON_CELL["atol"])
    p = torch.tensor(params, dtype=torch.float32, device="cuda", requires_grad=True)
    (clo(p).double() ** 2).sum().backward()
    g32 = p.grad.cpu().numpy().astype(np.float64)
    dts = clo.state.record.padded_dts().cpu().numpy().astype(np.float64)
    y64 = oracle.replay("rosenbrock23", "robertson", y0, params, dts, nthreads=8)
    _gy, g64 = oracle.replay_vjp("rosenbrock23", "robertson", y0, params, dts, 2.0 * y64,
                                 nthreads=8)
    rel, cos = rel_l2(g32, g64), cosine(g32, g64)
    print(f"robertson f32: grad rel-L2 {rel:.3e}, cosine 1 - {1 - cos:.2e}")
    assert rel <= GRAD_REL_L2_TOL
    assert cos >= 1 - GRAD_COSINE_TOL


def test_primal_error_vs_tight_reference_lorenz(gslib, cuda):
    import gradsolve_b200 as gsb
    y0, params = lorenz_batch(128)
    clo = gsb.grad_closure(Lorenz(), y0, params, precision="float32",
                           rtol=LORENZ_CELL["rtol"], atol=LORENZ_CELL["atol"])
    y32 = clo(torch.tensor(params, device="cuda")).cpu().numpy().astype(np.float64)
    ref = gsb.solve(Lorenz(), y0, params, rtol=1e-12, atol=1e-14).y_final
    err = np.max(np.linalg.norm(y32 - ref, axis=1) / np.linalg.norm(ref, axis=1))
    print(f"lorenz f32 primal error {err:.3e}")
    assert err <= PRIMAL_TOL_LORENZ


def test_primal_error_vs_tight_reference_robertson(gslib, cuda):
    import gradsolve_b200 as gsb
    y0, params = robertson_batch(8)
    clo = gsb.grad_closure(Robertson(), y0, params, precision="float32",
                           rtol=ROBERTSON_CELL["rtol"], atol=ROBERTSON_CELL["atol"])
    y32 = clo(torch.tensor(params, device="cuda")).cpu().numpy().astype(np.float64)
    # a tight float64 Rosenbrock23 solve (order 2: ~1e5 steps at this tolerance)
    ref = gsb.solve(Robertson(), y0, params, rtol=1e-9, atol=1e-11, max_steps=10**6).y_final
    err = np.max(np.abs(y32 - ref).sum(axis=1))  # y2 ~ 1e-5: absolute, as the reference
    print(f"robertson f32 primal error {err:.3e}")
    assert err <= PRIMAL_TOL_ROBERTSON


@pytest.mark.parametrize("method,field,problem,batch,kw", [
    ("tsit5", "lorenz", Lorenz(), lorenz_batch, dict(rtol=1e-6, atol=1e-9)),
    ("rosenbrock23", "robertson", Robertson(), robertson_batch, dict(rtol=1e-5, atol=1e-8))])
def test_replay_reproduces_the_recording_pass(gslib, cuda, method, field, problem, batch, kw):
    """The float32 replay evaluates the recording pass's expressions on its own mesh, so it
    lands on the recorded y_final bit for bit; and the reverse pass at K = 1 (every state
    stored) and K = 5 (recomputed segments) gives the same gradient."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    spec = field_spec(field)
    y0n, pn = batch(256)
    y0 = torch.tensor(y0n, device="cuda")
    p = torch.tensor(pn[:, : spec.nparam], device="cuda").contiguous()
    grads = []
    for K in (1, 5):
        r = engine.forward_record(method, spec, y0, p, t0=0.0, t1=float(problem.t1),
                                  checkpoint=K, precision="float32", **kw)
        assert (r.status == 0).all()
        assert r.rec.dtype == torch.float32
        yr = engine.replay(r, y0, p, precision="float32")
        assert torch.equal(yr, r.y_final)
        ybar = 2.0 * yr
        grads.append(engine.adjoint(r, p, ybar, precision="float32"))
    for a, b in zip(grads[0], grads[1]):
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) <= 1e-5


def test_float32_refusals(gslib, cuda):
    """Refused rather than served another way: other schedules, lanes and reverse-pass
    variants at the C ABI; fields above 8 components at the API."""
    import gradsolve_b200 as gsb
    from gradsolve_b200 import _lib, engine
    from gradsolve_b200.fields import field_spec
    spec = field_spec("lorenz")
    y0, params = lorenz_batch(64)
    y0t = torch.tensor(y0, device="cuda")
    pt = torch.tensor(params, device="cuda")
    with pytest.raises(_lib.GsolveError, match="one thread per trajectory"):
        engine.forward_record("tsit5", spec, y0t, pt, t0=0.0, t1=1.0, rtol=1e-6, atol=1e-9,
                              precision="float32", schedule="refill")
    r = engine.forward_record("tsit5", spec, y0t, pt, t0=0.0, t1=1.0, rtol=1e-6, atol=1e-9,
                              precision="float32", checkpoint=4)
    with pytest.raises(_lib.GsolveError, match="not float32-route options"):
        engine.adjoint(r, pt, y0t, precision="float32", variant="stages")
    spec8 = field_spec("lorenz96_8")
    y8 = torch.full((64, 8), 8.0, dtype=torch.float64, device="cuda")
    y8[:, 0] += 0.01
    p8 = torch.full((64, 1), 8.0, dtype=torch.float64, device="cuda")
    r8 = engine.forward_record("tsit5", spec8, y8, p8, t0=0.0, t1=0.5, rtol=1e-6, atol=1e-9,
                               precision="float32", checkpoint=4)
    with pytest.raises(_lib.GsolveError, match="GS_ADJ_PAIRS is built for"):
        engine.adjoint(r8, p8, y8, precision="float32", variant="pairs")

    class L96:
        name = "lorenz96_32"
        dim = 32
        t0 = 0.0
        t1 = 1.0
        is_stiff = False

    with pytest.raises(ValueError, match="at most 8 components"):
        gsb.grad_closure(L96(), np.ones((4, 32)), np.full((4, 1), 8.0), precision="float32")


@pytest.mark.parametrize("method,field,problem,batch,kw,ts", [
    ("tsit5", "lorenz", Lorenz(), lorenz_batch, dict(rtol=1e-6, atol=1e-9),
     np.linspace(0.0, 1.0, 17)),
    ("rosenbrock23", "robertson", Robertson(), robertson_batch, dict(rtol=1e-5, atol=1e-8),
     np.array([0.0, 1.0, 10.0, 100.0, 1000.0, 1.0e4]))])
def test_saveat_matches_f64_oracle_on_the_same_mesh(gslib, oracle, cuda, method, field,
                                                     problem, batch, kw, ts):
    """The float32 closure with saveat (the times float32, as the reference's f32 replay
    casts them): the saved states and dL/dparams of sum(ys**2) against the float64 oracle's
    dense-output replay and reverse pass over the same float32 mesh, at the reference's f32
    bars; the last saved state equals y_final bit for bit."""
    import gradsolve_b200 as gsb
    y0, params = batch(256)
    clo = gsb.grad_closure(problem, y0, params, precision="float32", saveat=ts, **kw)
    p = torch.tensor(params, dtype=torch.float32, device="cuda", requires_grad=True)
    ys = clo(p)
    assert ys.dtype == torch.float32 and ys.shape == (256, len(ts), 3)
    (ys.double() ** 2).sum().backward()
    g32 = p.grad.cpu().numpy().astype(np.float64)
    dts = clo.state.record.padded_dts().cpu().numpy().astype(np.float64)
    _yf, ys64 = oracle.replay_saveat(method, field, y0, params, dts, ts, nthreads=8)
    _gy, g64 = oracle.replay_saveat_vjp(method, field, y0, params, dts, ts, 2.0 * ys64,
                                        nthreads=8)
    y32 = ys.detach().cpu().numpy().astype(np.float64)
    scale = np.abs(ys64).max(axis=(1, 2), keepdims=True)
    ey = float(np.max(np.abs(y32 - ys64) / scale))
    rel, cos = rel_l2(g32, g64), cosine(g32, g64)
    print(f"{field} f32 saveat: ys row error {ey:.2e}, grad rel-L2 {rel:.3e}, "
          f"cosine 1 - {1 - cos:.2e}")
    assert ey <= 1e-4
    assert rel <= GRAD_REL_L2_TOL
    assert cos >= 1 - GRAD_COSINE_TOL
    # the final saved time is t1: its state is y_final itself
    from gradsolve_b200 import engine
    yf = engine.replay(clo.state.record, torch.tensor(y0, device="cuda"),
                       torch.tensor(params, device="cuda"), write_ckpt=False,
                       precision="float32")
    assert torch.equal(ys[:, -1].detach().double(), yf)


def test_uneven_end_times_per_row_saveat_and_wrt_y0(gslib, oracle, cuda):
    """The float32 route with per-trajectory end times, a row of saved times per trajectory
    (ending at its own t1) and the gradient with respect to y0 and the parameters together:
    against the float64 oracle's dense-output replay and reverse pass over the same float32
    mesh, at the reference's f32 bars."""
    import gradsolve_b200 as gsb
    n = 256
    y0, params = lorenz_batch(n)
    rng = np.random.default_rng(3)
    t1v = rng.uniform(0.5, 1.0, n)
    ts = t1v[:, None] * np.linspace(0.0, 1.0, 9)[None, :]
    clo = gsb.grad_closure(Lorenz(), y0, params, precision="float32", t1=t1v, saveat=ts,
                           wrt=("y0", "params"), rtol=1e-6, atol=1e-9)
    z = torch.tensor(y0, dtype=torch.float32, device="cuda", requires_grad=True)
    p = torch.tensor(params, dtype=torch.float32, device="cuda", requires_grad=True)
    ys = clo(z, p)
    assert ys.dtype == torch.float32 and ys.shape == (n, 9, 3)
    (ys.double() ** 2).sum().backward()
    dts = clo.state.record.padded_dts().cpu().numpy().astype(np.float64)
    _yf, ys64 = oracle.replay_saveat("tsit5", "lorenz", y0, params, dts, ts, nthreads=8)
    gy64, gp64 = oracle.replay_saveat_vjp("tsit5", "lorenz", y0, params, dts, ts, 2.0 * ys64,
                                          nthreads=8)
    y32 = ys.detach().cpu().numpy().astype(np.float64)
    ey = float(np.max(np.abs(y32 - ys64) / np.abs(ys64).max(axis=(1, 2), keepdims=True)))
    g32 = np.concatenate([z.grad.cpu().numpy().ravel(), p.grad.cpu().numpy().ravel()])
    g64 = np.concatenate([gy64.ravel(), gp64.ravel()])
    rel, cos = rel_l2(g32.astype(np.float64), g64), cosine(g32.astype(np.float64), g64)
    print(f"uneven f32 saveat: ys row error {ey:.2e}, grad rel-L2 {rel:.3e}, 1 - cos {1 - cos:.2e}")
    assert ey <= 1e-4
    assert rel <= GRAD_REL_L2_TOL
    assert cos >= 1 - GRAD_COSINE_TOL


@pytest.mark.parametrize("n,K,uneven", [(1, 2, False), (5, 3, True), (2048, 2, False),
                                        (4099, 1, True), (4099, 2, True), (4099, 8, False)])
def test_pairs_agree_with_one_trajectory_per_thread(gslib, cuda, n, K, uneven):
    """The float32 reverse pass two trajectories per thread (packed float32x2, the default for
    the built-in nonstiff fields) against one per thread on the same record: bit for bit
    equal (both evaluate each step with the same explicit contractions), for odd batches (a
    half without a trajectory), lanes ordered by step count (from 4096 trajectories),
    neighbours with different step counts (per-trajectory end times) and several checkpoint
    intervals."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    spec = field_spec("lorenz")
    rng = np.random.default_rng(n + K)
    y0 = torch.tensor(np.tile([1.0, 0.0, 0.0], (n, 1)) + 0.1 * rng.standard_normal((n, 3)),
                      device="cuda")
    p = torch.tensor(rng.uniform(20.0, 30.0, (n, 1)), device="cuda")
    t1v = torch.tensor(rng.uniform(0.2, 1.0, n), device="cuda") if uneven else None
    r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=1.0, t1v=t1v, rtol=1e-6,
                              atol=1e-9, precision="float32", checkpoint=K)
    ybar = 2.0 * r.y_final
    out = {}
    for variant in ("pairs", "recompute"):
        out[variant] = engine.adjoint(r, p, ybar, precision="float32", variant=variant)
    auto = engine.adjoint(r, p, ybar, precision="float32")
    for a, b, c in zip(out["pairs"], out["recompute"], auto):
        a, b, c = a.cpu().numpy(), b.cpu().numpy(), c.cpu().numpy()
        assert np.array_equal(a, c)  # auto is pairs for this field
        assert np.all(np.isfinite(a))
        assert np.array_equal(a, b), f"pairs vs one per thread: rel-L2 {rel_l2(a, b):.3e}"
