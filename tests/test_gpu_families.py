"""The reference's other fused-lane fields on the GPU, through the C ABI, against the oracle
and the reference's own outputs (tests/golden/, made by tests/golden/make_golden.py from the
reference's tsit5_adaptive and its numpy Rosenbrock23 oracle):

  * lorenz96_<D> and linear_ladder_<D> on the Tsit5 lane (gradsolve/warp/warp_ode.py:463-510):
    D = 5 (a library of its own, built on first use), 8 (one thread per trajectory), 10
    (two lanes of five components) and 32 (eight lanes of four components);
  * hires and a registered constant-matrix linstiff field on the Rosenbrock23 lane
    (gradsolve/warp/warp_rosenbrock.py:221-254);
  * the dimension limit (gradsolve/warp/warp_ode.py:649-664): refused before any launch.

Bars as for the other fields: counts exact against the reference, y_final within 1e-10 of
the reference (Tsit5) / of the oracle (Rosenbrock23; 1e-9 of the reference's LAPACK solves),
dts as check_dts; replay of the reference's dts within 1e-10 of the oracle's, gradients
within 1e-9 of the oracle's reverse pass and within 1e-6 (Tsit5) / 1e-5 (Rosenbrock23) of
frozen-mesh central differences.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu

TSIT5_CASES = [("lorenz96_5", "lorenz96_5"), ("lorenz96_8", "lorenz96_8"),
               ("lorenz96_32", "lorenz96_32"), ("linear_10", "linear_10"),
               ("linear_32", "linear_32")]
ROS_CASES = ["hires", "linstiff_4", "linstiff_8"]


def rel(a, b, floor=1e-300):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def rowrel(a, b):
    """Worst trajectory's max-norm error relative to its own row's max-norm: the measure for
    many-component states, whose chaotic mixing leaves some gradient components orders of
    magnitude below the row (an entrywise ratio would measure cancellation, not error)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-300)))


def _spec(field):
    from gradsolve_b200.fields import field_spec
    return field_spec(field)


def _ros_spec(case, oracle=None):
    """The field of a Rosenbrock23 case: hires is built in; a linstiff case registers its
    matrix (and points the oracle's linstiff field at it)."""
    g = load_golden(case)
    if case == "hires":
        return _spec("hires"), "hires", g
    import gradsolve_b200 as gsb
    spec = gsb.register_linstiff(f"linstiff_test_{g['A'].shape[0]}", g["A"])
    name = oracle.set_linstiff(g["A"]) if oracle is not None else None
    return spec, name, g


def _inputs(cuda, spec, g):
    y0 = torch.tensor(g["y0"], device=cuda)
    p = torch.tensor(g["params"][:, : spec.nparam], device=cuda).contiguous()
    return y0, p


@pytest.mark.parametrize("case,field", TSIT5_CASES)
def test_forward_record_matches_reference(gslib, cuda, case, field):
    from gradsolve_b200 import engine
    from test_gpu_tsit5 import check_dts
    g = load_golden(case)
    spec = _spec(field)
    y0, p = _inputs(cuda, spec, g)
    r = engine.forward_record("tsit5", spec, y0, p, t0=float(g["t0"]), t1=float(g["t1"]),
                              rtol=float(g["rtol"]), atol=float(g["atol"]), max_steps=100000)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(r.status.cpu().numpy(), g["status"])
    np.testing.assert_array_equal(r.n_acc.cpu().numpy(), g["n_acc"])
    np.testing.assert_array_equal(r.n_rej.cpu().numpy(), g["n_rej"])
    assert rel(r.y_final.cpu().numpy(), g["y_final"], 1e-12) <= 1e-10
    check_dts(r.padded_dts().cpu().numpy(), g["dts"], float(g["rtol"]))


@pytest.mark.parametrize("case,field", TSIT5_CASES)
def test_forward_value_equals_replay_value(gslib, cuda, case, field):
    """The recording pass and the replay evaluate the same expressions, the group's lanes
    included: y_final and every checkpoint bitwise equal."""
    from gradsolve_b200 import engine
    g = load_golden(case)
    spec = _spec(field)
    y0, p = _inputs(cuda, spec, g)
    r = engine.forward_record("tsit5", spec, y0, p, t0=float(g["t0"]), t1=float(g["t1"]),
                              rtol=float(g["rtol"]), atol=float(g["atol"]), checkpoint=3)
    yf, ck = r.y_final.clone(), r.ckpt.clone()
    yr = engine.replay(r, y0, p, write_ckpt=True)
    torch.cuda.synchronize()
    assert torch.equal(yf, yr)
    D = spec.dim
    CW = (D + 2) & ~1
    slots = (int(r.n_acc.max()) + 2) // 3 + 1
    a = ck[: slots * r.n * CW].view(slots, r.n, CW).cpu().numpy()
    b = r.ckpt[: slots * r.n * CW].view(slots, r.n, CW).cpu().numpy()
    n_acc = r.n_acc.cpu().numpy()
    for j in range(r.n):
        m = n_acc[j] // 3 + 1
        np.testing.assert_array_equal(a[:m, j, : D + 1], b[:m, j, : D + 1])


@pytest.mark.parametrize("checkpoint", [1, 2, 5, "sqrt"])
@pytest.mark.parametrize("case,field", TSIT5_CASES)
def test_adjoint_of_reference_dts(gslib, oracle, cuda, case, field, checkpoint):
    from gradsolve_b200 import engine
    g = load_golden(case)
    spec = _spec(field)
    dts = torch.tensor(g["dts"], device=cuda)
    r = engine.record_from_padded("tsit5", spec, dts, float(g["t0"]), checkpoint=checkpoint)
    y0, p = _inputs(cuda, spec, g)
    yf = engine.replay(r, y0, p, write_ckpt=True)
    ref = oracle.replay("tsit5", field, g["y0"], g["params"], g["dts"])
    assert rowrel(yf.cpu().numpy(), ref) <= 1e-10
    ybar = torch.linspace(-1.0, 1.5, yf.numel(), dtype=torch.float64,
                          device=cuda).reshape(yf.shape) * yf
    gy0, gp = engine.adjoint(r, p, ybar)
    torch.cuda.synchronize()
    oy, op = oracle.replay_vjp("tsit5", field, g["y0"], g["params"], g["dts"], ybar.cpu().numpy())
    assert rowrel(gy0.cpu().numpy(), oy) <= 1e-9
    if field.startswith("lorenz96_"):
        assert rel(gp.cpu().numpy(), op[:, :1], 1e-8) <= 1e-9


def test_checkpoint_interval_does_not_change_the_group_gradient(gslib, cuda):
    """Eight lanes per trajectory: the segments recompute the recorded states bit for bit,
    so every checkpoint interval gives the same gradient bit for bit."""
    from gradsolve_b200 import engine
    g = load_golden("lorenz96_32")
    spec = _spec("lorenz96_32")
    y0, p = _inputs(cuda, spec, g)
    outs = []
    for K in (1, 2, 7, 64):
        r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=float(g["t1"]),
                                  rtol=float(g["rtol"]), atol=float(g["atol"]), checkpoint=K)
        gy0, gp = engine.adjoint(r, p, 2.0 * r.y_final)
        outs.append((gy0.cpu().numpy(), gp.cpu().numpy()))
    for gy, gpp in outs[1:]:
        np.testing.assert_array_equal(gy, outs[0][0])
        np.testing.assert_array_equal(gpp, outs[0][1])


def test_group_gradient_vs_fd_and_torch(gslib, oracle, cuda):
    """d sum(y_final^2) / dF of Lorenz-96 with 32 components (eight lanes), against frozen-
    mesh central differences through the GPU replay and torch-float64 autograd."""
    from gradsolve_b200 import engine
    g = load_golden("lorenz96_32")
    spec = _spec("lorenz96_32")
    y0, p = _inputs(cuda, spec, g)
    dts = torch.tensor(g["dts"], device=cuda)
    r = engine.record_from_padded("tsit5", spec, dts, 0.0, checkpoint="sqrt")
    yf = engine.replay(r, y0, p, write_ckpt=True)
    gy0, gp = engine.adjoint(r, p, 2.0 * yf)
    ty, tp = oracle.torch_replay_grad("tsit5", "lorenz96_32", g["y0"], g["params"], g["dts"],
                                      2.0 * yf.cpu().numpy())
    # dL/dF sums 32 contributions of the size of the state sensitivities (~5e3 here), which
    # cancel to ~10: it is compared within the whole gradient row of the trajectory
    assert rowrel(np.hstack([gy0.cpu().numpy(), gp.cpu().numpy()]), np.hstack([ty, tp])) <= 1e-9

    def loss(q):
        qq = torch.tensor(q, device=cuda).contiguous()
        return float((engine.replay(r, y0, qq, write_ckpt=False) ** 2).sum().item())

    fd = oracle.fd_grad(loss, g["params"][:, :1].copy())
    assert rel(gp.cpu().numpy(), fd, 1e-8) < 1e-6


def test_group_paths_refuse_modes_not_built(gslib, cuda):
    from gradsolve_b200 import engine
    from gradsolve_b200._lib import GsolveError
    g = load_golden("lorenz96_32")
    spec = _spec("lorenz96_32")
    y0, p = _inputs(cuda, spec, g)
    with pytest.raises(GsolveError, match="float32-stage"):
        engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=0.5, rtol=1e-6, atol=1e-6,
                              precision="mixed")
    r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=0.5, rtol=1e-6, atol=1e-6)
    with pytest.raises(GsolveError, match="more than 8 components"):
        engine.replay_saveat(r, y0, p, torch.linspace(0.0, 0.5, 4, dtype=torch.float64,
                                                      device=cuda))


def test_dimension_limit_refused_before_launch(gslib, cuda):
    import gradsolve_b200 as gsb

    class Big:
        name = "lorenz96_65"
        dim = 65
        t0, t1 = 0.0, 1.0
        is_stiff = False

    y0 = np.ones((2, 65))
    with pytest.raises(RuntimeError, match="register-vector limit: dim=65 > 64"):
        gsb.solve(Big(), y0, np.full((2, 1), 8.0), device="cuda")
    with pytest.raises(RuntimeError, match="dim=65 > 64"):
        gsb.register_field("too_big", lambda t, y, p: [v for v in y], 65, 0)


@pytest.mark.parametrize("case", ROS_CASES)
def test_ros23_forward_matches_reference(gslib, oracle, cuda, case):
    from gradsolve_b200 import engine
    from test_gpu_tsit5 import check_dts
    spec, name, g = _ros_spec(case, oracle)
    y0, p = _inputs(cuda, spec, g)
    r = engine.forward_record("rosenbrock23", spec, y0, p, t0=float(g["t0"]), t1=float(g["t1"]),
                              rtol=float(g["rtol"]), atol=float(g["atol"]), max_steps=50000)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(r.status.cpu().numpy(), g["status"])
    np.testing.assert_array_equal(r.n_acc.cpu().numpy(), g["n_acc"])
    np.testing.assert_array_equal(r.n_rej.cpu().numpy(), g["n_rej"])
    yf = r.y_final.cpu().numpy()
    assert rel(yf, g["y_final"], 1e-10) <= 1e-9
    o = oracle.record("rosenbrock23", name, g["y0"], g["params"], float(g["t0"]),
                      float(g["t1"]), float(g["rtol"]), float(g["atol"]), max_steps=50000)
    assert rel(yf, o["y_final"], 1e-10) <= 1e-10
    check_dts(r.padded_dts().cpu().numpy(), o["dts"])


@pytest.mark.parametrize("checkpoint", [1, 2, 16])
@pytest.mark.parametrize("case", ROS_CASES)
def test_ros23_adjoint_of_reference_dts(gslib, oracle, cuda, case, checkpoint):
    from gradsolve_b200 import engine
    spec, name, g = _ros_spec(case, oracle)
    dts = torch.tensor(g["dts"], device=cuda)
    r = engine.record_from_padded("rosenbrock23", spec, dts, float(g["t0"]),
                                  checkpoint=checkpoint)
    y0, p = _inputs(cuda, spec, g)
    yf = engine.replay(r, y0, p)
    ref_y = oracle.replay("rosenbrock23", name, g["y0"], g["params"], g["dts"])
    assert rowrel(yf.cpu().numpy(), ref_y) <= 1e-10
    ybar = 2.0 * yf
    gy0, _gp = engine.adjoint(r, p, ybar)
    oy, _op = oracle.replay_vjp("rosenbrock23", name, g["y0"], g["params"], g["dts"],
                                ybar.cpu().numpy())
    assert rowrel(gy0.cpu().numpy(), oy) <= 1e-9


@pytest.mark.parametrize("case", ["hires", "linstiff_4"])
def test_ros23_gradient_vs_fd(gslib, oracle, cuda, case):
    """d sum(y_final^2) / dy0 through the frozen mesh against central differences (the
    parameters of these fields are placeholders, so the state is the input)."""
    from gradsolve_b200 import engine
    spec, name, g = _ros_spec(case, oracle)
    g = {k: (v[:2] if getattr(v, "ndim", 0) >= 1 and v.shape[0] == g["y0"].shape[0] else v)
         for k, v in g.items()}
    dts = torch.tensor(g["dts"], device=cuda)
    r = engine.record_from_padded("rosenbrock23", spec, dts, float(g["t0"]), checkpoint=4)
    y0, p = _inputs(cuda, spec, g)
    yf = engine.replay(r, y0, p)
    gy0, _gp = engine.adjoint(r, p, 2.0 * yf)

    def loss(z):
        zz = torch.tensor(z, device=cuda).contiguous()
        return float((engine.replay(r, zz, p, write_ckpt=False) ** 2).sum().item())

    # HIRES's 280 y5 y7 coupling curves the loss along y7 (~0.0057), where the usual step
    # 1e-6 max(1, |y|) is 1.8e-4 of the value: the central difference's own truncation error
    # there is 9.4e-5 (the oracle's gradient shows the same), falling as h^2 -- so HIRES
    # takes the step 1e-7 (truncation 9.4e-7)
    fd = oracle.fd_grad(loss, g["y0"].copy(), h_scale=1e-7 if case == "hires" else 1e-6)
    assert rowrel(gy0.cpu().numpy(), fd) < 1e-5


def test_public_api_routes_the_families(gslib, oracle, cuda):
    """solve / grad_closure by problem name: lorenz96_<D> and linear_ladder_<D> on the Tsit5
    engine (any D up to the limit), hires and a registered linstiff_* field on the
    Rosenbrock23 engine, with the reference's engine names accepted."""
    import gradsolve_b200 as gsb

    class L96:
        name = "lorenz96_32"
        dim = 32
        t0, t1 = 0.0, 2.0
        is_stiff = False

    class Hires:
        name = "hires"
        dim = 8
        t0, t1 = 0.0, 321.8122
        is_stiff = True

    g = load_golden("lorenz96_32")
    res = gsb.solve(L96(), g["y0"], g["params"], rtol=1e-8, atol=1e-8, engine="warp_ode")
    assert res.route.actual == "b200_tsit5"
    np.testing.assert_array_equal(res.accepted_steps, g["n_acc"])
    clo = gsb.grad_closure(L96(), g["y0"], g["params"], rtol=1e-8, atol=1e-8)
    pt = torch.tensor(g["params"], device="cuda", requires_grad=True)
    yf = clo(pt)
    (yf ** 2).sum().backward()
    dts = clo.state.record.padded_dts().cpu().numpy()
    ry = oracle.replay("tsit5", "lorenz96_32", g["y0"], g["params"], dts)
    _, rg = oracle.replay_vjp("tsit5", "lorenz96_32", g["y0"], g["params"], dts, 2.0 * ry)
    assert rel(pt.grad.cpu().numpy(), rg, 1e-8) <= 1e-9

    h = load_golden("hires")
    res = gsb.solve(Hires(), h["y0"], h["params"], rtol=1e-6, atol=1e-10, max_steps=50000)
    assert res.route.actual == "b200_rosenbrock23"
    np.testing.assert_array_equal(res.accepted_steps, h["n_acc"])

    A = load_golden("linstiff_4")["A"]
    spec = gsb.register_linstiff("linstiff_test_4", A)
    assert gsb.register_linstiff("linstiff_test_4", A) is spec and spec.stiff_ok

    class LS:
        name = "linstiff_test_4"
        dim = 4
        t0, t1 = 0.0, 1.0
        is_stiff = True

    ls = load_golden("linstiff_4")
    res = gsb.solve(LS(), ls["y0"], ls["params"], rtol=1e-6, atol=1e-9, engine="warp_rosenbrock")
    assert res.route.actual == "b200_rosenbrock23"
    np.testing.assert_array_equal(res.accepted_steps, ls["n_acc"])


@pytest.mark.parametrize("field", ["lorenz96_32", "linear_32"])
def test_every_built_group_size_matches_the_oracle(gslib, oracle, cuda, field):
    """Each group size the library builds for a 32-component field (8 lanes of 4 by default,
    4 of 8 and 16 of 2): the forward's counts exact and y_final against the reference, the
    replay and gradient of the reference's dts against the oracle; an unbuilt size (32 lanes
    of 1) is refused."""
    from gradsolve_b200 import engine
    from gradsolve_b200._lib import GsolveError
    from test_gpu_tsit5 import check_dts
    g = load_golden(field)
    spec = _spec(field)
    y0, p = _inputs(cuda, spec, g)
    choices = engine.lane_choices(spec)
    assert choices == [8, 4, 16]
    try:
        for G in choices:
            engine.set_lanes(spec, G)
            r = engine.forward_record("tsit5", spec, y0, p, t0=float(g["t0"]), t1=float(g["t1"]),
                                      rtol=float(g["rtol"]), atol=float(g["atol"]), checkpoint=3)
            np.testing.assert_array_equal(r.n_acc.cpu().numpy(), g["n_acc"])
            np.testing.assert_array_equal(r.n_rej.cpu().numpy(), g["n_rej"])
            assert rowrel(r.y_final.cpu().numpy(), g["y_final"]) <= 1e-10
            check_dts(r.padded_dts().cpu().numpy(), g["dts"], float(g["rtol"]))
            rr = engine.record_from_padded("tsit5", spec, torch.tensor(g["dts"], device=cuda),
                                           0.0, checkpoint=2)
            yf = engine.replay(rr, y0, p, write_ckpt=True)
            gy0, gp = engine.adjoint(rr, p, 2.0 * yf)
            oy, op = oracle.replay_vjp("tsit5", field, g["y0"], g["params"], g["dts"],
                                       2.0 * yf.cpu().numpy())
            # (dL/dF compared within the trajectory's whole gradient row: it sums cancelling
            # contributions of the state sensitivities' size)
            assert rowrel(np.hstack([gy0.cpu().numpy(), gp.cpu().numpy()]),
                          np.hstack([oy, op[:, :1]])) <= 1e-9
        with pytest.raises(ValueError, match="not built"):
            engine.set_lanes(spec, 32)
        engine._LANES[spec.key] = 32  # bypass the check: the library itself refuses
        with pytest.raises(GsolveError, match="32 lanes"):
            engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=0.5, rtol=1e-6, atol=1e-6,
                                  checkpoint=3)
    finally:
        engine.set_lanes(spec, None)
