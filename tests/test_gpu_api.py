"""The public API (solve / grad_closure) on the GPU: routing, .route, wrt variants, the
torch.autograd adapter, and gradients against the oracle and finite differences --
the reference's own API-level checks (tests/test_grad_closure_y0.py:144-185, 307-343;
tests/test_adjoint_replay.py:196-216) restated for the B200 engines."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu


class Lorenz:
    name = "diffeqgpu_lorenz"
    dim = 3
    t0 = 0.0
    t1 = 1.0
    is_stiff = False


class Lorenz3:
    name = "lorenz"
    dim = 3
    t0 = 0.0
    t1 = 1.0
    is_stiff = False


class VdP:
    name = "vdp"
    dim = 2
    t0 = 0.0
    t1 = 1.0
    is_stiff = False


class Unregistered:
    name = "my_custom_rhs"
    dim = 2
    t0 = 0.0
    t1 = 1.0
    is_stiff = False


def _rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_solve_matches_reference_counts(cuda):
    import gradsolve_b200 as gsb
    g = load_golden("lorenz_small")
    res = gsb.solve(Lorenz(), g["y0"], g["params"], rtol=1e-8, atol=1e-8, device="cuda")
    assert res.solver == "b200_tsit5"
    assert res.route.actual == "b200_tsit5" and res.route.requested == "auto"
    np.testing.assert_array_equal(res.accepted_steps, g["n_acc"])
    np.testing.assert_array_equal(res.rejected_steps, g["n_rej"])
    assert np.max(np.abs(res.y_final - g["y_final"]) / np.abs(g["y_final"])) <= 1e-10


def test_reference_engine_names_are_served(cuda):
    import gradsolve_b200 as gsb
    g = load_golden("vdp_batch")
    res = gsb.solve(VdP(), g["y0"], g["params"], engine="warp_replay", device="cuda")
    assert res.route.actual == "b200_tsit5"
    assert "served-by-b200_tsit5" in res.route.reason
    with pytest.raises(ValueError, match="unknown engine"):
        gsb.solve(VdP(), g["y0"], g["params"], engine="nope", device="cuda")


def test_unregistered_problem_and_cpu_device_raise(cuda):
    import gradsolve_b200 as gsb
    y0 = np.ones((2, 2))
    with pytest.raises(ValueError, match="no registered field"):
        gsb.grad_closure(Unregistered(), y0, np.ones((2, 1)), device="cuda")
    with pytest.raises(ValueError, match="CUDA devices only"):
        gsb.solve(VdP(), y0, np.ones((2, 1)), device="cpu")


@pytest.mark.parametrize("remat", [None, True, False])
def test_grad_closure_params_matches_oracle(oracle, cuda, remat):
    import gradsolve_b200 as gsb
    g = load_golden("lorenz_small")
    clo = gsb.grad_closure(Lorenz(), g["y0"], g["params"], rtol=1e-8, atol=1e-8, remat=remat)
    assert clo.route.actual == "b200_tsit5"
    p = torch.tensor(g["params"], device="cuda", requires_grad=True)
    yf = clo(p)
    (yf ** 2).sum().backward()
    ref_y = oracle.replay("tsit5", "lorenz", g["y0"], g["params"], g["dts"])
    assert np.max(np.abs(yf.detach().cpu().numpy() - ref_y) / np.abs(ref_y)) <= 1e-10
    _, ref_gp = oracle.replay_vjp("tsit5", "lorenz", g["y0"], g["params"], g["dts"], 2 * ref_y)
    assert np.max(np.abs(p.grad.cpu().numpy() - ref_gp) / np.abs(ref_gp)) <= 1e-9


def test_small_plain_config_through_grad_closure(oracle, cuda):
    """The small plain configuration exactly: Lorenz (sigma = 10, beta = 8/3, rho the
    parameter; the reference's 1-column diffeqgpu_lorenz problem), n = 1024, y0 = [1, 0, 0]
    for all, rho = linspace(20, 30, n) as (n, 1), t in [0, 1], Tsit5 rtol = atol = 1e-8,
    float64; forward solve plus the gradient of sum(y_final**2) w.r.t. rho through
    grad_closure, against the oracle: the oracle's own adaptive solve (step counts exact,
    y_final to 1e-10) and its reverse pass over the recorded mesh (1e-9)."""
    import gradsolve_b200 as gsb
    n = 1024
    y0 = np.tile(np.array([1.0, 0.0, 0.0]), (n, 1))
    rho = np.linspace(20.0, 30.0, n)[:, None]
    res = gsb.solve(Lorenz(), y0, rho, rtol=1e-8, atol=1e-8, device="cuda")
    ref = oracle.record("tsit5", "lorenz", y0, rho, 0.0, 1.0, 1e-8, 1e-8)
    np.testing.assert_array_equal(res.accepted_steps, ref["n_acc"])
    np.testing.assert_array_equal(res.rejected_steps, ref["n_rej"])
    assert np.max(np.abs(res.y_final - ref["y_final"]) / np.abs(ref["y_final"])) <= 1e-10
    clo = gsb.grad_closure(Lorenz(), y0, rho, rtol=1e-8, atol=1e-8, device="cuda")
    p = torch.tensor(rho, device="cuda", requires_grad=True)
    yf = clo(p)
    (yf ** 2).sum().backward()
    dts = clo.state.record.padded_dts().cpu().numpy()
    ry = oracle.replay("tsit5", "lorenz", y0, rho, dts)
    yfn = yf.detach().cpu().numpy()
    assert np.max(np.abs(yfn - ry) / np.abs(ry)) <= 1e-10
    _, rg = oracle.replay_vjp("tsit5", "lorenz", y0, rho, dts, 2.0 * ry)
    assert np.max(np.abs(p.grad.cpu().numpy() - rg) / np.abs(rg)) <= 1e-9
    # and against the oracle's gradient on its own recorded mesh (the reference's route)
    _, rg2 = oracle.replay_vjp("tsit5", "lorenz", y0, rho, ref["dts"], 2.0 * ref["y_final"])
    assert np.max(np.abs(p.grad.cpu().numpy() - rg2) / np.abs(rg2)) <= 1e-8


@pytest.mark.parametrize("wrt", ["y0", ("y0", "params")])
def test_grad_closure_y0_matches_fd(oracle, cuda, wrt):
    """Frozen-mesh FD of the y0 gradient, rel-L2 <= 1e-6 (tests/test_grad_closure_y0.py:145)."""
    import gradsolve_b200 as gsb
    n = 2
    y0 = np.tile(np.array([1.0, 0.0, 0.0]), (n, 1))
    y0[:, 0] += 0.1 * np.arange(n)
    params = np.tile(np.array([28.0]), (n, 1))
    clo = gsb.grad_closure(Lorenz(), y0, params, wrt=wrt)
    z = torch.tensor(y0, device="cuda", requires_grad=True)
    if wrt == "y0":
        out = clo(z)
    else:
        out = clo(z, torch.tensor(params, device="cuda"))
    (out ** 2).sum().backward()

    def loss(zz):
        with torch.no_grad():
            t = torch.tensor(zz, device="cuda")
            o = clo(t) if wrt == "y0" else clo(t, torch.tensor(params, device="cuda"))
            return float((o ** 2).sum().item())

    fd = oracle.fd_grad(loss, y0)
    assert _rel_l2(z.grad.cpu().numpy(), fd) <= 1e-6


def test_closure_off_the_recording_point_replays(oracle, cuda):
    """Perturbed params replay the SAME frozen mesh (the mesh is not re-recorded)."""
    import gradsolve_b200 as gsb
    g = load_golden("vdp_batch")
    clo = gsb.grad_closure(VdP(), g["y0"], g["params"])
    q = g["params"] * 1.01
    out = clo(torch.tensor(q, device="cuda")).cpu().numpy()
    ref = oracle.replay("tsit5", "vdp", g["y0"], q, g["dts"])
    assert np.max(np.abs(out - ref) / np.abs(ref)) <= 1e-10


def test_two_forwards_then_backward_uses_its_own_point(oracle, cuda):
    import gradsolve_b200 as gsb
    g = load_golden("vdp_batch")
    clo = gsb.grad_closure(VdP(), g["y0"], g["params"])
    p1 = torch.tensor(g["params"], device="cuda", requires_grad=True)
    p2 = torch.tensor(g["params"] * 1.02, device="cuda", requires_grad=True)
    y1 = clo(p1)
    y2 = clo(p2)          # rewrites the checkpoints
    (y1 ** 2).sum().backward()
    (y2 ** 2).sum().backward()
    for p, q in ((p1, g["params"]), (p2, g["params"] * 1.02)):
        ry = oracle.replay("tsit5", "vdp", g["y0"], q, g["dts"])
        _, rg = oracle.replay_vjp("tsit5", "vdp", g["y0"], q, g["dts"], 2 * ry)
        assert np.max(np.abs(p.grad.cpu().numpy() - rg) / np.abs(rg)) <= 1e-9


def test_lorenz3_gradient_covers_sigma_beta_rho(oracle, cuda):
    import gradsolve_b200 as gsb
    n = 4
    y0 = np.tile(np.array([1.0, 0.5, 0.2]), (n, 1))
    params = np.column_stack([np.full(n, 10.0), np.full(n, 8.0 / 3.0), np.linspace(20, 30, n)])
    clo = gsb.grad_closure(Lorenz3(), y0, params)
    p = torch.tensor(params, device="cuda", requires_grad=True)
    (clo(p) ** 2).sum().backward()

    def loss(q):
        with torch.no_grad():
            return float((clo(torch.tensor(q, device="cuda")) ** 2).sum().item())

    fd = oracle.fd_grad(loss, params)
    assert _rel_l2(p.grad.cpu().numpy(), fd) <= 1e-6
    assert np.all(np.abs(p.grad.cpu().numpy()) > 0)


def test_extra_param_columns_get_zero_gradient(cuda):
    import gradsolve_b200 as gsb
    g = load_golden("vdp_batch")
    params = np.column_stack([g["params"], np.ones(3)])
    clo = gsb.grad_closure(VdP(), g["y0"], params)
    p = torch.tensor(params, device="cuda", requires_grad=True)
    (clo(p) ** 2).sum().backward()
    assert torch.all(p.grad[:, 1] == 0)
    assert torch.all(p.grad[:, 0] != 0)


def test_max_steps_exhaustion_raises(cuda):
    import gradsolve_b200 as gsb
    y0 = np.array([[1.0]])
    with pytest.raises(RuntimeError, match="exhausted max_steps"):
        gsb.grad_closure(type("P", (), dict(name="linear_ladder_1", dim=1, t0=0.0, t1=1.0,
                                            is_stiff=False))(),
                         y0, np.zeros((1, 1)), max_steps=2)
