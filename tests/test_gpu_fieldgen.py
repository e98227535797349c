"""Generated fields on the GPU: a user field written like a built-in one gives the built-in's
results through its own library (Tsit5 and Rosenbrock23, forward and gradient), and a field
with transcendental functions is differentiated correctly (frozen-mesh finite differences)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu


def rowrel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b).max(axis=-1) / np.maximum(np.abs(b).max(axis=-1), 1e-300)))


def _user_lorenz(t, y, p):
    x, u, z = y
    return [10.0 * (u - x), p[0] * x - u - x * z, x * u - (8.0 / 3.0) * z]


def _user_robertson(t, y, p):
    a, b, c = y
    return [-p[0] * a + p[2] * b * c, p[0] * a - p[2] * b * c - p[1] * b * b, p[1] * b * b]


def _pendulum(t, y, p):
    return [y[1], -p[0] * np.sin(y[0]) - p[1] * y[1] + 0.1 * np.tanh(y[0] * y[1])]


@pytest.mark.parametrize("method,user,builtin,case,rtol,atol", [
    ("tsit5", _user_lorenz, "lorenz", "lorenz_scale", None, None),
    ("rosenbrock23", _user_robertson, "robertson", "robertson_stiff", None, None)])
def test_generated_field_matches_builtin(gslib, cuda, method, user, builtin, case, rtol, atol):
    import gradsolve_b200 as gsb
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    g = load_golden(case)
    ref = field_spec(builtin)
    spec = gsb.register_field(f"gen_{builtin}", user, ref.dim, ref.nparam,
                              stiff=method == "rosenbrock23")
    y0 = torch.tensor(g["y0"], device=cuda)
    p = torch.tensor(g["params"][:, : ref.nparam], device=cuda).contiguous()
    kw = dict(t0=float(g["t0"]), t1=float(g["t1"]), rtol=float(g["rtol"]), atol=float(g["atol"]),
              max_steps=100000, checkpoint=4)
    if "dt0" in g:
        kw["dt0"] = float(g["dt0"])
    outs = []
    for s in (ref, spec):
        r = engine.forward_record(method, s, y0, p, **kw)
        ybar = torch.zeros_like(r.y_final)
        ybar[:, -1] = 1.0
        gy0, gp = engine.adjoint(r, p, ybar)
        torch.cuda.synchronize()
        outs.append((r.n_acc.cpu(), r.n_rej.cpu(), r.y_final.cpu().numpy(),
                     r.padded_dts().cpu().numpy(), gy0.cpu().numpy(), gp.cpu().numpy()))
    (a0, b0, y_ref, d_ref, gy_ref, gp_ref), (a1, b1, y_gen, d_gen, gy_gen, gp_gen) = outs
    assert torch.equal(a0, a1) and torch.equal(b0, b1)
    assert rowrel(y_gen, y_ref) <= 1e-10
    # the two builds contract multiply-adds differently; the dts then differ as the GPU's and
    # the reference's do (the error estimate cancels), so the same bar applies
    from test_gpu_tsit5 import check_dts
    check_dts(d_gen, d_ref)
    assert rowrel(gy_gen, gy_ref) <= 1e-8
    assert rowrel(gp_gen, gp_ref) <= 1e-8


def test_generated_transcendental_field_gradient_vs_fd(gslib, cuda):
    import gradsolve_b200 as gsb
    from gradsolve_b200 import engine
    spec = gsb.register_field("gen_pendulum", _pendulum, 2, 2)
    rng = np.random.default_rng(3)
    n = 64
    y0 = torch.tensor(rng.uniform(-1, 1, (n, 2)), device=cuda)
    p = torch.tensor(np.c_[rng.uniform(5, 15, n), rng.uniform(0.05, 0.3, n)], device=cuda)
    r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=3.0, rtol=1e-9, atol=1e-9,
                              checkpoint=3)
    assert int((r.status != 0).sum()) == 0
    w = torch.tensor(rng.normal(size=(n, 2)), device=cuda)
    gy0, gp = engine.adjoint(r, p, w)
    torch.cuda.synchronize()

    def loss_rows(y0_, p_):
        return (engine.replay(r, y0_, p_, write_ckpt=False) * w).sum(dim=1)
    for k in range(2):  # central differences through the frozen mesh
        e = 1e-6
        pp, pm = p.clone(), p.clone()
        pp[:, k] += e
        pm[:, k] -= e
        fd = ((loss_rows(y0, pp) - loss_rows(y0, pm)) / (2 * e)).cpu().numpy()
        got = gp[:, k].cpu().numpy()
        assert np.max(np.abs(got - fd) / np.maximum(np.abs(fd), 1e-3)) <= 1e-5
        yp, ym = y0.clone(), y0.clone()
        yp[:, k] += e
        ym[:, k] -= e
        fd = ((loss_rows(yp, p) - loss_rows(ym, p)) / (2 * e)).cpu().numpy()
        got = gy0[:, k].cpu().numpy()
        assert np.max(np.abs(got - fd) / np.maximum(np.abs(fd), 1e-3)) <= 1e-5


def test_generated_field_through_the_public_api(gslib, cuda):
    import gradsolve_b200 as gsb
    gsb.register_field("gen_pendulum_api", _pendulum, 2, 2)

    class Pendulum:
        name = "gen_pendulum_api"
        dim = 2
        t0 = 0.0
        t1 = 2.0
        is_stiff = False
    rng = np.random.default_rng(5)
    y0 = rng.uniform(-1, 1, (32, 2))
    p = np.c_[rng.uniform(5, 15, 32), rng.uniform(0.05, 0.3, 32)]
    res = gsb.solve(Pendulum(), y0, p, rtol=1e-8, atol=1e-8)
    clo = gsb.grad_closure(Pendulum(), y0, p, rtol=1e-8, atol=1e-8)
    pt = torch.tensor(p, device=cuda, requires_grad=True)
    yf = clo(pt)
    np.testing.assert_allclose(yf.detach().cpu().numpy(), res.y_final, rtol=1e-12, atol=1e-14)
    (yf ** 2).sum().backward()
    assert torch.isfinite(pt.grad).all() and float(pt.grad.abs().sum()) > 0
