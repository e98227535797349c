"""Parity of the CUDA Rosenbrock23 path with the reference.

Bars (float64):
  * forward record vs the reference's own Rosenbrock23 specification
    (tests/_oracles/gradsolve_g2_spike_oracle.py:138-184, captured in tests/golden/):
    accepted/rejected counts identical, y_final within the LU rounding floor the
    reference documents (its test holds atol 1e-7; we hold 1e-9 relative), and within
    1e-10 relative of the oracle restatement of the fused kernel's arithmetic;
  * gradients of the replay within 1e-9 relative of the oracle's reverse pass and of
    torch-float64 autograd (which differentiates jacrev + linalg.solve), and within 1e-5
    of central finite differences (tests/test_adjoint_replay.py:272-317).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu

CASES = ["robertson_toy", "robertson_stiff"]


def rel(a, b, floor=1e-300):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def _spec():
    from gradsolve_b200.fields import field_spec
    return field_spec("robertson")


@pytest.mark.parametrize("case", CASES)
def test_forward_record_matches_reference(gslib, oracle, cuda, case):
    from gradsolve_b200 import engine
    g = load_golden(case)
    r = engine.forward_record("rosenbrock23", _spec(), torch.tensor(g["y0"], device=cuda),
                              torch.tensor(g["params"], device=cuda), t0=float(g["t0"]),
                              t1=float(g["t1"]), rtol=float(g["rtol"]), atol=float(g["atol"]),
                              max_steps=50000)
    np.testing.assert_array_equal(r.status.cpu().numpy(), g["status"])
    np.testing.assert_array_equal(r.n_acc.cpu().numpy(), g["n_acc"])
    np.testing.assert_array_equal(r.n_rej.cpu().numpy(), g["n_rej"])
    yf = r.y_final.cpu().numpy()
    assert rel(yf, g["y_final"], 1e-10) <= 1e-9
    o = oracle.record("rosenbrock23", "robertson", g["y0"], g["params"], float(g["t0"]),
                      float(g["t1"]), float(g["rtol"]), float(g["atol"]), max_steps=50000)
    assert rel(yf, o["y_final"], 1e-10) <= 1e-10
    from test_gpu_tsit5 import check_dts
    check_dts(r.padded_dts().cpu().numpy(), o["dts"])


# K = 64: the kept factors of a segment's replay no longer fit shared memory (D = 3), so the
# reverse pass recomputes every step's factors -- the other of its two code paths
@pytest.mark.parametrize("checkpoint", [1, 2, 16, 64, "sqrt"])
@pytest.mark.parametrize("case", CASES)
def test_adjoint_of_reference_dts(gslib, oracle, cuda, case, checkpoint):
    from gradsolve_b200 import engine
    g = load_golden(case)
    dts = torch.tensor(g["dts"], device=cuda)
    r = engine.record_from_padded("rosenbrock23", _spec(), dts, float(g["t0"]),
                                  checkpoint=checkpoint)
    y0 = torch.tensor(g["y0"], device=cuda)
    p = torch.tensor(g["params"], device=cuda)
    yf = engine.replay(r, y0, p)
    ref_y = oracle.replay("rosenbrock23", "robertson", g["y0"], g["params"], g["dts"])
    assert rel(yf.cpu().numpy(), ref_y, 1e-10) <= 1e-10
    ybar = torch.zeros_like(yf)
    ybar[:, 1] = 2.0 * yf[:, 1]  # loss sum(y[:,1]**2), the stiff intermediate species
    gy0, gp = engine.adjoint(r, p, ybar)
    oy, op = oracle.replay_vjp("rosenbrock23", "robertson", g["y0"], g["params"], g["dts"],
                               ybar.cpu().numpy())
    assert rel(gy0.cpu().numpy(), oy, 1e-8) <= 1e-9
    assert rel(gp.cpu().numpy(), op, 1e-12) <= 1e-9


def test_adjoint_vs_torch_autograd_and_fd(gslib, oracle, cuda):
    from gradsolve_b200 import engine
    g = load_golden("robertson_toy")
    dts = torch.tensor(g["dts"], device=cuda)
    r = engine.record_from_padded("rosenbrock23", _spec(), dts, 0.0)
    y0 = torch.tensor(g["y0"], device=cuda)
    p = torch.tensor(g["params"], device=cuda)
    yf = engine.replay(r, y0, p)
    ybar = torch.zeros_like(yf)
    ybar[:, 1] = 2.0 * yf[:, 1]
    gy0, gp = engine.adjoint(r, p, ybar)
    ty, tp = oracle.torch_replay_grad("rosenbrock23", "robertson", g["y0"], g["params"],
                                      g["dts"], ybar.cpu().numpy())
    assert rel(gy0.cpu().numpy(), ty, 1e-8) <= 1e-9
    assert rel(gp.cpu().numpy(), tp, 1e-12) <= 1e-9

    def loss(q):
        out = engine.replay(r, y0, torch.tensor(q, device=cuda).contiguous(), write_ckpt=False)
        return float((out[:, 1] ** 2).sum().item())

    fd = oracle.fd_grad(loss, g["params"].copy())
    assert rel(gp.cpu().numpy(), fd, 1e-8) < 1e-5


def test_stiff_grad_closure_canonical_robertson(oracle, cuda):
    """Canonical Robertson (0.04, 3e7, 1e4) through grad_closure, y0-gradient vs frozen-mesh
    FD (tests/test_grad_closure_y0.py:135-137, 307-343)."""
    import gradsolve_b200 as gsb

    class Robertson:
        name = "robertson"
        dim = 3
        t0 = 0.0
        t1 = 1.0
        is_stiff = True

    y0 = np.tile(np.array([1.0, 0.0, 0.0]), (2, 1))
    params = np.tile(np.array([0.04, 3.0e7, 1.0e4]), (2, 1))
    clo = gsb.grad_closure(Robertson(), y0, params, wrt="y0")
    assert clo.route.actual == "b200_rosenbrock23"
    z = torch.tensor(y0, device="cuda", requires_grad=True)
    (clo(z) ** 2).sum().backward()

    def loss(zz):
        with torch.no_grad():
            return float((clo(torch.tensor(zz, device="cuda")) ** 2).sum().item())

    fd = oracle.fd_grad(loss, y0)
    g = z.grad.cpu().numpy()
    assert float(np.linalg.norm(g - fd) / np.linalg.norm(fd)) <= 1e-6


@pytest.mark.parametrize("method,case,field", [("rosenbrock23", "robertson_stiff", "robertson"),
                                               ("tsit5", "lorenz_scale", "lorenz")])
def test_forward_only_solve_matches_recording_forward(gslib, cuda, method, case, field):
    """The forward-only solve (no record, no checkpoints: the store paths compiled out of
    the kernel) takes the recording forward's steps: the same counts and statuses, and
    y_final to rounding (another instance of the same expressions)."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    g = load_golden(case)
    spec = field_spec(field)
    y0 = torch.tensor(g["y0"], device=cuda)
    p = torch.tensor(g["params"][:, : spec.nparam], device=cuda).contiguous()
    kw = dict(t0=float(g["t0"]), t1=float(g["t1"]), rtol=float(g["rtol"]),
              atol=float(g["atol"]), max_steps=50000, schedule="static")
    if "dt0" in g:
        kw["dt0"] = float(g["dt0"])
    a = engine.forward_record(method, spec, y0, p, record=True, **kw)
    b = engine.forward_record(method, spec, y0, p, record=False, **kw)
    torch.cuda.synchronize()
    for x, y in ((a.n_acc, b.n_acc), (a.n_rej, b.n_rej), (a.status, b.status)):
        assert torch.equal(x, y)
    assert rel(b.y_final.cpu().numpy(), a.y_final.cpu().numpy(), 1e-12) <= 1e-12
