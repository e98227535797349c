"""The frozen-mesh replay, its cotangent and reverse pass captured as one CUDA graph
(engine.ReplayGraph), through the C ABI.

Bars: every re-launch gives bit for bit what replay + adjoint give called one by one at the
same point (two points in a row, so the second launch also shows the first left nothing
behind), on a reference golden batch and on a batch large enough for the ordered reverse
lanes and the occupancy instances; the gradient at a point away from the recording one
within 1e-9 (row-relative) of the oracle's reverse pass on the same mesh
(gradsolve/warp/warp_replay.py:186-237 is the reference's replay gradient).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _spec(field):
    from gradsolve_b200.fields import field_spec
    return field_spec(field)


def rowrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    num = np.max(np.abs(a - b), axis=1)
    den = np.maximum(np.max(np.abs(b), axis=1), 1e-300)
    return float(np.max(num / den)) if a.size else 0.0


def _eager(engine, r, y0, p, cot):
    yf = engine.replay(r, y0, p, write_ckpt=True)
    gy0, gp = engine.adjoint(r, p, cot(yf))
    torch.cuda.synchronize()
    return yf.cpu(), gy0.cpu(), gp.cpu()


def _check_against_eager(engine, r, y0, p, points):
    cot = lambda yf: 2.0 * yf  # noqa: E731  (d/dy of sum(y_final**2))
    g = engine.ReplayGraph(r, y0, p, cot)
    for y0k, pk in points:
        got = [t.cpu() for t in g(y0k, pk)]
        want = _eager(engine, r, y0k, pk, cot)
        for x, y in zip(got, want):
            assert torch.equal(x, y)
    return g


def test_replay_graph_golden(gslib, cuda, oracle):
    from gradsolve_b200 import engine
    gd = load_golden("lorenz_scale")
    spec = _spec("lorenz")
    y0 = torch.tensor(gd["y0"], device=cuda)
    p = torch.tensor(gd["params"][:, :1], device=cuda).contiguous()
    r = engine.forward_record("tsit5", spec, y0, p, t0=float(gd["t0"]), t1=float(gd["t1"]),
                              rtol=float(gd["rtol"]), atol=float(gd["atol"]), checkpoint=2)
    p2 = p * 1.001
    g = _check_against_eager(engine, r, y0, p, [(y0, p2), (y0 * 0.999, p)])
    yf, gy0, gp = (t.cpu().numpy() for t in g(y0, p2))
    dts = r.padded_dts().cpu().numpy()
    oy, op = oracle.replay_vjp("tsit5", "lorenz", gd["y0"], p2.cpu().numpy(), dts, 2.0 * yf,
                               t0=float(gd["t0"]))
    assert rowrel(np.hstack([gy0, gp]), np.hstack([oy, op[:, :1]])) <= 1e-9


def test_replay_graph_large_batch(gslib, cuda):
    """8192 trajectories: the reverse pass runs its ordered lanes and the occupancy instances
    inside the graph."""
    from gradsolve_b200 import engine
    spec = _spec("lorenz")
    rng = np.random.default_rng(11)
    n = 8192
    y0 = torch.tensor(np.array([1.0, 0.0, 0.0]) + rng.normal(0, 0.1, (n, 3)), device=cuda)
    p = torch.tensor(rng.uniform(20, 30, (n, 1)), device=cuda)
    r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=1.0, rtol=1e-8, atol=1e-8,
                              checkpoint=2)
    _check_against_eager(engine, r, y0, p, [(y0, p + 0.01), (y0, p - 0.01), (y0, p)])


def test_replay_graph_refusals(gslib, cuda):
    from gradsolve_b200 import engine
    gd = load_golden("lorenz_small")
    spec = _spec("lorenz")
    y0 = torch.tensor(gd["y0"], device=cuda)
    p = torch.tensor(gd["params"][:, :1], device=cuda).contiguous()
    r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=0.5, rtol=1e-6, atol=1e-6,
                              checkpoint=2, precision="float32")
    with pytest.raises(TypeError, match="float64"):
        engine.ReplayGraph(r, y0, p, lambda yf: yf)
    with pytest.raises(TypeError, match="single Record"):
        engine.ReplayGraph(object(), y0, p, lambda yf: yf)
