"""The CPU oracle against the reference's own outputs (tests/golden/, made by
tests/golden/make_golden.py from the reference's tsit5_adaptive and Rosenbrock23 oracle).

Tsit5: the oracle is a restatement of gradsolve/solvers/tsit5_replay.py:62-124 in the same
operation order, so accepted/rejected counts, every recorded dt and y_final must match
bit for bit.  Rosenbrock23: the reference oracle solves W with numpy's LAPACK LU while the
restatement follows the fused kernel's division-based elimination
(gradsolve/warp/_warp_rosenbrock.py:346-381); counts must match exactly and values agree at
the LU rounding level the reference documents (tests/test_adjoint_replay.py:232-254 uses
atol 1e-7; we hold 1e-12 relative on y_final, 1e-9 median and 1e-7 maximum on the dts).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden

TSIT5_CASES = [("lorenz_small", "lorenz"), ("lorenz_scale", "lorenz"), ("vdp_batch", "vdp"),
               ("lv_mixed", "lv"), ("linear3", "linear_3"), ("lorenz96_5", "lorenz96_5"),
               ("lorenz96_8", "lorenz96_8"), ("lorenz96_32", "lorenz96_32"),
               ("linear_10", "linear_10"), ("linear_32", "linear_32")]
ROS_CASES = [("robertson_toy", "robertson"), ("robertson_stiff", "robertson"),
             ("hires", "hires"), ("linstiff_4", "linstiff_4"), ("linstiff_8", "linstiff_8")]


def _run(oracle, method, field, g, nthreads=4):
    if field.startswith("linstiff_"):
        assert oracle.set_linstiff(g["A"]) == field
    return oracle.record(method, field, g["y0"], g["params"], float(g["t0"]), float(g["t1"]),
                         float(g["rtol"]), float(g["atol"]), max_steps=100000, nthreads=nthreads)


@pytest.mark.parametrize("case,field", TSIT5_CASES)
def test_tsit5_oracle_bitwise_vs_reference(oracle, case, field):
    g = load_golden(case)
    r = _run(oracle, "tsit5", field, g)
    np.testing.assert_array_equal(r["n_acc"], g["n_acc"])
    np.testing.assert_array_equal(r["n_rej"], g["n_rej"])
    np.testing.assert_array_equal(r["status"], g["status"])
    np.testing.assert_array_equal(r["dts"], g["dts"])
    np.testing.assert_array_equal(r["y_final"], g["y_final"])


@pytest.mark.parametrize("case,field", ROS_CASES)
def test_ros23_oracle_vs_reference(oracle, case, field):
    g = load_golden(case)
    r = _run(oracle, "rosenbrock23", field, g)
    np.testing.assert_array_equal(r["n_acc"], g["n_acc"])
    np.testing.assert_array_equal(r["n_rej"], g["n_rej"])
    np.testing.assert_array_equal(r["status"], g["status"])
    # the dts follow the error estimate (h/6)(k1 - 2 k2 + k3), which cancels, so LAPACK's LU
    # and the elimination move single dts by up to ~1e-7 relative on the ill-conditioned
    # linstiff operators (condition number 1e4); the median stays at the 1e-11 level
    m = g["dts"] > 0
    rel = np.abs(r["dts"][m] - g["dts"][m]) / g["dts"][m]
    assert np.all(r["dts"][~m] == 0)
    assert rel.max() <= 1e-7 and np.median(rel) <= 1e-9
    yrel = np.abs(r["y_final"] - g["y_final"]) / np.maximum(np.abs(g["y_final"]), 1e-12)
    assert yrel.max() <= 1e-12


def test_tableau_matches_reference_module(oracle):
    tab = load_golden("tableau")
    E = oracle.tsit5_error_weights()
    ref = np.array([tab[f"E{i}"] for i in range(1, 8)])
    np.testing.assert_array_equal(E, ref)


def test_padding_contract(oracle):
    """Rows past n_acc are exactly zero; accepted dts cover [t0, t1]
    (tests/test_tsit5_replay.py:56-88 of the reference)."""
    g = load_golden("lv_mixed")
    r = _run(oracle, "tsit5", "lv", g)
    for j in range(r["dts"].shape[0]):
        row = r["dts"][j]
        assert np.all(row[: r["n_acc"][j]] > 0)
        assert np.all(row[r["n_acc"][j]:] == 0)
        assert abs(row.sum() - (float(g["t1"]) - float(g["t0"]))) <= 1e-12


def test_replay_reproduces_forward_bitwise(oracle):
    """The replay (tsit5_step arithmetic, B7*k7 kept) of the recorded mesh reproduces the
    adaptive forward's y_final bit for bit."""
    g = load_golden("lorenz_scale")
    y = oracle.replay("tsit5", "lorenz", g["y0"], g["params"], g["dts"])
    np.testing.assert_array_equal(y, g["y_final"])


def test_max_steps_exhaustion_status(oracle):
    r = oracle.record("tsit5", "linear_1", np.array([[1.0]]), np.zeros((1, 1)), 0.0, 1.0, 1e-6,
                      1e-9, max_steps=2)
    assert r["status"][0] == 1


@pytest.mark.parametrize("method,field,case", [("tsit5", "vdp", "vdp_batch"),
                                               ("tsit5", "lorenz", "lorenz_small"),
                                               ("tsit5", "lv", "lv_mixed"),
                                               ("tsit5", "lorenz96_8", "lorenz96_8"),
                                               ("tsit5", "lorenz96_32", "lorenz96_32"),
                                               ("rosenbrock23", "robertson", "robertson_toy"),
                                               ("rosenbrock23", "hires", "hires")])
def test_oracle_vjp_vs_torch_autograd_and_fd(oracle, method, field, case):
    g = load_golden(case)
    y0, p, dts = g["y0"][:3], g["params"][:3], g["dts"][:3]
    yf = oracle.replay(method, field, y0, p, dts)
    gy, gp = oracle.replay_vjp(method, field, y0, p, dts, 2.0 * yf)
    ty, tp = oracle.torch_replay_grad(method, field, y0, p, dts, 2.0 * yf)

    def rel(a, b):
        return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-8)))

    # torch solves W with LAPACK's LU, the oracle by elimination: over HIRES's 2000 stiff
    # steps that rounding difference grows to ~1e-10
    tol = 1e-9 if field == "hires" else 1e-12
    assert rel(gy, ty) < tol
    assert rel(gp, tp) < tol
    fd = oracle.fd_grad(lambda q: float((oracle.replay(method, field, y0, q, dts) ** 2).sum()), p)
    assert rel(gp, fd) < (1e-6 if method == "tsit5" else 1e-5)
