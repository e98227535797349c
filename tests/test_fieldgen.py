"""The field generator (register_field / register_jax_field) on the CPU: the symbolic
derivatives against finite differences, the emitted code, the rejected constructs, and one
generated library built and loaded (its C ABI checked; no kernel runs without a GPU)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from gradsolve_b200 import fieldgen as G


def lorenz(t, y, p):
    x, u, z = y
    return [10.0 * (u - x), p[0] * x - u - x * z, x * u - (8.0 / 3.0) * z]


def robertson(t, y, p):
    a, b, c = y
    return [-p[0] * a + p[2] * b * c, p[0] * a - p[2] * b * c - p[1] * b * b, p[1] * b * b]


def exotic(t, y, p):
    x, v = y
    return [np.tanh(v) + G.sqrt(1.0 + x * x) * 0.25,
            -p[0] * np.sin(x) - p[1] * v + np.exp(-x * x) / (2.0 + np.cos(v)) + x ** 3
            + abs(v) * 0.1 + G.maximum(x, v) * 0.01 + (1.0 + v * v) ** p[1]]


CASES = [(lorenz, 3, 1, [1.3, -0.7, 20.0], [28.0]),
         (robertson, 3, 3, [0.9, 2e-5, 0.1], [0.04, 3e7, 1e4]),
         (exotic, 2, 2, [0.7, -0.3], [1.5, 0.2])]


def _num(fn, x, h):
    """Central differences of fn at x (each component scaled)."""
    cols = []
    for k in range(len(x)):
        e = max(abs(x[k]), 1.0) * h
        xp, xm = list(x), list(x)
        xp[k] += e
        xm[k] -= e
        cols.append((np.array(fn(xp)) - np.array(fn(xm))) / (2 * e))
    return np.array(cols).T  # d out / d x, (out, in)


@pytest.mark.parametrize("f,D,P,y,p", CASES)
def test_symbolic_derivatives_match_finite_differences(f, D, P, y, p):
    d = G.Derived(f, D, P, stiff=True)
    env = lambda yy, pp, w=None, g=None: {"y": yy, "p": pp, "w": w or [0.0] * D,  # noqa: E731
                                          "G": g or [0.0] * (D * D), "t": [0.0]}
    fval = lambda yy, pp: [G.evaluate(e, env(yy, pp)) for e in d.f]  # noqa: E731
    # the RHS is the function itself
    ref = f(0.0, [float(v) for v in y], [float(v) for v in p])  # the module's functions
    ref = [G.evaluate(r, {}) if isinstance(r, G.Expr) else float(r) for r in ref]  # fold floats
    np.testing.assert_allclose(fval(y, p), ref, rtol=1e-15)
    Jy = _num(lambda yy: fval(yy, p), y, 1e-6)
    Jp = _num(lambda pp: fval(y, pp), p, 1e-6)
    J = np.array([[G.evaluate(d.J[i][k], env(y, p)) for k in range(D)] for i in range(D)])
    np.testing.assert_allclose(J, Jy, rtol=1e-6, atol=1e-6 * np.abs(Jy).max())
    rng = np.random.default_rng(0)
    w = list(rng.normal(size=D))
    gy = [G.evaluate(e, env(y, p, w)) for e in d.gy]
    gp = [G.evaluate(e, env(y, p, w)) for e in d.gp]
    np.testing.assert_allclose(gy, np.array(w) @ Jy, rtol=1e-6, atol=1e-6 * np.abs(Jy).max())
    np.testing.assert_allclose(gp, np.array(w) @ Jp, rtol=1e-6, atol=1e-6 * np.abs(Jp).max())
    # grad of <Gm, J(y, p)> by differences of the symbolic J
    Gm = list(rng.normal(size=D * D))

    def contract(yy, pp):
        return [sum(Gm[i * D + k] * G.evaluate(d.J[i][k], env(yy, pp))
                    for i in range(D) for k in range(D))]
    hy = [G.evaluate(e, env(y, p, None, Gm)) for e in d.hy]
    hp = [G.evaluate(e, env(y, p, None, Gm)) for e in d.hp]
    ny = _num(lambda yy: contract(yy, p), y, 1e-6)[0]
    npp = _num(lambda pp: contract(y, pp), p, 1e-6)[0]
    scale = max(np.abs(ny).max(), np.abs(npp).max(), 1e-30)
    np.testing.assert_allclose(hy, ny, rtol=1e-5, atol=1e-6 * scale)
    np.testing.assert_allclose(hp, npp, rtol=1e-5, atol=1e-6 * scale)


def test_emitted_code_is_exact_and_shares_subexpressions():
    d = G.Derived(lorenz, 3, 1, stiff=False)
    src = G.emit_struct(d, "lz", 9001)
    assert "R(0x1.5555555555555p+1)" in src  # 8/3 to the last bit (hexadecimal literal)
    assert "jac(" not in src                 # only stiff fields get a Jacobian
    assert "#define GS_USER_STIFF 0" in src
    # the product x*y appears once in the RHS even if used twice
    d2 = G.Derived(lambda t, y, p: [y[0] * y[1] + 1.0, y[0] * y[1] * 2.0], 2, 0, False)
    body = G.emit_struct(d2, "s", 9002).split("rhs(")[1].split("}")[0]
    assert body.count("y[0] * y[1]") == 1


def test_rejected_constructs():
    with pytest.raises(G.UnsupportedRHS, match="comparison"):
        G.Derived(lambda t, y, p: [y[0] if y[0] > 0 else -y[0]], 1, 0, False)
    with pytest.raises(G.UnsupportedRHS, match="time-dependent"):
        G.Derived(lambda t, y, p: [t * y[0]], 1, 0, False)
    with pytest.raises(G.UnsupportedRHS, match="components"):
        G.Derived(lambda t, y, p: [y[0], y[0]], 1, 0, False)
    with pytest.raises(G.UnsupportedRHS):
        G.Derived(lambda t, y, p: [y[0] / 0.0], 1, 0, False)


def test_register_field_builds_a_library_with_the_full_abi(gslib):
    """One generated library, built with nvcc (cross-compiled for sm_100a), loads and exports
    every symbol of include/gsolve.h; registration is idempotent and routes by name."""
    import gradsolve_b200 as gsb
    from gradsolve_b200 import _lib
    from gradsolve_b200.fields import field_for

    spec = gsb.register_jax_field("pendulum_cpu_test",
                                  lambda t, y, p: [y[1], -p[0] * np.sin(y[0]) - p[1] * y[1]],
                                  2, 2, stiff=True)
    assert gsb.register_field("pendulum_cpu_test", lambda t, y, p: [y[0]], 1, 0) is spec
    assert spec.dim == 2 and spec.nparam == 2 and spec.stiff_ok and spec.lib

    class Prob:
        name = "pendulum_cpu_test"
    assert field_for(Prob()) is spec
    L = _lib.lib_for(spec)
    for sym in _lib.exported_symbols():
        assert hasattr(L, sym), sym
    import ctypes
    D, P = ctypes.c_int(), ctypes.c_int()
    assert L.gs_field_dims(spec.code, ctypes.byref(D), ctypes.byref(P)) == 0
    assert (D.value, P.value) == (2, 2)
    assert L.gs_field_dims(1, ctypes.byref(D), ctypes.byref(P)) != 0  # serves its field only
    assert math.isfinite(spec.code)
