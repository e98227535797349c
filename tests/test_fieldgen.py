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


# ---- the jaxpr walker (register_jax_field where JAX is installed) ---------------------------
# JAX is absent here, so the walker is driven with jaxprs built by hand in the shape
# jax.make_jaxpr produces (the attributes it reads: primitive.name, invars, outvars, params,
# Literal.val), written as JAX lowers these functions.
class _Var:
    pass


class Literal:  # the walker recognises literals by this class name, as in JAX
    def __init__(self, val):
        self.val = val


class _Prim:
    def __init__(self, name):
        self.name = name


class _Eqn:
    def __init__(self, name, invars, outvars, **params):
        self.primitive, self.invars, self.outvars, self.params = (_Prim(name), invars, outvars,
                                                                  params)


class _Jaxpr:
    def __init__(self, invars, eqns, outvars, constvars=()):
        self.invars, self.eqns, self.outvars, self.constvars = invars, eqns, outvars, constvars


class _Closed:
    def __init__(self, jaxpr, consts=()):
        self.jaxpr, self.consts = jaxpr, list(consts)


def _lorenz_jaxpr():
    """make_jaxpr of f(t, y, p) = jnp.stack([10*(y[1]-y[0]), p[0]*y[0]-y[1]-y[0]*y[2],
    y[0]*y[1]-(8/3)*y[2]]): static indexing is slice + squeeze, jnp.stack the stack
    primitive, and the arithmetic sits inside a pjit (jnp functions are jitted)."""
    t, y, p = _Var(), _Var(), _Var()
    eqns, v = [], {}

    def take(src, i, name):
        a, b = _Var(), _Var()
        eqns.append(_Eqn("slice", [src], [a], start_indices=(i,), limit_indices=(i + 1,),
                         strides=None))
        eqns.append(_Eqn("squeeze", [a], [b], dimensions=(0,)))
        v[name] = b

    take(y, 0, "x"), take(y, 1, "u"), take(y, 2, "z"), take(p, 0, "rho")

    def op(name, a, b):
        o = _Var()
        eqns.append(_Eqn(name, [a, b], [o]))
        return o

    f0 = op("mul", Literal(10.0), op("sub", v["u"], v["x"]))
    f1 = op("sub", op("sub", op("mul", v["rho"], v["x"]), v["u"]), op("mul", v["x"], v["z"]))
    f2 = op("sub", op("mul", v["x"], v["u"]), op("mul", Literal(8.0 / 3.0), v["z"]))
    # the stack sits in a jitted helper: inlined through the pjit's inner jaxpr
    a, b, c, o = _Var(), _Var(), _Var(), _Var()
    inner = _Jaxpr([a, b, c], [_Eqn("stack", [a, b, c], [o], axis=0)], [o])
    out = _Var()
    eqns.append(_Eqn("pjit", [f0, f1, f2], [out], jaxpr=_Closed(inner)))
    return _Closed(_Jaxpr([t, y, p], eqns, [out]))


def test_jaxpr_walker_gives_the_traced_field():
    ex = G.trace_jaxpr(_lorenz_jaxpr(), 3, 1)
    ref = G.trace(lambda t, y, p: [10.0 * (y[1] - y[0]), p[0] * y[0] - y[1] - y[0] * y[2],
                                   y[0] * y[1] - (8.0 / 3.0) * y[2]], 3, 1)
    rng = np.random.default_rng(3)
    for _ in range(5):
        env = {"y": list(rng.normal(size=3)), "p": [float(rng.uniform(20, 30))]}
        for a, b in zip(ex, ref):
            assert G.evaluate(a, env) == G.evaluate(b, env)
    d1 = G.Derived(None, 3, 1, True, exprs=ex)
    d0 = G.Derived(lambda t, y, p: [10.0 * (y[1] - y[0]), p[0] * y[0] - y[1] - y[0] * y[2],
                                    y[0] * y[1] - (8.0 / 3.0) * y[2]], 3, 1, True)
    assert G.emit_struct(d1, "x", 1) == G.emit_struct(d0, "x", 1)


def test_jaxpr_walker_matrix_field_and_refusals():
    """f = A @ y (dot_general) + reduce_sum(y) * p[0], built from broadcast_in_dim; then the
    refusals: a branch on the state and a primitive outside the table name themselves."""
    A = np.array([[-2.0, 1.0, 0.0], [0.5, -3.0, 0.25], [0.0, 1.5, -4.0]])
    t, y, p = _Var(), _Var(), _Var()
    ay, s, s1, pb, sp, sb, out, p0 = (_Var() for _ in range(8))
    Av = _Var()
    eqns = [
        _Eqn("dot_general", [Av, y], [ay], dimension_numbers=(((1,), (0,)), ((), ()))),
        _Eqn("reduce_sum", [y], [s], axes=(0,)),
        _Eqn("slice", [p], [p0], start_indices=(0,), limit_indices=(1,), strides=(1,)),
        _Eqn("squeeze", [p0], [s1], dimensions=(0,)),
        _Eqn("mul", [s, s1], [sp]),
        _Eqn("broadcast_in_dim", [sp], [sb], shape=(3,), broadcast_dimensions=()),
        _Eqn("add", [ay, sb], [out]),
    ]
    closed = _Closed(_Jaxpr([t, y, p], eqns, [out], constvars=[Av]), consts=[A])
    ex = G.trace_jaxpr(closed, 3, 1)
    yv = [0.3, -1.2, 2.0]
    for i in range(3):
        got = G.evaluate(ex[i], {"y": yv, "p": [0.7]})
        assert abs(got - (A[i] @ yv + sum(yv) * 0.7)) < 1e-14
    c = _Var()
    bad = _Closed(_Jaxpr([t, y, p], [_Eqn("gt", [y, Literal(0.0)], [c])], [c]))
    with pytest.raises(G.UnsupportedRHS, match="branch on the state"):
        G.trace_jaxpr(bad, 3, 1)
    w = _Var()
    bad = _Closed(_Jaxpr([t, y, p], [_Eqn("while", [y], [w])], [w]))
    with pytest.raises(G.UnsupportedRHS, match="'while'"):
        G.trace_jaxpr(bad, 3, 1)
