"""User fields: a right-hand side f(t, y, p) written in Python becomes a CUDA field.

Counterpart of ``register_jax_field`` (gradsolve/__init__.py:31-42,
gradsolve/warp/jax_field.py:393-560): the reference traces an ``f_jax`` to a jaxpr and emits
NVIDIA Warp code for the RHS (and, for stiff problems, the Jacobian).  Here the function is
traced with symbolic scalars (``Expr``) and this module emits the whole field contract the
kernels need (``gradsolve_b200/csrc/gs_fields.cuh``): the RHS, its float32 delta form, the
vector-Jacobian product, and for stiff fields the Jacobian and the gradient of <G, J(y, p)>,
all derived symbolically from the one traced graph.  The generated struct is compiled, with
the same kernel sources as the built-in fields, into a library of its own
(``gradsolve_b200/_fields/``, cached by content hash) that exports the same C ABI.

Supported: ``+ - * /``, unary ``-``, ``abs``, ``**`` (numeric or symbolic exponent), and the
functions of this module (``exp, log, sin, cos, tan, tanh, sqrt, sign, maximum, minimum``;
numpy's ``np.exp`` etc. dispatch to them for these objects).  Comparisons and branches on
values are not supported (the reference's translator accepts the same arithmetic subset);
fields must be autonomous (the kernels do not pass t).
"""
from __future__ import annotations

import hashlib
import math
import os
import shutil
import subprocess
import tempfile
from pathlib import Path
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
GEN_DIR = HERE / "_fields"
USER_CODE_BASE = 9000


class UnsupportedRHS(ValueError):
    """The traced function used something the field generator cannot express."""


# ---- the expression graph (hash-consed) ---------------------------------------------------
_TABLE: Dict[tuple, "Expr"] = {}


class Expr:
    __slots__ = ("op", "args", "val", "__weakref__")

    def __init__(self, op: str, args: tuple, val):
        self.op, self.args, self.val = op, args, val

    # arithmetic
    def __add__(self, o): return add(self, o)
    def __radd__(self, o): return add(o, self)
    def __sub__(self, o): return sub(self, o)
    def __rsub__(self, o): return sub(o, self)
    def __mul__(self, o): return mul(self, o)
    def __rmul__(self, o): return mul(o, self)
    def __truediv__(self, o): return div(self, o)
    def __rtruediv__(self, o): return div(o, self)
    def __neg__(self): return neg(self)
    def __pos__(self): return self
    def __pow__(self, o): return power(self, o)
    def __rpow__(self, o): return power(o, self)
    def __abs__(self): return absolute(self)

    # numpy ufuncs on object arrays call these
    def exp(self): return exp(self)
    def log(self): return log(self)
    def sin(self): return sin(self)
    def cos(self): return cos(self)
    def tan(self): return tan(self)
    def tanh(self): return tanh(self)
    def sqrt(self): return sqrt(self)
    def sign(self): return sign(self)

    def _cmp(self, *_):
        raise UnsupportedRHS("comparison: branches on values are not supported in a field")

    __lt__ = __le__ = __gt__ = __ge__ = _cmp

    def __bool__(self):
        raise UnsupportedRHS("truth value of a traced quantity (a branch on values)")

    def __repr__(self):
        return f"Expr({self.op}, {self.val})" if not self.args else f"Expr({self.op}, ...)"


def _mk(op: str, args: tuple = (), val=None) -> Expr:
    key = (op, tuple(id(a) for a in args), val)
    e = _TABLE.get(key)
    if e is None:
        e = Expr(op, args, val)
        _TABLE[key] = e
    return e


def const(v: float) -> Expr:
    v = float(v)
    if v == 0.0:
        v = 0.0  # one zero (no -0.0 constants)
    return _mk("c", (), v)


def var(kind: str, i: int) -> Expr:
    return _mk(kind, (), int(i))


def _e(x) -> Expr:
    if isinstance(x, Expr):
        return x
    if isinstance(x, (int, float)) and not isinstance(x, bool):
        return const(x)
    try:  # numpy scalars
        return const(float(x))
    except (TypeError, ValueError):
        raise UnsupportedRHS(f"value of type {type(x).__name__} in a field") from None


def _is(e: Expr, v: float) -> bool:
    return e.op == "c" and e.val == v


def add(a, b) -> Expr:
    a, b = _e(a), _e(b)
    if a.op == "c" and b.op == "c":
        return const(a.val + b.val)
    if _is(a, 0.0):
        return b
    if _is(b, 0.0):
        return a
    return _mk("add", (a, b))


def sub(a, b) -> Expr:
    a, b = _e(a), _e(b)
    if a.op == "c" and b.op == "c":
        return const(a.val - b.val)
    if _is(b, 0.0):
        return a
    if _is(a, 0.0):
        return neg(b)
    if a is b:
        return const(0.0)
    return _mk("sub", (a, b))


def mul(a, b) -> Expr:
    a, b = _e(a), _e(b)
    if a.op == "c" and b.op == "c":
        return const(a.val * b.val)
    if _is(a, 0.0) or _is(b, 0.0):
        return const(0.0)
    if _is(a, 1.0):
        return b
    if _is(b, 1.0):
        return a
    if _is(a, -1.0):
        return neg(b)
    if _is(b, -1.0):
        return neg(a)
    return _mk("mul", (a, b))


def div(a, b) -> Expr:
    a, b = _e(a), _e(b)
    if _is(b, 0.0):
        raise UnsupportedRHS("division by a constant zero")
    if a.op == "c" and b.op == "c":
        return const(a.val / b.val)
    if _is(a, 0.0):
        return const(0.0)
    if _is(b, 1.0):
        return a
    return _mk("div", (a, b))


def neg(a) -> Expr:
    a = _e(a)
    if a.op == "c":
        return const(-a.val)
    if a.op == "neg":
        return a.args[0]
    return _mk("neg", (a,))


def power(a, b) -> Expr:
    a, b = _e(a), _e(b)
    if b.op == "c":
        if b.val == 0.0:
            return const(1.0)
        if b.val == 1.0:
            return a
        if a.op == "c":
            return const(a.val ** b.val)
        return _mk("powc", (a,), b.val)
    return _mk("pow", (a, b))


def _unary(op: str, fn: Callable[[float], float]):
    def f(a) -> Expr:
        a = _e(a)
        if a.op == "c":
            return const(fn(a.val))
        return _mk(op, (a,))
    f.__name__ = op
    return f


exp = _unary("exp", math.exp)
log = _unary("log", math.log)
sin = _unary("sin", math.sin)
cos = _unary("cos", math.cos)
tan = _unary("tan", math.tan)
tanh = _unary("tanh", math.tanh)
sqrt = _unary("sqrt", math.sqrt)
absolute = _unary("abs", abs)
sign = _unary("sign", lambda v: float((v > 0) - (v < 0)))


def maximum(a, b) -> Expr:
    a, b = _e(a), _e(b)
    if a.op == "c" and b.op == "c":
        return const(max(a.val, b.val))
    return _mk("max", (a, b))


def minimum(a, b) -> Expr:
    a, b = _e(a), _e(b)
    if a.op == "c" and b.op == "c":
        return const(min(a.val, b.val))
    return _mk("min", (a, b))


def _select_ge(a: Expr, b: Expr, x: Expr, y: Expr) -> Expr:
    if x is y:
        return x
    return _mk("selge", (a, b, x, y))


# ---- symbolic differentiation ------------------------------------------------------------
def diff(e: Expr, v: Expr, memo: Optional[dict] = None) -> Expr:
    """d e / d v for a variable v (memoised per variable)."""
    if memo is None:
        memo = {}
    stack = [e]
    while stack:  # post-order without recursion limits
        node = stack[-1]
        if id(node) in memo:
            stack.pop()
            continue
        pending = [a for a in node.args if id(a) not in memo]
        if pending:
            stack.extend(pending)
            continue
        stack.pop()
        memo[id(node)] = _diff1(node, v, memo)
    return memo[id(e)]


def _diff1(e: Expr, v: Expr, memo: dict) -> Expr:
    op = e.op
    if op in ("c", "y", "p", "t", "w", "G"):
        return const(1.0) if e is v else const(0.0)
    d = [memo[id(a)] for a in e.args]
    a = e.args[0]
    if op == "add":
        return add(d[0], d[1])
    if op == "sub":
        return sub(d[0], d[1])
    if op == "mul":
        return add(mul(d[0], e.args[1]), mul(a, d[1]))
    if op == "div":  # (da - (a/b) db) / b
        return div(sub(d[0], mul(e, d[1])), e.args[1])
    if op == "neg":
        return neg(d[0])
    if op == "powc":
        c = e.val
        if c == 2.0:
            return mul(mul(const(2.0), a), d[0])
        return mul(mul(const(c), power(a, const(c - 1.0))), d[0])
    if op == "pow":
        b = e.args[1]
        return mul(e, add(mul(d[1], log(a)), div(mul(b, d[0]), a)))
    if op == "exp":
        return mul(e, d[0])
    if op == "log":
        return div(d[0], a)
    if op == "sin":
        return mul(cos(a), d[0])
    if op == "cos":
        return neg(mul(sin(a), d[0]))
    if op == "tan":
        return mul(add(const(1.0), mul(e, e)), d[0])
    if op == "tanh":
        return mul(sub(const(1.0), mul(e, e)), d[0])
    if op == "sqrt":
        return div(d[0], mul(const(2.0), e))
    if op == "abs":
        return mul(sign(a), d[0])
    if op == "sign":
        return const(0.0)
    if op == "max":
        return _select_ge(a, e.args[1], d[0], d[1])
    if op == "min":
        return _select_ge(e.args[1], a, d[0], d[1])
    if op == "selge":
        return _select_ge(e.args[0], e.args[1], d[2], d[3])
    raise UnsupportedRHS(f"no derivative rule for {op}")


# ---- tracing -----------------------------------------------------------------------------
class _Vec(list):
    """y and p as seen by the traced function: indexable, iterable, with a length."""


def trace(f: Callable, dim: int, n_params: int) -> List[Expr]:
    y = _Vec(var("y", i) for i in range(dim))
    p = _Vec(var("p", j) for j in range(max(n_params, 0)))
    t = var("t", 0)
    out = f(t, y, p)
    try:
        out = list(out)
    except TypeError:
        raise UnsupportedRHS("f must return a sequence of dim components") from None
    if len(out) != dim:
        raise UnsupportedRHS(f"f returns {len(out)} components, expected dim={dim}")
    out = [_e(o) for o in out]
    for o in out:
        if _depends(o, "t"):
            raise UnsupportedRHS("time-dependent field: the kernels integrate autonomous "
                                 "systems f(y, p)")
    return out


# ---- jaxpr walking: register_jax_field on a JAX function --------------------------------------
# A jaxpr value is a numpy object array of Expr (a scalar is a 0-d array).  The table maps
# jaxpr primitive names to what they do on such arrays -- the subset the reference's
# translator accepts (gradsolve/warp/jax_field.py:75-95, :196-330): elementwise arithmetic
# and transcendentals, integer_pow, element-type conversion, the shape primitives that
# indexing and jnp.stack / jnp.array lower to, dot_general and reduce_sum for matrix-vector
# fields, and call primitives (pjit / jit / closed_call), whose inner jaxpr is inlined.
# Comparisons fold on constants only; a branch on the state (select_n, while, cond, ...) is
# refused, as by the symbolic-scalar tracer.  trace_jaxpr reads only eqn.primitive.name,
# eqn.invars, eqn.outvars, eqn.params and Literal.val, so it needs no JAX import.
def _arr(x) -> np.ndarray:
    a = np.empty(np.shape(x), dtype=object)
    flat = np.asarray(x, dtype=object).reshape(-1)
    a.reshape(-1)[:] = [v if isinstance(v, Expr) else _e(float(v)) for v in flat]
    return a


def _ew(fn: Callable, nargs: int):
    uf = np.frompyfunc(fn, nargs, 1)

    def h(params, *xs):
        return _arr(uf(*xs))
    return h


def _folding_cmp(op: Callable[[float, float], bool]):
    def f(a, b):
        a, b = _e(a), _e(b)
        if a.op == "c" and b.op == "c":
            return const(1.0 if op(a.val, b.val) else 0.0)
        raise UnsupportedRHS("a comparison of state-dependent values (a branch on the state) "
                             "is not supported")
    return _ew(f, 2)


def _broadcast_in_dim(params, a):
    shape = tuple(params["shape"])
    inter = [1] * len(shape)
    for i, d in enumerate(params["broadcast_dimensions"]):
        inter[d] = a.shape[i]
    return _arr(np.broadcast_to(a.reshape(inter), shape))


def _slice(params, a):
    strides = params.get("strides") or [1] * len(params["start_indices"])
    idx = tuple(slice(b, e, st) for b, e, st in zip(params["start_indices"],
                                                    params["limit_indices"], strides))
    return _arr(a[idx])


def _iota(params):
    shape = tuple(params["shape"])
    return _arr(np.indices(shape)[params["dimension"]].astype(float))


def _dot_general(params, a, b):
    (lc, rc), (lb, rb) = params["dimension_numbers"]
    if len(lb) or len(rb):
        raise UnsupportedRHS("dot_general with batch dimensions is not supported")
    return _arr(np.tensordot(a, b, axes=(tuple(lc), tuple(rc))))


def _reduce_sum(params, a):
    return _arr(np.sum(a, axis=tuple(params["axes"])))


JAXPR_PRIMITIVES: Dict[str, Callable] = {
    "add": _ew(add, 2), "add_any": _ew(add, 2), "sub": _ew(sub, 2), "mul": _ew(mul, 2),
    "div": _ew(div, 2), "max": _ew(maximum, 2), "min": _ew(minimum, 2), "pow": _ew(power, 2),
    "neg": _ew(neg, 1), "abs": _ew(absolute, 1), "sign": _ew(sign, 1), "exp": _ew(exp, 1),
    "log": _ew(log, 1), "sin": _ew(sin, 1), "cos": _ew(cos, 1), "tan": _ew(tan, 1),
    "tanh": _ew(tanh, 1), "sqrt": _ew(sqrt, 1),
    "rsqrt": _ew(lambda a: div(1.0, sqrt(a)), 1), "square": _ew(lambda a: mul(a, a), 1),
    "integer_pow": lambda params, a: _arr(np.frompyfunc(
        lambda v: power(v, float(params["y"])), 1, 1)(a)),
    "lt": _folding_cmp(lambda a, b: a < b), "le": _folding_cmp(lambda a, b: a <= b),
    "gt": _folding_cmp(lambda a, b: a > b), "ge": _folding_cmp(lambda a, b: a >= b),
    "eq": _folding_cmp(lambda a, b: a == b), "ne": _folding_cmp(lambda a, b: a != b),
    "convert_element_type": lambda params, a: a, "copy": lambda params, a: a,
    "copy_p": lambda params, a: a,
    "squeeze": lambda params, a: _arr(np.squeeze(a, axis=tuple(params["dimensions"]))),
    "expand_dims": lambda params, a: _arr(np.expand_dims(a, tuple(params["dimensions"]))),
    "reshape": lambda params, a: _arr(a.reshape(tuple(params["new_sizes"]))),
    "broadcast_in_dim": _broadcast_in_dim,
    "slice": _slice,
    "concatenate": lambda params, *xs: _arr(np.concatenate(xs, axis=params["dimension"])),
    "stack": lambda params, *xs: _arr(np.stack(xs, axis=params["axis"])),
    "transpose": lambda params, a: _arr(np.transpose(a, tuple(params["permutation"]))),
    "iota": _iota,
    "dot_general": _dot_general,
    "reduce_sum": _reduce_sum,
}
_CALL_PRIMITIVES = ("pjit", "jit", "closed_call", "core_call")


def _walk_jaxpr(jaxpr, consts, args) -> list:
    env: Dict[int, np.ndarray] = {}

    def read(v):
        if type(v).__name__ == "Literal":
            return _arr(v.val)
        return env[id(v)]

    for v, c in zip(getattr(jaxpr, "constvars", ()), consts):
        env[id(v)] = _arr(c)
    for v, a in zip(jaxpr.invars, args):
        env[id(v)] = a
    for eqn in jaxpr.eqns:
        name = eqn.primitive.name
        ins = [read(v) for v in eqn.invars]
        if name in _CALL_PRIMITIVES:
            inner = eqn.params.get("jaxpr") or eqn.params.get("call_jaxpr")
            if inner is None:
                raise UnsupportedRHS(f"call primitive {name!r} without an inlinable jaxpr")
            outs = _walk_jaxpr(getattr(inner, "jaxpr", inner), getattr(inner, "consts", ()),
                               ins)
        elif name in JAXPR_PRIMITIVES:
            outs = [JAXPR_PRIMITIVES[name](eqn.params, *ins)]
        else:
            raise UnsupportedRHS(f"unsupported jaxpr primitive {name!r} in f_jax")
        for v, o in zip(eqn.outvars, outs):
            if type(v).__name__ != "DropVar":
                env[id(v)] = o
    return [read(v) for v in jaxpr.outvars]


def trace_jaxpr(closed_jaxpr, dim: int, n_params: int) -> List[Expr]:
    """The components of f(t, y, p) from the jaxpr of ``f_jax`` (what
    ``jax.make_jaxpr(f_jax)(0.0, zeros(dim), zeros(n_params))`` returns), as expressions of
    the symbolic state and parameters -- the same result ``trace`` gives for a function
    written with Python arithmetic."""
    jaxpr = getattr(closed_jaxpr, "jaxpr", closed_jaxpr)
    consts = getattr(closed_jaxpr, "consts", ())
    t = _arr(var("t", 0))
    y = _arr([var("y", i) for i in range(dim)])
    p = _arr([var("p", j) for j in range(max(n_params, 0))])
    outs = _walk_jaxpr(jaxpr, consts, [t, y, p])
    if len(outs) != 1:
        raise UnsupportedRHS(f"f_jax returns {len(outs)} arrays; expected one of length {dim}")
    flat = list(outs[0].reshape(-1))
    if len(flat) != dim:
        raise UnsupportedRHS(f"f_jax returns {len(flat)} components, expected dim={dim}")
    out = [_e(o) for o in flat]
    for o in out:
        if _depends(o, "t"):
            raise UnsupportedRHS("time-dependent field: the kernels integrate autonomous "
                                 "systems f(y, p)")
    return out


def _depends(e: Expr, kind: str) -> bool:
    seen, stack = set(), [e]
    while stack:
        n = stack.pop()
        if id(n) in seen:
            continue
        seen.add(id(n))
        if n.op == kind:
            return True
        stack.extend(n.args)
    return False


def evaluate(e: Expr, env: Dict[str, Sequence[float]]) -> float:
    """The float64 value of e with y, p, w, G bound (used by the tests)."""
    memo: Dict[int, float] = {}
    stack = [e]
    while stack:
        n = stack[-1]
        if id(n) in memo:
            stack.pop()
            continue
        pending = [a for a in n.args if id(a) not in memo]
        if pending:
            stack.extend(pending)
            continue
        stack.pop()
        memo[id(n)] = _eval1(n, [memo[id(a)] for a in n.args], env)
    return memo[id(e)]


def _eval1(n: Expr, a: list, env) -> float:
    op = n.op
    if op == "c":
        return n.val
    if op in ("y", "p", "w", "G", "t"):
        return float(env[op][n.val])
    f = {"add": lambda: a[0] + a[1], "sub": lambda: a[0] - a[1], "mul": lambda: a[0] * a[1],
         "div": lambda: a[0] / a[1], "neg": lambda: -a[0], "powc": lambda: a[0] ** n.val,
         "pow": lambda: a[0] ** a[1], "exp": lambda: math.exp(a[0]),
         "log": lambda: math.log(a[0]), "sin": lambda: math.sin(a[0]),
         "cos": lambda: math.cos(a[0]), "tan": lambda: math.tan(a[0]),
         "tanh": lambda: math.tanh(a[0]), "sqrt": lambda: math.sqrt(a[0]),
         "abs": lambda: abs(a[0]), "sign": lambda: float((a[0] > 0) - (a[0] < 0)),
         "max": lambda: max(a[0], a[1]), "min": lambda: min(a[0], a[1]),
         "selge": lambda: a[2] if a[0] >= a[1] else a[3]}[op]
    return f()


# ---- the field's derived quantities ------------------------------------------------------
class Derived:
    """f, its VJP, and (stiff) J and grad <G, J>, as expressions."""

    def __init__(self, f: Optional[Callable], dim: int, n_params: int, stiff: bool,
                 exprs: Optional[List[Expr]] = None):
        self.D, self.P, self.stiff = int(dim), max(int(n_params), 1), bool(stiff)
        self.f = list(exprs) if exprs is not None else trace(f, self.D, int(n_params))
        ys = [var("y", i) for i in range(self.D)]
        ps = [var("p", j) for j in range(self.P)]
        s = const(0.0)
        for i, fi in enumerate(self.f):
            s = add(s, mul(var("w", i), fi))
        self.gy = [diff(s, v) for v in ys]
        self.gp = [diff(s, v) for v in ps]
        self.J = self.s2 = self.hy = self.hp = None
        if self.stiff:
            self.J = [[diff(fi, yk) for yk in ys] for fi in self.f]
            s2 = const(0.0)
            for i in range(self.D):
                for k in range(self.D):
                    s2 = add(s2, mul(var("G", i * self.D + k), self.J[i][k]))
            self.hy = [diff(s2, v) for v in ys]
            self.hp = [diff(s2, v) for v in ps]


# ---- C++ emission ---------------------------------------------------------------------------
def _lit(v: float) -> str:
    if v == int(v) and abs(v) < 2 ** 53:
        return f"R({float(v)!r})"
    return f"R({float(v).hex()})"  # exact (C++17 hexadecimal floating literal)


def _emit_body(outputs: List[tuple]) -> List[str]:
    """Straight-line code computing the (target, expr, op) outputs, one temporary per shared
    node (the graph is hash-consed, so common subexpressions are computed once)."""
    names: Dict[int, str] = {}
    uses: Dict[int, int] = {}
    order: List[Expr] = []
    seen = set()
    for _t, e, _op in outputs:
        stack = [(e, False)]
        while stack:
            n, done = stack.pop()
            if done:
                order.append(n)
                continue
            uses[id(n)] = uses.get(id(n), 0) + 1
            if id(n) in seen:
                continue
            seen.add(id(n))
            stack.append((n, True))
            for a in reversed(n.args):
                stack.append((a, False))
    lines: List[str] = []

    def ref(n: Expr) -> str:
        if n.op == "c":
            return _lit(n.val)
        if n.op in ("y", "p", "w", "G"):
            return f"{n.op}[{n.val}]"
        return names[id(n)]

    for n in order:
        if n.op in ("c", "y", "p", "w", "G") or id(n) in names:
            continue
        a = [ref(x) for x in n.args]
        op = n.op
        if op == "add":
            s = f"{a[0]} + {a[1]}"
        elif op == "sub":
            s = f"{a[0]} - {a[1]}"
        elif op == "mul":
            s = f"{a[0]} * {a[1]}"
        elif op == "div":
            s = f"{a[0]} / {a[1]}"
        elif op == "neg":
            s = f"-{a[0]}"
        elif op == "powc":
            c = n.val
            s = (f"{a[0]} * {a[0]}" if c == 2.0 else f"{a[0]} * {a[0]} * {a[0]}" if c == 3.0
                 else f"sqrt({a[0]})" if c == 0.5 else f"R(1.0) / {a[0]}" if c == -1.0
                 else f"pow({a[0]}, {_lit(c)})")
        elif op == "pow":
            s = f"pow({a[0]}, {a[1]})"
        elif op in ("exp", "log", "sin", "cos", "tan", "tanh", "sqrt"):
            s = f"{op}({a[0]})"
        elif op == "abs":
            s = f"fabs({a[0]})"
        elif op == "sign":
            s = f"R(({a[0]} > R(0.0)) - ({a[0]} < R(0.0)))"
        elif op == "max":
            s = f"fmax({a[0]}, {a[1]})"
        elif op == "min":
            s = f"fmin({a[0]}, {a[1]})"
        elif op == "selge":
            s = f"({a[0]} >= {a[1]} ? {a[2]} : {a[3]})"
        else:
            raise UnsupportedRHS(f"cannot emit {op}")
        nm = f"v{len(names)}"
        names[id(n)] = nm
        lines.append(f"    const R {nm} = {s};")
    for target, e, how in outputs:
        lines.append(f"    {target} {how} {ref(e)};")
    return lines


def emit_struct(d: Derived, name: str, code: int) -> str:
    D, P = d.D, d.P
    out = [f"// generated by gradsolve_b200.fieldgen for the field {name!r}; do not edit",
           "#pragma once", "namespace gs {", "struct UserField {",
           f"  static constexpr int D = {D}, P = {P};",
           "  template <class R>",
           "  static GS_HD void rhs(const R* y, const R* p, R* dy) {"]
    out += _emit_body([(f"dy[{i}]", fi, "=") for i, fi in enumerate(d.f)])
    out += ["  }",
            "  // f(y + d) - f(y) by direct difference (no cancellation-free expansion)",
            "  template <class R>",
            "  static GS_HD void rhs_delta(const R* y, const R* p, const R* d, R* df) {",
            f"    R yd[{D}], a[{D}], b[{D}];",
            f"    for (int i = 0; i < {D}; ++i) yd[i] = y[i] + d[i];",
            "    rhs(yd, p, a);", "    rhs(y, p, b);",
            f"    for (int i = 0; i < {D}; ++i) df[i] = a[i] - b[i];", "  }",
            "  template <class R>",
            "  static GS_HD void vjp(const R* y, const R* p, const R* w, R* gy, R* gp) {"]
    outs = [(f"gy[{k}]", g, "+=") for k, g in enumerate(d.gy) if not _is(g, 0.0)]
    outs += [(f"gp[{j}]", g, "+=") for j, g in enumerate(d.gp) if not _is(g, 0.0)]
    out += _emit_body(outs) + ["    (void)y; (void)p; (void)w; (void)gy; (void)gp;", "  }"]
    if d.stiff:
        out += ["  template <class R>", "  static GS_HD void jac(const R* y, const R* p, R* J) {"]
        out += _emit_body([(f"J[{i * D + k}]", d.J[i][k], "=")
                           for i in range(D) for k in range(D)])
        out += ["    (void)y; (void)p;", "  }", "  template <class R>",
                "  static GS_HD void jac_contract_grad(const R* y, const R* p, const R* G, "
                "R* gy, R* gp) {"]
        outs = [(f"gy[{k}]", g, "+=") for k, g in enumerate(d.hy) if not _is(g, 0.0)]
        outs += [(f"gp[{j}]", g, "+=") for j, g in enumerate(d.hp) if not _is(g, 0.0)]
        out += _emit_body(outs) + ["    (void)y; (void)p; (void)G; (void)gy; (void)gp;", "  }"]
    out += ["};", "}  // namespace gs", f"#define GS_USER_FIELD_CODE {code}",
            f"#define GS_USER_STIFF {1 if d.stiff else 0}", ""]
    return "\n".join(out)


# ---- build ----------------------------------------------------------------------------------
def _sources_digest() -> str:
    h = hashlib.sha256()
    for p in sorted((HERE / "csrc").glob("*.cu*")) + [HERE.parent / "include" / "gsolve.h"]:
        h.update(p.read_bytes())
    return h.hexdigest()[:16]


def library_path(header: str) -> Path:
    """Where the library of a field header lives (named by the content of the header and of
    the kernel sources), built or not."""
    key = hashlib.sha256((header + _sources_digest()).encode()).hexdigest()[:20]
    return GEN_DIR / f"libgsfield_{key}.so"


# the built-in stencil families the core library carries at a few dimensions only; any other
# dimension gets a library of its own, compiled on first use: kind -> (code base, template)
FAMILIES = {"linear": (4000, "Linear"), "lorenz96": (5000, "Lorenz96")}


def family_header(kind: str, dim: int) -> str:
    """The field header of a built-in family member (Linear<D>, Lorenz96<D>) at dimension
    ``dim``: the hand-written field of gs_fields.cuh, instantiated, not traced."""
    base, tmpl = FAMILIES[kind]
    return "\n".join([
        f"// generated by gradsolve_b200.fieldgen: the built-in {kind} field at D = {dim}",
        "#pragma once", "namespace gs {", f"using UserField = {tmpl}<{int(dim)}>;",
        "}  // namespace gs", f"#define GS_USER_FIELD_CODE {base + int(dim)}",
        "#define GS_USER_STIFF 0", ""])


def family_library(kind: str, dim: int) -> Path:
    return build_field_library(family_header(kind, dim))


def build_field_library(header: str, *, force: bool = False) -> Path:
    """Compile the kernels and the C ABI for one generated field into its own library
    (cached by the content of the header and of the kernel sources)."""
    GEN_DIR.mkdir(exist_ok=True)
    out = library_path(header)
    key = out.stem[len("libgsfield_"):]
    if out.exists() and not force:
        return out
    hdr = GEN_DIR / f"field_{key}.cuh"
    hdr.write_text(header)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    with tempfile.TemporaryDirectory() as td:
        tmp = Path(td) / out.name
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
               "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
               f"-DGS_USER_FIELD_HEADER=\"{hdr}\"", "-o", str(tmp),
               str(HERE / "csrc" / "gs_abi.cu")]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for the generated field ({res.returncode}):\n"
                               f"{res.stderr[-4000:]}")
        os.replace(tmp, out)
    return out
