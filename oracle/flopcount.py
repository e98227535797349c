"""Counting oracle for the algorithmic work per unit (test infrastructure only).

Evaluates the reference's expressions once on a scalar type that counts operations:
``+ - * /`` count 1 each (a fused multiply-add therefore counts 2), ``sqrt``, ``pow``,
``abs`` and ``max`` count 1 each; negation, comparisons and min are free.

  F_att  one adaptive attempt (gradsolve/solvers/tsit5_replay.py:85-122 for Tsit5;
         tests/_oracles/gradsolve_g2_spike_oracle.py:161-181 for Rosenbrock23, with the
         3x3 elimination of gradsolve/warp/_warp_rosenbrock.py:346-381 done once)
  F_step one replay step (gradsolve/solvers/tsit5_step.py:80-102 without the dead k7
         stage, whose weight B7 is 0; gradsolve/solvers/rosenbrock23_step.py:47-66)
  F_vjp  the minimal transposed graph of that step (the backward sweep only; recomputing
         forward stage values is implementation overhead and is not counted)

gradsolve_b200/flops.py holds the resulting numbers; tests/test_flops.py checks they agree.
"""
from __future__ import annotations

import math


class Counter:
    n = 0


class Num:
    __slots__ = ("v",)

    def __init__(self, v):
        self.v = float(v.v if isinstance(v, Num) else v)

    def _bin(self, o, f):
        Counter.n += 1
        return Num(f(self.v, o.v if isinstance(o, Num) else float(o)))

    def __add__(self, o): return self._bin(o, lambda a, b: a + b)
    def __radd__(self, o): return self._bin(o, lambda a, b: b + a)
    def __sub__(self, o): return self._bin(o, lambda a, b: a - b)
    def __rsub__(self, o): return self._bin(o, lambda a, b: b - a)
    def __mul__(self, o): return self._bin(o, lambda a, b: a * b)
    def __rmul__(self, o): return self._bin(o, lambda a, b: b * a)
    def __truediv__(self, o): return self._bin(o, lambda a, b: a / b)
    def __rtruediv__(self, o): return self._bin(o, lambda a, b: b / a)
    def __neg__(self): return Num(-self.v)
    def __le__(self, o): return self.v <= (o.v if isinstance(o, Num) else o)
    def __lt__(self, o): return self.v < (o.v if isinstance(o, Num) else o)
    def __gt__(self, o): return self.v > (o.v if isinstance(o, Num) else o)


def c_sqrt(x):
    Counter.n += 1
    return Num(math.sqrt(x.v))


def c_pow(x, e):
    Counter.n += 1
    return Num(x.v ** e)


def c_abs(x):
    Counter.n += 1
    return Num(abs(x.v))


def c_max(a, b):
    Counter.n += 1
    return a if a.v >= b.v else b


# ---- fields (reference operation order) and their VJPs ----
def f_lorenz(y, p):
    s, b, r = 10.0, 8.0 / 3.0, p[0]
    return [s * (y[1] - y[0]), r * y[0] - y[1] - y[0] * y[2], y[0] * y[1] - b * y[2]]


def vjp_lorenz(y, p, w):
    s, b, r = 10.0, 8.0 / 3.0, p[0]
    gy = [-s * w[0] + (r - y[2]) * w[1] + y[1] * w[2], s * w[0] - w[1] + y[0] * w[2],
          -y[0] * w[1] - b * w[2]]
    return gy, [y[0] * w[1]]


def f_lv(y, p):
    x, u = y
    return [p[0] * x - p[1] * x * u, p[3] * x * u - p[2] * u]


def vjp_lv(y, p, w):
    x, u = y
    gy = [(p[0] - p[1] * u) * w[0] + p[3] * u * w[1], -p[1] * x * w[0] + (p[3] * x - p[2]) * w[1]]
    return gy, [x * w[0], -x * u * w[0], -u * w[1], x * u * w[1]]


def f_vdp(y, p):
    x, v = y
    return [v, p[0] * ((1.0 - x * x) * v - x)]


def vjp_vdp(y, p, w):
    x, v = y
    mu = p[0]
    return [w[1] * mu * (-2.0 * x * v - 1.0), w[0] + w[1] * mu * (1.0 - x * x)], \
        [w[1] * ((1.0 - x * x) * v - x)]


def f_rob(y, p):
    k1, k2, k3 = p
    a, b, c = y
    return [-k1 * a + k3 * b * c, k1 * a - k3 * b * c - k2 * b * b, k2 * b * b]


def jac_rob(y, p):
    k1, k2, k3 = p
    b, c = y[1], y[2]
    return [[-k1, k3 * c, k3 * b], [k1, -k3 * c - 2.0 * k2 * b, -k3 * b], [0.0, 2.0 * k2 * b, 0.0]]


def vjp_rob(y, p, w):
    k1, k2, k3 = p
    a, b, c = y
    gy = [-k1 * w[0] + k1 * w[1], k3 * c * w[0] + (-k3 * c - 2.0 * k2 * b) * w[1] + 2.0 * k2 * b * w[2],
          k3 * b * w[0] - k3 * b * w[1]]
    gp = [-a * w[0] + a * w[1], -b * b * w[1] + b * b * w[2], b * c * w[0] - b * c * w[1]]
    return gy, gp


def jcg_rob(y, p, G):
    k2, k3 = p[1], p[2]
    b, c = y[1], y[2]
    gy = [0.0, k3 * G[0][2] - 2.0 * k2 * G[1][1] - k3 * G[1][2] + 2.0 * k2 * G[2][1],
          k3 * G[0][1] - k3 * G[1][1]]
    gp = [-G[0][0] + G[1][0], -2.0 * b * G[1][1] + 2.0 * b * G[2][1],
          c * G[0][1] + b * G[0][2] - c * G[1][1] - b * G[1][2]]
    return gy, gp


def jac_vdp(y, p):
    x, v = y
    mu = p[0]
    return [[0.0, 1.0], [mu * (-2.0 * x * v - 1.0), mu * (1.0 - x * x)]]


def jcg_vdp(y, p, G):
    x, v = y
    mu = p[0]
    gy = [G[1][0] * mu * (-2.0 * v) + G[1][1] * mu * (-2.0 * x), G[1][0] * mu * (-2.0 * x)]
    gp = [G[1][0] * (-2.0 * x * v - 1.0) + G[1][1] * (1.0 - x * x)]
    return gy, gp


def f_l96(y, p):
    """lorenz96_<D> in the reference's order (gradsolve/warp/_warp_kernel.py:175-195)."""
    D = len(y)
    return [(y[(i + 1) % D] - y[(i - 2) % D]) * y[(i - 1) % D] - y[i] + p[0] for i in range(D)]


def vjp_l96(y, p, w):
    D = len(y)
    gy = [w[(j - 1) % D] * y[(j - 2) % D] - w[(j + 2) % D] * y[(j + 1) % D] +
          w[(j + 1) % D] * (y[(j + 2) % D] - y[(j - 1) % D]) - w[j] for j in range(D)]
    gF = w[0]
    for j in range(1, D):
        gF = gF + w[j]
    return gy, [gF]


def f_lin(y, p):
    """linear_<D> (gradsolve/warp/_warp_kernel.py:133-155): 1.01 y, the parameter unread."""
    return [1.01 * v for v in y]


def vjp_lin(y, p, w):
    return [1.01 * v for v in w], [0.0]


STIFF = {"robertson": (jac_rob, jcg_rob, [0.04, 3e7, 1e4]), "vdp": (jac_vdp, jcg_vdp, [50.0])}

FIELDS = {"lorenz": (f_lorenz, vjp_lorenz, 3, 1), "lv": (f_lv, vjp_lv, 2, 4),
          "vdp": (f_vdp, vjp_vdp, 2, 1), "robertson": (f_rob, vjp_rob, 3, 3),
          "lorenz96_32": (f_l96, vjp_l96, 32, 1), "linear_32": (f_lin, vjp_lin, 32, 1)}

# Tsit5 tableau (values only matter for the arithmetic to run; counts are structural)
A = [[0.161], [-0.0085, 0.3355], [2.897, -6.359, 4.362], [5.326, -11.749, 7.496, -0.0925],
     [5.861, -12.921, 8.159, -0.0716, -0.0283]]
B = [0.0965, 0.01, 0.4799, 1.379, -3.290, 2.325]
E = [0.00178, 0.000816, -0.00788, 0.1447, -0.5824, 0.458, -1.0 / 66.0]


def _lin(coefs, ks, i):
    acc = coefs[0] * ks[0][i]
    for c, k in zip(coefs[1:], ks[1:]):
        acc = acc + c * k[i]
    return acc


def _y(D, v=1.0):
    return [Num(v + 0.1 * i) for i in range(D)]


def count_tsit5(field):
    f, vjp, D, P = FIELDS[field]
    y, p, h = _y(D), _y(P, 0.7), Num(0.01)
    k1 = f(y, p)
    Counter.n = 0
    ks = [k1]
    for row in A:
        s = [y[i] + h * _lin(row, ks, i) for i in range(D)]
        ks.append(f(s, p))
    y5 = [y[i] + h * _lin(B, ks, i) for i in range(D)]
    k7 = f(y5, p)
    e = [h * _lin(E, ks + [k7], i) for i in range(D)]
    q = []
    for i in range(D):
        sc = 1e-8 + 1e-8 * c_max(c_abs(y[i]), c_abs(y5[i]))
        c = e[i] / sc
        q.append(c * c)
    acc = q[0]
    for v in q[1:]:
        acc = acc + v
    err = c_sqrt(acc / float(D))
    _dt = h * (0.9 * c_pow(c_max(err, Num(1e-10)), -0.2))
    f_att = Counter.n

    Counter.n = 0
    ks = [f(y, p)]
    for row in A:
        s = [y[i] + h * _lin(row, ks, i) for i in range(D)]
        ks.append(f(s, p))
    _yn = [y[i] + h * _lin(B, ks, i) for i in range(D)]
    f_step = Counter.n

    # backward sweep of the step: stage states S[m] are inputs (not counted)
    S = [_y(D, 0.5 + 0.01 * m) for m in range(6)]
    lam = _y(D, 0.3)
    Counter.n = 0
    g = [h * lam[i] for i in range(D)]
    kb = [[B[m] * g[i] for i in range(D)] for m in range(6)]
    yb = list(lam)
    for m in range(5, -1, -1):
        sb, _gp = vjp(S[m], p, kb[m])
        yb = [yb[i] + sb[i] for i in range(D)]
        if m > 0:
            u = [h * sb[i] for i in range(D)]
            for jj in range(m):
                kb[jj] = [kb[jj][i] + A[m - 1][jj] * u[i] for i in range(D)]
    f_vjp = Counter.n
    return dict(F_att=f_att, F_step=f_step, F_vjp=f_vjp)


def _lu_solve_count(W, b, D):
    # factor once (counted separately) -- here: forward + back substitution
    x = list(b)
    for k in range(D):
        for r in range(k + 1, D):
            x[r] = x[r] - W[r][k] * x[k]
    out = [None] * D
    for i in range(D - 1, -1, -1):
        s = x[i]
        for c in range(i + 1, D):
            s = s - W[i][c] * out[c]
        out[i] = s / W[i][i]
    return out


def _lu_factor_count(W, D):
    W = [list(r) for r in W]
    for col in range(D):
        for r in range(col + 1, D):
            _ = c_abs(W[r][col])
        for r in range(col + 1, D):
            fct = W[r][col] / W[col][col]
            W[r][col] = fct
            for c in range(col + 1, D):
                W[r][c] = W[r][c] - fct * W[col][c]
    return W


def count_ros23(field="robertson"):
    f, vjp, D, P = FIELDS[field]
    jac, jcg, pv = STIFF[field]
    y, p, h = _y(D), [Num(v) for v in pv], Num(0.01)
    d, e32 = 0.2928932188134525, 7.414213562373095

    def core(y, p, h):
        J = [[v if isinstance(v, Num) else Num(v) for v in row] for row in jac(y, p)]
        dh = h * (-d)                                   # W = I - d h J: 1 + 9 + 3 ops
        W = [[dh * J[i][c] for c in range(D)] for i in range(D)]
        for i in range(D):
            W[i][i] = W[i][i] + 1.0
        W = _lu_factor_count(W, D)
        F0 = f(y, p)
        k1 = _lu_solve_count(W, F0, D)
        s = [y[i] + 0.5 * h * k1[i] for i in range(D)]
        F1 = f(s, p)
        k2 = _lu_solve_count(W, [F1[i] - k1[i] for i in range(D)], D)
        k2 = [k2[i] + k1[i] for i in range(D)]
        yn = [y[i] + h * k2[i] for i in range(D)]
        return W, F0, k1, F1, k2, yn

    Counter.n = 0
    W, F0, k1, F1, k2, yn = core(y, p, h)
    F2 = f(yn, p)
    k3 = _lu_solve_count(W, [F2[i] - e32 * (k2[i] - F1[i]) - 2.0 * (k1[i] - F0[i]) for i in range(D)], D)
    ev = [(h / 6.0) * (k1[i] - 2.0 * k2[i] + k3[i]) for i in range(D)]
    q = []
    for i in range(D):
        sc = 1e-10 + 1e-6 * c_max(c_abs(y[i]), c_abs(yn[i]))
        c = ev[i] / sc
        q.append(c * c)
    acc = q[0]
    for v in q[1:]:
        acc = acc + v
    err = c_sqrt(acc / float(D))
    _dt = h * (0.9 * c_pow(c_max(err, Num(1e-10)), -1.0 / 3.0))
    f_att = Counter.n

    Counter.n = 0
    core(y, p, h)
    f_step = Counter.n

    # backward sweep: W factors, k1, k2', s1 are stored inputs (not counted)
    lam = _y(D, 0.3)
    k2p = _y(D, 0.2)
    s1 = _y(D, 0.4)
    Counter.n = 0
    k2b = [h * lam[i] for i in range(D)]
    k1b = list(k2b)
    r2b = _lu_solve_count(W, k2b, D)   # transposed solve has the same operation count
    scale = d * h
    G = [[scale * (r2b[i] * k2p[c]) for c in range(D)] for i in range(D)]
    k1b = [k1b[i] - r2b[i] for i in range(D)]
    s1b, _ = vjp(s1, p, r2b)
    yb = [lam[i] + s1b[i] for i in range(D)]
    k1b = [k1b[i] + 0.5 * h * s1b[i] for i in range(D)]
    r1b = _lu_solve_count(W, k1b, D)
    G = [[G[i][c] + scale * (r1b[i] * k1[c]) for c in range(D)] for i in range(D)]
    gyb, _ = vjp(y, p, r1b)
    yb = [yb[i] + gyb[i] for i in range(D)]
    jy, _ = jcg(y, p, G)
    yb = [yb[i] + jy[i] for i in range(D)]
    f_vjp = Counter.n
    return dict(F_att=f_att, F_step=f_step, F_vjp=f_vjp)


def all_counts():
    out = {("tsit5", k): count_tsit5(k) for k in ("lorenz", "lv", "vdp", "lorenz96_32",
                                                   "linear_32")}
    out[("rosenbrock23", "robertson")] = count_ros23("robertson")
    out[("rosenbrock23", "vdp")] = count_ros23("vdp")
    return out


if __name__ == "__main__":
    for k, v in all_counts().items():
        print(k, v)
