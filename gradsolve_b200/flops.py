"""Algorithmic work per unit, for roofline reporting.

Counted once per (method, field) by the counting oracle (``+ - * /`` = 1 each, so a fused
multiply-add = 2; ``sqrt``/``pow``/``abs``/``max`` = 1 each) on the reference's expressions:
  F_att  one adaptive attempt; F_step one replay step (the zero-weight k7 stage excluded);
  F_vjp  the backward sweep of one step (forward recomputation excluded).
Per trajectory:
  solve    F = (n_acc + n_rej) * F_att
  gradient F = (n_acc + n_rej) * F_att + n_acc * (F_step + F_vjp)
tests/test_flops.py re-derives the numbers.
"""
from __future__ import annotations

COUNTS = {
    ("tsit5", "lorenz"): dict(F_att=269, F_step=198, F_vjp=228),
    ("tsit5", "lv"): dict(F_att=193, F_step=144, F_vjp=204),
    ("tsit5", "vdp"): dict(F_att=175, F_step=126, F_vjp=186),
    ("tsit5", "lorenz96_32"): dict(F_att=3013, F_step=2304, F_vjp=3066),
    ("tsit5", "linear_32"): dict(F_att=2437, F_step=1728, F_vjp=1728),
    ("rosenbrock23", "robertson"): dict(F_att=205, F_step=115, F_vjp=191),
    ("rosenbrock23", "vdp"): dict(F_att=108, F_step=54, F_vjp=97),
}


def solve_flops(method: str, field: str, attempts: int) -> int:
    return COUNTS[(method, field)]["F_att"] * int(attempts)


def adjoint_flops(method: str, field: str, accepted: int) -> int:
    c = COUNTS[(method, field)]
    return (c["F_step"] + c["F_vjp"]) * int(accepted)


def gradient_flops(method: str, field: str, attempts: int, accepted: int) -> int:
    return solve_flops(method, field, attempts) + adjoint_flops(method, field, accepted)


def saveat_flops(method: str, field: str, resteps: int) -> int:
    """Dense output on the frozen mesh: each requested time inside (t0, t_fin) is one step of
    the method from the bracketing step's start (F_step) and, in the reverse pass, that
    step's VJP (F_vjp) -- the reference's bracket-and-re-step (gradsolve/solvers/dense.py:
    106-163); times at t0 or t_fin are copies."""
    c = COUNTS[(method, field)]
    return (c["F_step"] + c["F_vjp"]) * int(resteps)

