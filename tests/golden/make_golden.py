"""Generate the golden vectors under tests/golden/ from the reference's own code.

Runs only where the reference source tree is present (it is read from
``$GRADSOLVE_REFERENCE``, default: a ``reference`` directory beside the repository's root);
the GPU test runs never run this.
What it executes, verbatim, from the reference:

* ``gradsolve/solvers/tsit5_step.py`` -- imported by file path (it has no imports), for
  the tableau and controller constants;
* ``tsit5_adaptive`` -- the function body of ``gradsolve/solvers/tsit5_replay.py:62-124``
  extracted with ``ast`` (the module itself imports JAX, which is not installed); its one
  in-function import of ``fixed_step_tsit5`` is dropped and the same names are supplied
  from ``tsit5_step``, which is where ``fixed_step_tsit5`` takes them from;
* ``rosenbrock23_adaptive`` and ``robertson_jac`` from
  ``tests/_oracles/gradsolve_g2_spike_oracle.py`` (numpy only), the reference's own
  Rosenbrock23 specification.

RHS functions are written in the reference's operation order (Lorenz as
``gradsolve/warp/_warp_kernel.py:111-130``, VdP as ``tests/test_adjoint_replay.py:58-68``,
Robertson as ``tests/test_adjoint_replay.py:90-104``, Lotka-Volterra as
``alpha*x - beta*x*y``, ``delta*x*y - gamma*y``).

Output: one ``.npz`` per case holding inputs, ``dts`` (padded ``[n, S]``), ``n_acc``,
``n_rej``, ``status`` and ``y_final``, plus ``tableau.npz`` with the reference's constants.
"""
from __future__ import annotations

import ast
import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
REF = Path(os.environ.get("GRADSOLVE_REFERENCE", OUT.parent.parent.parent / "reference"))


def _load_module(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_reference():
    ts = _load_module(REF / "gradsolve/solvers/tsit5_step.py", "ref_tsit5_step")
    src = (REF / "gradsolve/solvers/tsit5_replay.py").read_text()
    tree = ast.parse(src)
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "tsit5_adaptive")
    fn.body = [st for st in fn.body if not isinstance(st, ast.ImportFrom)]
    mod = ast.Module(body=[fn], type_ignores=[])
    ns = {"np": np}
    for k in dir(ts):
        if k.startswith("_") and k[1:2].isupper() or k in ("SAFETY", "ERR_FLOOR", "FAC_MIN",
                                                            "FAC_MAX", "ORDER_EXP"):
            ns[k] = getattr(ts, k)
    exec(compile(mod, str(REF / "gradsolve/solvers/tsit5_replay.py"), "exec"), ns)
    ros = _load_module(REF / "tests/_oracles/gradsolve_g2_spike_oracle.py", "ref_ros_oracle")
    return ts, ns["tsit5_adaptive"], ros


def f_lorenz(t, y, p):
    sigma = 10.0
    beta = 8.0 / 3.0
    rho = p[0]
    return np.array([sigma * (y[1] - y[0]), rho * y[0] - y[1] - y[0] * y[2],
                     y[0] * y[1] - beta * y[2]], dtype=np.float64)


def f_vdp(t, y, p):
    x, v = float(y[0]), float(y[1])
    mu = float(p[0])
    return np.array([v, mu * ((1.0 - x * x) * v - x)], dtype=np.float64)


def f_lv(t, y, p):
    x, w = float(y[0]), float(y[1])
    a, b, g, d = (float(v) for v in p)
    return np.array([a * x - b * x * w, d * x * w - g * w], dtype=np.float64)


def f_linear(t, y, p):
    return 1.01 * y


def f_robertson(t, y, p):
    k1, k2, k3 = float(p[0]), float(p[1]), float(p[2])
    y0, y1, y2 = float(y[0]), float(y[1]), float(y[2])
    return np.array([-k1 * y0 + k3 * y1 * y2, k1 * y0 - k3 * y1 * y2 - k2 * y1 * y1,
                     k2 * y1 * y1], dtype=np.float64)


def f_lorenz96(t, y, p):
    # the reference's numpy form of its lorenz96 field (gradsolve/warp/_warp_kernel.py:175-182:
    # roll(-1) / roll(2) / roll(1) are y_{i+1} / y_{i-2} / y_{i-1})
    return (np.roll(y, -1) - np.roll(y, 2)) * np.roll(y, 1) - y + float(p[0])


def f_hires(t, y, p):
    # HIRES-8 in the operation order of gradsolve/warp/_warp_rosenbrock.py:164-184
    y0, y1, y2, y3, y4, y5, y6, y7 = (float(v) for v in y)
    return np.array([
        -1.71 * y0 + 0.43 * y1 + 8.32 * y2 + 0.0007,
        1.71 * y0 - 8.75 * y1,
        -10.03 * y2 + 0.43 * y3 + 0.035 * y4,
        8.32 * y1 + 1.71 * y2 - 1.12 * y3,
        -1.745 * y4 + 0.43 * y5 + 0.43 * y6,
        -280.0 * y5 * y7 + 0.69 * y3 + 1.71 * y4 - 0.43 * y5 + 0.69 * y6,
        280.0 * y5 * y7 - 1.81 * y6,
        -280.0 * y5 * y7 + 1.81 * y6], dtype=np.float64)


def linstiff_matrix(D: int, seed: int) -> np.ndarray:
    """A constant stiff operator A = Q diag(-lam) Q^T with eigenvalues spread over four
    decades and a random orthogonal Q (numpy default_rng(seed))."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(D, D)))
    lam = np.logspace(0.0, 4.0, D)
    return -(Q * lam) @ Q.T


def run_tsit5(tsit5_adaptive, f, y0, params, t0, t1, rtol, atol, max_steps=100000):
    n = y0.shape[0]
    dt0 = (t1 - t0) / 100.0
    outs = []
    for j in range(n):
        p = params[j]
        outs.append(tsit5_adaptive(lambda t, y, p=p: f(t, y, p), y0[j], t0, t1, rtol, atol, dt0,
                                   max_steps))
    return _pack(outs, y0, params, t0, t1, rtol, atol)


def run_ros23(ros, f, y0, params, t0, t1, rtol, atol, max_steps=50000, jac=None):
    n = y0.shape[0]
    dt0 = (t1 - t0) / 100.0
    jac = ros.robertson_jac if jac is None else jac
    outs = []
    for j in range(n):
        p = params[j]
        outs.append(ros.rosenbrock23_adaptive(
            lambda t, y, p=p: f(t, y, p), lambda y, _p, p=p: jac(y, p),
            y0[j], t0, t1, rtol, atol, dt0, max_steps))
    return _pack(outs, y0, params, t0, t1, rtol, atol)


def _pack(outs, y0, params, t0, t1, rtol, atol):
    n = len(outs)
    n_acc = np.array([o[1].shape[0] for o in outs], dtype=np.int64)
    S = int(n_acc.max()) if n else 0
    dts = np.zeros((n, S))
    for j, o in enumerate(outs):
        dts[j, : o[1].shape[0]] = o[1]
    return dict(
        y0=y0, params=params, t0=np.float64(t0), t1=np.float64(t1), rtol=np.float64(rtol),
        atol=np.float64(atol), dts=dts, n_acc=n_acc,
        n_rej=np.array([o[2] for o in outs], dtype=np.int64),
        status=np.array([o[3] for o in outs], dtype=np.int64),
        y_final=np.stack([np.asarray(o[0], dtype=np.float64) for o in outs]))


def family_cases(tsit5_adaptive, ros) -> dict:
    """The reference's other fused-lane fields (gradsolve/warp/warp_ode.py:463-510 and
    gradsolve/warp/warp_rosenbrock.py:221-254): lorenz96_<D> and linear_ladder_<D> on the
    Tsit5 lane (D = 5 and 8 one thread per trajectory, 10 and 32 on a group of lanes), hires
    and a constant-matrix linstiff field on the Rosenbrock23 lane."""
    cases = {}
    for D, n, seed in ((5, 4, 11), (8, 6, 12), (32, 6, 13)):
        rng = np.random.default_rng(seed)
        F = rng.uniform(7.5, 8.5, (n, 1))
        y0 = F + rng.normal(0.0, 0.5, (n, D))
        cases[f"lorenz96_{D}"] = run_tsit5(tsit5_adaptive, f_lorenz96, y0, F, 0.0, 2.0,
                                           1e-8, 1e-8)
    for D, n, seed in ((10, 3, 14), (32, 3, 15)):
        rng = np.random.default_rng(seed)
        y0 = rng.uniform(-2.0, 2.0, (n, D))
        cases[f"linear_{D}"] = run_tsit5(tsit5_adaptive, f_linear, y0, np.zeros((n, 1)), 0.0,
                                         4.0, 1e-10, 1e-10)
    # HIRES: the standard start (Hairer & Wanner IV.10) with its first and last components
    # scaled by 1 + U(-0.1, 0.1) per trajectory, t in [0, 321.8122]
    rng = np.random.default_rng(16)
    n = 4
    y0 = np.tile(np.array([1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0057]), (n, 1))
    y0[:, 0] *= 1.0 + rng.uniform(-0.1, 0.1, n)
    y0[:, 7] *= 1.0 + rng.uniform(-0.1, 0.1, n)
    cases["hires"] = run_ros23(ros, f_hires, y0, np.zeros((n, 1)), 0.0, 321.8122, 1e-6, 1e-10,
                               jac=ros.hires_jac)
    for D, seed in ((4, 17), (8, 18)):
        A = linstiff_matrix(D, seed)
        rng = np.random.default_rng(seed + 100)
        y0 = rng.uniform(-1.0, 1.0, (3, D))
        c = run_ros23(ros, lambda t, y, p, A=A: A @ y, y0, np.zeros((3, 1)), 0.0, 1.0, 1e-6,
                      1e-9, jac=ros.constant_jac(A))
        c["A"] = A
        cases[f"linstiff_{D}"] = c
    return cases


def main(only=None):
    ts, tsit5_adaptive, ros = load_reference()
    if only:  # regenerate just the named cases (the others are deterministic and kept)
        cases = {k: v for k, v in family_cases(tsit5_adaptive, ros).items() if k in only}
        _save(cases)
        return 0
    cases = {}

    # tableau, as the reference module evaluates it
    names = ["_C", "_A21", "_A31", "_A32", "_A41", "_A42", "_A43", "_A51", "_A52", "_A53", "_A54",
             "_A61", "_A62", "_A63", "_A64", "_A65", "_B1", "_B2", "_B3", "_B4", "_B5", "_B6",
             "_B7", "_E1", "_E2", "_E3", "_E4", "_E5", "_E6", "_E7"]
    tab = {}
    for nm in names:
        tab[nm.lstrip("_")] = np.asarray(getattr(ts, nm), dtype=np.float64)
    tab["controller"] = np.array([ts.SAFETY, ts.ERR_FLOOR, ts.FAC_MIN, ts.FAC_MAX, ts.ORDER_EXP])
    tab["ros"] = np.array([ros._D, ros._E32, ros.SAFETY, ros.ERR_FLOOR, ros.FAC_MIN, ros.FAC_MAX,
                           ros.ORDER_EXP])
    np.savez(OUT / "tableau.npz", **tab)

    # config "plain method, small": Lorenz n=1024, rho = linspace(20,30); every 8th row kept
    n = 1024
    rho = np.linspace(20.0, 30.0, n)[:, None][::8]
    y0 = np.tile(np.array([1.0, 0.0, 0.0]), (rho.shape[0], 1))
    cases["lorenz_small"] = run_tsit5(tsit5_adaptive, f_lorenz, y0, rho, 0.0, 1.0, 1e-8, 1e-8)

    # "differentiation at scale" inputs (seed 0, n = 2^20), 12 sampled rows, t in [0, 10]
    rng = np.random.default_rng(0)
    N = 1 << 20
    y0_all = np.array([1.0, 0.0, 0.0]) + rng.normal(0.0, 0.1, (N, 3))
    rho_all = rng.uniform(20.0, 30.0, (N, 1))
    rows = np.random.default_rng(1).choice(N, 12, replace=False)
    cases["lorenz_scale"] = run_tsit5(tsit5_adaptive, f_lorenz, y0_all[rows], rho_all[rows],
                                      0.0, 10.0, 1e-8, 1e-8)
    cases["lorenz_scale"]["rows"] = rows

    # Van der Pol batch of tests/test_adjoint_replay.py:131-135
    y0 = np.array([[2.0, 0.0], [1.5, -0.5], [0.6, 1.0]])
    mu = np.array([0.6, 1.2, 0.9]).reshape(-1, 1)
    cases["vdp_batch"] = run_tsit5(tsit5_adaptive, f_vdp, y0, mu, 0.0, 1.0, 1e-6, 1e-9)

    # Lotka-Volterra, seed 2, 24 rows, t in [0, 20], rtol 1e-6 atol 1e-8
    rng = np.random.default_rng(2)
    M = 1 << 22
    lvp = rng.uniform(0.5, 1.5, (M, 4))
    lvy = rng.uniform(0.5, 2.0, (M, 2))
    rows = np.random.default_rng(1).choice(M, 24, replace=False)
    cases["lv_mixed"] = run_tsit5(tsit5_adaptive, f_lv, lvy[rows], lvp[rows], 0.0, 20.0,
                                  1e-6, 1e-8)
    cases["lv_mixed"]["rows"] = rows

    # linear_3 (analytic exp(1.01 t))
    y0 = np.array([[1.0, 2.0, -0.5], [0.25, -1.0, 3.0]])
    cases["linear3"] = run_tsit5(tsit5_adaptive, f_linear, y0, np.zeros((2, 1)), 0.0, 1.0,
                                 1e-6, 1e-9)

    # Robertson-ish batch of tests/test_adjoint_replay.py:224-229 (t1 = 0.5)
    y0 = np.array([[1.0, 0.0, 0.0], [0.9, 0.05, 0.05], [0.8, 0.1, 0.1]])
    k = np.array([[0.4, 20.0, 5.0], [0.5, 25.0, 6.0], [0.35, 15.0, 4.0]])
    cases["robertson_toy"] = run_ros23(ros, f_robertson, y0, k, 0.0, 0.5, 1e-6, 1e-9)

    # "stiff" config: canonical rates scaled by 10^U(-0.5,0.5) (seed 4), 6 rows, t1 = 1e4
    rng = np.random.default_rng(4)
    M = 1 << 18
    scale = 10.0 ** rng.uniform(-0.5, 0.5, (M, 3))
    kk = np.array([0.04, 3.0e7, 1.0e4]) * scale
    rows = np.random.default_rng(1).choice(M, 6, replace=False)
    y0 = np.tile(np.array([1.0, 0.0, 0.0]), (6, 1))
    cases["robertson_stiff"] = run_ros23(ros, f_robertson, y0, kk[rows], 0.0, 1.0e4, 1e-6, 1e-10)
    cases["robertson_stiff"]["rows"] = rows

    cases.update(family_cases(tsit5_adaptive, ros))
    _save(cases)
    return 0


def _save(cases):
    for name, d in cases.items():
        np.savez_compressed(OUT / f"{name}.npz", **d)
        print(f"{name}: n={d['y0'].shape[0]} S={d['dts'].shape[1]} "
              f"acc {d['n_acc'].min()}..{d['n_acc'].max()} rej max {d['n_rej'].max()} "
              f"status {set(d['status'].tolist())}")


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
