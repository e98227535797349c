"""Python face of the CPU oracle (test infrastructure only).

Nothing in the product package ``gradsolve_b200`` imports this module.  It is loaded by
the tests, by ``__graft_entry__.smoke()`` and by the CPU legs of ``bench.py``, always as
the result compared against or the timed CPU baseline, never as the path being measured.

Three layers:

* ``libgs_oracle.so`` (``gs_oracle.c``): a plain-C restatement of the reference's
  ``tsit5_adaptive`` (gradsolve/solvers/tsit5_replay.py:62-124), its replay
  (gradsolve/warp/warp_replay.py:30-55 over gradsolve/solvers/tsit5_step.py:80-102), the
  fused Rosenbrock23 kernel's arithmetic (gradsolve/warp/_warp_rosenbrock.py:383-452) and
  its replay (gradsolve/solvers/rosenbrock23_step.py:47-66), plus hand-derived reverse
  passes of both replays.  Pinned against tests/golden/ (made by the reference's own code).
* ``torch_replay_grad``: an independent float64 ``torch.autograd`` restatement of the
  replay (the same per-step arithmetic, differentiated by autograd rather than by hand) --
  the stand-in for ``jax.grad`` through ``replay_solve_jax``, which cannot run without JAX.
* ``fd_grad``: frozen-mesh central differences (tests/test_adjoint_replay.py:109-123).
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libgs_oracle.so"

# field codes shared with the C oracle (linear_D is 4000 + D, lorenz96_D 5000 + D, the
# constant-matrix linstiff field 13000 + D with its matrix set by set_linstiff)
FIELDS = {"lorenz": 1, "vdp": 2, "lv": 3, "robertson": 10, "lorenz3": 11, "hires": 12}
METHODS = {"tsit5": 0, "rosenbrock23": 1}


def field_code(name: str) -> int:
    for prefix, base in (("linear_", 4000), ("lorenz96_", 5000), ("linstiff_", 13000)):
        if name.startswith(prefix):
            return base + int(name.rsplit("_", 1)[1])
    return FIELDS[name]


def set_linstiff(A) -> str:
    """Make the oracle's linstiff field f = A y (constant D x D matrix); returns its field
    name ``linstiff_<D>`` for the calls that follow."""
    A = np.ascontiguousarray(np.asarray(A, np.float64))
    D = A.shape[0]
    if A.shape != (D, D):
        raise ValueError(f"linstiff matrix must be square, got {A.shape}")
    if lib().gso_set_linstiff(D, _dp(A)):
        raise ValueError(f"linstiff dimension {D} out of range")
    return f"linstiff_{D}"


def build() -> Path:
    """Compile the oracle (make in this directory); returns the library path.  Concurrent
    callers (one process per GPU, parallel test workers) take an exclusive lock first, so one
    of them runs make and the others find the library up to date."""
    import fcntl
    with open(HERE / ".build.lock", "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        try:
            subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
        finally:
            fcntl.flock(lock, fcntl.LOCK_UN)
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.gso_record.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, dp, dp, ctypes.c_double,
                                 dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp, ip, ip, ip,
                                 ctypes.c_int]
        L.gso_replay.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, dp, dp, ctypes.c_double,
                                 dp, ctypes.c_long, dp, ctypes.c_int]
        L.gso_replay_vjp.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, dp, dp,
                                     ctypes.c_double, dp, ctypes.c_long, dp, dp, dp, ctypes.c_int]
        L.gso_field_info.argtypes = [ctypes.c_int, ip, ip]
        L.gso_tsit5_error_weights.argtypes = [dp]
        L.gso_set_linstiff.argtypes = [ctypes.c_int, dp]
        _LIB = L
    return _LIB


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def field_dims(field: str):
    D, P = ctypes.c_int(), ctypes.c_int()
    if lib().gso_field_info(field_code(field), ctypes.byref(D), ctypes.byref(P)):
        raise ValueError(f"oracle has no field {field!r}")
    return D.value, P.value


def _prep(field, y0, params):
    D, P = field_dims(field)
    y0 = np.ascontiguousarray(np.asarray(y0, dtype=np.float64).reshape(-1, D))
    n = y0.shape[0]
    params = np.asarray(params, dtype=np.float64)
    if params.size == 0:
        params = np.zeros((n, P))
    params = np.ascontiguousarray(params.reshape(n, -1))
    if params.shape[1] < P:
        params = np.ascontiguousarray(np.pad(params, ((0, 0), (0, P - params.shape[1]))))
    return y0, params[:, :P].copy(), n, D, P


def record(method, field, y0, params, t0, t1, rtol, atol, *, dt0=None, max_steps=100000,
           cap=None, t1v=None, nthreads=1):
    """Adaptive solve with the accepted dt's recorded. Returns a dict with y_final, dts
    (padded [n, S], S = max n_acc), n_acc, n_rej, status."""
    y0, params, n, D, P = _prep(field, y0, params)
    cap = int(max_steps if cap is None else cap)
    dts = np.zeros((n, cap))
    yf = np.zeros((n, D))
    n_acc = np.zeros(n, np.int32)
    n_rej = np.zeros(n, np.int32)
    status = np.zeros(n, np.int32)
    t1v_a = None if t1v is None else np.ascontiguousarray(np.asarray(t1v, np.float64))
    rc = lib().gso_record(METHODS[method], field_code(field), n, _dp(y0), _dp(params), float(t0),
                          _dp(t1v_a), float(t1), float(rtol), float(atol),
                          float(dt0) if dt0 is not None else -1.0, int(max_steps), cap, _dp(dts),
                          _dp(yf), _ip(n_acc), _ip(n_rej), _ip(status), int(nthreads))
    if rc:
        raise RuntimeError(f"oracle record failed ({rc})")
    S = int(n_acc.max()) if n else 0
    return dict(y_final=yf, dts=np.ascontiguousarray(dts[:, :S]), n_acc=n_acc.astype(np.int64),
                n_rej=n_rej.astype(np.int64), status=status.astype(np.int64))


def replay(method, field, y0, params, dts, t0=0.0, nthreads=1):
    y0, params, n, D, P = _prep(field, y0, params)
    dts = np.ascontiguousarray(np.asarray(dts, np.float64).reshape(n, -1))
    yf = np.zeros((n, D))
    rc = lib().gso_replay(METHODS[method], field_code(field), n, _dp(y0), _dp(params), float(t0),
                          _dp(dts), dts.shape[1], _dp(yf), int(nthreads))
    if rc:
        raise RuntimeError(f"oracle replay failed ({rc})")
    return yf


def replay_vjp(method, field, y0, params, dts, ybar, t0=0.0, nthreads=1):
    """(d/dy0, d/dp) of sum(ybar * replay(y0, p, dts)) with the dts frozen."""
    y0, params, n, D, P = _prep(field, y0, params)
    dts = np.ascontiguousarray(np.asarray(dts, np.float64).reshape(n, -1))
    ybar = np.ascontiguousarray(np.asarray(ybar, np.float64).reshape(n, D))
    gy0 = np.zeros((n, D))
    gp = np.zeros((n, P))
    rc = lib().gso_replay_vjp(METHODS[method], field_code(field), n, _dp(y0), _dp(params),
                              float(t0), _dp(dts), dts.shape[1], _dp(ybar), _dp(gy0), _dp(gp),
                              int(nthreads))
    if rc:
        raise RuntimeError(f"oracle replay_vjp failed ({rc})")
    return gy0, gp


def tsit5_error_weights():
    out = np.zeros(7)
    lib().gso_tsit5_error_weights(_dp(out))
    return out


# ------------------------------------------------------------------------------------
# torch float64 autograd restatement of the replay (the jax.grad stand-in)
# ------------------------------------------------------------------------------------

def _torch_tableau():
    w = tsit5_error_weights()  # noqa: F841  (the E's are not used by the replay)
    C = (161.0 / 1000.0, 327.0 / 1000.0, 9.0 / 10.0,
         0.9800255409045096857298102862870245954942137979563024768854764293221195950761080302604,
         1.0, 1.0)
    A = [
        [161.0 / 1000.0],
        [-0.8480655492356988544426874250230774675121177393430391537369234245294192976164141156943e-2,
         0.3354806554923569885444268742502307746751211773934303915373692342452941929761641411569],
        [2.897153057105493432130432594192938764924887287701866490314866693455023795137503079289,
         -6.359448489975074843148159912383825625952700647415626703305928850207288721235210244366,
         4.362295432869581411017727318190886861027813359713760212991062156752264926097707165077],
        [5.325864828439256604428877920840511317836476253097040101202360397727981648835607691791,
         -11.74888356406282787774717033978577296188744178259862899288666928009020615663593781589,
         7.495539342889836208304604784564358155658679161518186721010132816213648793440552049753,
         -0.9249506636175524925650207933207191611349983406029535244034750452930469056411389539635e-1],
        [5.861455442946420028659251486982647890394337666164814434818157239052507339770711679748,
         -12.92096931784710929170611868178335939541780751955743459166312250439928519268343184452,
         8.159367898576158643180400794539253485181918321135053305748355423955009222648673734986,
         -0.7158497328140099722453054252582973869127213147363544882721139659546372402303777878835e-1,
         -0.2826905039406838290900305721271224146717633626879770007617876201276764571291579142206e-1],
    ]
    B = [0.9646076681806522951816731316512876333711995238157997181903319145764851595234062815396e-1,
         1.0 / 100.0,
         0.4798896504144995747752495322905965199130404621990332488332634944254542060153074523509,
         1.379008574103741893192274821856872770756462643091360525934940067397245698027561293331,
         -3.290069515436080679901047585711363850115683290894936158531296799594813811049925401677,
         2.324710524099773982415355918398765796109060233222962411944060046314465391054716027841,
         0.0]
    return C, A, B


def torch_field(field):
    import torch

    if field == "lorenz":
        def f(y, p):
            return torch.stack([10.0 * (y[:, 1] - y[:, 0]),
                                p[:, 0] * y[:, 0] - y[:, 1] - y[:, 0] * y[:, 2],
                                y[:, 0] * y[:, 1] - (8.0 / 3.0) * y[:, 2]], dim=1)
    elif field == "lorenz3":
        def f(y, p):
            return torch.stack([p[:, 0] * (y[:, 1] - y[:, 0]),
                                p[:, 2] * y[:, 0] - y[:, 1] - y[:, 0] * y[:, 2],
                                y[:, 0] * y[:, 1] - p[:, 1] * y[:, 2]], dim=1)
    elif field == "vdp":
        def f(y, p):
            x, v = y[:, 0], y[:, 1]
            return torch.stack([v, p[:, 0] * ((1.0 - x * x) * v - x)], dim=1)
    elif field == "lv":
        def f(y, p):
            x, w = y[:, 0], y[:, 1]
            return torch.stack([p[:, 0] * x - p[:, 1] * x * w, p[:, 3] * x * w - p[:, 2] * w],
                               dim=1)
    elif field.startswith("linear_"):
        def f(y, p):
            return 1.01 * y
    elif field.startswith("lorenz96_"):
        def f(y, p):
            return ((torch.roll(y, -1, dims=1) - torch.roll(y, 2, dims=1)) *
                    torch.roll(y, 1, dims=1) - y + p[:, :1])
    elif field == "hires":
        def f(y, p):
            y0, y1, y2, y3, y4, y5, y6, y7 = (y[:, i] for i in range(8))
            return torch.stack([
                -1.71 * y0 + 0.43 * y1 + 8.32 * y2 + 0.0007, 1.71 * y0 - 8.75 * y1,
                -10.03 * y2 + 0.43 * y3 + 0.035 * y4, 8.32 * y1 + 1.71 * y2 - 1.12 * y3,
                -1.745 * y4 + 0.43 * y5 + 0.43 * y6,
                -280.0 * y5 * y7 + 0.69 * y3 + 1.71 * y4 - 0.43 * y5 + 0.69 * y6,
                280.0 * y5 * y7 - 1.81 * y6, -280.0 * y5 * y7 + 1.81 * y6], dim=1)
    elif field == "robertson":
        def f(y, p):
            k1, k2, k3 = p[:, 0], p[:, 1], p[:, 2]
            a, b, c = y[:, 0], y[:, 1], y[:, 2]
            return torch.stack([-k1 * a + k3 * b * c, k1 * a - k3 * b * c - k2 * b * b,
                                k2 * b * b], dim=1)
    else:
        raise ValueError(field)
    return f


def torch_replay(method, field, y0, params, dts):
    """Differentiable float64 replay (torch tensors in, tensor out)."""
    import torch

    f = torch_field(field)
    C, A, B = _torch_tableau()
    y = y0
    S = dts.shape[1]
    if method == "tsit5":
        for s in range(S):
            dt = dts[:, s:s + 1]
            k = [f(y, params)]
            for r in range(5):
                acc = A[r][0] * k[0]
                for c in range(1, r + 1):
                    acc = acc + A[r][c] * k[c]
                k.append(f(y + dt * acc, params))
            acc = B[0] * k[0]
            for c in range(1, 6):
                acc = acc + B[c] * k[c]
            k.append(f(y + dt * acc, params))
            acc = B[0] * k[0]
            for c in range(1, 7):
                acc = acc + B[c] * k[c]
            y = y + dt * acc
        return y
    # rosenbrock23_step with J from torch.func.jacrev of the per-trajectory field
    from torch.func import jacrev, vmap

    d = 1.0 / (2.0 + 2.0 ** 0.5)
    D = y.shape[1]

    def f1(yy, pp):
        return f(yy[None, :], pp[None, :])[0]

    jacf = vmap(jacrev(f1, argnums=0))
    eye = torch.eye(D, dtype=y.dtype)
    for s in range(S):
        dt = dts[:, s:s + 1]
        J = jacf(y, params)
        W = eye[None] - (dt * d)[:, :, None] * J
        F0 = f(y, params)
        k1 = torch.linalg.solve(W, F0)
        F1 = f(y + 0.5 * dt * k1, params)
        k2 = torch.linalg.solve(W, F1 - k1) + k1
        y = y + dt * k2
    return y


def torch_replay_grad(method, field, y0, params, dts, ybar):
    """(d/dy0, d/dp) of sum(ybar * replay) through torch float64 autograd."""
    import torch

    D, P = field_dims(field)
    y0_t = torch.tensor(np.asarray(y0, np.float64).reshape(-1, D), requires_grad=True)
    p_np = np.asarray(params, np.float64).reshape(y0_t.shape[0], -1)
    p_t = torch.tensor(p_np, requires_grad=True)
    dts_t = torch.tensor(np.asarray(dts, np.float64).reshape(y0_t.shape[0], -1))
    yf = torch_replay(method, field, y0_t, p_t, dts_t)
    loss = (yf * torch.tensor(np.asarray(ybar, np.float64).reshape(yf.shape))).sum()
    gy0, gp = torch.autograd.grad(loss, [y0_t, p_t], allow_unused=True)
    if gp is None:  # a field that reads no parameter (linear, hires, linstiff)
        gp = torch.zeros_like(p_t)
    return gy0.numpy(), gp.numpy()


def fd_grad(loss, x0, h_scale=1e-6):
    """Central differences with step h_scale*max(|x|,1) (tests/test_adjoint_replay.py:109-119)."""
    x0 = np.asarray(x0, dtype=np.float64)
    g = np.empty_like(x0)
    flat = x0.reshape(-1)
    gf = g.reshape(-1)
    for i in range(flat.size):
        h = h_scale * max(abs(flat[i]), 1.0)
        xp = flat.copy()
        xm = flat.copy()
        xp[i] += h
        xm[i] -= h
        gf[i] = (loss(xp.reshape(x0.shape)) - loss(xm.reshape(x0.shape))) / (2.0 * h)
    return g


# ------------------------------------------------------------------------------------
# saveat: restatement of gradsolve/solvers/dense.py:106-163 (bracket-and-re-step)
# ------------------------------------------------------------------------------------

def _saveat_rows(y0, dts, ts, t0):
    """For each (trajectory, requested time): the dt row whose replay gives that saved state,
    following scan_saveat_one's rules.  Returns rows (n*K, S+1) and their kinds."""
    n, S = dts.shape
    ts = np.asarray(ts, np.float64)
    if ts.ndim == 1:
        ts = np.broadcast_to(ts, (n, ts.shape[0]))
    K = ts.shape[1]
    rows = np.zeros((n * K, S + 1))
    for j in range(n):
        t = float(t0)
        starts = []
        for s in range(S):
            starts.append(t)
            t = t + dts[j, s]
        t_fin = t
        for k in range(K):
            tk = float(ts[j, k])
            r = rows[j * K + k]
            if tk >= t_fin:            # at or past the final accumulated time: y_final
                r[:S] = dts[j]
                continue
            hit = [s for s in range(S) if dts[j, s] > 0 and tk > starts[s]
                   and tk <= starts[s] + dts[j, s]]
            if not hit:               # never bracketed: y0
                continue
            s = hit[-1]
            r[:s] = dts[j, :s]
            r[s] = tk - starts[s]
    return rows, K


def replay_saveat(method, field, y0, params, dts, ts, t0=0.0, nthreads=4):
    """(y_final (n, D), ys (n, K, D)) of the frozen-mesh replay with dense output."""
    y0, params, n, D, P = _prep(field, y0, params)
    dts = np.ascontiguousarray(np.asarray(dts, np.float64).reshape(n, -1))
    rows, K = _saveat_rows(y0, dts, ts, t0)
    ys = replay(method, field, np.repeat(y0, K, axis=0), np.repeat(params, K, axis=0), rows,
                t0, nthreads)
    return replay(method, field, y0, params, dts, t0, nthreads), ys.reshape(n, K, D)


def replay_saveat_vjp(method, field, y0, params, dts, ts, ysbar, ybar=None, t0=0.0,
                      nthreads=4):
    """Gradient of sum(ysbar * ys) + sum(ybar * y_final) w.r.t. (y0, params)."""
    y0, params, n, D, P = _prep(field, y0, params)
    dts = np.ascontiguousarray(np.asarray(dts, np.float64).reshape(n, -1))
    rows, K = _saveat_rows(y0, dts, ts, t0)
    ysbar = np.asarray(ysbar, np.float64).reshape(n * K, D)
    gy, gp = replay_vjp(method, field, np.repeat(y0, K, axis=0), np.repeat(params, K, axis=0),
                        rows, ysbar, t0, nthreads)
    gy0 = gy.reshape(n, K, D).sum(axis=1)
    gpp = gp.reshape(n, K, P).sum(axis=1)
    if ybar is not None:
        a, b = replay_vjp(method, field, y0, params, dts, ybar, t0, nthreads)
        gy0 = gy0 + a
        gpp = gpp + b
    return gy0, gpp
