"""Bit-for-bit forward parity with the reference's tsit5_adaptive.

The exact-association instance (tests/exact/gs_exact.cu, built with -fmad=false) runs the
product's own stage helpers and fields with the reference's literal error norm and
controller, and takes the controller's power from the host libm (the reference's pow, which
CUDA's does not match in the last bit for every argument); on every Tsit5 golden made by the
reference's own code (tests/golden/) it must reproduce the accepted and rejected counts,
every recorded dt and y_final exactly.  The tuned
kernel's distance from those values is then measured here: it is what the tuned kernel's
own dt tolerance in tests/test_gpu_tsit5.py covers (fused multiply-adds and the pow-free
controller move a step by a few ulp of err; the chaotic cases amplify that).
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import ROOT, load_golden

pytestmark = pytest.mark.gpu

# (golden, field code of the exact instance, parameter count, product field name)
CASES = [("lorenz_small", 1, 1, "lorenz"), ("lorenz_scale", 1, 1, "lorenz"),
         ("vdp_batch", 2, 1, "vdp"), ("lv_mixed", 3, 4, "lv"), ("linear3", 4003, 1, "linear_3"),
         ("linear_10", 4010, 1, "linear_ladder_10"), ("linear_32", 4032, 1, "linear_ladder_32"),
         ("lorenz96_5", 5005, 1, "lorenz96_5"), ("lorenz96_8", 5008, 1, "lorenz96_8"),
         ("lorenz96_32", 5032, 1, "lorenz96_32")]


@pytest.fixture(scope="module")
def exact():
    import sys
    sys.path.insert(0, str(ROOT / "tests" / "exact"))
    import build as exact_build
    L = ctypes.CDLL(str(exact_build.build()))
    vp, d, ll, i = ctypes.c_void_p, ctypes.c_double, ctypes.c_longlong, ctypes.c_int
    L.gx_tsit5_record.argtypes = [i, ll, vp, vp, d, d, d, d, d, i, i, vp, vp, vp, vp, vp, vp,
                                  vp, i, vp]
    L.gx_tsit5_record.restype = i
    return L


def _params(g, P):
    n = g["y0"].shape[0]
    p = np.asarray(g["params"], np.float64).reshape(n, -1)
    if p.shape[1] < P:
        p = np.pad(p, ((0, 0), (0, P - p.shape[1])))
    return np.ascontiguousarray(p[:, :P])


def _run_exact(L, code, P, g, table=None, A=1):
    """One launch of the exact instance on a golden's inputs; returns dts (n, S), y_final,
    n_acc, n_rej, status and the (n, A, 2) log of (floored err, power used) per attempt."""
    dev = torch.device("cuda")
    y0 = torch.tensor(g["y0"], device=dev).contiguous()
    p = torch.tensor(_params(g, P), device=dev)
    n, D = y0.shape
    cap = max(1, g["dts"].shape[1])
    dts = torch.empty((n, cap), dtype=torch.float64, device=dev)
    yf = torch.empty_like(y0)
    n_acc, n_rej, status = (torch.empty(n, dtype=torch.int32, device=dev) for _ in range(3))
    tab = None if table is None else torch.tensor(table, device=dev).contiguous()
    log = torch.full((n, A, 2), float("nan"), dtype=torch.float64, device=dev)
    rc = L.gx_tsit5_record(code, n, y0.data_ptr(), p.data_ptr(), float(g["t0"]),
                           float(g["t1"]), float(g["rtol"]), float(g["atol"]), -1.0, 100000,
                           cap, dts.data_ptr(), yf.data_ptr(), n_acc.data_ptr(),
                           n_rej.data_ptr(), status.data_ptr(),
                           None if tab is None else tab.data_ptr(), log.data_ptr(), A,
                           torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    return (dts.cpu().numpy(), yf.cpu().numpy(), n_acc.cpu().numpy(), n_rej.cpu().numpy(),
            status.cpu().numpy(), log.cpu().numpy())


def _with_host_pow(L, code, P, g):
    """Run the exact instance with the reference's power, max(err, 1e-10) ** -0.2 on Python
    floats (the host libm's pow), at every attempt.  CUDA's pow is used except where a table
    overrides it; each round finds, per trajectory, the first attempt whose power differs
    from the host's for that attempt's own err, overrides it there and drops the overrides
    after it (they belonged to errors the correction changes).  A trajectory is settled when
    no attempt differs, so every round settles at least one more attempt of every unsettled
    trajectory.  Returns the settled run and the first run's share of controller arguments
    on which CUDA's pow and the host's differ."""
    A = int((np.asarray(g["n_acc"]) + np.asarray(g["n_rej"])).max()) + 8
    n = g["y0"].shape[0]
    over = np.full((n, A), np.nan)
    start = np.zeros(n, dtype=np.int64)  # attempts before start[j] are settled
    first_share = None
    for _ in range(A + 1):
        out = _run_exact(L, code, P, g, table=over, A=A)
        err, used = out[5][..., 0], out[5][..., 1]
        if first_share is None:
            m = np.isfinite(err)
            host = [float(e) ** -0.2 for e in err[m]]
            first_share = float(np.mean(used[m] != np.array(host))) if m.any() else 0.0
        changed = False
        for j in range(n):
            for it in range(int(start[j]), A):
                if not np.isfinite(err[j, it]):
                    start[j] = A
                    break
                hp = float(err[j, it]) ** -0.2
                if used[j, it] != hp:
                    over[j, it] = hp
                    over[j, it + 1:] = np.nan
                    start[j] = it + 1
                    changed = True
                    break
            else:
                start[j] = A
        if not changed:
            return out, first_share
    raise AssertionError("the powers did not settle")


@pytest.mark.parametrize("case,code,P,_name", CASES)
def test_exact_instance_reproduces_reference_bitwise(gslib, cuda, exact, case, code, P, _name):
    g = load_golden(case)
    (dts, yf, n_acc, n_rej, status, _log), cuda_vs_host = _with_host_pow(exact, code, P, g)
    print(f"{case}: CUDA's pow differs from the host libm's on {cuda_vs_host:.2%} of the "
          "controller's arguments")
    np.testing.assert_array_equal(status, g["status"])
    np.testing.assert_array_equal(n_acc, g["n_acc"])
    np.testing.assert_array_equal(n_rej, g["n_rej"])
    np.testing.assert_array_equal(dts, g["dts"])
    np.testing.assert_array_equal(yf, g["y_final"])


@pytest.mark.parametrize("case,code,P,name", CASES)
def test_tuned_kernel_distance_from_exact_instance(gslib, cuda, exact, case, code, P, name):
    """The tuned forward against the exact instance on the same inputs: identical step
    counts, dts within the tolerance tests/test_gpu_tsit5.py uses (max 1e-4 relative; the
    measured values are printed), y_final within 1e-9 relative of the row's scale."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    g = load_golden(case)
    (dts_x, yf_x, n_acc_x, n_rej_x, _st, _log), _ = _with_host_pow(exact, code, P, g)
    spec = field_spec(name)
    y0 = torch.tensor(g["y0"], device="cuda")
    p = torch.tensor(_params(g, spec.nparam), device="cuda")
    r = engine.forward_record("tsit5", spec, y0, p, t0=float(g["t0"]), t1=float(g["t1"]),
                              rtol=float(g["rtol"]), atol=float(g["atol"]), max_steps=100000)
    np.testing.assert_array_equal(r.n_acc.cpu().numpy(), n_acc_x)
    np.testing.assert_array_equal(r.n_rej.cpu().numpy(), n_rej_x)
    dts = r.padded_dts(dts_x.shape[1]).cpu().numpy()
    m = dts_x > 0
    q = np.abs(dts[m] - dts_x[m]) / dts_x[m]
    same = float(np.mean(q == 0))
    print(f"{case}: tuned vs exact dts: {same:.1%} identical, median {np.median(q):.1e}, "
          f"p99 {np.quantile(q, 0.99):.1e}, max {q.max():.1e}")
    assert q.max() <= 1e-4
    yr = r.y_final.cpu().numpy()
    assert np.max(np.abs(yr - yf_x).max(axis=1) / np.abs(yf_x).max(axis=1)) <= 1e-9
