"""Bit-for-bit forward parity with the reference's tsit5_adaptive.

The exact-association instance (tests/exact/gs_exact.cu, built with -fmad=false) runs the
product's own stage helpers and fields with the reference's literal error norm and
controller; on every Tsit5 golden made by the reference's own code (tests/golden/) it must
reproduce the accepted and rejected counts, every recorded dt and y_final exactly.  The tuned
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
    L.gx_tsit5_record.argtypes = [i, ll, vp, vp, d, d, d, d, d, i, i, vp, vp, vp, vp, vp, vp]
    L.gx_tsit5_record.restype = i
    return L


def _params(g, P):
    n = g["y0"].shape[0]
    p = np.asarray(g["params"], np.float64).reshape(n, -1)
    if p.shape[1] < P:
        p = np.pad(p, ((0, 0), (0, P - p.shape[1])))
    return np.ascontiguousarray(p[:, :P])


def _run_exact(L, code, P, g, cap=None):
    dev = torch.device("cuda")
    y0 = torch.tensor(g["y0"], device=dev).contiguous()
    p = torch.tensor(_params(g, P), device=dev)
    n, D = y0.shape
    cap = cap or max(1, g["dts"].shape[1])
    dts = torch.empty((n, cap), dtype=torch.float64, device=dev)
    yf = torch.empty_like(y0)
    n_acc, n_rej, status = (torch.empty(n, dtype=torch.int32, device=dev) for _ in range(3))
    rc = L.gx_tsit5_record(code, n, y0.data_ptr(), p.data_ptr(), float(g["t0"]),
                           float(g["t1"]), float(g["rtol"]), float(g["atol"]), -1.0, 100000,
                           cap, dts.data_ptr(), yf.data_ptr(), n_acc.data_ptr(),
                           n_rej.data_ptr(), status.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    return (dts.cpu().numpy(), yf.cpu().numpy(), n_acc.cpu().numpy(), n_rej.cpu().numpy(),
            status.cpu().numpy())


@pytest.mark.parametrize("case,code,P,_name", CASES)
def test_exact_instance_reproduces_reference_bitwise(gslib, cuda, exact, case, code, P, _name):
    g = load_golden(case)
    dts, yf, n_acc, n_rej, status = _run_exact(exact, code, P, g)
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
    dts_x, yf_x, n_acc_x, n_rej_x, _ = _run_exact(exact, code, P, g)
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
