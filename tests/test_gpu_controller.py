"""The forward kernels' controller (gs_tsit5.cuh step_from_sum: the accept test and the
reciprocal root on the sum of squares S -- a float32 first guess refined by one second-order
series step -- with host-computed constants for the state
dimension D) against the reference's formula on the mean m = S / D evaluated with CUDA's sqrt
and pow: accept iff sqrt(m) <= 1, factor 0.9 * max(sqrt(m), 1e-10)^(-1/q) clipped to
[0.2, 5] (gradsolve/solvers/tsit5_replay.py:122, gradsolve/warp/_warp_rosenbrock.py:448-450)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("D", [1, 2, 3, 8])
@pytest.mark.parametrize("order", [5, 3])
def test_step_factor_matches_pow(gslib, cuda, order, D):
    L = ctypes.CDLL(str(ROOT / "gradsolve_b200" / "libgsprobe.so"))
    rng = np.random.default_rng(order)
    m = np.concatenate([
        10.0 ** rng.uniform(-24, 9, 400000),
        np.nextafter(1.0, np.array([0.0, 2.0])),
        [1.0, 1.0 + 2 ** -52, 1.0 + 2 ** -51, 0.0, 3.570467226623999e-08, 3405062.8916015625,
         3.401222399999999e-05, 8303.765625],
        1.0 + rng.normal(0, 1e-12, 1000)])
    # sums of squares around every accept boundary D * (1 + k 2^-52), and D * m in general
    edge = np.array([D * (1.0 + k * 2.0 ** -52) for k in range(-4, 5)])
    m = np.concatenate([m * D, edge, np.nextafter(edge, 0.0), np.nextafter(edge, 10.0)])
    x = torch.tensor(m, device=cuda)
    n = x.numel()
    fast = torch.empty_like(x)
    ref = torch.empty_like(x)
    af = torch.empty(n, dtype=torch.int32, device=cuda)
    ar = torch.empty(n, dtype=torch.int32, device=cuda)
    assert L.gs_probe_step_factor(ctypes.c_void_p(x.data_ptr()), ctypes.c_longlong(n), order,
                                  D, ctypes.c_void_p(fast.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                  ctypes.c_void_p(af.data_ptr()), ctypes.c_void_p(ar.data_ptr()),
                                  None) == 0
    torch.cuda.synchronize()
    assert torch.equal(af, ar)  # the accept decision is unchanged, bit for bit
    f = fast.cpu().numpy()
    r = ref.cpu().numpy()
    ulp = np.abs(f - r) / np.spacing(r)
    # D = 1: the refined root agrees with pow to a few ulp; other D add the rounding of
    # 0.9 D^(1/K) and of the mean the reference forms
    assert ulp.max() <= (4 if D == 1 else 8), f"max {ulp.max()} ulp"
