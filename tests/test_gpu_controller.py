"""The forward kernels' step-size factor (Newton reciprocal root of the mean of squares,
gs_tsit5.cuh step_from_mean) against the reference's formula evaluated with CUDA's pow:
0.9 * max(sqrt(m), 1e-10)^(-1/q) clipped to [0.2, 5] (gradsolve/solvers/tsit5_replay.py:122,
gradsolve/warp/_warp_rosenbrock.py:448-450), and the accept test sqrt(m) <= 1."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [5, 3])
def test_step_factor_matches_pow(gslib, cuda, order):
    L = ctypes.CDLL(str(ROOT / "gradsolve_b200" / "libgsprobe.so"))
    rng = np.random.default_rng(order)
    m = np.concatenate([
        10.0 ** rng.uniform(-24, 9, 400000),
        np.nextafter(1.0, np.array([0.0, 2.0])),
        [1.0, 1.0 + 2 ** -52, 1.0 + 2 ** -51, 0.0, 3.570467226623999e-08, 3405062.8916015625,
         3.401222399999999e-05, 8303.765625],
        1.0 + rng.normal(0, 1e-12, 1000)])
    x = torch.tensor(m, device=cuda)
    n = x.numel()
    fast = torch.empty_like(x)
    ref = torch.empty_like(x)
    af = torch.empty(n, dtype=torch.int32, device=cuda)
    ar = torch.empty(n, dtype=torch.int32, device=cuda)
    assert L.gs_probe_step_factor(ctypes.c_void_p(x.data_ptr()), ctypes.c_longlong(n), order,
                                  ctypes.c_void_p(fast.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                  ctypes.c_void_p(af.data_ptr()), ctypes.c_void_p(ar.data_ptr()),
                                  None) == 0
    torch.cuda.synchronize()
    assert torch.equal(af, ar)  # the accept decision is unchanged, bit for bit
    f = fast.cpu().numpy()
    r = ref.cpu().numpy()
    ulp = np.abs(f - r) / np.spacing(r)
    assert ulp.max() <= 4, f"max {ulp.max()} ulp"
