"""gs_tsit5_vjp_static: the replay gradient for callers that cannot allocate device memory
(a custom call inside JAX/XLA whose memory XLA has already reserved, or a latency-critical
caller that cannot take cudaMalloc's device-wide synchronisation).

It must give the same y_final and gradients as the allocating entry points
(gs_record_from_padded + gs_tsit5_replay + gs_tsit5_adjoint on caller buffers), within the
tolerance the other gradient tests use, on two calls in a row -- the second on different
inputs, so contents the first call left in the shared scratch cannot leak into it -- and it
must refuse sizes beyond its scratch.  This file is collected last so a stop at the first
failure has already run every other test.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.cpu().numpy()
    b = b.cpu().numpy()
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-8)))


def _static_call(gslib, code, y0, p, dts, ybar):
    n, S = dts.shape
    yf = torch.empty_like(y0)
    gy0 = torch.empty_like(y0)
    gp = torch.empty_like(p)
    rc = gslib.lib().gs_tsit5_vjp_static(code, n, y0.data_ptr(), p.data_ptr(), 0.0,
                                         dts.data_ptr(), S, S, ybar.data_ptr(), yf.data_ptr(),
                                         gy0.data_ptr(), gp.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream)
    gslib.check(rc, "gs_tsit5_vjp_static")
    return yf, gy0, gp


def _allocating_call(method, field, y0, p, dts, ybar):
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    r = engine.record_from_padded(method, field_spec(field), dts, 0.0, checkpoint="sqrt")
    yf = engine.replay(r, y0, p, write_ckpt=True)
    gy0, gp = engine.adjoint(r, p, ybar)
    return yf, gy0, gp


@pytest.mark.parametrize("cases", [(("lorenz_scale", "lorenz"), ("vdp_batch", "vdp")),
                                   (("lv_mixed", "lv"), ("lorenz_small", "lorenz"))])
def test_static_vjp_matches_allocating_path_twice(gslib, cuda, cases):
    from gradsolve_b200.fields import field_spec
    for case, field in cases:  # two calls in a row, different sizes and fields
        g = load_golden(case)
        spec = field_spec(field)
        y0 = torch.tensor(g["y0"], device=cuda)
        p = torch.tensor(g["params"][:, : spec.nparam], device=cuda).contiguous()
        dts = torch.tensor(g["dts"], device=cuda)
        ybar = torch.linspace(-1.0, 2.0, y0.numel(), dtype=torch.float64,
                              device=cuda).reshape(y0.shape)
        s_yf, s_gy0, s_gp = _static_call(gslib, spec.code, y0, p, dts, ybar)
        a_yf, a_gy0, a_gp = _allocating_call("tsit5", field, y0, p, dts, ybar)
        torch.cuda.synchronize()
        assert _rel(s_yf, a_yf) <= 1e-10
        assert _rel(s_gy0, a_gy0) <= 1e-9
        assert _rel(s_gp, a_gp) <= 1e-9


def test_static_vjp_refuses_sizes_beyond_its_scratch(gslib, cuda):
    n, S = 1 << 16, 4096  # a 2 GiB record: far beyond the 64 MiB scratch
    small = torch.zeros(8, dtype=torch.float64, device=cuda)
    rc = gslib.lib().gs_tsit5_vjp_static(1, n, small.data_ptr(), small.data_ptr(), 0.0,
                                         small.data_ptr(), S, S, small.data_ptr(),
                                         small.data_ptr(), None, None, None)
    assert rc == -1
    msg = gslib.lib().gs_last_error().decode()
    assert "static scratch holds" in msg and str(64 << 20) in msg


def test_static_scratch_size_is_declared(gslib):
    hdr = (__import__("conftest").ROOT / "include" / "gsolve.h").read_text()
    assert "#define GS_STATIC_SCRATCH_BYTES (64ull << 20)" in hdr
    assert ctypes.sizeof(ctypes.c_double) == 8
