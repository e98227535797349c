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


def _static_call(gslib, code, y0, p, dts, ybar, *, want_y0=True, want_p=True):
    n, S = dts.shape
    yf = torch.empty_like(y0)
    gy0 = torch.empty_like(y0) if want_y0 else None
    gp = torch.empty_like(p) if want_p else None
    rc = gslib.lib().gs_tsit5_vjp_static(code, n, y0.data_ptr(), p.data_ptr(), 0.0,
                                         dts.data_ptr(), S, S, ybar.data_ptr(), yf.data_ptr(),
                                         None if gy0 is None else gy0.data_ptr(),
                                         None if gp is None else gp.data_ptr(),
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


@pytest.mark.parametrize("want", [(False, True), (True, False)])
def test_static_vjp_with_one_gradient_left_out(gslib, cuda, want):
    """gy0 or gp may be NULL: the other output is still the allocating path's."""
    from gradsolve_b200.fields import field_spec
    g = load_golden("lorenz_scale")
    spec = field_spec("lorenz")
    y0 = torch.tensor(g["y0"], device=cuda)
    p = torch.tensor(g["params"][:, :1], device=cuda).contiguous()
    dts = torch.tensor(g["dts"], device=cuda)
    ybar = 2.0 * torch.ones_like(y0)
    s_yf, s_gy0, s_gp = _static_call(gslib, spec.code, y0, p, dts, ybar, want_y0=want[0],
                                     want_p=want[1])
    a_yf, a_gy0, a_gp = _allocating_call("tsit5", "lorenz", y0, p, dts, ybar)
    torch.cuda.synchronize()
    assert _rel(s_yf, a_yf) <= 1e-10
    if want[0]:
        assert s_gp is None and _rel(s_gy0, a_gy0) <= 1e-9
    else:
        assert s_gy0 is None and _rel(s_gp, a_gp) <= 1e-9


@pytest.mark.parametrize("n", [48, 1024])
def test_static_vjp_long_record_intervals(gslib, cuda, n):
    """Records of more than 4096 steps.  At n = 48 the checkpoints fit the scratch at the
    shortest interval, K = 2 (the unrolled stage-keeping reverse pass); at n = 1024 they do
    not, and the entry point lengthens the segments until they fit (checked here with the
    library's own size functions), the shared-memory sizing of the longer segments included.
    Twice in a row, the second call with another cotangent."""
    from gradsolve_b200 import engine
    from gradsolve_b200.fields import field_spec
    spec = field_spec("lorenz")
    rng = np.random.default_rng(7)
    y0 = torch.tensor(np.array([1.0, 0.0, 0.0]) + rng.normal(0.0, 0.1, (n, 3)), device=cuda)
    p = torch.tensor(rng.uniform(20.0, 30.0, (n, 1)), device=cuda)
    r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=70.0, rtol=1e-8, atol=1e-8,
                              max_steps=100000)
    dts = r.padded_dts().contiguous()
    S = dts.shape[1]
    assert S >= 4096
    L = gslib.lib()

    def need(K):
        return L.gs_record_bytes(n, S) + L.gs_ckpt_bytes(spec.code, n, S, K)
    if n == 48:
        assert need(2) < (64 << 20)
    else:
        assert need(2) > (64 << 20) and need(64) < (64 << 20)
    for scale in (1.0, -3.0):
        ybar = scale * torch.linspace(-1.0, 2.0, y0.numel(), dtype=torch.float64,
                                      device=cuda).reshape(y0.shape)
        s_yf, s_gy0, s_gp = _static_call(gslib, spec.code, y0, p, dts, ybar)
        a_yf, a_gy0, a_gp = _allocating_call("tsit5", "lorenz", y0, p, dts, ybar)
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
    # sizes whose byte counts would overflow 64-bit products are refused before any is formed
    for n, S in ((1 << 62, 1), (1, 1 << 62), (1 << 40, 1 << 30)):
        rc = gslib.lib().gs_tsit5_vjp_static(1, n, small.data_ptr(), small.data_ptr(), 0.0,
                                             small.data_ptr(), S, S, small.data_ptr(),
                                             small.data_ptr(), None, None, None)
        assert rc == -1 and "does not fit" in gslib.lib().gs_last_error().decode()


def test_generated_field_libraries_carry_no_static_scratch():
    """Only libgsolve.so holds the 64 MiB array; a generated field's library (gs_abi.cu built
    with GS_USER_FIELD_HEADER) compiles the array out and refuses the entry point."""
    src = (__import__("conftest").ROOT / "gradsolve_b200" / "csrc" / "gs_abi.cu").read_text()
    decl = src.index("g_vjp_scratch[GS_STATIC_SCRATCH_BYTES]")
    guard = src.rfind("#ifndef GS_USER_FIELD_HEADER", 0, decl)
    assert guard >= 0 and src.find("#endif", guard, decl) < 0


def test_static_scratch_size_is_declared(gslib):
    hdr = (__import__("conftest").ROOT / "include" / "gsolve.h").read_text()
    assert "#define GS_STATIC_SCRATCH_BYTES (64ull << 20)" in hdr
    assert ctypes.sizeof(ctypes.c_double) == 8
