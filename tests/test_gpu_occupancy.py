"""Registers and occupancy of the float64 Tsit5 recording forward: the GS_OCC instances,
gs_occ_choices and the autotuner that picks one per field (engine.autotune_occupancy),
through the C ABI.

The instances differ only in the register bound the compiler is given (resident blocks of
128 threads per SM), so each must reproduce the default instance's record, final states,
counts and statuses bit for bit, and the gradients taken from its checkpoints too; on the
reference's golden batches the counts are also those of the reference's own tsit5_adaptive
(gradsolve/solvers/tsit5_replay.py:62-124).  Instances the library does not build, and the
flag on the paths it does not apply to, are refused.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu

CASES = [("lorenz_scale", "lorenz"), ("vdp_batch", "vdp"), ("lv_mixed", "lv"),
         ("linear3", "linear_3")]
GS_OCC_SHIFT = 15


def _spec(field):
    from gradsolve_b200.fields import field_spec
    return field_spec(field)


def _inputs(cuda, spec, g):
    y0 = torch.tensor(g["y0"], device=cuda)
    p = torch.tensor(g["params"][:, : spec.nparam], device=cuda).contiguous()
    return y0, p


def _solve(engine, spec, y0, p, g):
    r = engine.forward_record("tsit5", spec, y0, p, t0=float(g["t0"]), t1=float(g["t1"]),
                              rtol=float(g["rtol"]), atol=float(g["atol"]), checkpoint=2)
    gy0, gp = engine.adjoint(r, p, 2.0 * r.y_final)
    torch.cuda.synchronize()
    return [r.padded_dts().cpu(), r.y_final.cpu(), r.n_acc.cpu(), r.n_rej.cpu(),
            r.status.cpu(), gy0.cpu(), gp.cpu()]


@pytest.mark.parametrize("case,field", CASES)
def test_occupancy_instances_bitwise(gslib, cuda, case, field):
    from gradsolve_b200 import engine
    g = load_golden(case)
    spec = _spec(field)
    y0, p = _inputs(cuda, spec, g)
    fwd, rev = engine.occ_choices(spec, "forward"), engine.occ_choices(spec, "reverse")
    assert fwd == [0, 4, 5, 7, 8] and rev == [0, 3, 4, 6]
    saved = dict(engine._OCC), dict(engine._OCC_REV)
    outs = {}
    try:
        for pass_, choices in (("forward", fwd), ("reverse", rev)):
            for b in choices[1:] if pass_ == "reverse" else choices:
                engine.set_occupancy(spec, 0, "forward")
                engine.set_occupancy(spec, 0, "reverse")
                engine.set_occupancy(spec, b, pass_)
                outs[(pass_, b)] = _solve(engine, spec, y0, p, g)
    finally:
        _restore(engine, saved)
    base = outs[("forward", 0)]
    np.testing.assert_array_equal(base[2].numpy(), g["n_acc"])
    np.testing.assert_array_equal(base[3].numpy(), g["n_rej"])
    for key, out in outs.items():
        for x, y in zip(base, out):
            assert torch.equal(x, y), f"{key} differs from the default instances"


def _restore(engine, saved):
    engine._OCC.clear()
    engine._OCC.update(saved[0])
    engine._OCC_REV.clear()
    engine._OCC_REV.update(saved[1])


def test_occupancy_refusals(gslib, cuda):
    from gradsolve_b200 import _lib, engine
    from gradsolve_b200._lib import GsolveError
    g = load_golden("lorenz_small")
    spec = _spec("lorenz")
    y0, p = _inputs(cuda, spec, g)
    saved = dict(engine._OCC), dict(engine._OCC_REV)
    try:
        with pytest.raises(ValueError, match=r"3 blocks per SM .* built: \[0, 4, 5, 7, 8\]"):
            engine.set_occupancy(spec, 3)
        with pytest.raises(ValueError, match=r"reverse instance for 5 blocks .* \[0, 3, 4, 6\]"):
            engine.set_occupancy(spec, 5, "reverse")
        engine._OCC[("tsit5", spec.key)] = 3  # bypass the check: the library itself refuses
        with pytest.raises(GsolveError, match="GS_OCC"):
            engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=0.5, rtol=1e-6, atol=1e-6,
                                  checkpoint=2)
        engine._OCC[("tsit5", spec.key)] = 0
        engine._OCC_REV[("tsit5", spec.key)] = 7
        r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=0.5, rtol=1e-6, atol=1e-6,
                                  checkpoint=2)
        with pytest.raises(GsolveError, match="GS_OCC"):
            engine.adjoint(r, p, torch.ones_like(r.y_final))
        engine._OCC_REV[("tsit5", spec.key)] = 4  # applies at K = 2 only: other intervals ignore it
        r = engine.forward_record("tsit5", spec, y0, p, t0=0.0, t1=0.5, rtol=1e-6, atol=1e-6,
                                  checkpoint=3)
        engine.adjoint(r, p, torch.ones_like(r.y_final))
    finally:
        _restore(engine, saved)
    # fields above 4 components keep the compiler's allocation alone
    assert engine.occ_choices(_spec("lorenz96_8")) == [0]
    assert engine.occ_choices(_spec("lorenz96_8"), "reverse") == [0]
    # the flag on the paths it does not apply to: float32 stages, the float32 route, the
    # forward without a record, the refilled-lane schedule
    L = _lib.lib()
    n = y0.shape[0]
    cap, K = 4096, 2
    rec, ckpt = engine._alloc_record(n, cap, 3, K, y0.device, "float64")
    yf = torch.empty_like(y0)
    ints = [torch.empty(n, dtype=torch.int32, device=y0.device) for _ in range(3)]

    def call(mode, with_record=True):
        return L.gs_tsit5_fwd_record(
            spec.code, mode, n, y0.data_ptr(), p.data_ptr(), 0.0, None, 0.5, 1e-6, 1e-6,
            -1.0, 100000, cap, K, rec.data_ptr() if with_record else None,
            ckpt.data_ptr() if with_record else None, yf.data_ptr(),
            *(t.data_ptr() for t in ints), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))

    occ7 = 7 << GS_OCC_SHIFT
    assert call(occ7) == 0
    torch.cuda.synchronize()
    for mode, rec_on in ((1 | occ7, True), (2 | occ7, True), (occ7, False),
                         (0x200 | occ7, True)):
        assert call(mode, rec_on) == -1, hex(mode)


def test_occupancy_autotuner(gslib, cuda):
    """The autotuner keeps one of the built instances, runs on the first recording forward of
    a large enough batch, and what it keeps computes the default's values bit for bit."""
    from gradsolve_b200 import engine
    spec = _spec("lorenz")
    rng = np.random.default_rng(7)
    n = 8192
    y0 = torch.tensor(np.array([1.0, 0.0, 0.0]) + rng.normal(0, 0.1, (n, 3)), device=cuda)
    p = torch.tensor(rng.uniform(20, 30, (n, 1)), device=cuda)
    kw = dict(t0=0.0, t1=1.0, rtol=1e-8, atol=1e-8, checkpoint=2)
    saved = dict(engine._OCC), dict(engine._OCC_REV)
    try:
        engine._OCC.pop(("tsit5", spec.key), None)
        engine._OCC_REV.pop(("tsit5", spec.key), None)
        r = engine.forward_record("tsit5", spec, y0, p, **kw)
        assert engine._OCC.get(("tsit5", spec.key)) in engine.occ_choices(spec, "forward")
        assert engine._OCC_REV.get(("tsit5", spec.key)) in engine.occ_choices(spec, "reverse")
        f, b = engine.autotune_occupancy(spec, y0, p, t0=0.0, t1=1.0, rtol=1e-8, atol=1e-8,
                                         checkpoint=2)
        assert f in engine.occ_choices(spec, "forward")
        assert b in engine.occ_choices(spec, "reverse")
        ybar = torch.ones_like(r.y_final)
        tuned = [r.padded_dts().cpu(), r.y_final.cpu(), r.n_acc.cpu(),
                 *(x.cpu() for x in engine.adjoint(r, p, ybar))]
        engine.set_occupancy(spec, 0, "forward")
        engine.set_occupancy(spec, 0, "reverse")
        r0 = engine.forward_record("tsit5", spec, y0, p, **kw)
        plain = [r0.padded_dts().cpu(), r0.y_final.cpu(), r0.n_acc.cpu(),
                 *(x.cpu() for x in engine.adjoint(r0, p, ybar))]
        for x, y in zip(tuned, plain):
            assert torch.equal(x, y)
    finally:
        _restore(engine, saved)


@pytest.mark.parametrize("case", ["robertson_toy", "robertson_stiff"])
def test_ros23_occupancy_instances_bitwise(gslib, cuda, case):
    """Rosenbrock23: the forward's and the K = 2 reverse pass's instances against the
    defaults, bit for bit; counts those of the reference's Rosenbrock23 oracle."""
    from gradsolve_b200 import engine
    g = load_golden(case)
    spec = _spec("robertson")
    y0 = torch.tensor(g["y0"], device=cuda)
    p = torch.tensor(g["params"], device=cuda)
    fwd = engine.occ_choices(spec, "forward", "rosenbrock23")
    rev = engine.occ_choices(spec, "reverse", "rosenbrock23")
    assert fwd == [0, 4, 6] and rev == [0, 3, 5]
    saved = dict(engine._OCC), dict(engine._OCC_REV)

    def solve():
        r = engine.forward_record("rosenbrock23", spec, y0, p, t0=float(g["t0"]),
                                  t1=float(g["t1"]), rtol=float(g["rtol"]),
                                  atol=float(g["atol"]), max_steps=50000, checkpoint=2)
        gy0, gp = engine.adjoint(r, p, torch.ones_like(r.y_final))
        torch.cuda.synchronize()
        return [r.padded_dts().cpu(), r.y_final.cpu(), r.n_acc.cpu(), r.n_rej.cpu(),
                r.status.cpu(), gy0.cpu(), gp.cpu()]

    outs = {}
    try:
        for pass_, choices in (("forward", fwd), ("reverse", rev[1:])):
            for b in choices:
                engine.set_occupancy(spec, 0, "forward", "rosenbrock23")
                engine.set_occupancy(spec, 0, "reverse", "rosenbrock23")
                engine.set_occupancy(spec, b, pass_, "rosenbrock23")
                outs[(pass_, b)] = solve()
        engine._OCC_REV[("rosenbrock23", spec.key)] = 4  # not built: the library refuses
        with pytest.raises(Exception, match="GS_OCC"):
            solve()
    finally:
        _restore(engine, saved)
    base = outs[("forward", 0)]
    np.testing.assert_array_equal(base[2].numpy(), g["n_acc"])
    np.testing.assert_array_equal(base[3].numpy(), g["n_rej"])
    for key, out in outs.items():
        for x, y in zip(base, out):
            assert torch.equal(x, y), f"{key} differs from the default instances"


def test_mixed_reverse_occupancy_bitwise(gslib, cuda):
    """The float32-stage reverse pass's K = 2 instances against its default, bit for bit."""
    from gradsolve_b200 import engine
    g = load_golden("lorenz_scale")
    spec = _spec("lorenz")
    y0, p = _inputs(cuda, spec, g)
    rev = engine.occ_choices(spec, "reverse", engine.MIXED)
    assert rev == [0, 4, 5]
    saved = dict(engine._OCC), dict(engine._OCC_REV)
    try:
        r = engine.forward_record("tsit5", spec, y0, p, t0=float(g["t0"]), t1=float(g["t1"]),
                                  rtol=float(g["rtol"]), atol=float(g["atol"]), checkpoint=2,
                                  precision="mixed")
        ybar = 2.0 * r.y_final
        outs = {}
        for b in rev:
            engine.set_occupancy(spec, b, "reverse", engine.MIXED)
            outs[b] = [t.cpu() for t in engine.adjoint(r, p, ybar, precision="mixed")]
        engine._OCC_REV[(engine.MIXED, spec.key)] = 6  # not built: the library refuses
        with pytest.raises(Exception, match="GS_OCC"):
            engine.adjoint(r, p, ybar, precision="mixed")
    finally:
        _restore(engine, saved)
    for b in rev[1:]:
        for x, y in zip(outs[0], outs[b]):
            assert torch.equal(x, y), f"instance {b} differs from the default"
