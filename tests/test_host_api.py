"""Host-side API logic that needs no GPU: saveat validation, field routing, parameter
mapping, checkpoint policy."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from gradsolve_b200 import api
from gradsolve_b200.fields import field_for, field_spec, kernel_params


class P:
    def __init__(self, name):
        self.name = name


def test_validate_saveat_rules():
    ts = api.validate_saveat([0.0, 0.5, 0.5, 1.0], 0.0, 1.0)
    assert ts.dtype == np.float64 and ts.shape == (4,)
    with pytest.raises(ValueError, match="sorted"):
        api.validate_saveat([0.5, 0.1], 0.0, 1.0)
    with pytest.raises(ValueError, match="within the problem domain"):
        api.validate_saveat([0.0, 1.5], 0.0, 1.0)
    with pytest.raises(ValueError, match="non-finite"):
        api.validate_saveat([0.0, np.nan], 0.0, 1.0)
    with pytest.raises(ValueError, match="at least one"):
        api.validate_saveat([], 0.0, 1.0)
    # per-trajectory rows against per-trajectory end times
    rows = np.array([[0.0, 0.5], [0.0, 2.0]])
    api.validate_saveat(rows, 0.0, 2.0, t1v=np.array([1.0, 2.0]), n=2)
    with pytest.raises(ValueError, match="within the problem domain"):
        api.validate_saveat(rows, 0.0, 2.0, t1v=np.array([0.4, 2.0]), n=2)
    with pytest.raises(ValueError, match="rows"):
        api.validate_saveat(rows, 0.0, 2.0, n=3)


def test_field_routing_mirrors_reference_names():
    assert field_for(P("diffeqgpu_lorenz")).key == "lorenz"
    assert field_for(P("lorenz")).key == "lorenz3"
    assert field_for(P("vdp")).key == "vdp"
    assert field_for(P("lotka_volterra")).key == "lv"
    assert field_for(P("robertson")).stiff_ok
    assert field_for(P("linear_ladder_3")).dim == 3
    assert field_for(P("hires")).stiff_ok and field_for(P("hires")).dim == 8
    assert field_for(P("my_rhs")) is None
    # the families route for every dimension the reference routes (warp_ode.py:478-490):
    # in the core library at its built dimensions, else in a library built on first use
    s32, s5 = field_for(P("linear_ladder_32")), field_for(P("linear_ladder_5"))
    assert (s32.key, s32.dim, s32.lib, s32.family) == ("linear_32", 32, "", ())
    assert s5.dim == 5 and s5.family == ("linear", 5) and s5.lib.endswith(".so")
    l96 = field_for(P("lorenz96_40"))
    assert l96.code == 5040 and l96.family == ("lorenz96", 40) and not l96.stiff_ok
    assert field_for(P("lorenz96_32")).family == ()
    assert field_for(P("lorenz96_3")) is None  # D >= 4, as the reference requires
    assert field_for(P("linear_ladder_0")) is None and field_for(P("lorenz96_x")) is None
    # beyond the fused lanes' limit the name still routes, and use is refused before launch
    big = field_for(P("lorenz96_65"))
    assert big.dim == 65 and big.lib == ""
    with pytest.raises(RuntimeError, match="dim=65 > 64"):
        api._require_field(P("lorenz96_65"))


def test_group_size_rule():
    """Lanes per trajectory for a state of D components: 1 up to 8, then blocks of at most
    4 components where D allows, at least 2 (the stencil reaches two components into the
    next block), odd D on one thread -- the rule of coop_group in gs_fields.cuh, restated."""
    src = (Path(__file__).resolve().parent.parent / "gradsolve_b200" / "csrc" /
           "gs_fields.cuh").read_text()
    assert "constexpr int coop_group(int D)" in src

    def coop_group(D):
        if D <= 8:
            return 1
        best, g = 1, 2
        while g <= 32:
            if D % g == 0 and D // g >= 2:
                best = g
                if D // g <= 4:
                    return g
            g *= 2
        return best
    assert [coop_group(d) for d in (3, 8, 9, 10, 12, 16, 20, 32, 40, 64)] == \
        [1, 1, 1, 2, 4, 4, 4, 8, 8, 16]


def test_kernel_params_leading_columns_and_errors():
    spec = field_spec("lv")
    p = np.arange(10.0).reshape(2, 5)
    np.testing.assert_array_equal(kernel_params(spec, p), p[:, :4])
    with pytest.raises(ValueError, match="reads 4 parameter"):
        kernel_params(spec, p[:, :2])
    np.testing.assert_array_equal(kernel_params(field_spec("linear_2"), np.zeros((3, 0))),
                                  np.zeros((3, 1)))


def test_wrt_normalisation():
    assert api._normalize_wrt("params") == ("params",)
    assert api._normalize_wrt(["params", "y0"]) == ("y0", "params")
    with pytest.raises(ValueError, match="invalid wrt"):
        api._normalize_wrt("p")


def test_engine_resolution_and_aliases():
    reasons = []

    class S:
        name = "robertson"
        is_stiff = True

    assert api._resolve(S(), "auto", reasons) == "b200_rosenbrock23"
    assert api._resolve(S(), "warp_rosenbrock", reasons) == "b200_rosenbrock23"
    assert reasons == ["served-by-b200_rosenbrock23"]
    with pytest.raises(ValueError, match="unknown engine"):
        api._resolve(S(), "diffrax", [])


def test_float32_route_refusals():
    """precision="float32" is refused, before anything runs, where it has no float32 kernels:
    reference lanes without an f32 route (tests/test_f32_replay.py:171-192) and fields above 8
    components; an unknown precision names the known ones."""
    class Lz:
        name = "diffeqgpu_lorenz"
        dim = 3
        t0 = 0.0
        t1 = 1.0
        is_stiff = False

    class L96(Lz):
        name = "lorenz96_32"
        dim = 32

    y0, p = np.ones((4, 3)), np.full((4, 1), 28.0)
    with pytest.raises(ValueError, match="float32"):
        api.grad_closure(Lz(), y0, p, engine="tsit5_replay", precision="float32")
    with pytest.raises(ValueError, match="precision"):
        api.grad_closure(Lz(), y0, p, engine="warp_replay", precision="float16")
    with pytest.raises(ValueError, match="at most 8 components"):
        api.grad_closure(L96(), np.ones((4, 32)), np.full((4, 1), 8.0), precision="float32")
    with pytest.raises(ValueError, match="precision"):
        api.record(Lz(), y0, p, precision="mixed")


def test_checkpoint_policy(gslib):
    from gradsolve_b200.engine import choose_ckpt_every
    assert choose_ckpt_every("all", 3, 10, 700, None) == 1
    assert choose_ckpt_every("sqrt", 3, 10, 700, None) == 27
    assert choose_ckpt_every(5, 3, 10, 700, None) == 5
    # auto: the tuned segment length (8 before tuning), raised until the checkpoints fit
    assert choose_ckpt_every("auto", 3, 10, 700, budget_bytes=10**9) == 8
    assert choose_ckpt_every("auto", 3, 10, 700, budget_bytes=10**9, tuned=12) == 12
    assert choose_ckpt_every("auto", 3, 1 << 20, 700, budget_bytes=10**9) == 32
    with pytest.raises(ValueError):
        choose_ckpt_every(65, 3, 10, 700, None)


def test_record_row_gather_follows_the_chunked_layout():
    """Record.dts_rows reads step s of trajectory j at ((s//4)*n + j)*4 + s%4 and zero-pads
    past n_acc (the reference's padded layout, for a subset of rows)."""
    import torch

    from gradsolve_b200.engine import Record
    n, cap = 5, 9
    n_acc = np.array([0, 3, 9, 4, 7], np.int32)
    rec = np.full(((cap + 3) // 4) * n * 4, -1.0)
    for j in range(n):
        for s in range(n_acc[j]):
            rec[((s // 4) * n + j) * 4 + s % 4] = 100 * j + s + 1
    z = torch.zeros(n, dtype=torch.int32)
    r = Record("tsit5", field_spec("lorenz"), n, 0.0, cap, 1, torch.tensor(rec),
               torch.zeros(1), torch.zeros(n, 3, dtype=torch.float64),
               torch.tensor(n_acc), z, z)
    rows = torch.tensor([4, 0, 2])
    got = r.dts_rows(rows).numpy()
    assert got.shape == (3, 9)
    for k, j in enumerate([4, 0, 2]):
        want = np.zeros(9)
        want[: n_acc[j]] = 100 * j + np.arange(n_acc[j]) + 1
        np.testing.assert_array_equal(got[k], want)
    assert r.dts_rows(rows, S=12).shape == (3, 12)


def test_occupancy_flags_and_choice_rule():
    """Which calls carry GS_OCC, and the autotuner's keep-the-default margin (host logic; the
    instances themselves are checked bit for bit on the GPU)."""
    import re

    import torch

    from gradsolve_b200 import engine
    hdr = (Path(__file__).resolve().parents[1] / "include" / "gsolve.h").read_text()
    val = {m.group(1): int(m.group(2), 0)
           for m in re.finditer(r"#define (GS_\w+_MASK) (0x[0-9A-Fa-f]+)", hdr)}
    assert val["GS_OCC_MASK"] == 0x78000
    # the occupancy bits overlap no other flag field; the engine shifts by the header's shift
    for k, v in val.items():
        if k != "GS_OCC_MASK":
            assert v & val["GS_OCC_MASK"] == 0, k
    assert int(re.search(r"#define GS_OCC_SHIFT (\d+)", hdr).group(1)) == 15
    spec = field_spec("lorenz")
    saved = dict(engine._OCC), dict(engine._OCC_REV)
    try:
        engine._OCC[("tsit5", spec.key)] = 5
        engine._OCC_REV[("tsit5", spec.key)] = 4
        f = engine._occ_flag
        assert f("tsit5", spec, "float64", "auto", None, None) == 5 << 15
        assert f("tsit5", spec, "float64", "static", torch.zeros(1), None) == 5 << 15
        assert f("tsit5", spec, "float64", "auto", torch.zeros(1), None) == 0   # refilled
        assert f("tsit5", spec, "mixed", "auto", None, None) == 0
        assert f("tsit5", spec, "float32", "auto", None, None) == 0
        assert f("tsit5", spec, "float64", "auto", None, torch.zeros(2)) == 0   # saveat
        assert f("tsit5", spec, "float64", "refill", None, None) == 0
        assert f("rosenbrock23", spec, "float64", "auto", None, None) == 0    # not tuned

        class R:
            method, ckpt_every = "tsit5", 2
        R.spec = spec
        g = engine._occ_rev_flag
        assert g(R, "float64", "auto", "auto") == 4 << 15
        assert g(R, "float64", "static", "stages") == 4 << 15
        assert g(R, "float64", "auto", "recompute") == 0
        assert g(R, "float64", "refill", "auto") == 0
        assert g(R, "mixed", "auto", "auto") == 0
        R.ckpt_every = 3
        assert g(R, "float64", "auto", "auto") == 0
    finally:
        engine._OCC.clear()
        engine._OCC.update(saved[0])
        engine._OCC_REV.clear()
        engine._OCC_REV.update(saved[1])
    # another instance replaces the default only when faster by more than the margin
    m = engine.OCC_MARGIN
    assert engine._pick({0: 10.0, 5: 10.0 * (1 - m / 2)}) == 0
    assert engine._pick({0: 10.0, 5: 10.0 * (1 - 2 * m), 7: 10.5}) == 5
    assert engine._pick({0: 10.0, 4: 11.0}) == 0


def test_replay_graph_refuses_record_sets():
    from gradsolve_b200 import engine
    with pytest.raises(TypeError, match="single Record"):
        engine.ReplayGraph(object(), None, None, lambda yf: yf)
