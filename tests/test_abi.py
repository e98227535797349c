"""The C ABI (include/gsolve.h, libgsolve.so) without a GPU: the library loads, exports every
declared symbol, its host constants equal the reference's, size helpers are consistent,
and argument errors come back as status codes before anything is launched."""
from __future__ import annotations

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden

HEADER = ROOT / "include" / "gsolve.h"


def _declared_functions():
    src = HEADER.read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gs_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported(gslib):
    L = gslib.lib()
    names = _declared_functions()
    assert len(names) >= 15
    for nm in names:
        assert hasattr(L, nm), f"libgsolve.so does not export {nm}"
    # and the Python binding covers exactly the declared set
    assert sorted(gslib.exported_symbols()) == names


def test_host_tableau_equals_reference(gslib):
    tab = load_golden("tableau")
    out = (ctypes.c_double * 41)()
    assert gslib.lib().gs_tableau(out, 41) == 0
    v = np.array(out[:])
    ref = np.concatenate([
        tab["C"][:4],
        [tab[k] for k in ("A21", "A31", "A32", "A41", "A42", "A43", "A51", "A52", "A53", "A54",
                          "A61", "A62", "A63", "A64", "A65")],
        [tab[f"B{i}"] for i in range(1, 8)],
        [tab[f"E{i}"] for i in range(1, 8)],
        tab["controller"],
        tab["ros"][[0, 1, 6]],
    ])
    np.testing.assert_array_equal(v, ref)


def test_field_dims(gslib):
    L = gslib.lib()
    D, P = ctypes.c_int(), ctypes.c_int()
    expect = {1: (3, 1), 2: (2, 1), 3: (2, 4), 10: (3, 3), 11: (3, 3), 4001: (1, 1),
              4003: (3, 1), 4008: (8, 1)}
    for code, dp in expect.items():
        assert L.gs_field_dims(code, ctypes.byref(D), ctypes.byref(P)) == 0
        assert (D.value, P.value) == dp
    assert L.gs_field_dims(999, ctypes.byref(D), ctypes.byref(P)) == -2
    assert b"unknown field" in L.gs_last_error()


def test_workspace_sizes(gslib):
    L = gslib.lib()
    assert L.gs_record_bytes(10, 5) == 2 * 10 * 4 * 8
    assert L.gs_record_bytes(0, 5) == 0
    assert L.gs_ckpt_slots(100, 10) == 11
    assert L.gs_ckpt_slots(101, 10) == 12
    ctrl = 256  # control block of the persistent kernels after the slots
    assert L.gs_ckpt_bytes(1, 7, 100, 10) == 11 * 7 * 4 * 8 + ctrl     # lorenz: CW = 4
    assert L.gs_ckpt_bytes(2, 7, 100, 1) == 101 * 7 * 4 * 8 + ctrl     # vdp: CW = 4
    assert L.gs_ckpt_bytes(4008, 7, 100, 1) == 101 * 7 * 10 * 8 + ctrl  # linear_8: CW = 10
    assert L.gs_max_ckpt_every() == 64
    # the float32 route: 4-byte steps (exactly half the record) and 16-byte checkpoint rows
    F32 = gslib.GS_PREC_F32
    for n, cap in ((10, 5), (3, 1), (1000, 4099)):
        assert 2 * L.gs_record_bytes_prec(F32, n, cap) == L.gs_record_bytes(n, cap)
        assert L.gs_record_bytes_prec(0, n, cap) == L.gs_record_bytes(n, cap)
    assert L.gs_ckpt_bytes_prec(1, F32, 7, 100, 10) == 11 * 7 * 4 * 4 + ctrl     # lorenz: 4
    assert L.gs_ckpt_bytes_prec(4008, F32, 7, 100, 1) == 101 * 7 * 12 * 4 + ctrl  # linear_8: 12
    assert L.gs_ckpt_bytes_prec(4008, 0, 7, 100, 1) == L.gs_ckpt_bytes(4008, 7, 100, 1)


def test_argument_errors_are_status_codes(gslib):
    """Invalid calls fail on the host with GS_ERR_* and a message; nothing is launched."""
    L = gslib.lib()
    buf = (ctypes.c_double * 64)()
    ibuf = (ctypes.c_int * 64)()
    a = ctypes.addressof(buf)
    ia = ctypes.addressof(ibuf)
    # null y0
    rc = L.gs_tsit5_fwd_record(1, 0, 4, None, a, 0.0, None, 1.0, 1e-6, 1e-9, -1.0, 10, 8, 2,
                               a, a, a, ia, ia, ia, None)
    assert rc == -1 and b"required" in L.gs_last_error()
    # negative n
    rc = L.gs_tsit5_fwd_record(1, 0, -1, a, a, 0.0, None, 1.0, 1e-6, 1e-9, -1.0, 10, 8, 2,
                               a, a, a, ia, ia, ia, None)
    assert rc == -1
    # checkpoint interval out of range
    rc = L.gs_tsit5_fwd_record(1, 0, 4, a, a, 0.0, None, 1.0, 1e-6, 1e-9, -1.0, 10, 8, 65,
                               a, a, a, ia, ia, ia, None)
    assert rc == -1 and b"ckpt_every" in L.gs_last_error()
    # misaligned record
    rc = L.gs_tsit5_fwd_record(1, 0, 4, a, a, 0.0, None, 1.0, 1e-6, 1e-9, -1.0, 10, 8, 2,
                               a + 8, a, a, ia, ia, ia, None)
    assert rc == -1 and b"aligned" in L.gs_last_error()
    # unknown field
    rc = L.gs_tsit5_fwd_record(77, 0, 4, a, a, 0.0, None, 1.0, 1e-6, 1e-9, -1.0, 10, 8, 2,
                               a, a, a, ia, ia, ia, None)
    assert rc == -2
    # stiff engine on a field without Jacobian
    rc = L.gs_ros23_fwd_record(1, 0, 4, a, a, 0.0, None, 1.0, 1e-6, 1e-9, -1.0, 10, 8, 2,
                               a, a, a, ia, ia, ia, None)
    assert rc == -2 and b"Jacobian" in L.gs_last_error()
    # precision not built
    rc = L.gs_tsit5_adjoint(1, 7, 4, a, a, ia, 8, a, 2, a, a, a, None)
    assert rc == -4
    # the float32 route: one thread per trajectory only, no lanes, and of the reverse-pass
    # variants only the Tsit5 ones (pairs, one per thread), Rosenbrock23 included; fields
    # above 8 components refused
    rc = L.gs_tsit5_fwd_record(1, 2 | 0x200, 4, a, a, 0.0, None, 1.0, 1e-6, 1e-9, -1.0, 10, 8,
                               2, a, a, a, ia, ia, ia, None)
    assert rc == -1 and b"one thread per trajectory" in L.gs_last_error()
    rc = L.gs_tsit5_adjoint(1, 2 | 0x800, 4, a, a, ia, 8, a, 2, a, a, a, None)
    assert rc == -1 and b"not float32-route options" in L.gs_last_error()
    rc = L.gs_ros23_adjoint(10, 2 | 0xC00, 4, a, a, ia, 8, a, 2, a, a, a, None)
    assert rc == -1 and b"not float32-route options" in L.gs_last_error()
    rc = L.gs_ros23_adjoint(10, 2 | 0x300, 4, a, a, ia, 8, a, 2, a, a, a, None)
    assert rc == -1
    rc = L.gs_tsit5_replay(5032, 2 | 0x1000, 4, a, a, 0.0, a, ia, 8, 2, a, a, None)
    assert rc == -4
    # empty ensemble is a no-op success
    rc = L.gs_tsit5_fwd_record(1, 0, 0, a, a, 0.0, None, 1.0, 1e-6, 1e-9, -1.0, 10, 8, 2,
                               a, a, a, ia, ia, ia, None)
    assert rc == 0
    # padded-record conversion: S larger than the capacity
    rc = L.gs_record_from_padded(4, 9, a, 9, a, 8, ia, None)
    assert rc == -1


def test_lane_choices_per_field(gslib):
    """Host-only query: the group sizes built per field, the default first (the rule of
    coop_group and group_built in gs_fields.cuh): one thread for D <= 8, 8 / 4 / 16 lanes for
    D = 32, 2 lanes alone for D = 10 (5 components; neither 1 nor 4 lanes divide it well)."""
    import ctypes
    L = gslib.lib()
    buf = (ctypes.c_int * 8)()
    for code, want in ((1, [1]), (5008, [1]), (5032, [8, 4, 16]), (4032, [8, 4, 16]),
                       (4010, [2]), (12, [1])):
        k = L.gs_lane_choices(code, buf, 8)
        assert list(buf[:k]) == want, code
    assert L.gs_lane_choices(999, buf, 8) < 0
