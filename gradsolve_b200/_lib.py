"""ctypes binding of libgsolve.so (the C ABI declared in include/gsolve.h).

The library must have been built in-tree (``gradsolve_b200/csrc/build.py``); there is no
fallback path: every solve and gradient goes through these entry points, and a missing or
unloadable library raises immediately.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libgsolve.so"

GS_OK = 0
GS_PREC_F64 = 0
GS_PREC_MIXED = 1
GS_PREC_F32 = 2

c_int, c_ll, c_double, c_size_t, c_void_p = (ctypes.c_int, ctypes.c_longlong, ctypes.c_double,
                                             ctypes.c_size_t, ctypes.c_void_p)

# name -> (restype, argtypes).  Pointers to device memory travel as c_void_p integers.
_SIGS = {
    "gs_version": (c_int, []),
    "gs_launch_count": (ctypes.c_ulonglong, []),
    "gs_last_error": (ctypes.c_char_p, []),
    "gs_field_dims": (c_int, [c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
    "gs_tableau": (c_int, [ctypes.POINTER(c_double), c_int]),
    "gs_device_tableau": (c_int, [c_void_p, c_void_p]),
    "gs_record_bytes": (c_size_t, [c_ll, c_int]),
    "gs_ckpt_slots": (c_int, [c_int, c_int]),
    "gs_ckpt_bytes": (c_size_t, [c_int, c_ll, c_int, c_int]),
    "gs_record_bytes_prec": (c_size_t, [c_int, c_ll, c_int]),
    "gs_move_rows": (c_int, [c_int, c_int, c_void_p, c_void_p, c_ll, c_int, c_ll, c_void_p,
                             c_void_p, c_void_p]),
    "gs_adjoint_ordered": (c_int, [c_int, c_int, c_int, c_ll, c_void_p, c_void_p, c_void_p,
                                   c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                   c_void_p, c_void_p]),
    "gs_ckpt_bytes_prec": (c_size_t, [c_int, c_int, c_ll, c_int, c_int]),
    "gs_max_ckpt_every": (c_int, []),
    "gs_lane_choices": (c_int, [c_int, ctypes.POINTER(c_int), c_int]),
    "gs_occ_choices": (c_int, [c_int, c_int, ctypes.POINTER(c_int), c_int]),
    "gs_tsit5_fwd_record": (c_int, [c_int, c_int, c_ll, c_void_p, c_void_p, c_double, c_void_p,
                                    c_double, c_double, c_double, c_double, c_int, c_int, c_int,
                                    c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p]),
    "gs_tsit5_replay": (c_int, [c_int, c_int, c_ll, c_void_p, c_void_p, c_double, c_void_p,
                                c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "gs_tsit5_adjoint": (c_int, [c_int, c_int, c_ll, c_void_p, c_void_p, c_void_p, c_int,
                                 c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "gs_ros23_fwd_record": (c_int, [c_int, c_int, c_ll, c_void_p, c_void_p, c_double, c_void_p,
                                    c_double, c_double, c_double, c_double, c_int, c_int, c_int,
                                    c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p]),
    "gs_ros23_replay": (c_int, [c_int, c_int, c_ll, c_void_p, c_void_p, c_double, c_void_p,
                                c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "gs_ros23_adjoint": (c_int, [c_int, c_int, c_ll, c_void_p, c_void_p, c_void_p, c_int,
                                 c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "gs_record_from_padded": (c_int, [c_ll, c_ll, c_void_p, c_ll, c_void_p, c_int, c_void_p,
                                      c_void_p]),
    "gs_record_to_padded": (c_int, [c_ll, c_int, c_void_p, c_void_p, c_ll, c_void_p, c_void_p]),
    "gs_replay_saveat": (c_int, [c_int, c_int, c_int, c_ll, c_void_p, c_void_p, c_double,
                                 c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, c_ll,
                                 c_int, c_void_p, c_void_p, c_void_p]),
    "gs_fwd_record_saveat": (c_int, [c_int, c_int, c_int, c_ll, c_void_p, c_void_p, c_double,
                                     c_void_p, c_double, c_double, c_double, c_double, c_int,
                                     c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p, c_ll, c_int, c_void_p,
                                     c_void_p]),
    "gs_adjoint_saveat": (c_int, [c_int, c_int, c_int, c_ll, c_void_p, c_void_p, c_void_p,
                                  c_int, c_void_p, c_int, c_void_p, c_ll, c_int, c_void_p,
                                  c_void_p, c_void_p, c_void_p, c_void_p]),
    "gs_tsit5_vjp_static": (c_int, [c_int, c_ll, c_void_p, c_void_p, c_double, c_void_p, c_ll,
                                    c_ll, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
}

_LIB = None


class GsolveError(RuntimeError):
    """A libgsolve call returned a non-zero status."""


_FIELD_LIBS: dict = {}


def _load(path) -> ctypes.CDLL:
    L = ctypes.CDLL(str(path))
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def lib():
    """Load libgsolve.so (once).  Raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m gradsolve_b200.csrc.build` "
                "(gradsolve_b200 has no CPU fallback).")
        _LIB = _load(LIB_PATH)
    return _LIB


def lib_for(spec):
    """The library that serves a field: libgsolve.so, or a generated field's own library
    (same C ABI, built by gradsolve_b200.fieldgen; a built-in family member at a dimension
    the core library does not carry is compiled here on first use).  Fields beyond the fused
    lanes' dimension limit are refused before any launch."""
    from .fields import MAX_DIM, dim_limit_message
    if spec.dim > MAX_DIM:
        raise RuntimeError(dim_limit_message(spec.dim))
    path = getattr(spec, "lib", "")
    if not path:
        return lib()
    L = _FIELD_LIBS.get(path)
    if L is None:
        if spec.family and not Path(path).exists():
            from . import fieldgen
            built = fieldgen.family_library(*spec.family)
            if str(built) != path:
                raise RuntimeError(f"field library {built} is not the expected {path}")
        L = _FIELD_LIBS[path] = _load(path)
    return L


def launch_count() -> int:
    """Kernel launches issued so far by libgsolve.so and every field library loaded."""
    return int(lib().gs_launch_count()) + sum(int(L.gs_launch_count())
                                               for L in _FIELD_LIBS.values())


def check(rc: int, what: str, L=None) -> None:
    if rc != GS_OK:
        msg = (L or lib()).gs_last_error().decode(errors="replace")
        raise GsolveError(f"{what} failed ({rc}): {msg}")


def exported_symbols():
    """Names this binding expects the library to export."""
    return list(_SIGS)
