"""The XLA FFI handlers (gradsolve_b200/csrc/gs_xla_ffi.cc) against the C ABI.

JAX is not installed here, so the handlers are compiled (syntax and types only) against a
compile-only stand-in of XLA's FFI header (tests/xla_ffi_stub/): the compiler checks every
libgsolve call against the declarations of include/gsolve.h, and the stand-in's
XLA_FFI_DEFINE_HANDLER_SYMBOL checks every binding against its handler's parameters.  A
planted mismatch (an attribute bound with the wrong type) must fail the same compile.
"""
from __future__ import annotations

import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "gradsolve_b200" / "csrc" / "gs_xla_ffi.cc"
STUB = ROOT / "tests" / "xla_ffi_stub"
CUDA_INC = Path("/usr/local/cuda/include")

HANDLERS = ["GsTsit5Fwd", "GsRos23Fwd", "GsTsit5Solve", "GsTsit5Replay", "GsRos23Replay",
            "GsTsit5Adjoint", "GsRos23Adjoint", "GsTsit5VjpStatic"]


def _compile(src: Path, tmp: Path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None or not (CUDA_INC / "cuda_runtime.h").exists():
        pytest.skip("needs g++ and the CUDA runtime headers")
    return subprocess.run([cxx, "-std=c++17", "-fsyntax-only", "-Wall", "-Werror",
                           f"-I{STUB}", f"-I{CUDA_INC}", f"-I{ROOT / 'include'}", str(src)],
                          capture_output=True, text=True, cwd=tmp)


def test_handlers_type_check_against_the_abi(tmp_path):
    res = _compile(SRC, tmp_path)
    assert res.returncode == 0, res.stderr[-3000:]


def test_every_handler_is_defined_once():
    text = SRC.read_text()
    names = re.findall(r"XLA_FFI_DEFINE_HANDLER_SYMBOL\((\w+),", text)
    assert sorted(names) == sorted(HANDLERS)


def test_a_planted_binding_mismatch_fails_to_compile(tmp_path):
    """The check is real: binding one attribute with the wrong type is a compile error."""
    text = SRC.read_text()
    bad = text.replace('.Attr<double>("t0"));', '.Attr<int64_t>("t0"));', 1)
    assert bad != text
    src = tmp_path / "gs_xla_ffi_bad.cc"
    src.write_text(bad.replace('#include "../../include/gsolve.h"', '#include "gsolve.h"'))
    res = _compile(src, tmp_path)
    assert res.returncode != 0 and "does not match" in res.stderr
