"""Build libgsolve.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed).

    python -m gradsolve_b200.csrc.build [--verbose]

The library is written next to the package (``gradsolve_b200/libgsolve.so``) so it travels
with a copy of the repository; ``-Xptxas -v`` output (registers, stack, spills per kernel)
goes to ``gradsolve_b200/csrc/ptxas.log``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent
PKG = CSRC.parent
LIB = PKG / "libgsolve.so"
SOURCES = [CSRC / "gs_abi.cu"]
PROBE_LIB = PKG / "libgsprobe.so"
PROBE_SOURCES = [CSRC / "gs_probe.cu"]
HEADERS = sorted(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "gsolve.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libgsolve.so")
    return exe


def up_to_date(lib: Path, sources) -> bool:
    if not lib.exists():
        return False
    t = lib.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in list(sources) + HEADERS if p.exists())


def _compile(lib: Path, sources, log: str, verbose: bool) -> None:
    tmp = lib.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, *FLAGS, "-o", str(tmp), *map(str, sources)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    (CSRC / log).write_text(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stderr[-4000:]}")
    os.replace(tmp, lib)
    if verbose:
        print(res.stderr)


XLA_LIB = PKG / "libgsolve_xla.so"
XLA_SOURCES = [CSRC / "gs_xla_ffi.cc"]


def xla_ffi_include():
    """XLA's FFI headers as JAX ships them, or None where JAX is not installed."""
    try:
        import jax.ffi
        return jax.ffi.include_dir()
    except Exception:
        return None


def build_xla_ffi(force: bool = False):
    """The XLA FFI handlers (gs_xla_ffi.cc) as libgsolve_xla.so, linked to libgsolve.so;
    skipped (returns None) where JAX is not installed, as in this image."""
    inc = xla_ffi_include()
    if inc is None:
        return None
    if not force and up_to_date(XLA_LIB, XLA_SOURCES + [LIB]):
        return XLA_LIB
    cxx = shutil.which("g++") or "c++"
    cuda_inc = Path(nvcc()).resolve().parent.parent / "include"
    cmd = [cxx, "-std=c++17", "-O2", "-shared", "-fPIC", f"-I{inc}", f"-I{cuda_inc}",
           "-o", str(XLA_LIB), *map(str, XLA_SOURCES), f"-L{PKG}", "-lgsolve",
           "-Wl,-rpath,$ORIGIN"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"building the XLA FFI handlers failed:\n{res.stderr[-4000:]}")
    return XLA_LIB


def build(force: bool = False, verbose: bool = False) -> Path:
    """Build libgsolve.so (the solver), libgsprobe.so (the FMA peak probes) and, where JAX is
    installed, libgsolve_xla.so (the XLA FFI handlers)."""
    if force or not up_to_date(LIB, SOURCES):
        _compile(LIB, SOURCES, "ptxas.log", verbose)
    if force or not up_to_date(PROBE_LIB, PROBE_SOURCES):
        _compile(PROBE_LIB, PROBE_SOURCES, "ptxas_probe.log", verbose)
    build_xla_ffi(force)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
