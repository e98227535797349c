"""Build the test-only exact-association Tsit5 forward (tests/exact/libgsexact.so).

    python tests/exact/build.py

Compiled with -fmad=false so that float64 multiplies and adds are never fused: the kernel
then rounds every operation as numpy does (see gs_exact.cu).  Test infrastructure only; the
package never loads it.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
LIB = HERE / "libgsexact.so"
SOURCE = HERE / "gs_exact.cu"


def build(force: bool = False) -> Path:
    sys.path.insert(0, str(ROOT))
    from gradsolve_b200.csrc import build as product_build

    deps = [SOURCE] + product_build.HEADERS
    if not force and LIB.exists() and all(p.stat().st_mtime <= LIB.stat().st_mtime
                                          for p in deps if p.exists()):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [product_build.nvcc(), *product_build.ARCH, "-O3", "-fmad=false", "-std=c++17",
           "-Xcompiler", "-fPIC", "-shared", "-o", str(tmp), str(SOURCE)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stderr[-4000:]}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
