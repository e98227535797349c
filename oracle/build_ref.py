"""Recipe: build the reference's own hand-CUDA forward for the host, into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  Reads the templates gradsolve/cuda/kernels/tsit5_template.cu.in
and rosenbrock23_template.cu.in from the reference tree ($GRADSOLVE_REFERENCE, default: a
``reference`` directory beside the repository's root), fills them the way gradsolve/cuda/_codegen.py:32-55 and :65-100 do
(str.replace of the scalar type, the tableau #defines taken from the reference's own
tsit5_step.py / the Rosenbrock coefficients, the field bodies from the reference's own
gradsolve/cuda/_fields.py and _stiff_fields.py, D and P), and compiles each with
``g++ -O3 -ffp-contract=off`` (the host flags of gradsolve/cuda/_build.py:56) together with
oracle/ref_wrap.cpp.  Outputs (git-ignored, shipped with the tree):
    oracle/_ref/libref_tsit5_lorenz.so      ref_fwd(n, y0, rho, t1, rtol, atol, ...)
    oracle/_ref/libref_ros23_robertson.so   ref_fwd(n, y0, p, t1, rtol, atol, ...)
Nothing from the reference is copied into the repository: the filled sources live only
in oracle/_ref/.  Where the reference tree is absent the prebuilt outputs are used as-is.
"""
from __future__ import annotations

import importlib.util
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
REF = Path(os.environ.get("GRADSOLVE_REFERENCE", HERE.parent.parent / "reference"))

_A = ["A21", "A31", "A32", "A41", "A42", "A43", "A51", "A52", "A53", "A54", "A61", "A62", "A63",
      "A64", "A65"]
_B = ["B1", "B2", "B3", "B4", "B5", "B6"]
_E = ["E1", "E2", "E3", "E4", "E5", "E6", "E7"]


def _load(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _tsit5_source(field_key: str, D: int) -> str:
    ts = _load(REF / "gradsolve/solvers/tsit5_step.py", "ref_tsit5_step")
    fields = _load(REF / "gradsolve/cuda/_fields.py", "ref_cuda_fields")
    lines = [f"#define {nm} ((real){float(ts._C[i])!r})"
             for i, nm in enumerate(("C2", "C3", "C4", "C5", "C6"))]
    lines += [f"#define {nm} ((real){float(getattr(ts, '_' + nm))!r})" for nm in _A + _B + _E]
    src = (REF / "gradsolve/cuda/kernels/tsit5_template.cu.in").read_text()
    src = src.replace("@SCALAR@", "double").replace("@FFI_DTYPE@", "ffi::F64")
    src = src.replace("@TABLEAU@", "\n".join(lines))
    src = src.replace("@FIELD@", fields.emit_field(field_key, D))
    return src.replace("@D@", str(D))


def _ros23_source(field_key: str, D: int, P: int) -> str:
    import numpy as np

    stiff = _load(REF / "gradsolve/cuda/_stiff_fields.py", "ref_cuda_stiff_fields")
    d = 1.0 / (2.0 + np.sqrt(2.0))  # rosenbrock23_step.py:43-44 (jnp f64 == numpy f64 here)
    e32 = 6.0 + np.sqrt(2.0)
    tab = f"#define DCOEF ((real){float(d)!r})\n#define E32 ((real){float(e32)!r})"
    src = (REF / "gradsolve/cuda/kernels/rosenbrock23_template.cu.in").read_text()
    src = src.replace("@SCALAR@", "double").replace("@FFI_DTYPE@", "ffi::F64")
    src = src.replace("@TABLEAU@", tab)
    src = src.replace("@FIELD@", stiff.emit_stiff_field(field_key, D, None))
    src = src.replace("@JAC@", stiff.emit_stiff_jac(field_key, D, None))
    return src.replace("@D@", str(D)).replace("@P@", str(P))


def _compile(src: str, tag: str, define: str) -> Path:
    import tempfile

    OUT.mkdir(exist_ok=True)
    so = OUT / f"lib{tag}.so"
    with tempfile.TemporaryDirectory() as tmp:
        cpp = Path(tmp) / f"{tag}.cpp"  # the filled source is not kept
        cpp.write_text(src)
        cmd = ["g++", "-O3", "-ffp-contract=off", "-std=c++17", "-fPIC", "-shared",
               "-Wno-unknown-pragmas", f"-D{define}", f'-DREF_SOURCE="{cpp}"',
               str(HERE / "ref_wrap.cpp"), "-o", str(so), "-lpthread"]
        subprocess.run(cmd, check=True)
    return so


def build() -> list:
    if not (REF / "gradsolve/cuda/kernels").is_dir():
        have = sorted(OUT.glob("lib*.so")) if OUT.is_dir() else []
        if not have:
            print("build_ref: reference tree absent and no prebuilt oracle/_ref libraries",
                  file=sys.stderr)
        return have
    return [_compile(_tsit5_source("lorenz", 3), "ref_tsit5_lorenz", "REF_TSIT5"),
            _compile(_ros23_source("robertson", 3, 3), "ref_ros23_robertson", "REF_ROS23")]


if __name__ == "__main__":
    for p in build():
        print(p)
