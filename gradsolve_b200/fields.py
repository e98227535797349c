"""Problem-name -> kernel-field routing and parameter mapping.

Mirrors the reference's single sources of these rules:
  * ``gradsolve/warp/warp_ode.py:463-510`` (``_field_for`` / ``supports``) and
    ``:513-589`` (``_param_of`` / ``_rho_of``) for the non-stiff fields;
  * ``gradsolve/warp/warp_rosenbrock.py:221-273`` for the stiff ones.

Routing (problem.name -> field):
  ``diffeqgpu_lorenz``  -> lorenz, params (n, 1) = [rho]
  ``lorenz``            -> lorenz3, params (n, 3) = [sigma, beta, rho]; sigma/beta are read
                           from the params (all three columns get gradients)
  ``vdp``               -> vdp, params[:, 0] = mu
  ``lotka_volterra`` / ``lv`` -> Lotka-Volterra, params (n, 4) = [alpha, beta, gamma, delta]
  ``linear_ladder_<D>`` -> linear_<D> (dy = 1.01 y), any D > 0; params ignored
  ``lorenz96_<D>``      -> lorenz96_<D>, any D >= 4, params (n, 1) = [F]
  ``robertson``         -> robertson, params (n, 3) = [k1, k2, k3] (stiff)
  ``hires``             -> hires (stiff, D = 8, autonomous); params ignored
  a name given to ``register_field`` / ``register_jax_field`` / ``register_linstiff``
                        -> that generated field (``linstiff_*`` among them)

The core library carries linear_<D> for D in LINEAR_DIMS and lorenz96_<D> for D in
LORENZ96_DIMS; any other dimension of the two families gets a library of its own, compiled
on first use (``fieldgen.family_library``).  Above MAX_DIM the fused lanes refuse before any
launch, as the reference's GPU path does.

Params with more columns than a field reads keep the extra columns; their gradient is 0
(the field does not read them), as ``jax.grad`` through ``f_jax`` would give.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

FIELD_LORENZ = 1
FIELD_VDP = 2
FIELD_LOTKA_VOLTERRA = 3
FIELD_LINEAR = 4
FIELD_LORENZ96 = 5
FIELD_ROBERTSON = 10
FIELD_LORENZ3 = 11
FIELD_HIRES = 12

LINEAR_DIMS = (1, 2, 3, 4, 8, 10, 32)   # linear_<D> in libgsolve.so
STIFF_LINEAR_DIMS = (1, 2, 3, 4, 8)     # ... of which Rosenbrock23 serves these
LORENZ96_DIMS = (4, 8, 32)              # lorenz96_<D> in libgsolve.so
MAX_DIM = 64                            # gradsolve/warp/warp_ode.py:75-81 (_GPU_VEC_DIM_CEILING)


def dim_limit_message(dim: int) -> str:
    return (f"fused GPU register-vector limit: dim={dim} > {MAX_DIM}. The fused adaptive "
            "kernels are low-NVAR GPU engines (state and stages in registers, a group of "
            "lanes per trajectory above 8 components); larger systems are refused before "
            "any launch (gradsolve/warp/warp_ode.py:649-664).")


@dataclass(frozen=True)
class FieldSpec:
    key: str      # field key ("lorenz", "linear_3", ...)
    code: int     # libgsolve field code
    dim: int      # state dimension D
    nparam: int   # parameters the kernel reads (P)
    stiff_ok: bool  # has an analytic Jacobian (Rosenbrock23 capable)
    lib: str = ""   # the field's own library (empty: libgsolve.so)
    family: tuple = ()  # (kind, D) of a built-in family member whose library is built on use


# problem name -> FieldSpec of a generated field (register_field)
_USER: dict = {}


_STATIC = {
    "lorenz": FieldSpec("lorenz", FIELD_LORENZ, 3, 1, False),
    "lorenz3": FieldSpec("lorenz3", FIELD_LORENZ3, 3, 3, False),
    "vdp": FieldSpec("vdp", FIELD_VDP, 2, 1, True),
    "lv": FieldSpec("lv", FIELD_LOTKA_VOLTERRA, 2, 4, False),
    "robertson": FieldSpec("robertson", FIELD_ROBERTSON, 3, 3, True),
    "hires": FieldSpec("hires", FIELD_HIRES, 8, 1, True),
}


def _family_spec(kind: str, d: int) -> FieldSpec:
    """linear_<d> or lorenz96_<d>: in the core library at its built dimensions, else in a
    library of its own (compiled by ``_lib.lib_for`` on first use)."""
    base = FIELD_LINEAR if kind == "linear" else FIELD_LORENZ96
    key, code = f"{kind}_{d}", base * 1000 + d
    core = LINEAR_DIMS if kind == "linear" else LORENZ96_DIMS
    if d in core:
        return FieldSpec(key, code, d, 1, kind == "linear" and d in STIFF_LINEAR_DIMS)
    from . import fieldgen
    path = "" if d > MAX_DIM else str(fieldgen.library_path(fieldgen.family_header(kind, d)))
    return FieldSpec(key, code, d, 1, False, path, (kind, d))


def _suffix(name: str) -> int:
    try:
        return int(name.rsplit("_", 1)[1])
    except ValueError:
        return -1


def field_spec(key: str) -> FieldSpec:
    if key in _STATIC:
        return _STATIC[key]
    for spec in _USER.values():
        if spec.key == key:
            return spec
    if key.startswith("linear_") and _suffix(key) >= 1:
        return _family_spec("linear", _suffix(key))
    if key.startswith("lorenz96_") and _suffix(key) >= 4:
        return _family_spec("lorenz96", _suffix(key))
    raise KeyError(f"unknown field {key!r}; known: {sorted(_STATIC)} + linear_<D> (D >= 1) + "
                   f"lorenz96_<D> (D >= 4)")


def field_for(problem) -> FieldSpec | None:
    """The kernel field for ``problem`` (by name), or None when no field is registered."""
    nm = getattr(problem, "name", "")
    if nm in _USER:
        return _USER[nm]
    if nm == "diffeqgpu_lorenz":
        return _STATIC["lorenz"]
    if nm == "lorenz":
        return _STATIC["lorenz3"]
    if nm == "vdp":
        return _STATIC["vdp"]
    if nm in ("lotka_volterra", "lv"):
        return _STATIC["lv"]
    if nm in ("robertson", "hires"):
        return _STATIC[nm]
    if nm.startswith("linear_ladder_"):
        d = _suffix(nm)
        return _family_spec("linear", d) if d >= 1 else None
    if nm.startswith("lorenz96_"):
        d = _suffix(nm)
        return _family_spec("lorenz96", d) if d >= 4 else None
    return None


def kernel_params(spec: FieldSpec, params: np.ndarray) -> np.ndarray:
    """The (n, P) block of ``params`` the kernel reads (leading columns), validated.

    The reference's Warp kernel hard-codes sigma = 10, beta = 8/3 for the 3-column
    ``lorenz`` problem and guards them (gradsolve/warp/warp_ode.py:575-588); ``lorenz3``
    reads all three from the parameters instead, so no guard is needed and all three
    columns receive gradients."""
    params = np.asarray(params, dtype=np.float64)
    if params.ndim == 1:
        params = params[:, None]
    if params.ndim != 2:
        raise ValueError(f"params must be (n, P); got shape {params.shape}")
    n = params.shape[0]
    if spec.lib and params.shape[1] == 0:  # a generated field without parameters
        return np.zeros((n, spec.nparam))
    if spec.key.startswith("linear_") or spec.key == "hires":  # params read by nothing
        return np.zeros((n, 1)) if params.shape[1] == 0 else params[:, :1]
    if params.shape[1] < spec.nparam:
        raise ValueError(
            f"field {spec.key!r} reads {spec.nparam} parameter column(s); params has "
            f"{params.shape[1]}")
    return params[:, : spec.nparam]
