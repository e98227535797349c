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
  ``linear_ladder_<D>`` -> linear_<D> (dy = 1.01 y), D in 1, 2, 3, 4, 8; params ignored
  ``robertson``         -> robertson, params (n, 3) = [k1, k2, k3] (stiff)

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
FIELD_ROBERTSON = 10
FIELD_LORENZ3 = 11

LINEAR_DIMS = (1, 2, 3, 4, 8)


@dataclass(frozen=True)
class FieldSpec:
    key: str      # field key ("lorenz", "linear_3", ...)
    code: int     # libgsolve field code
    dim: int      # state dimension D
    nparam: int   # parameters the kernel reads (P)
    stiff_ok: bool  # has an analytic Jacobian (Rosenbrock23 capable)
    lib: str = ""   # the generated field's own library (empty: libgsolve.so)


# problem name -> FieldSpec of a generated field (register_field)
_USER: dict = {}


_STATIC = {
    "lorenz": FieldSpec("lorenz", FIELD_LORENZ, 3, 1, False),
    "lorenz3": FieldSpec("lorenz3", FIELD_LORENZ3, 3, 3, False),
    "vdp": FieldSpec("vdp", FIELD_VDP, 2, 1, True),
    "lv": FieldSpec("lv", FIELD_LOTKA_VOLTERRA, 2, 4, False),
    "robertson": FieldSpec("robertson", FIELD_ROBERTSON, 3, 3, True),
}


def field_spec(key: str) -> FieldSpec:
    if key in _STATIC:
        return _STATIC[key]
    for spec in _USER.values():
        if spec.key == key:
            return spec
    if key.startswith("linear_"):
        try:
            d = int(key.split("_", 1)[1])
        except ValueError:
            d = -1
        if d in LINEAR_DIMS:
            return FieldSpec(key, FIELD_LINEAR * 1000 + d, d, 1, True)
    raise KeyError(f"unknown field {key!r}; known: {sorted(_STATIC)} + linear_<D> for D in "
                   f"{LINEAR_DIMS}")


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
    if nm == "robertson":
        return _STATIC["robertson"]
    if nm.startswith("linear_ladder_"):
        try:
            d = int(nm.rsplit("_", 1)[1])
        except ValueError:
            return None
        if d in LINEAR_DIMS:
            return field_spec(f"linear_{d}")
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
    if spec.key.startswith("linear_"):
        return np.zeros((n, 1)) if params.shape[1] == 0 else params[:, :1]
    if params.shape[1] < spec.nparam:
        raise ValueError(
            f"field {spec.key!r} reads {spec.nparam} parameter column(s); params has "
            f"{params.shape[1]}")
    return params[:, : spec.nparam]
