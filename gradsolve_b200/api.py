"""Public API: ``solve`` and ``grad_closure`` with the reference's signatures and routing
contract, served by the B200 kernels.

Mirrors gradsolve/api.py:291-400 (``solve``) and :792-1030 (``grad_closure``):
  * ``engine="auto"`` picks the Rosenbrock23 engine for stiff problems and the Tsit5
    engine otherwise (gradsolve/dispatch.py:235-258); the reference's engine names for this
    path (``warp_replay``, ``tsit5_replay``, ``warp_ode``, ``cuda_tsit5``; ``warp_rosenbrock``,
    ``cuda_rosenbrock23``) are accepted and served by the matching B200 engine, which the
    ``.route`` records;
  * the closure records the accepted-dt mesh ONCE at (y0, params) and is differentiable in
    the inputs ``wrt`` selects (``"params"``, ``"y0"`` or ``("y0", "params")``,
    gradsolve/api.py:721-758); the gradient is the frozen-controller discrete adjoint;
  * every result and closure carries ``.route`` (gradsolve/base.py:116-140);
  * ``remat`` maps onto the checkpoint policy: True -> sqrt(N) segments, False -> every
    state stored, None -> chosen by the memory budget (gradsolve/dispatch.py:268-293 picks
    ``jax.checkpoint`` for the same trade).

Inputs may be numpy arrays or torch tensors; closures return float64 CUDA tensors and are
differentiated with ``torch.autograd`` (``loss.backward()`` / ``torch.autograd.grad``).
There is no CPU path: ``device`` must name a CUDA device.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np
import torch

from . import engine
from . import engine as engine_mod
from .base import Route, SolveResult
from .fields import MAX_DIM, FieldSpec, dim_limit_message, field_for, kernel_params
from .torch_adapter import ReplayState, replay_apply, saveat_apply

ENGINE_TSIT5 = "b200_tsit5"
ENGINE_ROS23 = "b200_rosenbrock23"

# reference engine names on this path -> the B200 engine that serves them
ALIASES = {
    "warp_replay": ENGINE_TSIT5, "tsit5_replay": ENGINE_TSIT5, "warp_ode": ENGINE_TSIT5,
    "cuda_tsit5": ENGINE_TSIT5,
    "warp_rosenbrock": ENGINE_ROS23, "cuda_rosenbrock23": ENGINE_ROS23,
}

DEFAULT_MAX_STEPS = {ENGINE_TSIT5: 4096, ENGINE_ROS23: 50000}  # warp_replay.py:121, :296


@dataclass(frozen=True)
class EngineSpec:
    """One engine (gradsolve/api.py:48-71): name, supports(problem), solve, reverse."""
    name: str
    method: str
    supports: Callable
    solve: Callable
    reverse: Optional[Callable] = None


def _supports_tsit5(problem) -> bool:
    return field_for(problem) is not None


def _supports_ros23(problem) -> bool:
    spec = field_for(problem)
    return spec is not None and spec.stiff_ok


def _device(device) -> torch.device:
    dev = torch.device(device if device is not None else "cuda")
    if dev.type != "cuda":
        raise ValueError(
            f"gradsolve_b200 runs on CUDA devices only (got device={device!r}); there is no "
            "CPU path")
    if not torch.cuda.is_available():
        raise RuntimeError("gradsolve_b200 needs a CUDA device, and none is visible")
    return dev


def _to_device(x: torch.Tensor, dev: torch.device) -> torch.Tensor:
    """A tensor as float64 on dev (the same tensor when it already is), on the current
    stream."""
    return x.to(device=dev, dtype=torch.float64, non_blocking=True)


def _as_tensor(x, dev: torch.device) -> torch.Tensor:
    """x as a float64 tensor on dev.  Host tensors are copied with non_blocking=True on the
    current stream (the kernels that read them follow on the same stream): from pinned memory
    the host goes on to launch those kernels while the copy runs, and the caller keeps the
    buffer unchanged until the stream has passed it, as with any asynchronous copy; pageable
    memory is staged before the call returns."""
    if isinstance(x, torch.Tensor):
        return _to_device(x, dev)
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device=dev)


def _require_field(problem) -> FieldSpec:
    spec = field_for(problem)
    if spec is None:
        raise ValueError(
            f"gradsolve_b200 has no registered field for problem {getattr(problem, 'name', '?')!r}"
            "; supported names: 'diffeqgpu_lorenz', 'lorenz', 'vdp', 'lotka_volterra', "
            "'linear_ladder_<D>', 'lorenz96_<D>' (D >= 4), 'robertson', 'hires', and names "
            "given to register_field / register_jax_field / register_linstiff")
    if spec.dim > MAX_DIM:
        raise RuntimeError(dim_limit_message(spec.dim))
    return spec


def _prepare(problem, y0, params, dev):
    spec = _require_field(problem)
    y0_np = y0 if isinstance(y0, torch.Tensor) else np.asarray(y0, dtype=np.float64)
    if y0_np.ndim == 1:
        y0_np = y0_np[None, :]
    if y0_np.shape[-1] != spec.dim:
        raise ValueError(f"y0 must be (n, {spec.dim}) for {problem.name!r}; got {tuple(y0_np.shape)}")
    if isinstance(params, torch.Tensor):
        p_t = _to_device(params, dev)
        if p_t.ndim == 1:
            p_t = p_t[:, None]
    else:
        p_np = np.asarray(params, dtype=np.float64)
        if p_np.ndim == 1:
            p_np = p_np[:, None]
        p_t = torch.as_tensor(p_np, device=dev)
    y0_t = _as_tensor(y0_np, dev).contiguous()
    if p_t.shape[0] != y0_t.shape[0]:
        raise ValueError(f"y0 has {y0_t.shape[0]} trajectories but params has {p_t.shape[0]}")
    if p_t.shape[1] < spec.nparam:
        if not spec.key.startswith("linear_"):
            kernel_params(spec, np.zeros((1, p_t.shape[1])))  # raises the column-count error
        p_t = torch.nn.functional.pad(p_t, (0, spec.nparam - p_t.shape[1]))
    pk = p_t[:, : spec.nparam].contiguous()
    return spec, y0_t, p_t.contiguous(), pk


def _resolve(problem, engine_name: str, reasons: list) -> str:
    if engine_name == "auto":
        return ENGINE_ROS23 if getattr(problem, "is_stiff", False) else ENGINE_TSIT5
    if engine_name in ENGINE_REGISTRY:
        return engine_name
    if engine_name in ALIASES:
        reasons.append(f"served-by-{ALIASES[engine_name]}")
        return ALIASES[engine_name]
    raise ValueError(f"unknown engine {engine_name!r}; known: {sorted(ENGINE_REGISTRY)} + "
                     f"reference names {sorted(ALIASES)}")


def _t1_arg(problem, t1, dev):
    if t1 is None:
        return float(problem.t1), None
    t1a = np.asarray(t1, dtype=np.float64)
    if t1a.ndim == 0:
        return float(t1a), None
    return float(t1a.max()), torch.as_tensor(t1a, device=dev).contiguous()


def _engine_solve(name):
    method = ENGINE_REGISTRY[name].method

    def run(problem, y0, params, *, rtol, atol, device="cuda", max_steps=None, t1=None):
        dev = _device(device)
        spec, y0_t, _p, pk = _prepare(problem, y0, params, dev)
        t1s, t1v = _t1_arg(problem, t1, dev)
        ms = int(max_steps or 100000)
        r = engine.forward_record(method, spec, y0_t, pk, t0=float(problem.t0), t1=t1s,
                                  t1v=t1v, rtol=rtol, atol=atol, max_steps=ms, record=False)
        yf = r.y_final.cpu().numpy()
        st = r.status.cpu().numpy()
        yf[st != 0] = np.nan  # failed rows NaN'd, as the reference driver does (warp_ode.py:319)
        return SolveResult(y_final=yf, accepted_steps=r.n_acc.cpu().numpy().astype(np.int64),
                           rejected_steps=r.n_rej.cpu().numpy().astype(np.int64), solver=name)
    return run


def solve(problem, y0, params, *, saveat=None, engine: str = "auto", rtol: float = 1e-6,
          atol: float = 1e-9, device: str = "cuda", max_steps: Optional[int] = None,
          t1=None, **unused) -> SolveResult:
    """Forward ensemble solve (gradsolve/api.py:291-400).  Routes like the reference and
    returns a host ``SolveResult`` with true per-trajectory accepted/rejected counts.
    ``t1`` (optional) overrides ``problem.t1`` with a scalar or per-trajectory end times."""
    reasons: list[str] = []
    _require_field(problem)
    name = _resolve(problem, engine, reasons)
    spec = ENGINE_REGISTRY[name]
    if not spec.supports(problem):
        raise ValueError(f"engine {name!r} does not support problem {problem.name!r}")
    if saveat is not None:
        res = _solve_saveat(name, problem, y0, params, saveat, rtol=rtol, atol=atol,
                            device=device, max_steps=max_steps, t1=t1)
        res.route = Route(requested=engine, actual=name, reason="; ".join(reasons) or None)
        return res
    res = spec.solve(problem, y0, params, rtol=rtol, atol=atol, device=device,
                     max_steps=max_steps, t1=t1)
    res.solver = name
    res.route = Route(requested=engine, actual=name, reason="; ".join(reasons) or None)
    return res


def validate_saveat(saveat, t0: float, t1: float, t1v=None, n: Optional[int] = None):
    """Validate requested output times (gradsolve/solvers/dense.py:81-103): finite, sorted
    non-decreasing, inside [t0, t1].  A (k,) grid is shared by every trajectory; an (n, k)
    array gives each trajectory its own row (checked against its own end time when
    per-trajectory end times are given).  Returns float64 numpy."""
    ts = np.asarray(saveat.detach().cpu() if isinstance(saveat, torch.Tensor) else saveat,
                    dtype=np.float64)
    if ts.ndim not in (1, 2):
        raise ValueError(f"saveat must be (k,) or (n, k); got shape {ts.shape}")
    if ts.shape[-1] == 0:
        raise ValueError("saveat must contain at least one time")
    if not np.all(np.isfinite(ts)):
        raise ValueError("saveat contains non-finite times")
    if np.any(np.diff(ts, axis=-1) < 0):
        raise ValueError("saveat must be sorted non-decreasing")
    if ts.ndim == 2 and n is not None and ts.shape[0] != n:
        raise ValueError(f"per-trajectory saveat has {ts.shape[0]} rows for {n} trajectories")
    hi = np.asarray(t1v, dtype=np.float64) if t1v is not None else np.float64(t1)
    last = ts[..., -1]
    if np.any(ts[..., 0] < t0) or np.any(last > (hi if ts.ndim == 2 else np.min(hi))):
        raise ValueError(f"saveat times must lie within the problem domain [t0, t1] "
                         f"(t0={t0}); got [{ts.min()}, {ts.max()}]")
    return ts


def _solve_saveat(name, problem, y0, params, saveat, *, rtol, atol, device, max_steps, t1):
    """solve(..., saveat=ts): record the mesh, replay it with dense output
    (gradsolve/api.py:438-536)."""
    method = ENGINE_REGISTRY[name].method
    dev = _device(device)
    spec, y0_t, _p, pk = _prepare(problem, y0, params, dev)
    t1s, t1v = _t1_arg(problem, t1, dev)
    ts = validate_saveat(saveat, float(problem.t0), t1s,
                         None if t1v is None else t1v.cpu().numpy(), y0_t.shape[0])
    ms = int(max_steps or DEFAULT_MAX_STEPS[name])
    # the forward re-steps each saved time as it integrates: no replay pass
    r = engine.forward_record(method, spec, y0_t, pk, t0=float(problem.t0), t1=t1s, t1v=t1v,
                              rtol=rtol, atol=atol, max_steps=ms, checkpoint="sqrt",
                              saveat_ts=torch.as_tensor(ts, device=dev))
    engine.raise_on_failed(r, ms, t1s)
    yf, ys = r.y_final, r.ys
    return SolveResult(y_final=yf.cpu().numpy(), y_saved=ys.cpu().numpy(), ts_saved=ts,
                       accepted_steps=r.n_acc.cpu().numpy().astype(np.int64),
                       rejected_steps=r.n_rej.cpu().numpy().astype(np.int64), solver=name)


_VALID_WRT = "'params', 'y0', or ('y0', 'params')"


def _normalize_wrt(wrt) -> tuple:
    if wrt == "params":
        return ("params",)
    if wrt == "y0":
        return ("y0",)
    if isinstance(wrt, (tuple, list, set, frozenset)) and set(wrt) == {"y0", "params"}:
        return ("y0", "params")
    raise ValueError(f"invalid wrt={wrt!r}; expected {_VALID_WRT}")


def build_replay_state(problem, y0, params, *, method: str, rtol: float, atol: float,
                       device="cuda", max_steps: Optional[int] = None, checkpoint="auto",
                       t1=None, precision: str = "float64", saveat=None):
    """Record the mesh once and return (ReplayState, y0 tensor, params tensor).  With saveat
    (validated times on the device) the recording pass also keeps the saved states, which the
    closure returns at the recording point instead of replaying."""
    dev = _device(device)
    spec, y0_t, p_t, pk = _prepare(problem, y0, params, dev)
    t1s, t1v = _t1_arg(problem, t1, dev)
    ms = int(max_steps or 100000)
    r = engine.forward_record(method, spec, y0_t, pk, t0=float(problem.t0), t1=t1s, t1v=t1v,
                              rtol=rtol, atol=atol, max_steps=ms, checkpoint=checkpoint,
                              precision=precision,
                              # the float32 route records without dense output: its closure
                              # replays the saved states at the recording point
                              saveat_ts=None if precision == "float32" else saveat)
    engine.raise_on_failed(r, ms, t1s)
    # queued after the checks' synchronisation, so the sort runs on the device while the host
    # goes on to the closure call and the cotangent; the reverse pass picks it up
    engine.prepare_lane_order(r)
    state = ReplayState(r, y0_t, pk, spec.nparam, precision=precision,
                        ts_rec=None if precision == "float32" else saveat)
    return state, y0_t, p_t


def _lib_max_ckpt_every() -> int:
    from . import _lib
    return _lib.lib().gs_max_ckpt_every()


def record(problem, y0, params, *, rtol: float = 1e-6, atol: float = 1e-9,
           max_steps: Optional[int] = None, device: str = "cuda", precision: str = "float64",
           engine: str = "auto"):
    """The recording forward alone: ``(y_final (n, dim), n_acc (n,), dts_padded (n, S))`` as
    host numpy arrays, ``S = max(n_acc)``, row j trajectory j's accepted dts zero-padded past
    ``n_acc[j]`` -- the return of gradsolve/warp/warp_replay.py:120-182 (``record``, Tsit5) and
    :295-337 (``record_rosenbrock``, for a stiff problem or ``engine="warp_rosenbrock"``).
    ``precision="float32"`` records with the float32 kernels: the dts come back float32 and
    y_final holds float32 values.  Trajectories that did not reach t1 raise."""
    if precision not in ("float64", "float32"):
        raise ValueError(f"unknown precision {precision!r}; known: ['float64', 'float32']")
    spec = _require_field(problem)
    if precision == "float32":
        _check_float32_route(engine, spec)
    name = _resolve(problem, engine, [])
    ms = int(max_steps or DEFAULT_MAX_STEPS[name])
    # (the checkpoints are not returned: the longest interval keeps them smallest)
    state, _y0, _p = build_replay_state(problem, y0, params, method=ENGINE_REGISTRY[name].method,
                                        rtol=rtol, atol=atol, device=device, max_steps=ms,
                                        checkpoint=int(_lib_max_ckpt_every()),
                                        precision=precision)
    r = state.record
    yf = r.y_final.cpu().numpy()
    if precision == "float32":
        yf = yf.astype(np.float32)
    return yf, r.n_acc.cpu().numpy(), r.padded_dts().cpu().numpy()


def _make_reverse(name):
    method = ENGINE_REGISTRY[name].method

    def reverse(problem, y0, params, *, rtol, atol, device="cuda", remat=None, wrt=("params",),
                max_steps=None, checkpoint=None, t1=None, precision="float64", saveat=None):
        if checkpoint is None:
            checkpoint = "auto" if remat is None else ("sqrt" if remat else "all")
        ms = max_steps or DEFAULT_MAX_STEPS[name]
        ts = None
        if saveat is not None:
            dev0 = _device(device)
            t1s, t1v = _t1_arg(problem, t1, dev0)
            n = np.asarray(y0).shape[0] if not isinstance(y0, torch.Tensor) else y0.shape[0]
            ts = torch.as_tensor(
                validate_saveat(saveat, float(problem.t0), t1s,
                                None if t1v is None else t1v.cpu().numpy(), n),
                device=dev0)
        state, y0_t, p_t = build_replay_state(problem, y0, params, method=method, rtol=rtol,
                                              atol=atol, device=device, max_steps=ms,
                                              checkpoint=checkpoint, t1=t1,
                                              precision=precision, saveat=ts)
        dev = y0_t.device
        if saveat is not None:

            def kernel(z, p):  # the dense time series (n, k, dim), gradsolve/api.py:748-752
                ys = saveat_apply(state, _as_tensor(z, dev), _as_tensor(p, dev), ts)
                return ys.to(torch.float32) if precision == "float32" else ys
        elif precision == "float32":
            def kernel(z, p):  # float32 values; the closure's output is float32
                return replay_apply(state, _as_tensor(z, dev),
                                    _as_tensor(p, dev)).to(torch.float32)
        else:
            def kernel(z, p):
                return replay_apply(state, _as_tensor(z, dev), _as_tensor(p, dev))

        if wrt == ("y0",):
            fn = lambda z: kernel(z, p_t)  # noqa: E731
        elif wrt == ("params",):
            fn = lambda p: kernel(y0_t, p)  # noqa: E731
        else:
            fn = lambda z, p: kernel(z, p)  # noqa: E731
        fn.state = state
        return fn
    return reverse


# Reference engine names whose lane has an f32 route (the registered-field record-and-replay
# lanes, gradsolve/api.py:253-274); a general-RHS lane asked for float32 raises.
F32_ENGINES = frozenset({"auto", ENGINE_TSIT5, ENGINE_ROS23, "warp_ode", "warp_replay",
                         "warp_rosenbrock"})
F32_MAX_DIM = 8


def _check_float32_route(engine_name: str, spec: FieldSpec) -> None:
    """precision="float32": the record, the replay (dense output included) and the reverse
    pass all in float32 (gradsolve/api.py:253-274, 876-887).  Refused, as the reference
    refuses it, on lanes without an f32 route, and here also for fields above 8 components,
    which the float32 kernels do not cover."""
    if engine_name not in F32_ENGINES:
        raise ValueError(
            f"precision='float32' is not supported on lane {engine_name!r}: the float32 "
            "adjoint covers the registered-field record-and-replay lanes ('warp_replay', "
            "'warp_ode', 'warp_rosenbrock'). Use one of those, or precision='float64'.")
    if spec.dim > F32_MAX_DIM:
        raise ValueError(f"precision='float32' is built for fields of at most {F32_MAX_DIM} "
                         f"components; {spec.key!r} has {spec.dim}. Use precision='float64'.")


def grad_closure(problem, y0, params, *, wrt="params", saveat=None, precision: str = "float64",
                 engine: str = "auto", rtol: float = 1e-6, atol: float = 1e-9,
                 device: str = "cuda", remat: Optional[bool] = None,
                 max_steps: Optional[int] = None, checkpoint=None, t1=None, **unused):
    """Record the frozen step mesh at (y0, params) and return a differentiable closure
    (gradsolve/api.py:792-1030).  ``closure(params) -> y_final`` (n, dim) for the default
    ``wrt="params"``; ``closure(y0)`` for ``wrt="y0"``; ``closure(y0, params)`` for both.
    The closure carries ``.route`` and ``.state`` (the device record)."""
    wrt_t = _normalize_wrt(wrt)
    reasons: list[str] = []
    if precision not in ("float64", "mixed", "float32"):
        raise ValueError(f"unknown precision {precision!r}; known: 'float64', 'mixed', "
                         "'float32'")
    fs = _require_field(problem)
    if precision == "float32":
        _check_float32_route(engine, fs)
    name = _resolve(problem, engine, reasons)
    spec = ENGINE_REGISTRY[name]
    if not spec.supports(problem):
        raise ValueError(f"engine {name!r} does not support problem {problem.name!r}")
    if precision == "mixed" and spec.method != engine_mod.METHOD_TSIT5:
        raise ValueError("precision='mixed' is available on the Tsit5 engine only")
    fn = spec.reverse(problem, y0, params, rtol=rtol, atol=atol, device=device, remat=remat,
                      wrt=wrt_t, max_steps=max_steps, checkpoint=checkpoint, t1=t1,
                      precision=precision, saveat=saveat)
    fn.route = Route(requested=engine, actual=name, reason="; ".join(reasons) or None)
    return fn


ENGINE_REGISTRY: dict[str, EngineSpec] = {}
for _name, _method, _sup in ((ENGINE_TSIT5, engine.METHOD_TSIT5, _supports_tsit5),
                             (ENGINE_ROS23, engine.METHOD_ROS23, _supports_ros23)):
    ENGINE_REGISTRY[_name] = EngineSpec(_name, _method, _sup, None, None)
for _name in list(ENGINE_REGISTRY):
    _s = ENGINE_REGISTRY[_name]
    ENGINE_REGISTRY[_name] = EngineSpec(_s.name, _s.method, _s.supports, _engine_solve(_name),
                                        _make_reverse(_name))

__all__ = ["solve", "grad_closure", "register_field", "register_jax_field", "register_linstiff",
           "ENGINE_REGISTRY", "ALIASES", "FieldSpec"]


def register_field(name: str, f, dim: int, n_params: int, *, stiff: bool = False,
                   exprs=None) -> FieldSpec:
    """Register a Python right-hand side ``f(t, y, p) -> dy`` (autonomous: t unused) so that
    a Problem of that ``name`` routes to the B200 kernels like a built-in field.

    Same contract as the reference's ``register_jax_field(name, f_jax, dim, n_params, *,
    stiff=False)`` (gradsolve/__init__.py:31-42, gradsolve/warp/jax_field.py:517-560):
    idempotent per name; ``stiff=True`` also derives the Jacobian so the Rosenbrock23 engine
    can serve it.  ``f`` is traced once with symbolic scalars (``gradsolve_b200.fieldgen``);
    the RHS, its VJP and (stiff) Jacobian and second-order term are generated as CUDA and
    compiled into the field's own library (cached on disk by content)."""
    from . import fieldgen
    from . import fields as F
    if name in F._USER:
        return F._USER[name]
    if int(dim) > MAX_DIM:
        raise RuntimeError(dim_limit_message(int(dim)))
    d = fieldgen.Derived(f, dim, n_params, stiff, exprs=exprs)
    code = fieldgen.USER_CODE_BASE + (sum(name.encode()) * 7919) % 90000
    path = fieldgen.build_field_library(fieldgen.emit_struct(d, name, code))
    spec = FieldSpec(f"user_{name}", code, d.D, d.P, bool(stiff), str(path))
    F._USER[name] = spec
    return spec


def register_jax_field(name: str, f_jax, dim: int, n_params: int, *,
                       stiff: bool = False) -> FieldSpec:
    """The reference's registration entry point (gradsolve/__init__.py:31-42,
    gradsolve/warp/jax_field.py:517-560), same signature and contract as ``register_field``.
    Where JAX is importable, ``f_jax`` is walked as its jaxpr (``jax.make_jaxpr``) through
    ``fieldgen.JAXPR_PRIMITIVES``, as the reference's translator walks it; without JAX (this
    image) the function is traced with symbolic scalars, which accepts the same expressions
    written with Python arithmetic and numpy ufuncs."""
    from . import fields as F
    from . import fieldgen
    if name in F._USER:
        return F._USER[name]
    try:
        import jax
        import jax.numpy as jnp
    except ImportError:
        return register_field(name, f_jax, dim, n_params, stiff=stiff)
    closed = jax.make_jaxpr(f_jax)(0.0, jnp.zeros(int(dim)), jnp.zeros(int(n_params)))
    exprs = fieldgen.trace_jaxpr(closed, int(dim), int(n_params))
    return register_field(name, None, dim, n_params, stiff=stiff, exprs=exprs)


def register_linstiff(key: str, A) -> FieldSpec:
    """Register the constant-matrix linear stiff field f(y) = A y under ``key`` (a
    ``linstiff_*`` name by the reference's convention), so a Problem of that name routes to
    the Rosenbrock23 engine (and the Tsit5 one).  The reference's
    ``warp_rosenbrock.register_linstiff(key, A)`` (gradsolve/warp/warp_rosenbrock.py:88-95,
    gradsolve/warp/_warp_rosenbrock.py:219-252): A is (D, D), baked into the field as exact
    constants, Jacobian = A, parameters ignored; idempotent per key.  The field is generated
    like any registered one (its own library; zero entries of A are left out of the sums)."""
    from . import fields as F
    if key in F._USER:
        return F._USER[key]
    A = np.asarray(A, dtype=np.float64)
    if A.ndim != 2 or A.shape[0] != A.shape[1]:
        raise ValueError(f"linstiff A must be square (D, D); got {A.shape}")
    if not np.all(np.isfinite(A)):
        raise ValueError("linstiff A must be finite")
    rows = [[float(v) for v in row] for row in A]
    D = len(rows)

    def f(t, y, p):
        out = []
        for i in range(D):
            acc = 0.0
            for k in range(D):
                if rows[i][k] != 0.0:
                    acc = acc + rows[i][k] * y[k]
            out.append(acc)
        return out

    return register_field(key, f, D, 0, stiff=True)
