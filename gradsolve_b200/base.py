"""Result and routing types of the public API.

Same fields and meaning as the reference's contracts (gradsolve/base.py:116-197), so code
written against ``gradsolve.SolveResult`` / ``gradsolve.Route`` reads these unchanged.
``Problem`` is duck-typed exactly as there (gradsolve/base.py:61-113): anything with
``name``, ``dim``, ``t0``, ``t1`` and ``is_stiff`` works; the engine routes by ``name``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Protocol

import numpy as np


class Problem(Protocol):
    name: str
    dim: int
    t0: float
    t1: float
    is_stiff: bool


@dataclass(frozen=True)
class Route:
    """Where a ``solve`` or ``grad_closure`` request actually went (gradsolve/base.py:116-140).

    ``requested`` is the ``engine=`` argument, ``actual`` the engine that ran, ``reason``
    why they differ (``None`` when the request was honoured)."""
    requested: str
    actual: str
    reason: Optional[str] = None


@dataclass
class SolveResult:
    """Result of one batched ensemble solve (gradsolve/base.py:143-197).

    ``accepted_steps`` / ``rejected_steps`` are the true per-trajectory counts from the
    kernel.  ``y_saved`` / ``ts_saved`` are set only for ``saveat`` requests."""
    y_final: np.ndarray
    accepted_steps: np.ndarray = field(default_factory=lambda: np.empty(0))
    rejected_steps: np.ndarray = field(default_factory=lambda: np.empty(0))
    solver: str = ""
    y_saved: Optional[np.ndarray] = None
    ts_saved: Optional[np.ndarray] = None
    route: Optional[Route] = None
