"""gradsolve_b200 -- B200-native ensemble adaptive ODE solve and record-and-replay adjoint.

A drop-in for the Tsit5 and Rosenbrock23 record-and-replay engines of gradsolve
(``tsit5_replay`` / ``warp_replay`` and ``warp_rosenbrock``) behind ``solve`` and
``grad_closure``.  The work runs in hand-written sm_100a CUDA kernels exposed through the C
ABI of ``libgsolve.so`` (include/gsolve.h); PyTorch provides device memory, streams and
autograd plumbing.
"""
from .api import (ALIASES, ENGINE_REGISTRY, grad_closure, record,  # noqa: F401
                  register_field, register_jax_field, register_linstiff, solve)
from .base import Problem, Route, SolveResult  # noqa: F401
from .fields import field_for, field_spec  # noqa: F401

__version__ = "0.1.0"
