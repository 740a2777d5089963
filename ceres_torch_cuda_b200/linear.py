"""Optional-backend registry and the registry-routed part of ``solve_linear_system``
with ceres-torch's names and calling convention (linear.py:12-23, :82-103,
:106-371, :1311-1328).

A backend is called as ``fn(A, b, **kwargs)`` with the dense Jacobian ``A``
[m, n], ``b`` [m] and the solver options as keywords. It may raise
``OptionalBackendUnavailable`` to decline; a ``TypeError`` is retried without
keywords, as in ceres-torch. The structured bundle-adjustment path of
``solve`` does not go through this registry: it never forms a dense Jacobian.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Callable, Iterable, Optional, Sequence

import torch

from .types import LinearSolverType, PreconditionerType, VisibilityClusteringType


@dataclass
class LinearSolverSummary:
    residual_norm: float
    num_iterations: int
    success: bool
    message: str = ""


@dataclass
class LinearSolverResult:
    x: torch.Tensor
    summary: LinearSolverSummary


class OptionalBackendUnavailable(RuntimeError):
    pass


OptionalBackend = Callable[..., "torch.Tensor | LinearSolverResult"]
_optional_backends: dict[str, OptionalBackend] = {}


def register_optional_backend(name: str, backend: OptionalBackend) -> None:
    _optional_backends[name] = backend


def unregister_optional_backend(name: str) -> None:
    _optional_backends.pop(name, None)


def clear_optional_backends() -> None:
    _optional_backends.clear()


def get_optional_backend(name: str) -> Optional[OptionalBackend]:
    return _optional_backends.get(name)


def _summarize(A: torch.Tensor, b: torch.Tensor, x: torch.Tensor, iterations: int, message: str,
               success: bool = True) -> LinearSolverResult:
    r = A @ x.reshape(-1) - b.reshape(-1)
    return LinearSolverResult(x.reshape(-1), LinearSolverSummary(float(torch.linalg.norm(r)), iterations, success,
                                                                  message))


def _try_backend(name: str, A: torch.Tensor, b: torch.Tensor, **kwargs: Any) -> Optional[LinearSolverResult]:
    backend = get_optional_backend(name)
    if backend is None:
        return None
    try:
        raw = backend(A, b, **kwargs)
    except TypeError:
        raw = backend(A, b)
    except OptionalBackendUnavailable:
        return None
    if isinstance(raw, LinearSolverResult):
        return raw
    return _summarize(A, b, raw, 1, f"optional {name} backend")


_ROUTES = {
    LinearSolverType.DENSE_SCHUR: ("dense_schur", "block_schur"),
    LinearSolverType.ITERATIVE_SCHUR: ("iterative_schur", "block_schur"),
    LinearSolverType.SPARSE_SCHUR: ("sparse_schur", "block_schur", "sparse_cholesky"),
    LinearSolverType.SPARSE_NORMAL_CHOLESKY: ("sparse_normal_cholesky", "sparse_cholesky"),
}


def solve_linear_system(
    A: torch.Tensor,
    b: torch.Tensor,
    *,
    solver_type: LinearSolverType = LinearSolverType.DENSE_QR,
    damping: Optional[torch.Tensor] = None,
    num_eliminate: int = 0,
    min_iterations: int = 0,
    max_iterations: int = 500,
    tolerance: float = 1e-10,
    preconditioner_type: PreconditionerType = PreconditionerType.JACOBI,
    block_sizes: Optional[Sequence[int]] = None,
    use_mixed_precision: bool = False,
    max_refinement_iterations: int = 0,
    max_num_spse_iterations: int = 5,
    use_spse_initialization: bool = False,
    spse_tolerance: float = 0.1,
    visibility: Optional[Sequence[Iterable[int]]] = None,
    visibility_clustering_type: VisibilityClusteringType = VisibilityClusteringType.CANONICAL_VIEWS,
) -> LinearSolverResult:
    """Route a dense linear least-squares system to the registered backends in
    ceres-torch's order. Types without a registered backend raise
    NotImplementedError: this package's solvers are the CUDA backends."""
    if A.ndim != 2:
        raise ValueError("A must be a 2D matrix")
    b = b.reshape(-1)
    if b.numel() != A.shape[0]:
        raise ValueError("b must have one entry per row of A")
    if A.shape[1] == 0:
        return LinearSolverResult(b.new_zeros(0), LinearSolverSummary(float(torch.linalg.norm(b)), 0, True,
                                                                      "zero-column system"))
    if A.shape[0] == 0:
        return LinearSolverResult(b.new_zeros(A.shape[1]), LinearSolverSummary(0.0, 0, True, "empty-row system"))
    kwargs = dict(damping=damping, num_eliminate=num_eliminate, solver_type=solver_type, block_sizes=block_sizes,
                  min_iterations=min_iterations, max_iterations=max_iterations, tolerance=tolerance,
                  preconditioner_type=preconditioner_type, max_num_spse_iterations=max_num_spse_iterations,
                  use_spse_initialization=use_spse_initialization, spse_tolerance=spse_tolerance,
                  visibility=visibility, visibility_clustering_type=visibility_clustering_type)
    routes = _ROUTES.get(solver_type, ())
    if solver_type is LinearSolverType.ITERATIVE_SCHUR and num_eliminate <= 0:
        routes = ()
    for name in routes:
        result = _try_backend(name, A, b, **kwargs)
        if result is not None:
            return result
    raise NotImplementedError(
        f"no registered backend handled {solver_type.value}; call register_cuda_sparse_backends() and pass CUDA "
        "tensors")
