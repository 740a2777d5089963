"""Drop-in behind ceres-torch's own API.

``install(ceres_torch)`` leaves the user's ``import ceres_torch`` in place and

* registers this package's backends in ceres-torch's linear-solver registry
  (``register_optional_backend``, linear.py:90-91) under the names
  ceres-torch's ``register_cuda_sparse_backends`` uses (cuda_backends.py:158-183),
  plus ``iterative_schur`` (tried first for ITERATIVE_SCHUR, linear.py:191-210);
* puts a pre-dispatch in front of ceres-torch's ``solve`` (solver.py:28-32): a
  trust-region Levenberg-Marquardt solve with ITERATIVE_SCHUR, SPARSE_SCHUR or
  DENSE_SCHUR whose residual blocks are all ``SnavelyReprojectionError`` over CUDA
  tensors runs on the sm_100a path; anything else runs ceres-torch's own solver,
  unchanged.

Options, losses and summaries cross the boundary by field and enum-member name, so
ceres-torch's own ``SolverOptions`` and loss objects are accepted and the caller gets
ceres-torch's own ``SolverSummary`` back.
"""
from __future__ import annotations

import dataclasses
import importlib
from dataclasses import dataclass, field
from enum import Enum
from typing import Any, Callable

import torch

from . import cuda_backends as _cb
from .linear import LinearSolverResult as _OwnResult
from .linear import OptionalBackendUnavailable as _OwnUnavailable
from .types import SolverOptions, SolverSummary

SCHUR_SOLVERS = ("ITERATIVE_SCHUR", "SPARSE_SCHUR", "DENSE_SCHUR")
GPU_PRECONDITIONERS = ("IDENTITY", "JACOBI", "SCHUR_JACOBI", "SCHUR_POWER_SERIES_EXPANSION", "CLUSTER_JACOBI",
                       "CLUSTER_TRIDIAGONAL")


def options_from(options: Any) -> SolverOptions:
    """This package's SolverOptions from any object with ceres-torch's SolverOptions
    fields (ceres-torch's own included); enum members are matched by name."""
    if isinstance(options, SolverOptions):
        return options
    values = {f.name: getattr(options, f.name) for f in dataclasses.fields(SolverOptions) if hasattr(options, f.name)}
    return SolverOptions(**values)


def _to_enum(value: Any, cls: type) -> Any:
    return value if isinstance(value, cls) else getattr(cls, getattr(value, "name", str(value)))


def _convert_dataclass(obj: Any, cls: type) -> Any:
    """An instance of dataclass ``cls`` with the fields of ``obj`` (enums by name)."""
    kwargs = {}
    for f in dataclasses.fields(cls):
        if not hasattr(obj, f.name):
            continue
        v = getattr(obj, f.name)
        default = f.default if f.default is not dataclasses.MISSING else None
        enum_cls = type(default) if isinstance(default, Enum) else None
        kwargs[f.name] = _to_enum(v, enum_cls) if enum_cls is not None and v is not None else v
    return cls(**kwargs)


def summary_to(module: Any, summary: SolverSummary) -> Any:
    """``module``'s SolverSummary (ceres-torch's, types.py:361-468) with the fields of
    ``summary``; the GPU-path additions (precision, time_to_tolerance_in_seconds)
    are kept as attributes."""
    out = _convert_dataclass(summary, module.SolverSummary)
    out.iterations = [_convert_dataclass(it, module.IterationSummary) for it in summary.iterations]
    out.precision = summary.precision
    out.time_to_tolerance_in_seconds = summary.time_to_tolerance_in_seconds
    return out


def _is_cuda_problem(problem: Any) -> bool:
    blocks = getattr(problem, "parameter_blocks", None)
    return bool(blocks) and all(getattr(b, "tensor", torch.empty(0)).is_cuda for b in blocks)


def _has_bounds_or_manifolds(problem: Any) -> bool:
    for b in problem.parameter_blocks:
        if getattr(b, "lower_bound", None) is not None or getattr(b, "upper_bound", None) is not None:
            return True
        if getattr(b, "has_explicit_manifold", False) and type(b.manifold).__name__ != "EuclideanManifold":
            return True
    return False


def route(options: Any, problem: Any) -> tuple[bool, str]:
    """Whether ``solve(options, problem)`` runs on the sm_100a path, and why not."""
    name = lambda v: getattr(v, "name", str(v))  # noqa: E731
    if name(options.minimizer_type) != "TRUST_REGION":
        return False, "not a trust-region solve"
    if name(options.trust_region_strategy_type) != "LEVENBERG_MARQUARDT":
        return False, "not Levenberg-Marquardt"
    if name(options.linear_solver_type) not in SCHUR_SOLVERS:
        return False, "not a Schur linear solver"
    if (name(options.linear_solver_type) == "ITERATIVE_SCHUR"
            and name(options.preconditioner_type) not in GPU_PRECONDITIONERS):
        return False, f"{name(options.preconditioner_type)} is not a GPU preconditioner"
    if options.use_inner_iterations or options.check_gradients:
        return False, "inner iterations / gradient checking"
    if not hasattr(problem, "residual_blocks") or not problem.residual_blocks:
        return False, "no residual blocks"
    if not _is_cuda_problem(problem):
        return False, "parameter blocks are not CUDA tensors"
    if _has_bounds_or_manifolds(problem):
        return False, "bounds or non-Euclidean manifolds"
    from .problem import extract_bundle_adjustment

    try:
        extract_bundle_adjustment(problem)
    except NotImplementedError as exc:
        return False, str(exc)
    return True, "bundle adjustment on CUDA"


def _wrap_backend(module: Any, fn: Callable, name: str) -> Callable:
    """A registry entry with ceres-torch's calling convention (linear.py:1311-1328):
    results as ``module``'s LinearSolverResult, unavailability as ``module``'s
    OptionalBackendUnavailable (so ceres-torch falls through to its own path)."""
    unavailable = module.OptionalBackendUnavailable

    def backend(A: torch.Tensor, b: torch.Tensor, **kwargs: Any):
        try:
            res = fn(A, b, **kwargs)
        except _OwnUnavailable as exc:
            raise unavailable(str(exc)) from exc
        if isinstance(res, _OwnResult):
            s = res.summary
            return module.LinearSolverResult(res.x, module.LinearSolverSummary(s.residual_norm, s.num_iterations,
                                                                                s.success, s.message))
        return res

    backend.__name__ = f"ceres_b200_{name}"
    backend.__qualname__ = backend.__name__
    backend._ceres_b200 = True  # noqa: SLF001 - marks this package's registry entries
    return backend


def _iterative_schur_dense(A: torch.Tensor, b: torch.Tensor, **_: Any):
    """Dense-Jacobian ITERATIVE_SCHUR requests: the structured path takes bundle
    adjustment before any dense Jacobian exists (the solve pre-dispatch); a dense A
    is left to the next registry entry (block_schur), as ceres-torch does when this
    name is not registered."""
    raise _OwnUnavailable("dense-Jacobian ITERATIVE_SCHUR: served by the structured solve path only")


@dataclass
class Installation:
    """What ``install`` changed in a ceres-torch module; ``uninstall()`` undoes it."""

    module: Any
    precision: str
    registered: tuple[str, ...]
    original_solve: Callable
    replaced: list[tuple[Any, str, Any]] = field(default_factory=list)
    routed: int = 0
    fell_through: int = 0
    last_reason: str = ""

    def uninstall(self) -> None:
        for owner, attr, old in reversed(self.replaced):
            setattr(owner, attr, old)
        self.replaced.clear()
        for name in self.registered:
            entry = self.module.get_optional_backend(name)
            if entry is not None and getattr(entry, "_ceres_b200", False):
                self.module.unregister_optional_backend(name)
        if getattr(self.module, "_ceres_b200_installation", None) is self:
            delattr(self.module, "_ceres_b200_installation")


def install(module: Any = None, *, precision: str = "fp64", overwrite: bool = True) -> Installation:
    """Route ceres-torch's bundle-adjustment Schur solves on CUDA to this package.

    ``module``: the ceres-torch package (imported as ``ceres_torch`` when omitted).
    ``precision``: "fp64" or "mixed" for the structured path. Installing again
    replaces the previous installation."""
    if precision not in ("fp64", "mixed"):
        raise ValueError("precision must be 'fp64' or 'mixed'")
    ct = module if module is not None else importlib.import_module("ceres_torch")
    prev = getattr(ct, "_ceres_b200_installation", None)
    if prev is not None:
        prev.uninstall()
    solver_mod = importlib.import_module(ct.__name__ + ".solver")
    original = solver_mod.solve
    table = {
        "sparse_normal_cholesky": _cb.cuda_sparse_normal_cholesky,
        "sparse_cholesky": _cb.cuda_sparse_normal_cholesky,
        "sparse_schur": _cb.cuda_block_schur,
        "block_schur": _cb.cuda_block_schur,
        "iterative_schur": _iterative_schur_dense,
    }
    registered = []
    for name, fn in table.items():
        if overwrite or ct.get_optional_backend(name) is None:
            ct.register_optional_backend(name, _wrap_backend(ct, fn, name))
            registered.append(name)
    inst = Installation(ct, precision, tuple(registered), original)

    def solve(options, problem):
        ok, why = route(options, problem)
        registry_name = "iterative_schur" if getattr(options.linear_solver_type, "name", "") == "ITERATIVE_SCHUR" \
            else "block_schur"
        entry = ct.get_optional_backend(registry_name)
        if ok and not (entry is not None and getattr(entry, "_ceres_b200", False)):
            ok, why = False, f"{registry_name} is not registered to the sm_100a path"
        inst.last_reason = why
        if not ok:
            inst.fell_through += 1
            return original(options, problem)
        inst.routed += 1
        from .solver import solve as gpu_solve

        own = options_from(options)
        return summary_to(ct, gpu_solve(own, problem, precision=precision))

    solve.__doc__ = original.__doc__
    solve.__wrapped__ = original
    for owner in (ct, solver_mod):
        inst.replaced.append((owner, "solve", getattr(owner, "solve")))
        setattr(owner, "solve", solve)
    ct._ceres_b200_installation = inst  # noqa: SLF001
    return inst


__all__ = ["Installation", "install", "options_from", "route", "summary_to"]
