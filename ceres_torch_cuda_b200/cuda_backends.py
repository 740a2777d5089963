"""CUDA backend registration with ceres-torch's interface (cuda_backends.py:21-355).

``register_cuda_sparse_backends()`` registers the dense-Jacobian backends
(``sparse_normal_cholesky``, ``sparse_cholesky``, ``sparse_schur``,
``block_schur``) under the same names as ceres-torch, backed by the sm_100a
library, and selects the precision of the structured bundle-adjustment path
that ``solve`` uses for ITERATIVE_SCHUR / SPARSE_SCHUR / DENSE_SCHUR on CUDA
tensors: ``precision="fp64"`` (default) or ``"mixed"`` (FP32 Jacobian store and
PCG, float64 cost, gain ratio and refinement).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any

import torch

from . import _lib
from .build import CSRC, SOURCES
from .linear import (LinearSolverResult, LinearSolverSummary, OptionalBackendUnavailable, get_optional_backend,
                     register_optional_backend, unregister_optional_backend)

CUDA_BACKEND_NAMES = ("sparse_normal_cholesky", "sparse_cholesky", "sparse_schur", "block_schur")

_STATE = {"precision": "fp64", "registered": False}


@dataclass(frozen=True)
class CudaExtensionInfo:
    available: bool
    backend: str
    registered: tuple[str, ...]
    source_paths: tuple[str, ...]
    message: str


def cuda_extension_source_paths() -> tuple[str, ...]:
    return tuple(str(CSRC / s) for s in SOURCES)


def torch_cuda_backend_available() -> bool:
    return torch.version.cuda is not None and torch.cuda.is_available()


def _info(backend: str, registered=(), message: str | None = None) -> CudaExtensionInfo:
    paths = cuda_extension_source_paths()
    if torch.version.cuda is None:
        return CudaExtensionInfo(False, backend, (), paths, "PyTorch is not CUDA-enabled.")
    if not torch.cuda.is_available():
        return CudaExtensionInfo(False, backend, (), paths, "No CUDA device is available.")
    try:
        _lib.load()
    except _lib.NativeLibraryError as exc:
        return CudaExtensionInfo(False, backend, (), paths, str(exc))
    return CudaExtensionInfo(True, backend, tuple(registered), paths,
                             message or "sm_100a bundle-adjustment library is available.")


def get_torch_cuda_backend_info() -> CudaExtensionInfo:
    return _info("torch-cuda")


def get_cuda_extension_info() -> CudaExtensionInfo:
    return _info("cuda-extension")


def cuda_extension_build_available() -> bool:
    return get_cuda_extension_info().available


def load_cuda_extension(*, verbose: bool | None = None, force: bool = False) -> Any:
    """The loaded sm_100a library (ctypes handle)."""
    del verbose, force
    try:
        return _lib.load()
    except _lib.NativeLibraryError as exc:
        raise OptionalBackendUnavailable(str(exc)) from exc


def get_ba_precision() -> str:
    return _STATE["precision"]


def register_cuda_sparse_backends(*, overwrite: bool = True, backend: str = "torch",
                                  precision: str = "fp64") -> CudaExtensionInfo:
    if backend not in ("torch", "extension"):
        raise ValueError("backend must be 'torch' or 'extension'")
    if precision not in ("fp64", "mixed"):
        raise ValueError("precision must be 'fp64' or 'mixed'")
    info = _info("torch-cuda" if backend == "torch" else "cuda-extension")
    if not info.available:
        return info
    table = {
        "sparse_normal_cholesky": cuda_sparse_normal_cholesky,
        "sparse_cholesky": cuda_sparse_normal_cholesky,
        "sparse_schur": cuda_block_schur,
        "block_schur": cuda_block_schur,
    }
    registered = []
    for name, fn in table.items():
        if overwrite or get_optional_backend(name) is None:
            register_optional_backend(name, fn)
            registered.append(name)
    _STATE["precision"] = precision
    _STATE["registered"] = True
    return CudaExtensionInfo(True, info.backend, tuple(registered), info.source_paths,
                             f"Registered sm_100a sparse/block-Schur backends ({precision}).")


def register_cuda_extension_backends(*, overwrite: bool = True, precision: str = "fp64") -> CudaExtensionInfo:
    return register_cuda_sparse_backends(overwrite=overwrite, backend="extension", precision=precision)


def unregister_cuda_sparse_backends() -> None:
    for name in CUDA_BACKEND_NAMES:
        unregister_optional_backend(name)
    _STATE["registered"] = False
    _STATE["precision"] = "fp64"


def _require_cuda_tensor(t: torch.Tensor, name: str) -> None:
    if t.device.type != "cuda":
        raise OptionalBackendUnavailable(f"{name} must be a CUDA tensor for the CUDA extension backend.")
    if t.dtype not in (torch.float32, torch.float64):
        raise OptionalBackendUnavailable(f"{name} must be float32 or float64 for the CUDA extension backend.")


def _normal_solve(A: torch.Tensor, b: torch.Tensor, damping: torch.Tensor | None) -> torch.Tensor:
    """(A^T A + diag(d)) x = A^T b: the product with cuBLAS, the solve with the
    library's Cholesky kernels (float64)."""
    lib = load_cuda_extension()
    A64 = A.to(torch.float64)
    H = (A64.T @ A64).contiguous()
    if damping is not None:
        H.diagonal().add_(damping.reshape(-1).to(H))
    rhs = (A64.T @ b.reshape(-1).to(torch.float64)).contiguous()
    x = torch.empty_like(rhs)
    flags = torch.zeros(4, dtype=torch.int32, device=A.device)
    stream = torch.cuda.current_stream(A.device).cuda_stream
    with torch.cuda.device(A.device):
        _lib.check(lib.ceres_b200_dense_cholesky_solve(H.data_ptr(), rhs.data_ptr(), x.data_ptr(),
                                                         ctypes.c_int64(H.shape[0]), flags.data_ptr(), stream),
                   "dense Cholesky solve")
    if int(flags[3]) & _lib.DEVERR_NOT_PD:
        raise RuntimeError("normal equations are not positive definite")
    return x.to(A.dtype)


def _summary(A, b, x, damping, message):
    r = A @ x.reshape(-1) - b.reshape(-1).to(A)
    sq = torch.sum(r * r)
    if damping is not None:
        sq = sq + torch.sum(torch.clamp(damping.reshape(-1).to(A), min=0.0) * x.reshape(-1) ** 2)
    return LinearSolverSummary(float(torch.sqrt(torch.clamp(sq, min=0.0))), 1, True, message)


def cuda_sparse_normal_cholesky(A: torch.Tensor, b: torch.Tensor, *, damping: torch.Tensor | None = None,
                                **_: Any) -> LinearSolverResult:
    _require_cuda_tensor(A, "A")
    _require_cuda_tensor(b, "b")
    if damping is not None:
        _require_cuda_tensor(damping, "damping")
    x = _normal_solve(A, b, damping)
    return LinearSolverResult(x, _summary(A, b, x, damping, "cuda sparse normal equations (sm_100a cholesky)"))


def cuda_block_schur(A: torch.Tensor, b: torch.Tensor, *, damping: torch.Tensor | None = None,
                     num_eliminate: int = 0, **_: Any) -> LinearSolverResult:
    """The block-Schur split of H at ``num_eliminate`` solves the same normal
    equations exactly; one Cholesky of H gives that solution."""
    _require_cuda_tensor(A, "A")
    _require_cuda_tensor(b, "b")
    if damping is not None:
        _require_cuda_tensor(damping, "damping")
    del num_eliminate
    x = _normal_solve(A, b, damping)
    return LinearSolverResult(x, _summary(A, b, x, damping, "cuda block schur (sm_100a cholesky)"))


cuda_extension_sparse_normal_cholesky = cuda_sparse_normal_cholesky
cuda_extension_block_schur = cuda_block_schur
