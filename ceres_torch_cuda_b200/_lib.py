"""ctypes binding of the C ABI in ``include/ceres_b200.h``.

The shared library is the only compute path of this package: if it cannot be
loaded, every solve raises ``NativeLibraryError``. There is no fallback.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

from . import build as _build

c_int32 = ctypes.c_int32
c_int64 = ctypes.c_int64
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p

ABI_VERSION = 5

OK = 0
EINVAL = -1
ECUDA = -2
ESMEM = -3
ECOOP = -4
ETOOBIG = -5
_ERRORS = {EINVAL: "invalid argument", ECUDA: "CUDA error", ESMEM: "shared memory limit", ECOOP: "cooperative launch failed",
           ETOOBIG: "size above capacity"}

DEVERR_LOSS = 1
DEVERR_BARRIER = 2
DEVERR_NOT_PD = 4

LOSS_TRIVIAL, LOSS_HUBER, LOSS_SOFTLONE, LOSS_CAUCHY, LOSS_ARCTAN, LOSS_TOLERANT, LOSS_TUKEY = range(7)
PRECOND_IDENTITY, PRECOND_JACOBI, PRECOND_SCHUR_JACOBI, PRECOND_SCHUR_POWER_SERIES, PRECOND_CLUSTER = range(5)
PRECOND_FLAG_SPSE_BASE = 0x100  # camera_assemble: also build the Hbb blocks of the SPSE initial point
FP64, FP32 = 0, 1
CAM_ITEM = 256  # CERES_B200_CAM_ITEM: entries per camera work item

(STAT_COST, STAT_GMAX_P, STAT_GSQ_P, STAT_GMAX_C, STAT_GSQ_C, STAT_CAND_COST, STAT_MODEL, STAT_STEP_SQ_P,
 STAT_STEP_SQ_C, STAT_NONFINITE, STAT_PCG_ITERS, STAT_PCG_SUCCESS, STAT_PCG_RNORM, STAT_ERROR, STAT_RHS_NORM,
 STAT_REFINE_RNORM, STAT_CAND_STATE_SQ_P, STAT_CAND_STATE_SQ_C) = range(18)
NSTATS = 18
CTL_BYTES = 256          # stats (float64) at 0, counters (uint32 x 16) at CTL_COUNTERS
CTL_COUNTERS = 192


class NativeLibraryError(RuntimeError):
    """The sm_100a library is missing, failed to load, or a call failed."""


class BAStruct(ctypes.Structure):
    """Mirror of ``ceres_b200_ba_t``."""

    _fields_ = [
        ("num_cameras", c_int32), ("num_observations", c_int32), ("num_points", c_int32),
        ("num_slices", c_int32), ("num_slots", c_int32), ("max_slice_len", c_int32),
        ("precision", c_int32), ("has_duplicate_cameras", c_int32), ("loss_kind", c_int32),
        ("loss_a", c_double), ("loss_b", c_double), ("loss_scale", c_double),
        ("inner_loss_kind", c_int32), ("pad0", c_int32),
        ("inner_a", c_double), ("inner_b", c_double), ("inner_scale", c_double),
        ("slice_base", c_void_p), ("slice_len", c_void_p), ("slot_cam", c_void_p), ("slot_obs", c_void_p),
        ("cam_offsets", c_void_p), ("cam_entries", c_void_p), ("cam_const", c_void_p), ("pt_const", c_void_p),
        ("cameras", c_void_p), ("points", c_void_p), ("cand_cameras", c_void_p), ("cand_points", c_void_p),
        ("jac", c_void_p), ("res", c_void_p),
        ("point_raw", c_void_p), ("winv", c_void_p), ("winv_ga", c_void_p), ("step_points", c_void_p),
        ("cam_diag", c_void_p), ("precond", c_void_p), ("rhs", c_void_p), ("step_cameras", c_void_p),
        ("pcg_x", c_void_p), ("pcg_r", c_void_p), ("pcg_z", c_void_p), ("pcg_p", c_void_p), ("pcg_ap", c_void_p),
        ("slot_pos", c_void_p), ("cm_jac", c_void_p), ("cam_items", c_void_p), ("items", c_void_p),
        ("num_items", c_int32), ("max_camera_obs", c_int32),
        ("scratch", c_void_p), ("scratch_bytes", c_int64),
        ("counters", c_void_p), ("stats", c_void_p),
        ("schur_blocks", c_void_p), ("schur_block_start", c_void_p), ("schur_contrib", c_void_p),
        ("num_schur_blocks", c_int64),
    ]


_P = ctypes.POINTER(BAStruct)

# batched solves (ceres_b200_batch_t)
BATCH_RESULT = 16
BATCH_TRACE = 10
(BR_INITIAL_COST, BR_FINAL_COST, BR_RECORDS, BR_TERMINATION, BR_MESSAGE, BR_SUCCESSFUL, BR_UNSUCCESSFUL,
 BR_JACOBIAN_EVALS, BR_RESIDUAL_EVALS, BR_LINEAR_SOLVES, BR_ERROR, BR_FINAL_GMAX) = range(12)
(BT_COST, BT_COST_CHANGE, BT_GMAX, BT_GNORM, BT_STEP_NORM, BT_RHO, BT_RADIUS, BT_LINEAR_ITERATIONS,
 BT_FLAGS) = range(9)
TERM_CONVERGENCE, TERM_NO_CONVERGENCE, TERM_FAILURE = range(3)
MESSAGES = ("Gradient tolerance reached.", "Maximum iterations reached.", "Too many invalid trust-region steps.",
            "Parameter tolerance reached.", "Function tolerance reached.", "Minimum trust-region radius reached.")


class BatchStruct(ctypes.Structure):
    """Mirror of ``ceres_b200_batch_t``."""

    _fields_ = [
        ("num_problems", c_int32), ("precision", c_int32), ("max_cameras", c_int32),
        ("has_duplicate_cameras", c_int32), ("loss_kind", c_int32), ("inner_loss_kind", c_int32),
        ("loss_a", c_double), ("loss_b", c_double), ("loss_scale", c_double),
        ("inner_a", c_double), ("inner_b", c_double), ("inner_scale", c_double),
        ("max_num_iterations", c_int32), ("min_linear_solver_iterations", c_int32),
        ("max_linear_solver_iterations", c_int32), ("preconditioner", c_int32),
        ("jacobi_scaling", c_int32), ("max_consecutive_invalid_steps", c_int32),
        ("max_refinements", c_int32), ("max_trace", c_int32),
        ("function_tolerance", c_double), ("gradient_tolerance", c_double), ("parameter_tolerance", c_double),
        ("min_relative_decrease", c_double), ("initial_radius", c_double), ("max_radius", c_double),
        ("min_radius", c_double), ("min_lm_diagonal", c_double), ("max_lm_diagonal", c_double), ("eta", c_double),
        ("cam_off", c_void_p), ("slice_off", c_void_p),
        ("slice_base", c_void_p), ("slice_len", c_void_p), ("slot_cam", c_void_p), ("slot_obs", c_void_p),
        ("cam_offsets", c_void_p), ("cam_entries", c_void_p), ("cam_const", c_void_p), ("pt_const", c_void_p),
        ("cameras", c_void_p), ("points", c_void_p), ("cand_cameras", c_void_p), ("cand_points", c_void_p),
        ("jac", c_void_p), ("res", c_void_p), ("point_raw", c_void_p), ("winv", c_void_p), ("winv_ga", c_void_p),
        ("step_points", c_void_p), ("cam_diag", c_void_p), ("precond", c_void_p), ("rhs", c_void_p),
        ("step_cameras", c_void_p), ("cam_acc", c_void_p), ("frames", c_void_p), ("pcg", c_void_p),
        ("result", c_void_p), ("trace", c_void_p), ("queue", c_void_p),
    ]


_PB = ctypes.POINTER(BatchStruct)


class ClusterStruct(ctypes.Structure):
    """ceres_b200_clusters_t: the visibility-cluster preconditioner's index arrays and
    storage (device pointers)."""
    _fields_ = [
        ("num_components", c_int32), ("num_pairs", c_int32), ("max_dim", c_int32), ("tridiagonal", c_int32),
        ("num_elements", c_int64),
        ("pairs", c_void_p), ("entries", c_void_p), ("cam_comp", c_void_p), ("cam_pos", c_void_p),
        ("cam_cluster", c_void_p), ("comp_cams", c_void_p), ("comp_cam_off", c_void_p), ("comp_base", c_void_p),
        ("comp_piv", c_void_p), ("inv", c_void_p), ("piv", c_void_p), ("flags", c_void_p),
    ]


_PC = ctypes.POINTER(ClusterStruct)

# name -> (restype, argtypes); every symbol include/ceres_b200.h declares
SIGNATURES = {
    "ceres_b200_abi_version": (c_int32, []),
    "ceres_b200_ba_struct_bytes": (c_int32, []),
    "ceres_b200_launch_count": (ctypes.c_uint64, []),
    "ceres_b200_scratch_bytes": (c_int32, [_P, ctypes.POINTER(c_int64)]),
    "ceres_b200_ba_evaluate": (c_int32, [_P, c_int32, c_void_p]),
    "ceres_b200_ba_evaluate_noalloc": (c_int32, [_P, c_int32, c_void_p]),
    "ceres_b200_ba_point_assemble": (c_int32, [_P, c_double, c_double, c_double, c_int32, c_void_p]),
    "ceres_b200_ba_camera_assemble": (c_int32, [_P, c_double, c_double, c_double, c_int32, c_int32, c_void_p]),
    "ceres_b200_ba_pcg": (c_int32, [_P, c_int32, c_int32, c_int32, c_double, c_int32, c_void_p]),
    "ceres_b200_ba_pcg_spse": (c_int32, [_P, c_int32, c_int32, c_int32, c_double, c_int32, c_int32, c_double, c_int32,
                                         c_void_p]),
    "ceres_b200_ba_schur_matvec": (c_int32, [_P, c_void_p, c_void_p, c_void_p]),
    "ceres_b200_ba_step": (c_int32, [_P, c_void_p]),
    "ceres_b200_dense_schur_bytes": (c_int32, [_P, ctypes.POINTER(c_int64)]),
    "ceres_b200_ba_dense_schur_solve": (c_int32, [_P, c_void_p, c_void_p]),
    "ceres_b200_dense_cholesky_solve": (c_int32, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    "ceres_b200_batch_struct_bytes": (c_int32, []),
    "ceres_b200_batch_solve": (c_int32, [_PB, c_int32, c_int32, c_int32, c_void_p]),
    "ceres_b200_debug_barrier_timeout": (c_int32, [c_void_p, ctypes.c_uint32, c_void_p]),
    "ceres_b200_ba_schur_matrix": (c_int32, [_P, c_void_p, c_void_p]),
    "ceres_b200_dense_spd_inverse": (c_int32, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    "ceres_b200_clusters_struct_bytes": (c_int32, []),
    "ceres_b200_ba_cluster_factor": (c_int32, [_P, _PC, c_void_p]),
    "ceres_b200_ba_pcg_cluster": (c_int32, [_P, _PC, c_int32, c_int32, c_double, c_int32, c_void_p]),
}

_LIB: ctypes.CDLL | None = None


def library_path() -> Path:
    override = os.environ.get("CERES_B200_LIBRARY")
    return Path(override) if override else _build.library_path()


def load(*, build_if_missing: bool = False) -> ctypes.CDLL:
    """Load the library (once). Raises NativeLibraryError when it is unavailable."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not path.exists() and build_if_missing:
        _build.build()
    if not path.exists():
        raise NativeLibraryError(
            f"{path} is missing: build it with `python -m ceres_torch_cuda_b200.build` (nvcc, sm_100a)")
    try:
        lib = ctypes.CDLL(str(path))
    except OSError as exc:  # pragma: no cover - depends on the host
        raise NativeLibraryError(f"cannot load {path}: {exc}") from exc
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.ceres_b200_abi_version() != ABI_VERSION:
        raise NativeLibraryError(f"{path} has ABI {lib.ceres_b200_abi_version()}, expected {ABI_VERSION}")
    if lib.ceres_b200_ba_struct_bytes() != ctypes.sizeof(BAStruct):
        raise NativeLibraryError("ceres_b200_ba_t layout differs between the library and this binding")
    if lib.ceres_b200_batch_struct_bytes() != ctypes.sizeof(BatchStruct):
        raise NativeLibraryError("ceres_b200_batch_t layout differs between the library and this binding")
    if lib.ceres_b200_clusters_struct_bytes() != ctypes.sizeof(ClusterStruct):
        raise NativeLibraryError("ceres_b200_clusters_t layout differs between the library and this binding")
    _LIB = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc != OK:
        raise NativeLibraryError(f"{what} failed: {_ERRORS.get(rc, rc)}")
