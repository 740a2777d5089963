"""``solve(options, problem)`` with ceres-torch's signature (solver.py:28-32).

Bundle-adjustment problems (a ``Problem`` of SnavelyReprojectionError blocks or
a ``BundleAdjustmentProblem``) on CUDA tensors with a Schur linear solver run
on the GPU: evaluation, Schur assembly, the linear solve and the LM step are
sm_100a kernels and the trust-region loop of ceres-torch runs on the host over
a 256-byte control block per iteration. Anything else raises
NotImplementedError; there is no CPU path.
"""
from __future__ import annotations

import os
import time

import torch

from . import cuda_backends
from .engine import BAEngine, linear_solver_kind, run_lm
from .problem import BundleAdjustmentProblem, Problem, extract_bundle_adjustment, write_back
from .types import LinearSolverType, MinimizerType, SolverOptions, SolverSummary, TrustRegionStrategyType


def _effective_linear_solver(requested: LinearSolverType) -> LinearSolverType:
    """solver.py:788-795: SPARSE_* requests run their dense counterparts."""
    if requested is LinearSolverType.SPARSE_NORMAL_CHOLESKY:
        return LinearSolverType.DENSE_NORMAL_CHOLESKY
    if requested is LinearSolverType.SPARSE_SCHUR:
        return LinearSolverType.DENSE_SCHUR
    return requested


def _new_summary(options: SolverOptions) -> SolverSummary:
    return SolverSummary(
        minimizer_type=options.minimizer_type,
        linear_solver_type_given=options.linear_solver_type,
        linear_solver_type_used=_effective_linear_solver(options.linear_solver_type),
        trust_region_strategy_type=options.trust_region_strategy_type,
        dogleg_type=options.dogleg_type,
        line_search_direction_type=options.line_search_direction_type,
        line_search_type=options.line_search_type,
        line_search_interpolation_type=options.line_search_interpolation_type,
        nonlinear_conjugate_gradient_type=options.nonlinear_conjugate_gradient_type,
        preconditioner_type=options.preconditioner_type,
        max_lbfgs_rank=options.max_lbfgs_rank,
        dense_linear_algebra_library_type=options.dense_linear_algebra_library_type,
        sparse_linear_algebra_library_type=options.sparse_linear_algebra_library_type,
    )


def _check_supported(options: SolverOptions) -> None:
    if options.minimizer_type is not MinimizerType.TRUST_REGION:
        raise NotImplementedError("the GPU path implements the TRUST_REGION minimizer")
    if options.trust_region_strategy_type is not TrustRegionStrategyType.LEVENBERG_MARQUARDT:
        raise NotImplementedError("the GPU path implements the LEVENBERG_MARQUARDT strategy")
    if options.use_inner_iterations:
        raise NotImplementedError("inner iterations are not implemented on the GPU path")
    if options.check_gradients:
        raise NotImplementedError("check_gradients is not implemented on the GPU path")
    linear_solver_kind(options)


def solve(options: SolverOptions, problem, *, precision: str | None = None, max_refinements: int = 1,
          target_cost: float | None = None, stop_at_target: bool = False, return_engine: bool = False,
          profile: bool = False, autotune: bool | None = None):
    """Solve ``problem`` in place and return the SolverSummary.

    ``precision`` overrides the registered precision ("fp64" or "mixed").
    ``target_cost`` records the wall time at which the best cost first reaches it
    (``summary.time_to_tolerance_in_seconds``); ``stop_at_target`` ends the solve there.
    ``profile`` brackets every library call with CUDA events (no extra
    synchronisation) and puts the per-entry-point device times in
    ``summary.kernel_profile``.
    ``autotune`` (default: the CERES_B200_AUTOTUNE environment variable) picks the
    camera-major copy and the camera work-item length by timing them on this problem
    (``autotune.tune``, cached per size class); the choice is in
    ``summary.kernel_config``.
    """
    if not isinstance(options, SolverOptions):
        from .dropin import options_from

        options = options_from(options)
    options.validate()
    _check_supported(options)
    start = time.perf_counter()
    summary = _new_summary(options)
    prec = precision or cuda_backends.get_ba_precision()
    if isinstance(problem, BundleAdjustmentProblem):
        ba = problem
        cams, pts = ba.cameras, ba.points
        cam_const = ba.camera_constant
        pt_const = ba.point_constant
        obs, ci, pi, loss = ba.observations, ba.camera_index, ba.point_index, ba.loss
        summary.num_parameter_blocks = ba.num_cameras + ba.num_points
        summary.num_parameters = 9 * ba.num_cameras + 3 * ba.num_points
        n_cc = int(cam_const.sum()) if cam_const is not None else 0
        n_pc = int(pt_const.sum()) if pt_const is not None else 0
        summary.num_effective_parameters = 9 * (ba.num_cameras - n_cc) + 3 * (ba.num_points - n_pc)
        summary.num_residual_blocks = ba.num_observations
        summary.num_residuals = 2 * ba.num_observations
        extracted = None
    elif isinstance(problem, Problem) or (hasattr(problem, "residual_blocks") and hasattr(problem, "parameter_blocks")):
        # this package's Problem, or one with ceres-torch's Problem structure
        extracted = extract_bundle_adjustment(problem)
        cams, pts = extracted.cameras, extracted.points
        cam_const, pt_const = extracted.camera_constant, extracted.point_constant
        obs, ci, pi, loss = (extracted.observations, extracted.camera_index, extracted.point_index,
                             extracted.loss)
        summary.num_parameter_blocks = problem.num_parameter_blocks()
        summary.num_parameters = problem.num_parameters()
        summary.num_effective_parameters = problem.num_effective_parameters()
        summary.num_residual_blocks = problem.num_residual_blocks()
        summary.num_residuals = problem.num_residuals()
    else:
        raise TypeError("problem must be a Problem or a BundleAdjustmentProblem")
    if cams.device.type != "cuda":
        raise NotImplementedError("the solver runs on CUDA tensors only; move the parameter blocks to a CUDA device")
    if autotune is None:
        autotune = os.environ.get("CERES_B200_AUTOTUNE", "0") == "1"
    kernel_config = {"camera_copy": None, "item_size": None, "autotuned": False}
    if autotune and obs.shape[0] > 0 and cams.shape[0] > 0:
        from . import autotune as _at

        cfg = _at.tune(cams, pts, obs, ci, pi, loss=loss, camera_constant=cam_const, point_constant=pt_const,
                       precision=prec, options=options)
        kernel_config = dict(cfg.as_dict(), autotuned=True)
        engine = BAEngine(cams, pts, obs, ci, pi, loss=loss, camera_constant=cam_const, point_constant=pt_const,
                          precision=prec, camera_copy=cfg.camera_copy, item_size=cfg.item_size)
    else:
        engine = BAEngine(cams, pts, obs, ci, pi, loss=loss, camera_constant=cam_const, point_constant=pt_const,
                          precision=prec)
    kernel_config["camera_copy"] = engine.camera_copy
    kernel_config["item_size"] = engine.item_size
    n_active = summary.num_effective_parameters
    if profile:
        engine.enable_profiling()
    summary.preprocessor_time_in_seconds = time.perf_counter() - start

    def on_state(eng, which):
        c, p = eng.get_parameters(which)
        _store(problem, extracted, c, p)

    result = run_lm(engine, options, summary, start=start, num_active_columns=n_active,
                    max_refinements=max_refinements, target_cost=target_cost, stop_at_target=stop_at_target,
                    on_state=on_state)
    c, p = engine.get_parameters("current")
    _store(problem, extracted, c, p)
    torch.cuda.current_stream(engine.device).synchronize()
    summary.total_time_in_seconds = time.perf_counter() - start
    summary.time_to_tolerance_in_seconds = result.time_to_tolerance
    summary.precision = prec
    summary.kernel_config = kernel_config
    if profile:
        summary.kernel_profile = engine.profile_report()
    if return_engine:
        return summary, engine
    return summary


def _store(problem, extracted, cams: torch.Tensor, pts: torch.Tensor) -> None:
    with torch.no_grad():
        if extracted is None:
            problem.cameras.copy_(cams.to(problem.cameras.dtype))
            problem.points.copy_(pts.to(problem.points.dtype))
        else:
            write_back(extracted.camera_blocks, cams)
            write_back(extracted.point_blocks, pts)
