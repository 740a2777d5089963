"""Option, enum and summary types with the same names, fields and defaults as
ceres-torch's ``types.py`` (enums :16-131, IterationSummary :135-161,
SolverOptions :165-357, SolverSummary :361-468), so user code written against
ceres-torch keeps working. Enum values are the member names, as in ceres-torch.
"""
from __future__ import annotations

from dataclasses import dataclass, field, fields
from enum import Enum
from typing import Callable


class _NamedEnum(Enum):
    def __str__(self) -> str:
        return self.value


def _enum(name: str, members: str) -> type:
    return _NamedEnum(name, [(m, m) for m in members.split()])


LinearSolverType = _enum("LinearSolverType", "DENSE_NORMAL_CHOLESKY DENSE_QR SPARSE_NORMAL_CHOLESKY DENSE_SCHUR "
                                             "SPARSE_SCHUR ITERATIVE_SCHUR CGNR")
PreconditionerType = _enum("PreconditionerType", "IDENTITY JACOBI SCHUR_JACOBI SCHUR_POWER_SERIES_EXPANSION "
                                                 "CLUSTER_JACOBI CLUSTER_TRIDIAGONAL SUBSET")
VisibilityClusteringType = _enum("VisibilityClusteringType", "CANONICAL_VIEWS SINGLE_LINKAGE")
SparseLinearAlgebraLibraryType = _enum("SparseLinearAlgebraLibraryType",
                                       "SUITE_SPARSE EIGEN_SPARSE ACCELERATE_SPARSE CUDA_SPARSE NO_SPARSE")
LinearSolverOrderingType = _enum("LinearSolverOrderingType", "AMD NESDIS")
DenseLinearAlgebraLibraryType = _enum("DenseLinearAlgebraLibraryType", "EIGEN LAPACK CUDA")
LoggingType = _enum("LoggingType", "SILENT PER_MINIMIZER_ITERATION")
MinimizerType = _enum("MinimizerType", "LINE_SEARCH TRUST_REGION")
LineSearchDirectionType = _enum("LineSearchDirectionType", "STEEPEST_DESCENT NONLINEAR_CONJUGATE_GRADIENT LBFGS BFGS")
NonlinearConjugateGradientType = _enum("NonlinearConjugateGradientType",
                                       "FLETCHER_REEVES POLAK_RIBIERE HESTENES_STIEFEL")
LineSearchType = _enum("LineSearchType", "ARMIJO WOLFE")
TrustRegionStrategyType = _enum("TrustRegionStrategyType", "LEVENBERG_MARQUARDT DOGLEG")
DoglegType = _enum("DoglegType", "TRADITIONAL_DOGLEG SUBSPACE_DOGLEG")
TerminationType = _enum("TerminationType", "CONVERGENCE NO_CONVERGENCE FAILURE USER_SUCCESS USER_FAILURE")
CallbackReturnType = _enum("CallbackReturnType", "SOLVER_CONTINUE SOLVER_ABORT SOLVER_TERMINATE_SUCCESSFULLY")
DumpFormatType = _enum("DumpFormatType", "CONSOLE TEXTFILE")
NumericDiffMethodType = _enum("NumericDiffMethodType", "CENTRAL FORWARD RIDDERS")
LineSearchInterpolationType = _enum("LineSearchInterpolationType", "BISECTION QUADRATIC CUBIC")
CovarianceAlgorithmType = _enum("CovarianceAlgorithmType", "DENSE_SVD SPARSE_QR")

DYNAMIC = -1


@dataclass
class IterationSummary:
    iteration: int = 0
    step_is_valid: bool = False
    step_is_nonmonotonic: bool = False
    step_is_successful: bool = False
    cost: float = 0.0
    cost_change: float = 0.0
    gradient_max_norm: float = 0.0
    gradient_norm: float = 0.0
    step_norm: float = 0.0
    relative_decrease: float = 0.0
    trust_region_radius: float = 0.0
    eta: float = 0.0
    step_size: float = 0.0
    line_search_function_evaluations: int = 0
    line_search_gradient_evaluations: int = 0
    line_search_iterations: int = 0
    line_search_direction_restarts: int = 0
    linear_solver_iterations: int = 0
    residual_evaluation_time_in_seconds: float = 0.0
    jacobian_evaluation_time_in_seconds: float = 0.0
    linear_solver_time_in_seconds: float = 0.0
    line_search_time_in_seconds: float = 0.0
    inner_iteration_time_in_seconds: float = 0.0
    iteration_time_in_seconds: float = 0.0
    step_solver_time_in_seconds: float = 0.0
    cumulative_time_in_seconds: float = 0.0


@dataclass
class SolverOptions:
    minimizer_type: MinimizerType = MinimizerType.TRUST_REGION
    line_search_direction_type: LineSearchDirectionType = LineSearchDirectionType.LBFGS
    line_search_type: LineSearchType = LineSearchType.WOLFE
    nonlinear_conjugate_gradient_type: NonlinearConjugateGradientType = NonlinearConjugateGradientType.FLETCHER_REEVES
    max_lbfgs_rank: int = 20
    use_approximate_eigenvalue_bfgs_scaling: bool = False
    line_search_interpolation_type: LineSearchInterpolationType = LineSearchInterpolationType.CUBIC
    min_line_search_step_size: float = 1e-9
    line_search_sufficient_function_decrease: float = 1e-4
    max_line_search_step_contraction: float = 1e-3
    min_line_search_step_contraction: float = 0.6
    max_num_line_search_step_size_iterations: int = 20
    max_num_line_search_direction_restarts: int = 5
    line_search_sufficient_curvature_decrease: float = 0.9
    max_line_search_step_expansion: float = 10.0
    trust_region_strategy_type: TrustRegionStrategyType = TrustRegionStrategyType.LEVENBERG_MARQUARDT
    dogleg_type: DoglegType = DoglegType.TRADITIONAL_DOGLEG
    use_nonmonotonic_steps: bool = False
    max_consecutive_nonmonotonic_steps: int = 5
    max_num_iterations: int = 50
    max_solver_time_in_seconds: float = 1e9
    num_threads: int = 1
    initial_trust_region_radius: float = 1e4
    max_trust_region_radius: float = 1e16
    min_trust_region_radius: float = 1e-32
    min_relative_decrease: float = 1e-3
    min_lm_diagonal: float = 1e-6
    max_lm_diagonal: float = 1e32
    max_num_consecutive_invalid_steps: int = 5
    function_tolerance: float = 1e-6
    gradient_tolerance: float = 1e-10
    parameter_tolerance: float = 1e-8
    linear_solver_type: LinearSolverType = LinearSolverType.DENSE_QR
    preconditioner_type: PreconditionerType = PreconditionerType.JACOBI
    visibility_clustering_type: VisibilityClusteringType = VisibilityClusteringType.CANONICAL_VIEWS
    dense_linear_algebra_library_type: DenseLinearAlgebraLibraryType = DenseLinearAlgebraLibraryType.EIGEN
    sparse_linear_algebra_library_type: SparseLinearAlgebraLibraryType = SparseLinearAlgebraLibraryType.NO_SPARSE
    linear_solver_ordering_type: LinearSolverOrderingType = LinearSolverOrderingType.AMD
    use_explicit_schur_complement: bool = False
    dynamic_sparsity: bool = False
    use_mixed_precision_solves: bool = False
    max_num_refinement_iterations: int = 0
    min_linear_solver_iterations: int = 0
    max_linear_solver_iterations: int = 500
    max_num_spse_iterations: int = 5
    use_spse_initialization: bool = False
    spse_tolerance: float = 0.1
    eta: float = 1e-1
    jacobi_scaling: bool = True
    use_inner_iterations: bool = False
    inner_iteration_tolerance: float = 1e-3
    logging_type: LoggingType = LoggingType.PER_MINIMIZER_ITERATION
    minimizer_progress_to_stdout: bool = False
    check_gradients: bool = False
    gradient_check_relative_precision: float = 1e-8
    gradient_check_numeric_derivative_relative_step_size: float = 1e-6
    update_state_every_iteration: bool = False
    callbacks: list[Callable[[IterationSummary], CallbackReturnType]] = field(default_factory=list)

    def __post_init__(self) -> None:
        # enum members of another module with the same member names (ceres-torch's own
        # SolverOptions passed field by field) become this module's members
        for f in fields(self):
            default = f.default
            if isinstance(default, Enum):
                v = getattr(self, f.name)
                if not isinstance(v, type(default)):
                    try:
                        setattr(self, f.name, type(default)[getattr(v, "name", str(v))])
                    except KeyError as exc:
                        raise ValueError(f"{f.name}: {v!r} is not a {type(default).__name__} member") from exc

    def _rules(self):
        """(condition, message) pairs; the messages are the ones ceres-torch raises."""
        ls_min = 0 if self.minimizer_type is MinimizerType.TRUST_REGION else 1
        cg = self.check_gradients
        yield self.max_num_iterations >= 0, "max_num_iterations must be >= 0"
        yield self.max_solver_time_in_seconds >= 0, "max_solver_time_in_seconds must be >= 0"
        yield self.function_tolerance >= 0, "function_tolerance must be >= 0"
        yield self.gradient_tolerance >= 0, "gradient_tolerance must be >= 0"
        yield self.parameter_tolerance >= 0, "parameter_tolerance must be >= 0"
        yield self.num_threads > 0, "num_threads must be > 0"
        yield (not cg) or self.gradient_check_relative_precision > 0, \
            "gradient_check_relative_precision must be > 0 when check_gradients is enabled"
        yield (not cg) or self.gradient_check_numeric_derivative_relative_step_size > 0, \
            "gradient_check_numeric_derivative_relative_step_size must be > 0 when check_gradients is enabled"
        yield self.initial_trust_region_radius > 0, "initial_trust_region_radius must be > 0"
        yield self.min_trust_region_radius > 0, "min_trust_region_radius must be > 0"
        yield self.max_trust_region_radius > 0, "max_trust_region_radius must be > 0"
        yield (self.min_trust_region_radius <= self.initial_trust_region_radius <= self.max_trust_region_radius), \
            "trust region radii must satisfy min <= initial <= max"
        yield self.min_relative_decrease >= 0, "min_relative_decrease must be >= 0"
        yield self.min_lm_diagonal >= 0, "min_lm_diagonal must be >= 0"
        yield self.max_lm_diagonal >= 0, "max_lm_diagonal must be >= 0"
        yield self.min_lm_diagonal <= self.max_lm_diagonal, "min_lm_diagonal must be <= max_lm_diagonal"
        yield self.max_num_consecutive_invalid_steps >= 0, "max_num_consecutive_invalid_steps must be >= 0"
        yield self.eta > 0, "eta must be > 0"
        yield self.min_linear_solver_iterations >= 0, "min_linear_solver_iterations must be >= 0"
        yield self.max_linear_solver_iterations >= 0, "max_linear_solver_iterations must be >= 0"
        yield self.min_linear_solver_iterations <= self.max_linear_solver_iterations, \
            "min_linear_solver_iterations must be <= max_linear_solver_iterations"
        yield (not self.use_inner_iterations) or self.inner_iteration_tolerance >= 0, \
            "inner_iteration_tolerance must be >= 0 when use_inner_iterations is enabled"
        yield (not self.use_nonmonotonic_steps) or self.max_consecutive_nonmonotonic_steps > 0, \
            "max_consecutive_nonmonotonic_steps must be > 0 when use_nonmonotonic_steps is enabled"
        yield self.max_lbfgs_rank > 0, "max_lbfgs_rank must be > 0"
        yield self.min_line_search_step_size > 0, "min_line_search_step_size must be > 0"
        yield self.max_line_search_step_contraction > 0, "max_line_search_step_contraction must be > 0"
        yield self.max_line_search_step_contraction < 1, "max_line_search_step_contraction must be < 1"
        yield self.max_line_search_step_contraction < self.min_line_search_step_contraction, \
            "max_line_search_step_contraction must be < min_line_search_step_contraction"
        yield self.min_line_search_step_contraction <= 1, "min_line_search_step_contraction must be <= 1"
        yield self.max_num_line_search_step_size_iterations >= ls_min, \
            "max_num_line_search_step_size_iterations is too small for the minimizer type"
        yield self.max_num_line_search_direction_restarts >= 0, "max_num_line_search_direction_restarts must be >= 0"
        yield self.line_search_sufficient_function_decrease > 0, "line_search_sufficient_function_decrease must be > 0"
        yield self.line_search_sufficient_function_decrease < self.line_search_sufficient_curvature_decrease, \
            "line_search_sufficient_function_decrease must be < line_search_sufficient_curvature_decrease"
        yield self.line_search_sufficient_curvature_decrease < 1, "line_search_sufficient_curvature_decrease must be < 1"
        yield self.max_line_search_step_expansion > 1, "max_line_search_step_expansion must be > 1"
        yield self.max_num_refinement_iterations >= 0, "max_num_refinement_iterations must be >= 0"
        lst = self.linear_solver_type
        yield not (self.trust_region_strategy_type is TrustRegionStrategyType.DOGLEG
                   and lst in (LinearSolverType.CGNR, LinearSolverType.ITERATIVE_SCHUR)), \
            "DOGLEG only supports exact factorization based linear solvers"
        yield not (self.line_search_direction_type in (LineSearchDirectionType.BFGS, LineSearchDirectionType.LBFGS)
                   and self.line_search_type is not LineSearchType.WOLFE), \
            "line_search_type must be WOLFE when using BFGS or LBFGS"
        yield not (lst is LinearSolverType.DENSE_QR and self.use_mixed_precision_solves), \
            "use_mixed_precision_solves cannot be used with DENSE_QR"
        yield not (lst in (LinearSolverType.DENSE_SCHUR, LinearSolverType.SPARSE_SCHUR,
                           LinearSolverType.ITERATIVE_SCHUR, LinearSolverType.CGNR) and self.dynamic_sparsity), \
            "dynamic_sparsity is only supported with SPARSE_NORMAL_CHOLESKY"
        if lst is LinearSolverType.ITERATIVE_SCHUR:
            if self.use_explicit_schur_complement:
                yield self.preconditioner_type is PreconditionerType.SCHUR_JACOBI, \
                    "use_explicit_schur_complement only supports SCHUR_JACOBI"
                yield not self.use_spse_initialization, \
                    "use_explicit_schur_complement does not support use_spse_initialization"
            if self.use_spse_initialization or self.preconditioner_type is PreconditionerType.SCHUR_POWER_SERIES_EXPANSION:
                yield self.max_num_spse_iterations >= 1, "max_num_spse_iterations must be >= 1"
                yield self.spse_tolerance >= 0, "spse_tolerance must be >= 0"
            yield not self.use_mixed_precision_solves, "use_mixed_precision_solves cannot be used with ITERATIVE_SCHUR"
            yield self.preconditioner_type is not PreconditionerType.SUBSET, \
                "SUBSET preconditioner cannot be used with ITERATIVE_SCHUR"
        if lst is LinearSolverType.CGNR:
            yield self.preconditioner_type in (PreconditionerType.IDENTITY, PreconditionerType.JACOBI,
                                               PreconditionerType.SUBSET), \
                "CGNR only supports IDENTITY, JACOBI, or SUBSET preconditioners"
            yield not self.use_mixed_precision_solves, "use_mixed_precision_solves cannot be used with CGNR"

    def validate(self) -> None:
        for ok, message in self._rules():
            if not ok:
                raise ValueError(message)


@dataclass
class SolverSummary:
    minimizer_type: MinimizerType = MinimizerType.TRUST_REGION
    termination_type: TerminationType = TerminationType.FAILURE
    message: str = "torch_ceres.solve was not called."
    initial_cost: float = -1.0
    final_cost: float = -1.0
    fixed_cost: float = 0.0
    iterations: list[IterationSummary] = field(default_factory=list)
    num_successful_steps: int = 0
    num_unsuccessful_steps: int = 0
    num_residual_evaluations: int = 0
    num_jacobian_evaluations: int = 0
    num_linear_solves: int = 0
    num_inner_iteration_steps: int = 0
    num_line_search_steps: int = 0
    num_line_search_function_evaluations: int = 0
    num_line_search_gradient_evaluations: int = 0
    num_line_search_direction_restarts: int = 0
    line_search_total_time_in_seconds: float = 0.0
    preprocessor_time_in_seconds: float = 0.0
    minimizer_time_in_seconds: float = 0.0
    postprocessor_time_in_seconds: float = 0.0
    residual_evaluation_time_in_seconds: float = 0.0
    jacobian_evaluation_time_in_seconds: float = 0.0
    linear_solver_time_in_seconds: float = 0.0
    inner_iteration_time_in_seconds: float = 0.0
    total_time_in_seconds: float = 0.0
    num_parameter_blocks: int = 0
    num_parameters: int = 0
    num_effective_parameters: int = 0
    num_residual_blocks: int = 0
    num_residuals: int = 0
    linear_solver_type_given: LinearSolverType = LinearSolverType.DENSE_QR
    linear_solver_type_used: LinearSolverType = LinearSolverType.DENSE_QR
    trust_region_strategy_type: TrustRegionStrategyType = TrustRegionStrategyType.LEVENBERG_MARQUARDT
    dogleg_type: DoglegType = DoglegType.TRADITIONAL_DOGLEG
    line_search_direction_type: LineSearchDirectionType = LineSearchDirectionType.LBFGS
    line_search_type: LineSearchType = LineSearchType.WOLFE
    line_search_interpolation_type: LineSearchInterpolationType = LineSearchInterpolationType.CUBIC
    nonlinear_conjugate_gradient_type: NonlinearConjugateGradientType = NonlinearConjugateGradientType.FLETCHER_REEVES
    preconditioner_type: PreconditionerType = PreconditionerType.JACOBI
    max_lbfgs_rank: int = 20
    dense_linear_algebra_library_type: DenseLinearAlgebraLibraryType = DenseLinearAlgebraLibraryType.EIGEN
    sparse_linear_algebra_library_type: SparseLinearAlgebraLibraryType = SparseLinearAlgebraLibraryType.NO_SPARSE
    # GPU-path additions: the arithmetic of the Schur solve and, when a target
    # cost was given, the wall time until the best cost first reached it
    precision: str = "fp64"
    time_to_tolerance_in_seconds: float | None = None
    kernel_profile: dict | None = None
    kernel_config: dict | None = None   # camera-major copy and work-item length used (autotune.py)

    def IsSolutionUsable(self) -> bool:  # noqa: N802 - ceres-torch API name
        return self.termination_type in (TerminationType.CONVERGENCE, TerminationType.NO_CONVERGENCE,
                                         TerminationType.USER_SUCCESS)

    def BriefReport(self) -> str:  # noqa: N802
        return (f"ceres-torch Solver Report: Iterations: {len(self.iterations)}, "
                f"Initial cost: {self.initial_cost:.6e}, Final cost: {self.final_cost:.6e}, "
                f"Termination: {self.termination_type.value}")

    def FullReport(self) -> str:  # noqa: N802
        rows = [
            ("Minimizer", self.minimizer_type.value), ("Linear solver", self.linear_solver_type_used.value),
            ("Preconditioner", self.preconditioner_type.value),
            ("Trust region strategy", self.trust_region_strategy_type.value), ("Dogleg type", self.dogleg_type.value),
            ("Line search direction", self.line_search_direction_type.value),
            ("Line search type", self.line_search_type.value),
            ("Line search interpolation", self.line_search_interpolation_type.value),
            ("Nonlinear conjugate gradient", self.nonlinear_conjugate_gradient_type.value),
            ("LBFGS rank", self.max_lbfgs_rank),
            ("Dense linear algebra library", self.dense_linear_algebra_library_type.value),
            ("Sparse linear algebra library", self.sparse_linear_algebra_library_type.value),
            ("Parameter blocks", self.num_parameter_blocks), ("Parameters", self.num_parameters),
            ("Effective parameters", self.num_effective_parameters), ("Residual blocks", self.num_residual_blocks),
            ("Residuals", self.num_residuals), ("Initial cost", f"{self.initial_cost:.12e}"),
            ("Final cost", f"{self.final_cost:.12e}"), ("Fixed cost", f"{self.fixed_cost:.12e}"),
            ("Successful steps", self.num_successful_steps), ("Unsuccessful steps", self.num_unsuccessful_steps),
            ("Linear solves", self.num_linear_solves), ("Inner iteration steps", self.num_inner_iteration_steps),
            ("Line search steps", self.num_line_search_steps),
            ("Line search function evaluations", self.num_line_search_function_evaluations),
            ("Line search gradient evaluations", self.num_line_search_gradient_evaluations),
            ("Line search direction restarts", self.num_line_search_direction_restarts),
            ("Residual evaluation time (s)", f"{self.residual_evaluation_time_in_seconds:.6f}"),
            ("Jacobian evaluation time (s)", f"{self.jacobian_evaluation_time_in_seconds:.6f}"),
            ("Linear solver time (s)", f"{self.linear_solver_time_in_seconds:.6f}"),
            ("Line search time (s)", f"{self.line_search_total_time_in_seconds:.6f}"),
            ("Inner iteration time (s)", f"{self.inner_iteration_time_in_seconds:.6f}"),
            ("Preprocessor time (s)", f"{self.preprocessor_time_in_seconds:.6f}"),
            ("Minimizer time (s)", f"{self.minimizer_time_in_seconds:.6f}"),
            ("Postprocessor time (s)", f"{self.postprocessor_time_in_seconds:.6f}"),
            ("Total time (s)", f"{self.total_time_in_seconds:.6f}"),
            ("Termination", f"{self.termination_type.value} ({self.message})"),
        ]
        return "\n".join(["Solver Summary (ceres-torch)", ""] + [f"{k}: {v}" for k, v in rows])
