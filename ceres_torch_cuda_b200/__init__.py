"""B200-native (sm_100a) Schur-complement bundle adjustment behind ceres-torch's
``Problem`` / ``solve`` / ``SolverOptions`` / ``register_cuda_sparse_backends``
surface.

    import ceres_torch_cuda_b200 as tc
    tc.register_cuda_sparse_backends(precision="mixed")
    summary = tc.solve(tc.SolverOptions(linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR,
                                        preconditioner_type=tc.PreconditionerType.SCHUR_JACOBI), problem)
"""
from .cuda_backends import (CUDA_BACKEND_NAMES, CudaExtensionInfo, cuda_block_schur, cuda_extension_block_schur,
                            cuda_extension_build_available, cuda_extension_source_paths,
                            cuda_extension_sparse_normal_cholesky, cuda_sparse_normal_cholesky, get_ba_precision,
                            get_cuda_extension_info, get_torch_cuda_backend_info, load_cuda_extension,
                            register_cuda_extension_backends, register_cuda_sparse_backends,
                            torch_cuda_backend_available, unregister_cuda_sparse_backends)
from .batch import BatchSolver, build_batch_layout, solve_batch
from .engine import BAEngine, build_layout
from .linear import (LinearSolverResult, LinearSolverSummary, OptionalBackendUnavailable, clear_optional_backends,
                     get_optional_backend, register_optional_backend, solve_linear_system,
                     unregister_optional_backend)
from .losses import (ArctanLoss, CauchyLoss, ComposedLoss, HuberLoss, LossFunction, LossFunctionWrapper, ScaledLoss,
                     SoftLOneLoss, TolerantLoss, TrivialLoss, TukeyLoss)
from .problem import (BundleAdjustmentProblem, CostFunction, ParameterBlock, Problem, ProblemOptions, ResidualBlock,
                      SnavelyReprojectionError, snavely_project)
from .solver import solve
from .dropin import install
from .covariance import Covariance, CovarianceOptions, CovarianceSummary
from .types import (DYNAMIC, CallbackReturnType, DenseLinearAlgebraLibraryType, DoglegType, IterationSummary,
                    LinearSolverType, LineSearchDirectionType, LineSearchInterpolationType, LineSearchType,
                    LoggingType, MinimizerType, NonlinearConjugateGradientType, PreconditionerType, SolverOptions,
                    SolverSummary, SparseLinearAlgebraLibraryType, TerminationType, TrustRegionStrategyType,
                    VisibilityClusteringType)

__all__ = [name for name in globals() if not name.startswith("_")]
