"""The drop-in on CUDA: a ceres-torch Problem built as ceres-torch's BAL example builds it
(examples/simple_bundle_adjuster.py:82-112, with this package's cost class) on CUDA
tensors, solved by calling ceres-torch's own ``solve`` after
``ceres_torch_cuda_b200.install(ceres_torch)``, must give the reference's recorded
solves (fixtures made by running ceres-torch), and this package's registry entries
must satisfy ceres-torch's backend contract on CUDA tensors
(tests/test_cuda_extensions.py:60-110 of ceres-torch)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import ceres_torch_cuda_b200 as b200
from tests import _golden as G
from tests._reference import reference_module
from tests.test_dropin import _bal_problem

ct = reference_module()
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(ct is None, reason="ceres-torch is not installed in baseline/_ref")]

DEV = "cuda"


def _ref_loss(spec):
    kind = spec[0]
    if kind == "trivial":
        return None
    return {"huber": ct.HuberLoss, "cauchy": ct.CauchyLoss}[kind](float(spec[1]))


@pytest.mark.parametrize("name,precision,rtol", [("ba_small_sparse", "fp64", 1e-9), ("config1_small", "fp64", 1e-9),
                                                 ("ba_cauchy", "fp64", 1e-9), ("ba_cauchy", "mixed", 1e-6),
                                                 ("ba_cluster_tridiagonal", "fp64", 1e-9)])
def test_reference_solve_routes_to_the_gpu_and_matches_its_fixture(name, precision, rtol):
    d = G.load(name)
    meta = d["meta"]
    problem, cams, pts = _bal_problem(d, device=DEV, loss=_ref_loss(G.loss_spec(meta["loss"])))
    opts = ct.SolverOptions(max_num_iterations=meta["max_num_iterations"],
                            linear_solver_type=getattr(ct.LinearSolverType, meta["solver"]),
                            preconditioner_type=getattr(ct.PreconditionerType, meta["preconditioner"]))
    inst = b200.install(ct, precision=precision)
    try:
        lib = b200._lib.load()
        before = lib.ceres_b200_launch_count()
        s = ct.solve(opts, problem)
        launched = lib.ceres_b200_launch_count() - before
    finally:
        inst.uninstall()
    assert inst.routed == 1, inst.last_reason
    assert launched > 0  # the sm_100a kernels ran
    assert isinstance(s, ct.SolverSummary) and s.precision == precision
    assert s.termination_type is getattr(ct.TerminationType, meta["termination"])
    tol_it = 0 if precision == "fp64" else 2
    assert abs(len(s.iterations) - meta["num_iterations"]) <= tol_it
    np.testing.assert_allclose(s.final_cost, meta["final_cost"], rtol=rtol)
    if precision == "fp64":
        np.testing.assert_allclose(cams.cpu().numpy(), d["final_cameras"], rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(pts.cpu().numpy(), d["final_points"], rtol=1e-5, atol=1e-7)


def test_registry_entries_on_cuda_tensors():
    """ceres-torch's backend contract through its own registry on CUDA tensors: the
    normal-equations and block-Schur entries match ceres-torch's dense solvers, and a
    dense ITERATIVE_SCHUR request falls through to block_schur."""
    A = torch.tensor([[3.0, 0.0, 1.0], [0.0, 4.0, -1.0], [2.0, 0.0, 0.0], [0.0, -1.0, 5.0]], dtype=torch.float64,
                     device=DEV)
    expected = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float64, device=DEV)
    b = A @ expected
    damping = torch.tensor([0.1, 0.2, 0.3], dtype=torch.float64, device=DEV)
    A2 = torch.tensor([[2.0, 0.0, 1.0], [0.0, 3.0, -1.0], [1.0, -1.0, 2.0], [0.5, 0.0, 1.0]], dtype=torch.float64,
                      device=DEV)
    b2 = torch.tensor([1.0, -2.0, 0.5, 3.0], dtype=torch.float64, device=DEV)
    inst = b200.install(ct)
    try:
        normal = ct.solve_linear_system(A, b, solver_type=ct.LinearSolverType.SPARSE_NORMAL_CHOLESKY, damping=damping)
        schur = ct.solve_linear_system(A2, b2, solver_type=ct.LinearSolverType.SPARSE_SCHUR, num_eliminate=1)
        iterative = ct.solve_linear_system(A2, b2, solver_type=ct.LinearSolverType.ITERATIVE_SCHUR, num_eliminate=1)
    finally:
        inst.uninstall()
    dense_n = ct.solve_linear_system(A, b, solver_type=ct.LinearSolverType.DENSE_NORMAL_CHOLESKY, damping=damping)
    dense_s = ct.solve_linear_system(A2, b2, solver_type=ct.LinearSolverType.DENSE_SCHUR, num_eliminate=1)
    assert isinstance(normal, ct.LinearSolverResult) and "sm_100a" in normal.summary.message
    torch.testing.assert_close(normal.x, dense_n.x, atol=1e-10, rtol=1e-10)
    assert "sm_100a" in schur.summary.message
    torch.testing.assert_close(schur.x, dense_s.x, atol=1e-10, rtol=1e-10)
    assert "block schur" in iterative.summary.message
    torch.testing.assert_close(iterative.x, dense_s.x, atol=1e-10, rtol=1e-10)
