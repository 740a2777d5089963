"""The drop-in behind ceres-torch's own API, on CPU: option, loss and summary
conversion, registry entries with ceres-torch's calling convention, and the solve
pre-dispatch, which leaves everything that is not bundle adjustment on CUDA to
ceres-torch's own solver (checked here on CPU tensors, where ceres-torch's result
must come out unchanged). The CUDA side is tests/test_gpu_dropin.py."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import ceres_torch_cuda_b200 as b200
from ceres_torch_cuda_b200 import dropin
from tests import _golden as G
from tests._reference import reference_module

ct = reference_module()
pytestmark = pytest.mark.skipif(ct is None, reason="ceres-torch is not installed in baseline/_ref")


def _bal_problem(d, device="cpu", loss=None):
    """ceres-torch's own Problem built as its BAL example does
    (examples/simple_bundle_adjuster.py:82-112), with this package's cost class."""
    cams = torch.tensor(d["cameras"], dtype=torch.float64, device=device)
    pts = torch.tensor(d["points"], dtype=torch.float64, device=device)
    problem = ct.Problem()
    cb = [cams[i] for i in range(cams.shape[0])]
    pb = [pts[i] for i in range(pts.shape[0])]
    for i, c in enumerate(cb):
        problem.AddParameterBlock(c)
        if i in d["meta"]["constant_cameras"]:
            problem.SetParameterBlockConstant(c)
    for p in pb:
        problem.AddParameterBlock(p)
        problem.SetParameterBlockOrderingGroup(p, 0)
    for c, p, o in zip(d["camera_index"].tolist(), d["point_index"].tolist(), d["observations"]):
        problem.AddResidualBlock(b200.SnavelyReprojectionError(o[0], o[1]), loss, [cb[c], pb[p]])
    return problem, cams, pts


def test_reference_options_convert_by_member_name():
    o = ct.SolverOptions(linear_solver_type=ct.LinearSolverType.ITERATIVE_SCHUR,
                         preconditioner_type=ct.PreconditionerType.SCHUR_JACOBI, eta=0.05, max_num_iterations=7)
    for own in (b200.SolverOptions(**vars(o)), dropin.options_from(o)):
        assert own.linear_solver_type is b200.LinearSolverType.ITERATIVE_SCHUR
        assert own.preconditioner_type is b200.PreconditionerType.SCHUR_JACOBI
        assert own.minimizer_type is b200.MinimizerType.TRUST_REGION
        assert own.eta == 0.05 and own.max_num_iterations == 7
        own.validate()
        from ceres_torch_cuda_b200.engine import linear_solver_kind

        assert linear_solver_kind(own) == "iterative"
    with pytest.raises(ValueError, match="linear_solver_type"):
        b200.SolverOptions(linear_solver_type="NOT_A_SOLVER")


def test_reference_losses_convert():
    from ceres_torch_cuda_b200.losses import as_loss, device_loss

    assert as_loss(ct.CauchyLoss(2.0)) == b200.CauchyLoss(2.0)
    assert as_loss(ct.TolerantLoss(1.0, 0.5)) == b200.TolerantLoss(1.0, 0.5)
    assert device_loss(ct.HuberLoss(1.5)) == device_loss(b200.HuberLoss(1.5))
    composed = ct.ScaledLoss(ct.ComposedLoss(ct.CauchyLoss(1.0), ct.HuberLoss(2.0)), 3.0)
    assert device_loss(composed) == device_loss(b200.ScaledLoss(b200.ComposedLoss(b200.CauchyLoss(1.0),
                                                                                  b200.HuberLoss(2.0)), 3.0))
    assert as_loss(None) is None


def test_summary_converts_to_the_reference_classes():
    s = b200.SolverSummary(termination_type=b200.TerminationType.CONVERGENCE, message="Function tolerance reached.",
                           initial_cost=10.0, final_cost=1.0,
                           linear_solver_type_given=b200.LinearSolverType.SPARSE_SCHUR,
                           linear_solver_type_used=b200.LinearSolverType.DENSE_SCHUR, precision="mixed")
    s.iterations.append(b200.IterationSummary(iteration=0, cost=10.0, step_is_valid=True))
    r = dropin.summary_to(ct, s)
    assert isinstance(r, ct.SolverSummary)
    assert r.termination_type is ct.TerminationType.CONVERGENCE
    assert r.linear_solver_type_used is ct.LinearSolverType.DENSE_SCHUR
    assert isinstance(r.iterations[0], ct.IterationSummary) and r.iterations[0].cost == 10.0
    assert r.precision == "mixed" and r.IsSolutionUsable()


def test_install_registers_every_name_and_uninstall_restores():
    original = ct.solve
    inst = b200.install(ct)
    try:
        for name in ("sparse_normal_cholesky", "sparse_cholesky", "sparse_schur", "block_schur", "iterative_schur"):
            entry = ct.get_optional_backend(name)
            assert entry is not None and getattr(entry, "_ceres_b200", False), name
        import ceres_torch.solver as ref_solver

        assert ct.solve is not original and ref_solver.solve is ct.solve
        assert ct.solve.__wrapped__ is original
    finally:
        inst.uninstall()
    assert ct.solve is original
    assert ct.get_optional_backend("iterative_schur") is None


def test_registry_entries_follow_the_reference_contract_on_cpu():
    """CPU tensors: this package's entries report themselves unavailable with
    ceres-torch's own exception class, so ceres-torch falls through to its own solver
    (tests/test_cuda_extensions.py:26-34 of ceres-torch, through the registry)."""
    A = torch.tensor([[2.0, 0.0, 1.0], [0.0, 3.0, -1.0], [1.0, -1.0, 2.0], [0.5, 0.0, 1.0]], dtype=torch.float64)
    b = torch.tensor([1.0, -2.0, 0.5, 3.0], dtype=torch.float64)
    inst = b200.install(ct)
    try:
        with pytest.raises(ct.OptionalBackendUnavailable, match="CUDA tensor"):
            ct.get_optional_backend("block_schur")(A, b, num_eliminate=1)
        with pytest.raises(ct.OptionalBackendUnavailable):
            ct.get_optional_backend("iterative_schur")(A, b, num_eliminate=1)
        via_registry = ct.solve_linear_system(A, b, solver_type=ct.LinearSolverType.SPARSE_SCHUR, num_eliminate=1)
    finally:
        inst.uninstall()
    dense = ct.solve_linear_system(A, b, solver_type=ct.LinearSolverType.DENSE_SCHUR, num_eliminate=1)
    torch.testing.assert_close(via_registry.x, dense.x, atol=1e-12, rtol=1e-12)


def test_route_decisions():
    d = G.load("ba_fixed_cameras")
    problem, _, _ = _bal_problem(d)
    ok, why = dropin.route(ct.SolverOptions(linear_solver_type=ct.LinearSolverType.DENSE_SCHUR), problem)
    assert not ok and "CUDA" in why
    ok, why = dropin.route(ct.SolverOptions(linear_solver_type=ct.LinearSolverType.DENSE_QR), problem)
    assert not ok and "Schur" in why
    ok, why = dropin.route(ct.SolverOptions(linear_solver_type=ct.LinearSolverType.ITERATIVE_SCHUR,
                                            preconditioner_type=ct.PreconditionerType.CLUSTER_TRIDIAGONAL), problem)
    assert not ok and "CUDA" in why  # the preconditioner is a GPU one; the tensors are not on a GPU
    ok, why = dropin.route(ct.SolverOptions(linear_solver_type=ct.LinearSolverType.CGNR,
                                            preconditioner_type=ct.PreconditionerType.SUBSET), problem)
    assert not ok and "Schur" in why
    ok, why = dropin.route(ct.SolverOptions(minimizer_type=ct.MinimizerType.LINE_SEARCH,
                                            linear_solver_type=ct.LinearSolverType.DENSE_SCHUR), problem)
    assert not ok
    # the extraction the GPU path uses reads ceres-torch's Problem (the cost class
    # behind ceres-torch's CallableCostFunction wrapper, its loss objects)
    from ceres_torch_cuda_b200.problem import extract_bundle_adjustment

    c = G.load("ba_cauchy")
    cp, _, _ = _bal_problem(c, loss=ct.CauchyLoss(2.0))
    ex = extract_bundle_adjustment(cp)
    assert ex.loss == b200.CauchyLoss(2.0)
    np.testing.assert_array_equal(ex.observations.numpy(), c["observations"])
    np.testing.assert_array_equal(ex.camera_index.numpy(), c["camera_index"])


def test_cpu_problem_runs_the_reference_solver_unchanged():
    """The pre-dispatch sends a CPU problem to ceres-torch's own solver: the result is
    the reference's recorded solve of the same fixture."""
    d = G.load("ba_fixed_cameras")
    meta = d["meta"]
    problem, cams, pts = _bal_problem(d)
    inst = b200.install(ct)
    try:
        s = ct.solve(ct.SolverOptions(max_num_iterations=meta["max_num_iterations"],
                                      linear_solver_type=ct.LinearSolverType.DENSE_SCHUR), problem)
    finally:
        inst.uninstall()
    assert inst.routed == 0 and inst.fell_through == 1
    assert isinstance(s, ct.SolverSummary)
    assert len(s.iterations) == meta["num_iterations"]
    np.testing.assert_allclose(s.final_cost, meta["final_cost"], rtol=1e-9)
    np.testing.assert_allclose(pts.numpy(), d["final_points"], rtol=1e-5, atol=1e-7)
