"""Host-side behaviour of the ceres-torch-compatible surface (no GPU needed):
option validation, the backend registry contract, loss functions, the LM
radius/step-quality logic, problem recognition and error paths."""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import ceres_torch_cuda_b200 as tc
from ceres_torch_cuda_b200.engine import _LMRadius, _StepEvaluator
from ceres_torch_cuda_b200.problem import extract_bundle_adjustment, write_back
from ceres_torch_cuda_b200.solver import _effective_linear_solver


def test_solver_options_defaults_and_validation_messages():
    o = tc.SolverOptions()
    assert o.eta == 0.1 and o.max_linear_solver_iterations == 500 and o.initial_trust_region_radius == 1e4
    assert o.linear_solver_type is tc.LinearSolverType.DENSE_QR and o.max_num_iterations == 50
    o.validate()
    with pytest.raises(ValueError, match="use_mixed_precision_solves cannot be used with ITERATIVE_SCHUR"):
        tc.SolverOptions(linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR, use_mixed_precision_solves=True).validate()
    with pytest.raises(ValueError, match="eta must be > 0"):
        tc.SolverOptions(eta=0.0).validate()
    with pytest.raises(ValueError, match="DOGLEG only supports exact factorization"):
        tc.SolverOptions(trust_region_strategy_type=tc.TrustRegionStrategyType.DOGLEG,
                         linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR).validate()
    with pytest.raises(ValueError, match="SUBSET preconditioner cannot be used with ITERATIVE_SCHUR"):
        tc.SolverOptions(linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR,
                         preconditioner_type=tc.PreconditionerType.SUBSET).validate()


def test_enum_values_are_member_names():
    assert tc.LinearSolverType.SPARSE_SCHUR.value == "SPARSE_SCHUR"
    assert str(tc.PreconditionerType.SCHUR_JACOBI) == "SCHUR_JACOBI"
    assert _effective_linear_solver(tc.LinearSolverType.SPARSE_SCHUR) is tc.LinearSolverType.DENSE_SCHUR
    assert _effective_linear_solver(tc.LinearSolverType.ITERATIVE_SCHUR) is tc.LinearSolverType.ITERATIVE_SCHUR


def test_summary_reports():
    s = tc.SolverSummary(termination_type=tc.TerminationType.CONVERGENCE, initial_cost=2.0, final_cost=1.0)
    assert s.IsSolutionUsable()
    assert "Termination: CONVERGENCE" in s.BriefReport()
    rep = s.FullReport()
    assert "Preconditioner" in rep and "Preprocessor time" in rep and "Inner iteration steps" in rep


def test_registry_passes_all_options_to_backend():
    """Mirrors the reference's backend contract test: every keyword reaches the backend."""
    A = torch.tensor([[2.0, 0.0, 1.0], [0.0, 3.0, -1.0], [1.0, 1.0, 2.0]], dtype=torch.float64)
    b = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float64)
    captured = []

    def backend(A, b, **kwargs):
        captured.append(kwargs)
        return torch.linalg.lstsq(A, b).solution.reshape(-1)

    tc.register_optional_backend("iterative_schur", backend)
    try:
        result = tc.solve_linear_system(A, b, solver_type=tc.LinearSolverType.ITERATIVE_SCHUR, num_eliminate=1,
                                        min_iterations=2, max_iterations=7, tolerance=1e-5,
                                        preconditioner_type=tc.PreconditionerType.SCHUR_POWER_SERIES_EXPANSION,
                                        block_sizes=[1, 2], max_num_spse_iterations=4, use_spse_initialization=True,
                                        spse_tolerance=0.25)
    finally:
        tc.unregister_optional_backend("iterative_schur")
    kw = captured[0]
    assert kw["solver_type"] is tc.LinearSolverType.ITERATIVE_SCHUR and kw["num_eliminate"] == 1
    assert kw["min_iterations"] == 2 and kw["max_iterations"] == 7 and kw["tolerance"] == 1e-5
    assert kw["block_sizes"] == [1, 2] and kw["use_spse_initialization"] is True and kw["spse_tolerance"] == 0.25
    assert "optional iterative_schur backend" in result.summary.message


def test_registry_fallthrough_and_typeerror_retry():
    A = torch.eye(2, dtype=torch.float64)
    b = torch.ones(2, dtype=torch.float64)

    def declines(A, b, **kwargs):
        raise tc.OptionalBackendUnavailable("no")

    calls = []

    def positional_only(A, b):
        calls.append(1)
        return b.clone()

    tc.register_optional_backend("sparse_schur", declines)
    tc.register_optional_backend("block_schur", positional_only)
    try:
        r = tc.solve_linear_system(A, b, solver_type=tc.LinearSolverType.SPARSE_SCHUR, num_eliminate=1)
    finally:
        tc.clear_optional_backends()
    assert calls == [1] and "optional block_schur backend" in r.summary.message
    with pytest.raises(NotImplementedError):
        tc.solve_linear_system(A, b, solver_type=tc.LinearSolverType.SPARSE_SCHUR, num_eliminate=1)


def test_cuda_backends_reject_cpu_tensors_and_registration_is_safe():
    A = torch.eye(2, dtype=torch.float64)
    b = torch.ones(2, dtype=torch.float64)
    with pytest.raises(tc.OptionalBackendUnavailable, match="CUDA tensor"):
        tc.cuda_sparse_normal_cholesky(A, b)
    with pytest.raises(tc.OptionalBackendUnavailable, match="CUDA tensor"):
        tc.cuda_block_schur(A, b, num_eliminate=1)
    info = tc.register_cuda_sparse_backends()
    try:
        if info.available:
            assert {"sparse_normal_cholesky", "sparse_schur", "block_schur"} <= set(info.registered)
        else:
            assert info.registered == () and info.message
            assert tc.get_optional_backend("block_schur") is None
    finally:
        tc.unregister_cuda_sparse_backends()
    with pytest.raises(ValueError):
        tc.register_cuda_sparse_backends(precision="fp16")
    assert tc.get_cuda_extension_info().source_paths


def test_losses_known_answers_and_device_encoding():
    s = torch.tensor(4.0, dtype=torch.float64)
    r0, r1, r2 = tc.HuberLoss(1.0).evaluate(s)
    assert float(r0) == 3.0 and float(r1) == 0.5 and float(r2) < 0
    r0, r1, r2 = tc.TrivialLoss().evaluate(torch.tensor(2.0, dtype=torch.float64))
    assert float(r0) == 2.0 and float(r1) == 1.0 and float(r2) == 0.0
    from ceres_torch_cuda_b200.losses import device_loss
    d = device_loss(tc.ScaledLoss(tc.CauchyLoss(2.0), 3.0))
    assert d["loss_kind"] == 3 and d["loss_a"] == 2.0 and d["loss_scale"] == 3.0 and d["inner_loss_kind"] == -1
    d = device_loss(tc.ComposedLoss(tc.CauchyLoss(2.0), tc.SoftLOneLoss(1.0)))
    assert d["loss_kind"] == 3 and d["inner_loss_kind"] == 2
    assert device_loss(None)["loss_kind"] == 0


def test_lm_radius_matches_reference_strategy():
    """The known answers of the reference's LM radius test."""
    st = _LMRadius(2.0, 20.0)
    assert st.rejected() == 1.0
    assert st.rejected() == 0.25
    assert math.isclose(st.accepted(1.0), 0.75)
    assert math.isclose(st.accepted(1.0), 2.25)
    assert math.isclose(st.accepted(0.25), 2.0)
    assert math.isclose(st.accepted(1.0), 6.0)
    assert math.isclose(st.accepted(1.0), 18.0)
    assert math.isclose(st.accepted(1.0), 20.0)


def test_nonmonotonic_step_evaluator_matches_reference():
    ev = _StepEvaluator(10.0, 2)
    assert math.isclose(ev.step_quality(9.0, 2.0), 0.5)
    ev.step_accepted(9.0, 2.0)
    assert math.isclose(ev.step_quality(9.5, 1.0), 1.0 / 6.0)
    ev.step_accepted(9.5, 1.0)
    assert math.isclose(ev.step_quality(9.4, 1.0), 0.15)
    ev.step_accepted(9.4, 1.0)
    assert math.isclose(ev.step_quality(9.6, 1.0), -0.05)


def _bal_problem(cams, pts, ci, pi, obs, group_points=True):
    problem = tc.Problem()
    cb = [cams[i] for i in range(cams.shape[0])]
    pb = [pts[i] for i in range(pts.shape[0])]
    for c in cb:
        problem.AddParameterBlock(c)
    for p in pb:
        problem.AddParameterBlock(p)
        if group_points:
            problem.SetParameterBlockOrderingGroup(p, 0)
    for c, p, o in zip(ci, pi, obs):
        problem.AddResidualBlock(tc.SnavelyReprojectionError(float(o[0]), float(o[1])), tc.HuberLoss(1.0),
                                 [cb[c], pb[p]])
    return problem, cb, pb


def test_problem_recognition_and_write_back():
    rng = np.random.default_rng(0)
    cams = torch.tensor(rng.normal(size=(3, 9)))
    pts = torch.tensor(rng.normal(size=(5, 3)))
    ci = [0, 1, 2, 0, 1]
    pi = [0, 1, 2, 3, 4]
    obs = rng.normal(size=(5, 2))
    problem, cb, pb = _bal_problem(cams, pts, ci, pi, obs)
    problem.SetParameterBlockConstant(cb[1])
    ex = extract_bundle_adjustment(problem)
    np.testing.assert_array_equal(ex.camera_index.numpy(), ci)
    np.testing.assert_array_equal(ex.point_index.numpy(), pi)
    np.testing.assert_allclose(ex.observations.numpy(), obs)
    assert ex.camera_constant.tolist() == [False, True, False]
    assert isinstance(ex.loss, tc.HuberLoss)
    new = torch.arange(15, dtype=torch.float64).reshape(5, 3)
    write_back(ex.point_blocks, new)
    np.testing.assert_array_equal(pts.numpy(), new.numpy())
    assert problem.NumResiduals() == 10 and problem.NumEffectiveParameters() == 9 * 2 + 15


def test_unsupported_problems_fail_loudly():
    class Other(tc.CostFunction):
        parameter_block_sizes = [1]
        num_residuals = 1

    x = torch.zeros(1, dtype=torch.float64)
    p = tc.Problem()
    p.AddResidualBlock(Other(), None, [x])
    opts = tc.SolverOptions(linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR)
    with pytest.raises(NotImplementedError, match="SnavelyReprojectionError"):
        tc.solve(opts, p)
    rng = np.random.default_rng(1)
    problem, _, _ = _bal_problem(torch.tensor(rng.normal(size=(2, 9))), torch.tensor(rng.normal(size=(2, 3))),
                                 [0, 1], [0, 1], rng.normal(size=(2, 2)))
    with pytest.raises(NotImplementedError, match="CUDA"):
        tc.solve(opts, problem)  # CPU tensors: no CPU path
    with pytest.raises(NotImplementedError, match="SCHUR"):
        tc.solve(tc.SolverOptions(linear_solver_type=tc.LinearSolverType.DENSE_QR), problem)
    with pytest.raises(NotImplementedError, match="CUDA"):  # a GPU preconditioner, CPU tensors
        tc.solve(tc.SolverOptions(linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR,
                                  preconditioner_type=tc.PreconditionerType.CLUSTER_JACOBI), problem)


def test_snavely_residual_matches_generator_projection():
    from ceres_torch_cuda_b200 import synthetic as S
    d = S.make_small_ba(3, 10, 2, seed=3)
    cost = tc.SnavelyReprojectionError(*d.observations[0])
    r = cost.residuals(torch.tensor(d.cameras[d.camera_index[0]]), torch.tensor(d.points[d.point_index[0]]))
    expect = S.project(d.cameras[d.camera_index[:1]], d.points[d.point_index[:1]])[0] - d.observations[0]
    np.testing.assert_allclose(r.numpy(), expect, rtol=1e-12)


def test_bal_text_round_trip_and_errors():
    """BAL parsing (the format of examples/simple_bundle_adjuster.py:33-70) on CPU tensors."""
    import numpy as np
    import pytest

    import ceres_torch_cuda_b200 as tc
    from ceres_torch_cuda_b200 import synthetic as S

    d = S.make_small_ba(3, 7, 2, seed=1)
    lines = [f"{d.num_cameras} {d.num_points} {d.num_observations}"]
    lines += [f"{int(c)} {int(p)} {float(x)!r} {float(y)!r}"
              for c, p, (x, y) in zip(d.camera_index, d.point_index, d.observations)]
    lines += [repr(float(v)) for v in d.cameras.ravel()] + [repr(float(v)) for v in d.points.ravel()]
    text = "\n".join(lines) + "\n"
    bal = tc.BundleAdjustmentProblem.from_bal_text(text, device="cpu")
    np.testing.assert_array_equal(bal.cameras.numpy(), d.cameras)
    np.testing.assert_array_equal(bal.points.numpy(), d.points)
    np.testing.assert_array_equal(bal.observations.numpy(), d.observations)
    np.testing.assert_array_equal(bal.camera_index.numpy(), d.camera_index)
    np.testing.assert_array_equal(bal.point_index.numpy(), d.point_index)
    with pytest.raises(ValueError, match="trailing"):
        tc.BundleAdjustmentProblem.from_bal_text(text + " 1.0", device="cpu")
    with pytest.raises(ValueError, match="truncated"):
        tc.BundleAdjustmentProblem.from_bal_text(text.rsplit("\n", 2)[0], device="cpu")
