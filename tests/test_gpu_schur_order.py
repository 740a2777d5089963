"""The explicit reduced camera matrix summed in a fixed order on the GPU.

ceres_b200_ba_schur_matrix and ceres_b200_ba_dense_schur_solve (the reference's dense
Schur route, linear.py:667-699) sum S block by block in the order of
engine.schur_contributions when the struct carries it:

* the ordered S equals the float64-atomic S within 1e-12 (same terms, other order) and
  two ordered assemblies give the same bits, with duplicate observations, constant
  cameras and constant points;
* two DENSE_SCHUR solves give the same bits in both precisions, and the fp64 solve still
  follows the oracle's trace (tests/test_gpu_parity.py holds the reference traces);
* the covariance (built on the explicit S) is bit-reproducible.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import ba_oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _tc():
    import ceres_torch_cuda_b200 as tc

    return tc


def _data(dup=True):
    from ceres_torch_cuda_b200 import synthetic as S

    d = S.make_small_ba(12, 400, 4, seed=31)
    ci, pi, ob = d.camera_index, d.point_index, d.observations
    if dup:
        rep = np.arange(0, ci.size, 9)
        ci, pi = np.concatenate([ci, ci[rep]]), np.concatenate([pi, pi[rep]])
        ob = np.concatenate([ob, ob[rep] + 0.25])
    return d, ci, pi, ob


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ordered_matrix_matches_atomic_and_repeats(precision):
    tc = _tc()
    from ceres_torch_cuda_b200 import _lib

    d, ci, pi, ob = _data()
    t = lambda a, dt=torch.float64: torch.as_tensor(a).to(DEV, dt)  # noqa: E731
    cc = torch.zeros(12, dtype=torch.bool)
    cc[[0, 7]] = True
    pc = torch.zeros(400, dtype=torch.bool)
    pc[[3, 50, 51]] = True
    eng = tc.BAEngine(t(d.cameras), t(d.points), t(ob), t(ci, torch.int64), t(pi, torch.int64),
                      camera_constant=cc.to(DEV), point_constant=pc.to(DEV), precision=precision)
    assert eng.layout.has_duplicate_cameras
    eng.evaluate(True)
    eng.assemble(1e4, tc.SolverOptions(), _lib.PRECOND_SCHUR_JACOBI)
    a = eng.schur_matrix(ordered=False)
    b = eng.schur_matrix()
    c = eng.schur_matrix()
    eng.read_stats()
    assert eng._schur_order
    assert torch.equal(b, c)
    assert torch.equal(b, b.T)
    np.testing.assert_allclose(b.cpu().numpy(), a.cpu().numpy(), rtol=1e-12, atol=1e-12 * float(a.abs().max()))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_schur_solves_repeat_bit_for_bit(precision):
    tc = _tc()
    d, ci, pi, ob = _data()
    runs = []
    for _ in range(2):
        prob = tc.BundleAdjustmentProblem.from_arrays(d.cameras, d.points, ob, ci, pi)
        s = tc.solve(tc.SolverOptions(linear_solver_type=tc.LinearSolverType.DENSE_SCHUR, max_num_iterations=15),
                     prob, precision=precision)
        runs.append(([it.cost for it in s.iterations], prob.cameras.cpu().numpy(), prob.points.cpu().numpy()))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1]) and np.array_equal(runs[0][2], runs[1][2])
    if precision == "fp64":
        ref = O.solve(O.OracleProblem(d.cameras, d.points, ob, ci, pi),
                      O.OracleOptions(linear_solver_type="DENSE_SCHUR", max_num_iterations=15))
        assert len(runs[0][0]) == len(ref.iterations)
        np.testing.assert_allclose(runs[0][0], [it.cost for it in ref.iterations], rtol=1e-9)


def test_covariance_repeats_bit_for_bit():
    from ceres_torch_cuda_b200.covariance import Covariance
    from tests import _golden as G
    from tests.test_gpu_covariance import _problem

    d = G.load("ba_covariance")
    free, pts = d["meta"]["free_cameras"], d["meta"]["points"]
    out = []
    for _ in range(2):
        problem, cb, pb = _problem(d)
        pairs = [(cb[i], cb[j]) for a, i in enumerate(free) for j in free[a:]]
        pairs += [(pb[q], pb[q]) for q in pts] + [(cb[free[0]], pb[q]) for q in pts]
        cov = Covariance()
        assert cov.compute(pairs, problem), cov.summary.message
        out.append([cov.get_covariance_block(x, y).cpu().numpy() for x, y in pairs])
        assert cov._engine._schur_order
    for x, y in zip(*out):
        assert np.array_equal(x, y)
