"""CLUSTER_JACOBI / CLUSTER_TRIDIAGONAL on the GPU (linear.py:498-521, :1032-1085).

* The component inverses that ceres_b200_ba_cluster_factor builds equal the inverse of
  the explicit reduced camera matrix (ceres_b200_ba_schur_matrix) kept on the oracle's
  cluster block pairs (1e-9 relative).
* Whole solves reproduce the reference's LM traces for these preconditioners
  (tests/golden ba_cluster_*: same termination, iteration and linear-iteration counts,
  costs 1e-9, parameters 1e-5) in float64; the mixed path reaches the same final cost
  within 1e-6 with iteration counts within 2. (Through ceres-torch's own solve:
  tests/test_gpu_dropin.py.)
* Two solves give the same bits (the kept blocks are summed in point order, the
  inverses by a fixed sweep, the apply by a fixed shuffle tree).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import ba_oracle as O
from tests import _golden as G

pytestmark = pytest.mark.gpu
DEV = "cuda"
CLUSTER_CASES = ["ba_cluster_jacobi", "ba_cluster_tridiagonal", "ba_cluster_single_linkage", "ba_cluster_uniform"]


def _tc():
    import ceres_torch_cuda_b200 as tc

    return tc


def _loss_obj(spec):
    tc = _tc()
    if spec[0] == "trivial":
        return None
    return {"huber": tc.HuberLoss, "cauchy": tc.CauchyLoss}[spec[0]](float(spec[1]))


def _problem(d):
    tc = _tc()
    meta = d["meta"]
    nc = d["cameras"].shape[0]
    t = lambda a, dt=torch.float64: torch.as_tensor(a).to(DEV, dt)  # noqa: E731
    return tc.BundleAdjustmentProblem(t(d["cameras"]), t(d["points"]), t(d["observations"]),
                                      t(d["camera_index"], torch.int64), t(d["point_index"], torch.int64),
                                      loss=_loss_obj(G.loss_spec(meta["loss"])),
                                      camera_constant=t(G.constant_mask(nc, meta["constant_cameras"]), torch.bool))


def _options(meta, **kw):
    tc = _tc()
    return tc.SolverOptions(max_num_iterations=meta["max_num_iterations"],
                            linear_solver_type=getattr(tc.LinearSolverType, meta["solver"]),
                            preconditioner_type=getattr(tc.PreconditionerType, meta["preconditioner"]),
                            **meta.get("spse", {}), **kw)


@pytest.mark.parametrize("name", CLUSTER_CASES)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cluster_inverses_match_masked_schur_matrix(name, precision):
    tc = _tc()
    from ceres_torch_cuda_b200 import _lib

    d = G.load(name)
    meta = d["meta"]
    prob = _problem(d)
    eng = tc.BAEngine(prob.cameras, prob.points, prob.observations, prob.camera_index, prob.point_index,
                      loss=prob.loss, camera_constant=prob.camera_constant, precision=precision)
    opts = _options(meta)
    tri = meta["preconditioner"] == "CLUSTER_TRIDIAGONAL"
    assert eng.setup_clusters(tri, meta.get("spse", {}).get("visibility_clustering_type", "CANONICAL_VIEWS"))
    eng.evaluate(True)
    eng.assemble(1e3, opts, _lib.PRECOND_CLUSTER)
    S = torch.zeros((9 * eng.nc, 9 * eng.nc), dtype=torch.float64, device=DEV)
    eng._call("ceres_b200_ba_schur_matrix", S.data_ptr())
    eng.read_stats()
    flags = eng.cluster_flags()
    assert flags[2] == 0 and flags[5] == 0
    S = S.cpu().numpy()
    # the oracle's clusters over the active cameras, mapped to camera ids
    op = O.OracleProblem(d["cameras"], d["points"], d["observations"], d["camera_index"], d["point_index"],
                         G.loss_spec(meta["loss"]), camera_constant=G.constant_mask(d["cameras"].shape[0],
                                                                                    meta["constant_cameras"]))
    st = O.cluster_structure(O.schur_visibility(op), tridiagonal=tri,
                             clustering=meta.get("spse", {}).get("visibility_clustering_type", "CANONICAL_VIEWS"))
    act = op.active_cams
    keep = np.zeros((eng.nc, eng.nc), dtype=bool)
    for a, b in st.block_pairs:
        keep[act[a], act[b]] = keep[act[b], act[a]] = True
    member = np.full(eng.nc, -1)
    member[act] = st.membership
    M = np.where(np.kron(keep, np.ones((9, 9), bool)), S, 0.0)
    if flags[0]:  # not positive definite: the blocks between clusters halved (linear.py:1059-1072)
        cross = keep & (member[:, None] != member[None, :])
        M = np.where(np.kron(cross, np.ones((9, 9), bool)), 0.5 * M, M)
    plan = eng.clusters
    for comp, inv in zip(plan.components, plan.matrices()):
        cams = act[comp]
        idx = (9 * cams[:, None] + np.arange(9)[None, :]).reshape(-1)
        ref = np.linalg.inv(M[np.ix_(idx, idx)])
        got = inv.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


@pytest.mark.parametrize("name", CLUSTER_CASES)
def test_cluster_solve_matches_reference_trace(name):
    tc = _tc()
    d = G.load(name)
    meta = d["meta"]
    prob = _problem(d)
    s = tc.solve(_options(meta), prob, precision="fp64")
    assert s.termination_type.value == meta["termination"]
    assert len(s.iterations) == meta["num_iterations"]
    np.testing.assert_allclose(s.initial_cost, meta["initial_cost"], rtol=1e-11)
    np.testing.assert_allclose(s.final_cost, meta["final_cost"], rtol=1e-9)
    np.testing.assert_allclose([it.cost for it in s.iterations], d["trace"][:, 1], rtol=1e-9)
    np.testing.assert_array_equal([it.linear_solver_iterations for it in s.iterations], d["trace"][:, 7].astype(int))
    np.testing.assert_allclose(prob.cameras.cpu().numpy(), d["final_cameras"], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(prob.points.cpu().numpy(), d["final_points"], rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("name", CLUSTER_CASES)
def test_cluster_mixed_precision_reaches_reference_cost(name):
    tc = _tc()
    d = G.load(name)
    meta = d["meta"]
    s = tc.solve(_options(meta), _problem(d), precision="mixed")
    assert s.precision == "mixed"
    assert s.termination_type.value == meta["termination"]
    assert abs(len(s.iterations) - meta["num_iterations"]) <= 2
    np.testing.assert_allclose(s.final_cost, meta["final_cost"], rtol=1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cluster_solves_are_reproducible(precision):
    tc = _tc()
    d = G.load("ba_cluster_tridiagonal")
    meta = d["meta"]
    runs = []
    for _ in range(2):
        prob = _problem(d)
        s = tc.solve(_options(meta), prob, precision=precision)
        runs.append(([it.cost for it in s.iterations], prob.cameras.cpu().numpy(), prob.points.cpu().numpy()))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1]) and np.array_equal(runs[0][2], runs[1][2])


@pytest.mark.parametrize("tridiagonal", [False, True])
def test_cluster_inverses_with_repeated_observations(tridiagonal):
    """A camera that sees a point twice: the kept blocks sum over all of the camera's
    observations of each shared point (the diagonal block from the camera reduction's
    duplicate-aware sums), so the inverses still equal those of the masked explicit S."""
    tc = _tc()
    from ceres_torch_cuda_b200 import _lib
    from ceres_torch_cuda_b200 import clustering as C
    from ceres_torch_cuda_b200 import synthetic as S

    d = S.make_sequence_ba(10, 150, 3, seed=21)
    rep = np.arange(0, d.num_observations, 7)  # every 7th observation recorded twice
    ci = np.concatenate([d.camera_index, d.camera_index[rep]])
    pi = np.concatenate([d.point_index, d.point_index[rep]])
    ob = np.concatenate([d.observations, d.observations[rep] + 0.5])
    t = lambda a, dt=torch.float64: torch.as_tensor(a).to(DEV, dt)  # noqa: E731
    eng = tc.BAEngine(t(d.cameras), t(d.points), t(ob), t(ci, torch.int64), t(pi, torch.int64), precision="fp64")
    assert eng.layout.has_duplicate_cameras
    assert eng.setup_clusters(tridiagonal)
    eng.evaluate(True)
    eng.assemble(1e3, tc.SolverOptions(), _lib.PRECOND_CLUSTER)
    S_ = torch.zeros((9 * eng.nc, 9 * eng.nc), dtype=torch.float64, device=DEV)
    eng._call("ceres_b200_ba_schur_matrix", S_.data_ptr())
    eng.read_stats()
    flags = eng.cluster_flags()
    S_ = S_.cpu().numpy()
    st = C.cluster_structure(tridiagonal=tridiagonal, incidence=C.incidence_from_observations(eng.nc, ci, pi))
    keep = np.zeros((eng.nc, eng.nc), dtype=bool)
    for a, b in st.block_pairs():
        keep[a, b] = keep[b, a] = True
    M = np.where(np.kron(keep, np.ones((9, 9), bool)), S_, 0.0)
    if flags[0]:
        cross = keep & (st.membership[:, None] != st.membership[None, :])
        M = np.where(np.kron(cross, np.ones((9, 9), bool)), 0.5 * M, M)
    for comp, inv in zip(eng.clusters.components, eng.clusters.matrices()):
        idx = (9 * comp[:, None] + np.arange(9)[None, :]).reshape(-1)
        ref = np.linalg.inv(M[np.ix_(idx, idx)])
        np.testing.assert_allclose(inv.cpu().numpy(), ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
