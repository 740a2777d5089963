"""Camera, point and camera-point covariance blocks through the reduced camera system on
the GPU (ceres_b200_ba_schur_matrix + ceres_b200_dense_spd_inverse) against the
reference's own dense-SVD Covariance (covariance.py:86-445) at the reference's solution
(fixtures made by running ceres-torch): blocks within 1e-6 relative; a free gauge is
reported as the reference reports it."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from tests import _golden as G

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _problem(d):
    import ceres_torch_cuda_b200 as tc

    meta = d["meta"]
    cams = torch.tensor(d["solved_cameras"], device=DEV)
    pts = torch.tensor(d["solved_points"], device=DEV)
    problem = tc.Problem()
    cb = [cams[i] for i in range(cams.shape[0])]
    pb = [pts[i] for i in range(pts.shape[0])]
    for i, c in enumerate(cb):
        problem.AddParameterBlock(c)
        if i in meta["constant_cameras"]:
            problem.SetParameterBlockConstant(c)
    for p in pb:
        problem.AddParameterBlock(p)
        problem.SetParameterBlockOrderingGroup(p, 0)
    kind = meta["loss"][0]
    loss = None if kind == "trivial" else {"cauchy": tc.CauchyLoss, "huber": tc.HuberLoss}[kind](float(meta["loss"][1]))
    for c, p, o in zip(d["camera_index"].tolist(), d["point_index"].tolist(), d["observations"]):
        problem.AddResidualBlock(tc.SnavelyReprojectionError(o[0], o[1]), loss, [cb[c], pb[p]])
    return problem, cb, pb


@pytest.mark.parametrize("name", ["ba_covariance", "ba_covariance_cauchy"])
def test_covariance_blocks_match_reference(name):
    from ceres_torch_cuda_b200.covariance import Covariance

    d = G.load(name)
    meta = d["meta"]
    problem, cb, pb = _problem(d)
    free, pts = meta["free_cameras"], meta["points"]
    pairs = [(cb[i], cb[j]) for a, i in enumerate(free) for j in free[a:]]
    pairs += [(pb[q], pb[q]) for q in pts] + [(cb[free[0]], pb[q]) for q in pts]
    cov = Covariance()
    assert cov.compute(pairs, problem), cov.summary.message
    assert cov.summary.rank == meta["rank"] and cov.summary.nullity == 0
    scale = np.abs(d["cov_cameras"]).max()
    for a, i in enumerate(free):
        for b, j in enumerate(free):
            got = cov.get_covariance_block(cb[i], cb[j]).cpu().numpy()
            np.testing.assert_allclose(got, d["cov_cameras"][a, b], rtol=1e-6, atol=1e-8 * scale)
    for k, q in enumerate(pts):
        np.testing.assert_allclose(cov.get_covariance_block(pb[q], pb[q]).cpu().numpy(), d["cov_points"][k],
                                   rtol=1e-6, atol=1e-8 * np.abs(d["cov_points"]).max())
        np.testing.assert_allclose(cov.get_covariance_block(cb[free[0]], pb[q]).cpu().numpy(),
                                   d["cov_camera_point"][k], rtol=1e-6,
                                   atol=1e-8 * np.abs(d["cov_camera_point"]).max())
        np.testing.assert_allclose(cov.get_covariance_block(pb[q], cb[free[0]]).cpu().numpy(),
                                   d["cov_camera_point"][k].T, rtol=1e-6,
                                   atol=1e-8 * np.abs(d["cov_camera_point"]).max())
    # a block that was not requested raises
    const = meta["constant_cameras"][0]
    assert not cov.has_covariance_block(cb[const], cb[const])
    with pytest.raises(KeyError):
        cov.get_covariance_block(cb[const], cb[const])
    # the symmetric matrix of the free cameras
    m = cov.get_covariance_matrix([cb[i] for i in free]).cpu().numpy()
    np.testing.assert_allclose(m, m.T, rtol=0, atol=1e-12 * np.abs(m).max())


def test_free_gauge_is_reported_rank_deficient():
    from ceres_torch_cuda_b200.covariance import Covariance

    d = G.load("ba_covariance_gauge")
    meta = d["meta"]
    problem, cb, _ = _problem(d)
    cov = Covariance()
    assert not cov.compute([cb[0], cb[1]], problem)
    assert cov.summary.message == meta["message"] == "Jacobian is rank deficient."
    assert cov.summary.nullity >= 1
    with pytest.raises(RuntimeError):
        cov.get_covariance_block(cb[0], cb[1])
