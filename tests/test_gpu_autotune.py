"""The single-problem autotuner (ceres_torch_cuda_b200/autotune.py): it times every
candidate (camera-major copy on/off x camera work-item lengths) on the problem, picks
one of them and caches it per size class; every candidate gives the same PCG solution
to rounding (the copy changes no bit, the item length only the grouping of the camera
pass's sums), and an autotuned solve reports its choice and ends where the default one
does."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _ring(seed=41):
    from ceres_torch_cuda_b200 import synthetic as S

    d = S.make_ring_ba(60, 3000, seed=seed)
    t = lambda a, dt=torch.float64: torch.as_tensor(a).to(DEV, dt)  # noqa: E731
    return d, (t(d.cameras), t(d.points), t(d.observations), t(d.camera_index, torch.int64),
               t(d.point_index, torch.int64))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_candidate_gives_the_same_pcg_solution(precision):
    import ceres_torch_cuda_b200 as tc
    from ceres_torch_cuda_b200 import _lib, autotune

    _, arrays = _ring()
    opts = tc.SolverOptions()
    ref = None
    layout = None
    for copy in (True, False):
        eng = tc.BAEngine(*arrays, loss=tc.CauchyLoss(2.0), precision=precision, camera_copy=copy, layout=layout)
        layout = eng.layout
        for item in autotune.ITEM_SIZES:
            eng.retile_items(item)
            eng.evaluate(True)
            eng.assemble(1e3, opts, _lib.PRECOND_SCHUR_JACOBI)
            eng.pcg(_lib.PRECOND_SCHUR_JACOBI, 10, 10, 0.0, 0)
            eng.read_stats()
            x = eng.step_cameras[: eng.nc].cpu().numpy().copy()
            if ref is None:
                ref = x
            np.testing.assert_allclose(x, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())


def test_tuner_picks_a_candidate_and_caches_it():
    import ceres_torch_cuda_b200 as tc
    from ceres_torch_cuda_b200 import autotune

    autotune.clear_cache()
    _, arrays = _ring(seed=42)
    cfg = autotune.tune(*arrays, loss=tc.CauchyLoss(2.0), precision="mixed")
    assert (cfg.camera_copy, cfg.item_size) in cfg.timings
    assert len(cfg.timings) == 2 * len(autotune.ITEM_SIZES)
    assert all(t["estimate"] > 0 for t in cfg.timings.values())
    best = min(t["estimate"] for t in cfg.timings.values())
    assert cfg.estimate_ms <= (1.0 + autotune.MARGIN) * best
    if (cfg.camera_copy, cfg.item_size) != (True, 256):  # left the default: clearly faster
        assert cfg.estimate_ms == best
    assert autotune.tune(*arrays, loss=tc.CauchyLoss(2.0), precision="mixed") is cfg  # cached


def test_autotuned_solve_reports_its_choice_and_matches_the_default():
    import ceres_torch_cuda_b200 as tc
    from ceres_torch_cuda_b200 import autotune

    autotune.clear_cache()
    d, _ = _ring(seed=43)
    t = lambda a, dt=torch.float64: torch.as_tensor(a).to(DEV, dt)  # noqa: E731
    runs = []
    for at in (False, True):
        prob = tc.BundleAdjustmentProblem(t(d.cameras), t(d.points), t(d.observations),
                                          t(d.camera_index, torch.int64), t(d.point_index, torch.int64),
                                          loss=tc.CauchyLoss(2.0))
        s = tc.solve(tc.SolverOptions(max_num_iterations=8, linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR),
                     prob, precision="fp64", autotune=at)
        assert s.kernel_config["autotuned"] is at
        runs.append(s)
    assert runs[1].kernel_config["item_size"] in autotune.ITEM_SIZES
    assert len(runs[0].iterations) == len(runs[1].iterations)
    np.testing.assert_allclose(runs[1].final_cost, runs[0].final_cost, rtol=1e-10)
