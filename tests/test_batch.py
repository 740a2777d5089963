"""Batched solves (one persistent launch for many problems).

CPU: the concatenated layout gives every problem the layout its single-problem
solve would use (same slices, same slot order, same camera-major lists).
GPU: each problem of a batch ends where its own ``tc.solve`` ends (float64: final
cost 1e-8 relative, termination and iteration count equal up to +-2, parameters
1e-5; mixed: final cost within 1e-6 of the float64 single solve), and a problem's
result in a batch of one equals its result in the mix (1e-8 relative). Clusters of
1 to 16 CTAs per problem give the same results.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from ceres_torch_cuda_b200 import synthetic as S
from ceres_torch_cuda_b200.batch import build_batch_layout
from ceres_torch_cuda_b200.engine import build_layout


def _concat(datas):
    cam_counts = np.array([d.num_cameras for d in datas], dtype=np.int64)
    pt_counts = np.array([d.num_points for d in datas], dtype=np.int64)
    co = np.concatenate([[0], np.cumsum(cam_counts)])
    po = np.concatenate([[0], np.cumsum(pt_counts)])
    ci = torch.cat([torch.as_tensor(d.camera_index, dtype=torch.int64) + int(co[i]) for i, d in enumerate(datas)])
    pi = torch.cat([torch.as_tensor(d.point_index, dtype=torch.int64) + int(po[i]) for i, d in enumerate(datas)])
    obs = torch.cat([torch.as_tensor(d.observations) for d in datas])
    return cam_counts, pt_counts, co, po, ci, pi, obs


def test_batch_layout_matches_single_problem_layouts():
    datas = S.make_batched_instances(5, seed=3, max_points=150)
    cam_counts, pt_counts, co, po, ci, pi, obs = _concat(datas)
    L = build_batch_layout(cam_counts, pt_counts, ci, pi, obs)
    soff = L.slice_off.numpy()
    assert (L.cam_off.numpy() == co).all()
    for b, d in enumerate(datas):
        one = build_layout(torch.as_tensor(d.camera_index), torch.as_tensor(d.point_index),
                           torch.as_tensor(d.observations), d.num_cameras, d.num_points)
        s0, s1 = soff[b], soff[b + 1]
        assert s1 - s0 == one.num_slices
        np.testing.assert_array_equal(L.slice_len.numpy()[s0:s1], one.slice_len.numpy())
        base0 = int(L.slice_base.numpy()[s0])
        np.testing.assert_array_equal(L.slice_base.numpy()[s0:s1] - base0, one.slice_base.numpy())
        nslot = one.num_slots
        np.testing.assert_array_equal(L.slot_cam.numpy()[base0:base0 + nslot], one.slot_cam.numpy()[:nslot])
        np.testing.assert_array_equal(L.slot_obs.numpy()[base0:base0 + nslot], one.slot_obs.numpy()[:nslot])
        lp = L.lane_point.numpy()[32 * s0:32 * s1]
        ref = one.lane_point.numpy()
        np.testing.assert_array_equal(np.where(lp >= 0, lp - po[b], -1), ref)
        off = L.cam_offsets.numpy()
        ent = L.cam_entries.numpy()
        for c in range(d.num_cameras):
            e = ent[off[co[b] + c]:off[co[b] + c + 1]]
            e1 = one.cam_entries.numpy()[one.cam_offsets.numpy()[c]:one.cam_offsets.numpy()[c + 1]]
            np.testing.assert_array_equal(e[:, 0] - base0, e1[:, 0])
            np.testing.assert_array_equal(e[:, 1] - 32 * s0, e1[:, 1])


def _problems(datas, loss=None):
    import ceres_torch_cuda_b200 as tc
    return [tc.BundleAdjustmentProblem.from_arrays(d.cameras, d.points, d.observations, d.camera_index,
                                                   d.point_index, loss=loss) for d in datas]


def _options(max_iterations=30):
    import ceres_torch_cuda_b200 as tc
    return tc.SolverOptions(linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR,
                            preconditioner_type=tc.PreconditionerType.SCHUR_JACOBI,
                            max_num_iterations=max_iterations)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,cluster", [("fp64", 1), ("mixed", 1), ("fp64", 4), ("mixed", 8), ("fp64", 16)])
def test_batch_matches_single_solves(precision, cluster):
    import ceres_torch_cuda_b200 as tc
    datas = S.make_batched_instances(6, seed=11, max_points=300)
    singles = _problems(datas)
    ref = [tc.solve(_options(), p, precision="fp64") for p in singles]
    batch = _problems(datas)
    got = tc.solve_batch(_options(), batch, precision=precision, cluster_size=cluster)
    for r, g, ps, pb in zip(ref, got, singles, batch):
        if precision == "fp64":
            np.testing.assert_allclose(g.final_cost, r.final_cost, rtol=1e-8)
            assert g.termination_type == r.termination_type
            assert abs(len(g.iterations) - len(r.iterations)) <= 2
            np.testing.assert_allclose(pb.cameras.cpu().numpy(), ps.cameras.cpu().numpy(), rtol=1e-5, atol=1e-7)
            np.testing.assert_allclose(pb.points.cpu().numpy(), ps.points.cpu().numpy(), rtol=1e-5, atol=1e-7)
        else:
            assert g.final_cost <= r.final_cost * (1 + 1e-6)
            assert g.final_cost >= r.final_cost * (1 - 1e-6)
        assert g.initial_cost == pytest.approx(r.initial_cost, rel=1e-12)
        assert g.iterations[0].cost == pytest.approx(r.iterations[0].cost, rel=1e-12)


@pytest.mark.gpu
def test_batch_result_alone_equals_result_in_the_mix():
    import ceres_torch_cuda_b200 as tc
    datas = S.make_batched_instances(8, seed=5, max_points=200)
    mix = tc.solve_batch(_options(), _problems(datas), precision="fp64")
    for k in (0, 5):
        alone = tc.solve_batch(_options(), _problems([datas[k]]), precision="fp64")[0]
        np.testing.assert_allclose(alone.final_cost, mix[k].final_cost, rtol=1e-8)
        assert abs(len(alone.iterations) - len(mix[k].iterations)) <= 2


@pytest.mark.gpu
def test_batch_with_loss_and_constant_camera():
    import ceres_torch_cuda_b200 as tc
    datas = S.make_batched_instances(3, seed=21, max_points=120)
    singles = _problems(datas, loss=tc.CauchyLoss(2.0))
    batch = _problems(datas, loss=tc.CauchyLoss(2.0))
    for p in singles + batch:
        p.camera_constant = torch.zeros(p.num_cameras, dtype=torch.bool, device=p.cameras.device)
        p.camera_constant[0] = True
    ref = [tc.solve(_options(), p, precision="fp64") for p in singles]
    got = tc.solve_batch(_options(), batch, precision="fp64")
    for r, g, pb, ps in zip(ref, got, batch, singles):
        np.testing.assert_allclose(g.final_cost, r.final_cost, rtol=1e-8)
        np.testing.assert_array_equal(pb.cameras[0].cpu().numpy(), ps.cameras[0].cpu().numpy())


def _oracle_solve(d, loss_spec=("trivial",), max_iterations=30):
    from oracle import ba_oracle as O
    p = O.OracleProblem(d.cameras, d.points, d.observations, d.camera_index, d.point_index, loss_spec)
    return O.solve(p, O.OracleOptions(linear_solver_type="ITERATIVE_SCHUR", preconditioner_type="SCHUR_JACOBI",
                                      max_num_iterations=max_iterations))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_the_reference_fixtures(precision):
    """Each batched problem against the reference's own recorded solve of it (ceres-torch's
    float64 tc.solve, ITERATIVE_SCHUR + SCHUR_JACOBI, default tolerances): the same
    termination, iteration count within +-2 and final cost within 1e-8 (float64) or 1e-6
    (mixed) relative. Problems sharing a loss form one batch."""
    import ceres_torch_cuda_b200 as tc
    from tests import _golden as G

    groups = {("trivial",): ["ba_small_iterative"], ("cauchy", 2.0): ["ba_cauchy", "config2_small"],
              ("huber", 1.0): ["config1_small"]}
    rtol = 1e-8 if precision == "fp64" else 1e-6
    for spec, names in groups.items():
        loss = None if spec[0] == "trivial" else (tc.CauchyLoss if spec[0] == "cauchy" else tc.HuberLoss)(spec[1])
        ds = [G.load(n) for n in names]
        probs = [tc.BundleAdjustmentProblem.from_arrays(d["cameras"], d["points"], d["observations"],
                                                        d["camera_index"], d["point_index"], loss=loss) for d in ds]
        opts = tc.SolverOptions(linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR,
                                preconditioner_type=tc.PreconditionerType.SCHUR_JACOBI,
                                max_num_iterations=ds[0]["meta"]["max_num_iterations"])
        got = tc.solve_batch(opts, probs, precision=precision)
        for name, d, g in zip(names, ds, got):
            meta = d["meta"]
            assert g.termination_type.value == meta["termination"], (name, g.message)
            assert abs(len(g.iterations) - meta["num_iterations"]) <= 2, (name, len(g.iterations))
            np.testing.assert_allclose(g.final_cost, meta["final_cost"], rtol=rtol, err_msg=name)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_of_configuration3_size_instances_matches_the_oracle(precision):
    """Eight instances drawn like configuration 3 at its full size range (3-32 cameras,
    up to 2,000 points, tracks of 3-8) in one launch against the float64 oracle:
    final cost within 1e-8 (float64) or 1e-6 (mixed) relative, iteration count within
    +-2."""
    import ceres_torch_cuda_b200 as tc

    datas = S.make_batched_instances(8, seed=33, max_points=2000)
    assert max(d.num_points for d in datas) > 1000 and max(d.num_cameras for d in datas) > 16
    got = tc.solve_batch(_options(), _problems(datas), precision=precision)
    rtol = 1e-8 if precision == "fp64" else 1e-6
    for d, g in zip(datas, got):
        ref = _oracle_solve(d)
        np.testing.assert_allclose(g.final_cost, ref.final_cost, rtol=rtol)
        assert abs(len(g.iterations) - len(ref.iterations)) <= 2


@pytest.mark.gpu
def test_batch_autotune_shapes_give_the_same_float64_results():
    """Every CTA shape the autotuner chooses from gives the same float64 solves (final
    cost 1e-10 relative), and autotune returns one of them."""
    import ceres_torch_cuda_b200 as tc
    from ceres_torch_cuda_b200 import batch as B

    datas = S.make_batched_instances(4, seed=44, max_points=200)
    results = {}
    for shape in B.SHAPES:
        solver = tc.BatchSolver(_problems(datas), _options(), precision="fp64")
        solver.launch(*shape)
        results[shape] = [s.final_cost for s in solver.summaries()]
    first = next(iter(results.values()))
    for shape, costs in results.items():
        np.testing.assert_allclose(costs, first, rtol=1e-10, err_msg=str(shape))
    chosen = B.autotune(_options(), _problems(datas), precision="fp64")
    assert tuple(chosen) in {tuple(s) for s in B.SHAPES}


def test_batch_layout_from_host_track_stats():
    """With each problem's largest track and duplicate flag known on the host, the slot
    count comes from the bound sum_p (32 max_track_p + no_p) and no device read is made;
    every array equals the one built with the read (the extra slots are padding)."""
    datas = S.make_batched_instances(7, seed=5, max_points=200)
    cam_counts, pt_counts, co, po, ci, pi, obs = _concat(datas)
    ref = build_batch_layout(cam_counts, pt_counts, ci, pi, obs)
    stats, counts = [], []
    for d in datas:
        track = np.bincount(d.point_index, minlength=d.num_points)
        stats.append((int(track.max()), False))
        counts.append(d.num_observations)
    L = build_batch_layout(cam_counts, pt_counts, ci, pi, obs, obs_counts=np.array(counts), track_stats=stats)
    assert L.num_slots >= ref.num_slots
    assert L.num_slots == sum(32 * t + n for (t, _), n in zip(stats, counts))
    assert L.has_duplicate_cameras == ref.has_duplicate_cameras
    for name in ("slice_base", "slice_len", "cam_offsets", "cam_entries", "lane_point", "cam_off", "slice_off"):
        np.testing.assert_array_equal(getattr(L, name).numpy(), getattr(ref, name).numpy())
    n = ref.num_slots
    np.testing.assert_array_equal(L.slot_cam.numpy()[:n], ref.slot_cam.numpy()[:n])
    np.testing.assert_array_equal(L.slot_obs.numpy()[:n], ref.slot_obs.numpy()[:n])
    assert (L.slot_cam.numpy()[n:] == -1).all()


def test_track_stats_follow_the_index_tensors():
    import ceres_torch_cuda_b200 as tc

    d = S.make_small_ba(6, 80, 3, seed=2)
    ci = np.concatenate([d.camera_index, d.camera_index[:1]])
    pi = np.concatenate([d.point_index, d.point_index[:1]])
    ob = np.concatenate([d.observations, d.observations[:1]])
    p = tc.BundleAdjustmentProblem.from_arrays(d.cameras, d.points, ob, ci, pi, device="cpu", track_stats=True)
    assert p.track_stats == (int(np.bincount(pi).max()), True)
    assert tc.BundleAdjustmentProblem.from_arrays(d.cameras, d.points, ob, ci, pi, device="cpu").track_stats is None
    q = tc.BundleAdjustmentProblem.from_arrays(d.cameras, d.points, d.observations, d.camera_index,
                                               d.point_index, device="cpu", track_stats=True)
    assert q.track_stats == (int(np.bincount(d.point_index).max()), False)
    q.point_index[0] = 1  # an in-place change drops the statistics
    assert q.track_stats is None


@pytest.mark.parametrize("seed", range(20))
def test_slot_bound_holds_for_any_track_lengths(seed):
    """The host slot bound used without a device read: for track lengths sorted in
    descending order and cut into slices of 32, 32 * sum of the slice maxima is at most
    32 * max_track + no (each slice after the first is no longer than the mean of the
    slice before it)."""
    rng = np.random.default_rng(seed)
    npts = int(rng.integers(1, 3000))
    kind = seed % 4
    if kind == 0:
        c = rng.integers(1, 8, npts)
    elif kind == 1:
        c = rng.geometric(0.2, npts)
    elif kind == 2:  # one very long track among short ones
        c = np.ones(npts, dtype=np.int64)
        c[rng.integers(npts)] = int(rng.integers(50, 5000))
    else:  # steps just across slice boundaries
        c = np.repeat(rng.integers(1, 40, (npts + 32) // 33), 33)[:npts]
    c = np.sort(c)[::-1]
    pad = np.zeros(32 * ((npts + 31) // 32), dtype=np.int64)
    pad[:npts] = c
    slots = 32 * int(pad.reshape(-1, 32).max(axis=1).sum())
    assert slots <= 32 * int(c.max()) + int(c.sum())
