"""Generate golden fixtures by running the ceres-torch reference itself.

Run where the reference is checked out (read-only is fine), naming its root:

    python tests/golden/make_golden.py --reference <ceres-torch checkout> [--big]

Each fixture is an ``.npz`` holding the inputs (seeded synthetic BA problem),
what ceres-torch's own ``Problem.evaluate`` returns at the initial point
(cost, corrected residuals, the per-observation camera/point Jacobian blocks
cut out of its dense Jacobian, gradient), the Schur visibility it computes,
and what ``tc.solve`` returns (initial/final cost, iteration count and
per-iteration trace, termination, final parameters). ``losses.npz`` and
``rotation.npz`` pin the loss functions and the angle-axis rotation.

The problems are built exactly as the reference's BAL example builds them
(``examples/simple_bundle_adjuster.py:82-112``): one AutoDiff residual block per
observation calling the example's ``snavely_reprojection``, cameras added
first, points in ordering group 0. Nothing here is needed at test time; the
tests only read the ``.npz`` files.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from ceres_torch_cuda_b200 import synthetic as S  # noqa: E402


def _load_reference(root: Path):
    sys.path.insert(0, str(root / "src"))
    import ceres_torch as tc  # noqa: F401
    spec = importlib.util.spec_from_file_location("ref_simple_ba", root / "examples" / "simple_bundle_adjuster.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return tc, mod


def _loss_obj(tc, spec):
    kind = spec[0]
    if kind == "trivial":
        return None
    return {"huber": tc.HuberLoss, "cauchy": tc.CauchyLoss, "softlone": tc.SoftLOneLoss,
            "arctan": tc.ArctanLoss}[kind](float(spec[1]))


def _build(tc, ex, data, constant_cameras=()):
    import torch

    cams = torch.tensor(data.cameras, dtype=torch.float64)
    pts = torch.tensor(data.points, dtype=torch.float64)
    problem = tc.Problem()
    cam_blocks = [cams[i] for i in range(cams.shape[0])]
    pt_blocks = [pts[i] for i in range(pts.shape[0])]
    for i, c in enumerate(cam_blocks):
        problem.AddParameterBlock(c)
        if i in constant_cameras:
            problem.SetParameterBlockConstant(c)
    for p in pt_blocks:
        problem.AddParameterBlock(p)
        problem.SetParameterBlockOrderingGroup(p, 0)
    loss = _loss_obj(tc, data.loss)
    obs = torch.tensor(data.observations, dtype=torch.float64)
    for ci, pi, o in zip(data.camera_index.tolist(), data.point_index.tolist(), obs):
        problem.AddResidualBlock(
            tc.AutoDiffCostFunction(lambda camera, point, observation=o: ex.snavely_reprojection(camera, point) - observation,
                                    [9, 3], 2),
            loss,
            [cam_blocks[ci], pt_blocks[pi]],
        )
    return problem, cams, pts


def _evaluate_blocks(tc, problem, data, constant_cameras):
    """Initial-point evaluation, dense J cut into per-observation blocks."""
    from ceres_torch.solver import _linear_solver_parameter_order, _num_eliminate_for_schur, _schur_visibility_from_residual_blocks

    order = _linear_solver_parameter_order(problem)
    ev = problem.evaluate(tc.EvaluateOptions(parameter_blocks=order), compute_jacobian=True)
    J = ev.jacobian.numpy()
    npts = data.num_points
    nc = data.num_cameras
    active_cams = [c for c in range(nc) if c not in constant_cameras]
    cam_col = {c: 3 * npts + 9 * k for k, c in enumerate(active_cams)}
    no = data.num_observations
    Jc = np.zeros((no, 2, 9))
    Jp = np.zeros((no, 2, 3))
    for i, (c, p) in enumerate(zip(data.camera_index.tolist(), data.point_index.tolist())):
        Jp[i] = J[2 * i:2 * i + 2, 3 * p:3 * p + 3]
        if c in cam_col:
            Jc[i] = J[2 * i:2 * i + 2, cam_col[c]:cam_col[c] + 9]
    ne = _num_eliminate_for_schur(order, tc.LinearSolverType.ITERATIVE_SCHUR)
    vis = _schur_visibility_from_residual_blocks(problem, order, ne)
    vis_flat = np.array([p for t in vis for p in t], dtype=np.int64) if vis else np.zeros(0, np.int64)
    vis_len = np.array([len(t) for t in vis], dtype=np.int64) if vis else np.zeros(0, np.int64)
    return dict(eval_cost=float(ev.cost), eval_residuals=ev.residuals.numpy().reshape(-1, 2), eval_Jc=Jc, eval_Jp=Jp,
                eval_gradient=ev.gradient.numpy(), num_eliminate=ne, visibility_flat=vis_flat, visibility_len=vis_len)


def make_case(tc, ex, name, data, *, solver, preconditioner="SCHUR_JACOBI", constant_cameras=(), max_iter=50, out=HERE,
              spse=None, clustering=None):
    """``spse``: further SolverOptions fields (stored in meta["spse"], which the tests pass
    back); ``clustering``: the visibility_clustering_type name (stored there as a string)."""
    t0 = time.time()
    problem, cams, pts = _build(tc, ex, data, constant_cameras)
    blocks = _evaluate_blocks(tc, problem, data, constant_cameras)
    spse = dict(spse or {})
    extra = dict(spse)
    if clustering is not None:
        extra["visibility_clustering_type"] = getattr(tc.VisibilityClusteringType, clustering)
        spse["visibility_clustering_type"] = clustering
    opts = tc.SolverOptions(
        max_num_iterations=max_iter,
        linear_solver_type=getattr(tc.LinearSolverType, solver),
        preconditioner_type=getattr(tc.PreconditionerType, preconditioner),
        **extra,
    )
    summary = tc.solve(opts, problem)
    trace = np.array([[it.iteration, it.cost, it.cost_change, it.gradient_max_norm, it.step_norm,
                       it.relative_decrease, it.trust_region_radius, it.linear_solver_iterations,
                       float(it.step_is_successful)] for it in summary.iterations])
    meta = dict(name=name, solver=solver, preconditioner=preconditioner, loss=list(data.loss),
                constant_cameras=list(constant_cameras), max_num_iterations=max_iter, spse=spse,
                termination=summary.termination_type.value, message=summary.message,
                initial_cost=summary.initial_cost, final_cost=summary.final_cost,
                num_iterations=len(summary.iterations), num_successful_steps=summary.num_successful_steps,
                num_unsuccessful_steps=summary.num_unsuccessful_steps, description=data.description,
                seconds=time.time() - t0)
    np.savez_compressed(
        out / f"{name}.npz",
        cameras=data.cameras, points=data.points, observations=data.observations,
        camera_index=data.camera_index, point_index=data.point_index,
        final_cameras=cams.numpy(), final_points=pts.numpy(), trace=trace,
        meta=np.array(json.dumps(meta)), **blocks,
    )
    print(f"{name}: {meta['termination']} '{meta['message']}' iters={meta['num_iterations']} "
          f"cost {meta['initial_cost']:.6e} -> {meta['final_cost']:.6e} ({meta['seconds']:.1f}s)", flush=True)


def make_losses(tc, out=HERE):
    import torch

    s = torch.tensor([0.0, 1e-6, 0.25, 0.9, 1.0, 1.1, 4.0, 9.0, 100.0, 1e4], dtype=torch.float64)
    specs = {
        "trivial": tc.TrivialLoss(), "huber_1": tc.HuberLoss(1.0), "huber_2": tc.HuberLoss(2.0),
        "softlone_1": tc.SoftLOneLoss(1.0), "cauchy_1": tc.CauchyLoss(1.0), "cauchy_2": tc.CauchyLoss(2.0),
        "arctan_1": tc.ArctanLoss(1.0), "tolerant_1_1": tc.TolerantLoss(1.0, 1.0), "tukey_2": tc.TukeyLoss(2.0),
        "scaled_cauchy_2_3": tc.ScaledLoss(tc.CauchyLoss(2.0), 3.0),
        "composed_cauchy2_softlone1": tc.ComposedLoss(tc.CauchyLoss(2.0), tc.SoftLOneLoss(1.0)),
    }
    arrays = {"s": s.numpy()}
    for k, loss in specs.items():
        r0, r1, r2 = loss.evaluate(s)
        arrays[k] = np.stack([r0.numpy(), r1.numpy(), r2.numpy()])
    # corrector (losses.py:158-193) on a few residual/Jacobian pairs
    rng = np.random.default_rng(5)
    res = rng.normal(0, 2.0, size=(6, 2))
    jac = rng.normal(0, 1.0, size=(6, 2, 12))
    for k in ("huber_1", "cauchy_2", "tolerant_1_1", "softlone_1"):
        rows = []
        for i in range(res.shape[0]):
            c, r, J = _robustify(k, specs, res[i], jac[i])
            rows.append(np.concatenate([[float(c)], r.numpy(), J.numpy().reshape(-1)]))
        arrays[f"corrector_{k}"] = np.array(rows)
    arrays["corrector_residuals"] = res
    arrays["corrector_jacobians"] = jac
    np.savez_compressed(out / "losses.npz", **arrays)
    print("losses.npz written", flush=True)


def _robustify(k, specs, r, J):
    import torch
    from ceres_torch.losses import robustify_residual_and_jacobian

    return robustify_residual_and_jacobian(specs[k], torch.tensor(r), torch.tensor(J))


def make_rotation(tc, out=HERE):
    import torch

    rng = np.random.default_rng(11)
    aa = rng.normal(0.0, 1.0, size=(32, 3))
    aa[0] = 0.0
    aa[1] = [1e-17, 0.0, 0.0]
    aa[2] = [0.0, 0.0, np.pi / 2]
    aa[3] = [np.pi, 0.0, 0.0]
    X = rng.normal(0.0, 2.0, size=(32, 3))
    out_pts = np.stack([tc.angle_axis_rotate_point(torch.tensor(a), torch.tensor(x)).numpy() for a, x in zip(aa, X)])
    np.savez_compressed(out / "rotation.npz", angle_axis=aa, points=X, rotated=out_pts)
    print("rotation.npz written", flush=True)


def make_covariance(tc, ex, name, data, *, constant_cameras, out=HERE, point_blocks=5):
    """Solve with the reference (DENSE_SCHUR, its default tolerances), then its own
    Covariance (covariance.py:86-445, DENSE_SVD, default options) of every free camera
    pair, the first ``point_blocks`` points and camera-point pairs at the solution."""
    problem, cams, pts = _build(tc, ex, data, constant_cameras)
    t0 = time.time()
    summary = tc.solve(tc.SolverOptions(linear_solver_type=tc.LinearSolverType.DENSE_SCHUR), problem)
    blocks = problem.parameter_blocks
    cam_blocks, pt_blocks = blocks[:data.num_cameras], blocks[data.num_cameras:]
    free = [i for i in range(data.num_cameras) if i not in constant_cameras]
    chosen_pts = list(range(min(point_blocks, data.num_points)))
    pairs = [(cam_blocks[i], cam_blocks[j]) for a, i in enumerate(free) for j in free[a:]]
    pairs += [(pt_blocks[q], pt_blocks[q]) for q in chosen_pts]
    pairs += [(cam_blocks[free[0]], pt_blocks[q]) for q in chosen_pts] if free else []
    cov = tc.Covariance()
    ok = cov.compute(pairs, problem)
    cc = np.zeros((len(free), len(free), 9, 9))
    pp = np.zeros((len(chosen_pts), 3, 3))
    cp = np.zeros((len(chosen_pts), 9, 3))
    if ok:
        for a, i in enumerate(free):
            for b, j in enumerate(free):
                cc[a, b] = cov.get_covariance_block(cam_blocks[i], cam_blocks[j]).numpy()
        for k, q in enumerate(chosen_pts):
            pp[k] = cov.get_covariance_block(pt_blocks[q], pt_blocks[q]).numpy()
            if free:
                cp[k] = cov.get_covariance_block(cam_blocks[free[0]], pt_blocks[q]).numpy()
    meta = {"name": name, "loss": list(data.loss), "constant_cameras": list(constant_cameras), "free_cameras": free,
            "points": chosen_pts, "success": bool(cov.summary.success), "message": cov.summary.message,
            "rank": int(cov.summary.rank), "nullity": int(cov.summary.nullity),
            "tangent_dimension": int(cov.summary.tangent_dimension), "final_cost": float(summary.final_cost),
            "seconds": time.time() - t0}
    np.savez_compressed(out / f"{name}.npz", meta=json.dumps(meta), cameras=data.cameras, points=data.points,
                        observations=data.observations, camera_index=data.camera_index,
                        point_index=data.point_index, solved_cameras=cams.numpy(), solved_points=pts.numpy(),
                        cov_cameras=cc, cov_points=pp, cov_camera_point=cp)
    print(f"{name}: success={cov.summary.success} rank={cov.summary.rank} ({meta['seconds']:.1f} s)", flush=True)


def _visibility(nc, camera_index, point_index):
    vis = [set() for _ in range(nc)]
    for c, p in zip(np.asarray(camera_index).tolist(), np.asarray(point_index).tolist()):
        vis[c].add(int(p))
    return [sorted(v) for v in vis]


def make_clustering(tc, out=HERE):
    """The reference's visibility clustering (linear.py:842-1028) on visibility lists of
    capture sequences, uniform problems and hand-made edge cases, for both clustering
    types and both cluster preconditioners: membership, cluster pairs, kept block pairs
    and the two similarity graphs."""
    from ceres_torch.linear import build_visibility_cluster_structure

    cases = {}
    for nc, npts, w, closed, seed in ((12, 200, 3, False, 5), (10, 150, 4, True, 6), (16, 300, 3, False, 7),
                                      (30, 600, 4, False, 8), (40, 500, 2, True, 9)):
        d = S.make_sequence_ba(nc, npts, w, seed=seed, closed=closed)
        cases[f"sequence_{nc}_{w}{'_closed' if closed else ''}"] = _visibility(nc, d.camera_index, d.point_index)
    for nc, npts, t, seed in ((8, 60, 3, 1), (20, 300, 4, 2), (6, 10, 2, 3), (25, 80, 2, 4)):
        d = S.make_small_ba(nc, npts, t, seed=seed)
        cases[f"uniform_{nc}_{npts}_{t}"] = _visibility(nc, d.camera_index, d.point_index)
    cases["edge_empty_and_duplicates"] = [[0, 1, 2, 2], [2, 3], [], [0, 1, 2], [5], [5, 6]]
    cases["edge_identical_views"] = [[0, 1, 2], [0, 1, 2], [0, 1, 2], [7, 8], [7, 8], [9]]
    cases["edge_single_camera"] = [[0, 1, 2]]
    cases["edge_disjoint"] = [[0], [1], [2], [3]]
    results = {}
    for cname, vis in cases.items():
        for pre in ("CLUSTER_JACOBI", "CLUSTER_TRIDIAGONAL"):
            for kind in ("CANONICAL_VIEWS", "SINGLE_LINKAGE"):
                st = build_visibility_cluster_structure(
                    vis, preconditioner_type=getattr(tc.PreconditionerType, pre),
                    visibility_clustering_type=getattr(tc.VisibilityClusteringType, kind))
                results[f"{cname}|{pre}|{kind}"] = dict(
                    membership=list(st.membership), num_clusters=st.num_clusters,
                    cluster_pairs=[list(p) for p in st.cluster_pairs], block_pairs=[list(p) for p in st.block_pairs],
                    camera_graph_edges=[list(e) for e in st.camera_graph_edges],
                    cluster_graph_edges=[list(e) for e in st.cluster_graph_edges])
    np.savez_compressed(out / "clustering.npz", visibility=np.array(json.dumps(cases)),
                        results=np.array(json.dumps(results)))
    print(f"clustering.npz written ({len(results)} structures)", flush=True)


def make_bal(ex, name, data, out=HERE):
    """BAL text of ``data`` (the format BALProblem.from_text reads,
    examples/simple_bundle_adjuster.py:33-70) and what the reference parser returns."""
    lines = [f"{data.num_cameras} {data.num_points} {data.num_observations}"]
    for c, q, o in zip(data.camera_index.tolist(), data.point_index.tolist(), data.observations.tolist()):
        lines.append(f"{c} {q} {o[0]!r} {o[1]!r}")
    lines += [repr(float(v)) for v in data.cameras.reshape(-1)]
    lines += [repr(float(v)) for v in data.points.reshape(-1)]
    text = "\n".join(lines) + "\n"
    bal = ex.BALProblem.from_text(text)
    np.savez_compressed(out / f"{name}.npz", meta=json.dumps({"name": name}), text=np.array(text),
                        camera_indices=np.array(bal.camera_indices, dtype=np.int64),
                        point_indices=np.array(bal.point_indices, dtype=np.int64),
                        observations=bal.observations.numpy(), cameras=bal.cameras.numpy(), points=bal.points.numpy())
    print(f"{name}: {bal.num_cameras} cameras, {bal.num_points} points, {bal.num_observations} observations", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of a ceres-torch checkout (src/, examples/)")
    ap.add_argument("--big", action="store_true", help="also run config0 at full size (minutes)")
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    tc, ex = _load_reference(Path(args.reference))
    only = set(filter(None, args.only.split(",")))

    def want(n):
        return not only or n in only

    if want("losses"):
        make_losses(tc)
    if want("rotation"):
        make_rotation(tc)
    small = S.make_small_ba(4, 30, 3, seed=1)
    if want("ba_small_iterative"):
        make_case(tc, ex, "ba_small_iterative", small, solver="ITERATIVE_SCHUR")
    if want("ba_small_dense"):
        make_case(tc, ex, "ba_small_dense", small, solver="DENSE_SCHUR")
    if want("ba_small_sparse"):
        make_case(tc, ex, "ba_small_sparse", small, solver="SPARSE_SCHUR")
    if want("ba_huber_outliers"):
        hub = S.make_small_ba(5, 40, 3, seed=2, loss=("huber", 1.0), outlier_fraction=0.1)
        make_case(tc, ex, "ba_huber_outliers", hub, solver="ITERATIVE_SCHUR")
    if want("ba_cauchy"):
        cau = S.make_small_ba(5, 40, 3, seed=3, loss=("cauchy", 2.0), outlier_fraction=0.05)
        make_case(tc, ex, "ba_cauchy", cau, solver="ITERATIVE_SCHUR")
    if want("ba_const_camera_jacobi"):
        cc = S.make_small_ba(3, 20, 3, seed=4)
        cc.cameras[1, 0:3] = 0.0  # theta == 0 branch of the angle-axis conversion
        make_case(tc, ex, "ba_const_camera_jacobi", cc, solver="ITERATIVE_SCHUR", preconditioner="JACOBI",
                  constant_cameras=(0,))
    if want("ba_fixed_cameras"):
        fx = S.make_small_ba(2, 6, 2, seed=6)
        make_case(tc, ex, "ba_fixed_cameras", fx, solver="DENSE_SCHUR", constant_cameras=(0, 1), max_iter=40)
    if want("ba_spse"):
        sp = S.make_small_ba(5, 40, 3, seed=7)
        make_case(tc, ex, "ba_spse", sp, solver="ITERATIVE_SCHUR", preconditioner="SCHUR_POWER_SERIES_EXPANSION")
    if want("ba_spse_cauchy"):
        sc = S.make_small_ba(6, 50, 3, seed=8, loss=("cauchy", 2.0), outlier_fraction=0.05)
        make_case(tc, ex, "ba_spse_cauchy", sc, solver="ITERATIVE_SCHUR", preconditioner="SCHUR_POWER_SERIES_EXPANSION",
                  spse=dict(max_num_spse_iterations=8, spse_tolerance=0.01))
    if want("ba_spse_init"):
        si = S.make_small_ba(5, 40, 3, seed=9)
        make_case(tc, ex, "ba_spse_init", si, solver="ITERATIVE_SCHUR",
                  spse=dict(use_spse_initialization=True, max_num_spse_iterations=3))
    if want("ba_covariance"):
        cv = S.make_small_ba(6, 40, 4, seed=10)
        make_covariance(tc, ex, "ba_covariance", cv, constant_cameras=(0, 1))
    if want("ba_covariance_cauchy"):
        cvc = S.make_small_ba(5, 40, 4, seed=11, loss=("cauchy", 2.0), outlier_fraction=0.05)
        make_covariance(tc, ex, "ba_covariance_cauchy", cvc, constant_cameras=(0, 2))
    if want("ba_covariance_gauge"):
        cvg = S.make_small_ba(4, 30, 3, seed=12)
        make_covariance(tc, ex, "ba_covariance_gauge", cvg, constant_cameras=())
    if want("bal_text"):
        make_bal(ex, "bal_text", S.make_small_ba(7, 60, 3, seed=13))
    if want("clustering"):
        make_clustering(tc)
    if want("ba_cluster_jacobi"):
        make_case(tc, ex, "ba_cluster_jacobi", S.make_sequence_ba(12, 200, 3, seed=14), solver="ITERATIVE_SCHUR",
                  preconditioner="CLUSTER_JACOBI")
    if want("ba_cluster_tridiagonal"):
        make_case(tc, ex, "ba_cluster_tridiagonal", S.make_sequence_ba(16, 240, 3, seed=15, loss=("cauchy", 2.0)),
                  solver="ITERATIVE_SCHUR", preconditioner="CLUSTER_TRIDIAGONAL")
    if want("ba_cluster_single_linkage"):
        make_case(tc, ex, "ba_cluster_single_linkage", S.make_sequence_ba(10, 150, 4, seed=16, closed=True),
                  solver="ITERATIVE_SCHUR", preconditioner="CLUSTER_TRIDIAGONAL", clustering="SINGLE_LINKAGE",
                  constant_cameras=(0,))
    if want("ba_cluster_uniform"):
        make_case(tc, ex, "ba_cluster_uniform", S.make_small_ba(8, 80, 3, seed=17), solver="ITERATIVE_SCHUR",
                  preconditioner="CLUSTER_JACOBI", clustering="SINGLE_LINKAGE")
    if args.big and want("config0_dense"):
        make_case(tc, ex, "config0_dense", S.ba_config(0), solver="DENSE_SCHUR")
    if args.big and want("config1_small"):
        make_case(tc, ex, "config1_small", S.ba_config(1, scale=0.005), solver="ITERATIVE_SCHUR")
    if args.big and want("config2_small"):
        make_case(tc, ex, "config2_small", S.ba_config(2, scale=0.0004), solver="ITERATIVE_SCHUR")


if __name__ == "__main__":
    main()
