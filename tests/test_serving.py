"""Serving loop: continuous batching with admission by device footprint.

Requests submitted in a burst run as several overlapping batches; each result is the
same request solved alone in its own launch, bit for bit (one cluster per problem with
the same cluster size and CTA shape, and every sum of the batched kernel in a fixed
order), and the in-flight footprint never exceeds the budget.
"""
from __future__ import annotations

import numpy as np
import pytest

from ceres_torch_cuda_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _setup(count=12, seed=4):
    import ceres_torch_cuda_b200 as tc
    arrivals, datas = S.make_serving_requests(count, seed=seed, max_cameras=12, points_per_camera=40)
    opts = tc.SolverOptions(linear_solver_type=tc.LinearSolverType.ITERATIVE_SCHUR,
                            preconditioner_type=tc.PreconditionerType.SCHUR_JACOBI, max_num_iterations=30)

    def probs():
        return [tc.BundleAdjustmentProblem.from_arrays(d.cameras, d.points, d.observations, d.camera_index,
                                                       d.point_index) for d in datas]
    return tc, opts, arrivals, probs


def test_server_results_equal_alone_and_batches_overlap():
    tc, opts, _, probs = _setup()
    from ceres_torch_cuda_b200.serving import BAServer
    ps = probs()
    cut = int(np.median([p.num_observations for p in ps]))
    classes = ((cut, 1), (None, 2))  # two size classes, so batches of both cluster sizes run
    server = BAServer(opts, precision="fp64", max_inflight=3, max_batch=3, cluster_size=0, size_classes=classes,
                      min_batch=1)
    reqs = [server.submit(p) for p in ps]
    server.drain()
    assert server.launches >= 4
    assert server.peak_inflight >= 2
    # the same CTA shape as the server's (the shape fixes the order of the block sums)
    alone = [tc.solve_batch(opts, [p], precision="fp64", cluster_size=1 if p.num_observations < cut else 2,
                            threads_per_cta=server.threads_per_cta, ctas_per_sm=server.ctas_per_sm)[0]
             for p in probs()]
    for r, a in zip(reqs, alone):
        assert r.summary is not None and r.latency is not None and r.latency >= 0
        assert r.summary.final_cost == a.final_cost
        assert [it.cost for it in r.summary.iterations] == [it.cost for it in a.iterations]


def test_server_respects_memory_budget_and_stream_replay():
    tc, opts, arrivals, probs = _setup(count=10, seed=6)
    from ceres_torch_cuda_b200.serving import BAServer, footprint_bytes, run_stream
    ps = probs()
    biggest = max(footprint_bytes(p, "mixed") for p in ps)
    server = BAServer(opts, precision="mixed", memory_budget=2 * biggest, max_inflight=4, cluster_size=1,
                      min_batch=1)
    stats = run_stream(server, arrivals * 0.0 + np.linspace(0.0, 0.01, len(ps)), ps)
    assert server.peak_bytes <= 2 * biggest
    assert stats["requests"] == len(ps)
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    for r in stats["requests_list"]:
        assert r.summary.termination_type in (tc.TerminationType.CONVERGENCE, tc.TerminationType.NO_CONVERGENCE)


def test_mixed_server_results_equal_alone():
    """Mixed precision in the served mix: each request's result is the same request solved
    alone in its own launch, bit for bit, with several batches overlapping on the GPU."""
    tc, opts, _, probs = _setup(count=12, seed=8)
    from ceres_torch_cuda_b200.serving import BAServer
    server = BAServer(opts, precision="mixed", max_inflight=3, max_batch=3, cluster_size=1, min_batch=1)
    reqs = [server.submit(p) for p in probs()]
    server.drain()
    assert server.peak_inflight >= 2
    alone = [tc.solve_batch(opts, [p], precision="mixed", cluster_size=1, threads_per_cta=server.threads_per_cta,
                            ctas_per_sm=server.ctas_per_sm)[0] for p in probs()]
    for r, a in zip(reqs, alone):
        assert r.summary.final_cost == a.final_cost
        assert [it.cost for it in r.summary.iterations] == [it.cost for it in a.iterations]
