"""The host side of the trust-region loop (engine.run_lm) on the CPU.

run_lm drives the device kernels through a small engine interface (evaluate, assemble,
pcg or dense_solve, step, read_stats, accept, save_best, restore_best). Here that
interface is backed by the oracle's float64 numerics (evaluation, damped Schur solve,
candidate cost, model decrease), so the loop's decisions can be checked against the
oracle's own restatement of solver.py:35-357 (oracle.ba_oracle.solve), which is pinned
to the reference's traces: the same costs, radii, step validity and acceptance, linear
iteration counts, counters and termination, including the pipelined evaluation after an
accepted step (its gradient test runs before anything of the next iteration is used).
"""
from __future__ import annotations

import time

import numpy as np
import pytest

from ceres_torch_cuda_b200 import _lib
from ceres_torch_cuda_b200 import engine as E
from ceres_torch_cuda_b200 import synthetic as S
from ceres_torch_cuda_b200 import types as T
from oracle import ba_oracle as O


class OracleEngine:
    """The engine interface of run_lm over the oracle's numerics (statistics slots as the
    device writes them: the evaluation's and the step's are disjoint)."""

    precision = "fp64"

    def __init__(self, prob: O.OracleProblem, opts: O.OracleOptions):
        self.prob, self.opts = prob, opts
        self.cams, self.pts = prob.cameras.copy(), prob.points.copy()
        self.nc = prob.cameras.shape[0]
        self.stats = np.zeros(_lib.NSTATS)
        self.best = None
        self.calls: list[str] = []

    def setup_clusters(self, tridiagonal, clustering):
        return False

    def evaluate(self, jacobian):
        self.calls.append("evaluate")
        self.ev = O.evaluate(self.prob, self.cams, self.pts)
        g = O._gradient(self.prob, self.ev)
        n_p = 3 * self.prob.active_pts.size
        gp, gc = g[:n_p], g[n_p:]
        st = self.stats
        st[_lib.STAT_COST] = self.ev.cost
        st[_lib.STAT_GMAX_P] = float(np.max(np.abs(gp))) if gp.size else 0.0
        st[_lib.STAT_GMAX_C] = float(np.max(np.abs(gc))) if gc.size else 0.0
        st[_lib.STAT_GSQ_P] = float(gp @ gp)
        st[_lib.STAT_GSQ_C] = float(gc @ gc)

    def assemble(self, radius, options, precond, spse_base=False):
        self.calls.append("assemble")
        self.radius = radius

    def pcg(self, *args, **kwargs):
        self.calls.append("pcg")
        self.xa, self.xb, its = O.solve_step(self.prob, self.ev, self.radius, self.opts,
                                             explicit_limit=self.opts.explicit_schur_limit)
        self.stats[_lib.STAT_PCG_ITERS] = its

    def dense_solve(self):
        self.calls.append("dense")
        self.xa, self.xb, _ = O.solve_step(self.prob, self.ev, self.radius, self.opts)

    def step(self):
        self.calls.append("step")
        st, prob, ev = self.stats, self.prob, self.ev
        step = np.concatenate([self.xa.reshape(-1), self.xb.reshape(-1)])
        if not np.all(np.isfinite(step)):
            st[_lib.STAT_NONFINITE] = 1.0
            return
        st[_lib.STAT_NONFINITE] = 0.0
        self.cand_cams, self.cand_pts = self.cams.copy(), self.pts.copy()
        self.cand_pts[prob.active_pts] += self.xa
        self.cand_cams[prob.active_cams] += self.xb
        st[_lib.STAT_CAND_COST] = O.evaluate(prob, self.cand_cams, self.cand_pts, jacobians=False).cost
        pt = prob.pt_col[prob.point_index]
        cam = prob.cam_col[prob.camera_index]
        jd = np.zeros_like(ev.r)
        m = pt >= 0
        jd[m] += np.einsum("nij,nj->ni", ev.Jp[m], self.xa[pt[m]])
        m = cam >= 0
        jd[m] += np.einsum("nij,nj->ni", ev.Jc[m], self.xb[cam[m]])
        after = (ev.r + jd).reshape(-1)
        st[_lib.STAT_MODEL] = 0.5 * float(ev.r.reshape(-1) @ ev.r.reshape(-1)) - 0.5 * float(after @ after)
        st[_lib.STAT_STEP_SQ_P] = float(np.sum(self.xa ** 2))
        st[_lib.STAT_STEP_SQ_C] = float(np.sum(self.xb ** 2))
        st[_lib.STAT_CAND_STATE_SQ_P] = float(np.sum(self.cand_pts ** 2))
        st[_lib.STAT_CAND_STATE_SQ_C] = float(np.sum(self.cand_cams ** 2))

    def read_stats(self):
        self.calls.append("read")
        return self.stats.copy()

    def accept(self):
        self.cams, self.pts = self.cand_cams, self.cand_pts

    def save_best(self):
        self.best = (self.cams.copy(), self.pts.copy())

    def restore_best(self):
        self.cams, self.pts = (a.copy() for a in self.best)


def _run(d, loss=("trivial",), constant_cameras=(), **kw):
    cc = np.zeros(d.num_cameras, dtype=bool)
    cc[list(constant_cameras)] = True
    prob = O.OracleProblem(d.cameras, d.points, d.observations, d.camera_index, d.point_index, loss,
                           camera_constant=cc)
    okw = {k: v for k, v in kw.items()}
    oopts = O.OracleOptions(**okw)
    ref = O.solve(prob, oopts)
    tkw = dict(okw)
    tkw["linear_solver_type"] = getattr(T.LinearSolverType, okw.get("linear_solver_type", "ITERATIVE_SCHUR"))
    tkw["preconditioner_type"] = getattr(T.PreconditionerType, okw.get("preconditioner_type", "SCHUR_JACOBI"))
    tkw.pop("explicit_schur_limit", None)
    opts = T.SolverOptions(**tkw)
    eng = OracleEngine(prob, oopts)
    summary = T.SolverSummary()
    ncols = 3 * prob.active_pts.size + 9 * prob.active_cams.size
    res = E.run_lm(eng, opts, summary, start=time.perf_counter(), num_active_columns=ncols)
    return ref, res.summary, eng


def _compare(ref, s):
    assert s.termination_type.value == ref.termination and s.message == ref.message
    assert len(s.iterations) == len(ref.iterations)
    for a, b in zip(s.iterations, ref.iterations):
        assert a.iteration == b.iteration
        assert a.cost == b.cost
        assert a.trust_region_radius == b.trust_region_radius
        assert (a.step_is_valid, a.step_is_successful) == (b.step_is_valid, b.step_is_successful)
        assert a.gradient_max_norm == pytest.approx(b.gradient_max_norm, rel=1e-12, abs=0.0, nan_ok=True)
        if a.iteration:
            assert a.linear_solver_iterations == b.linear_solver_iterations
            assert a.relative_decrease == b.relative_decrease
            assert a.step_norm == pytest.approx(b.step_norm, rel=1e-12, nan_ok=True)
    assert s.initial_cost == ref.initial_cost and s.final_cost == ref.final_cost
    assert s.num_successful_steps == ref.num_successful_steps
    assert s.num_unsuccessful_steps == ref.num_unsuccessful_steps


CASES = [
    dict(data=(8, 200, 3, 1), kw=dict(max_num_iterations=25)),
    dict(data=(10, 300, 4, 2), kw=dict(max_num_iterations=30, function_tolerance=1e-12), loss=("cauchy", 2.0)),
    dict(data=(6, 150, 3, 3), kw=dict(linear_solver_type="DENSE_SCHUR", max_num_iterations=20)),
    dict(data=(9, 250, 4, 4), kw=dict(max_num_iterations=30, use_nonmonotonic_steps=True,
                                      max_consecutive_nonmonotonic_steps=3, function_tolerance=1e-14),
         loss=("huber", 1.0)),
    dict(data=(7, 180, 3, 5), kw=dict(max_num_iterations=40, initial_trust_region_radius=1e10,
                                      function_tolerance=1e-15, parameter_tolerance=1e-14)),
    dict(data=(8, 200, 3, 6), kw=dict(max_num_iterations=4)),
    dict(data=(8, 220, 3, 7), kw=dict(max_num_iterations=30, gradient_tolerance=1e-2, function_tolerance=1e-16)),
    dict(data=(8, 220, 3, 8), kw=dict(max_num_iterations=30, parameter_tolerance=1e-3), constant=(0, 1)),
]


@pytest.mark.parametrize("case", CASES, ids=[f"case{i}" for i in range(len(CASES))])
def test_run_lm_decides_like_the_oracle_loop(case):
    d = S.make_small_ba(*case["data"][:3], seed=case["data"][3])
    ref, s, eng = _run(d, case.get("loss", ("trivial",)), case.get("constant", ()), **case["kw"])
    _compare(ref, s)
    # the best state is what the solve leaves behind
    assert np.array_equal(eng.cams, ref.cameras) and np.array_equal(eng.pts, ref.points)


def test_one_read_per_iteration():
    """The loop reads the statistics once per LM iteration (the evaluation after an
    accepted step is queued behind the next linear solve and step), plus the first
    evaluation's read and the last accepted point's gradient test."""
    d = S.make_small_ba(8, 200, 3, seed=1)
    ref, s, eng = _run(d, max_num_iterations=25)
    _compare(ref, s)
    assert eng.calls.count("read") <= len(s.iterations) + 1
    # an evaluation never waits for its own read: the next pcg and step come first
    for k, c in enumerate(eng.calls[:-3]):
        if c == "evaluate" and k > 0:
            assert eng.calls[k + 1:k + 4] == ["assemble", "pcg", "step"]


def test_invalid_steps_end_the_solve_like_the_oracle_loop():
    """A camera whose focal length overflows every step: non-finite steps are invalid
    (radius halved, then quartered ...) until max_num_consecutive_invalid_steps of them
    end the solve with FAILURE (solver.py:168-190)."""
    d = S.make_small_ba(3, 20, 3, seed=13)
    d.cameras[0, 6] = 1e308
    with np.errstate(over="ignore", invalid="ignore"):
        ref, s, eng = _run(d, max_num_iterations=10)
    assert s.termination_type.value == "FAILURE" and ref.termination == "FAILURE"
    _compare(ref, s)
