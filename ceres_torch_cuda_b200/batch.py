"""Batched solves: many independent bundle-adjustment problems in one persistent launch.

``solve_batch(options, problems)`` concatenates the problems into one device
layout (each problem keeps its own slices, cameras and points) and calls
``ceres_b200_batch_solve`` once: every CTA takes whole problems from a work
counter and runs their complete Levenberg-Marquardt solves on the device (the
decisions of ceres-torch's solver.py:35-357, monotonic steps, ITERATIVE_SCHUR).
A problem's result does not depend on the rest of the batch. The reference has no
batched API; each problem there is one ``tc.solve`` call.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .engine import _PRECOND
from .losses import device_loss
from .problem import BundleAdjustmentProblem
from .solver import _new_summary
from .types import (IterationSummary, LinearSolverType, MinimizerType, PreconditionerType, SolverOptions,
                    SolverSummary, TerminationType, TrustRegionStrategyType)

_TERMS = {_lib.TERM_CONVERGENCE: TerminationType.CONVERGENCE, _lib.TERM_NO_CONVERGENCE: TerminationType.NO_CONVERGENCE,
          _lib.TERM_FAILURE: TerminationType.FAILURE}


@dataclass
class BatchLayout:
    """Concatenated sliced-ELL layout of a batch (see include/ceres_b200.h)."""

    num_problems: int
    cam_off: torch.Tensor        # int32 [B+1]
    slice_off: torch.Tensor      # int32 [B+1]
    slice_base: torch.Tensor     # int32 [S]
    slice_len: torch.Tensor      # int32 [S]
    slot_cam: torch.Tensor       # int32 [slots], camera index local to the problem, -1 padding
    slot_obs: torch.Tensor       # float64 [slots, 2]
    cam_offsets: torch.Tensor    # int32 [C+1]
    cam_entries: torch.Tensor    # int32 [no, 2] (global slot, global sorted point)
    lane_point: torch.Tensor     # int64 [32 S] global input point id of each lane, -1 padding
    num_slots: int
    has_duplicate_cameras: bool
    max_cameras: int
    num_slices: int


def batch_ints(cam_counts: np.ndarray, pt_counts: np.ndarray) -> np.ndarray:
    """The per-problem integers build_batch_layout needs on the device, in its order."""
    B = len(cam_counts)
    pt_off_in = np.zeros(B + 1, dtype=np.int64)
    pt_off_in[1:] = np.cumsum(pt_counts)
    cam_off = np.zeros(B + 1, dtype=np.int64)
    cam_off[1:] = np.cumsum(cam_counts)
    slice_off = np.zeros(B + 1, dtype=np.int64)
    slice_off[1:] = np.cumsum((pt_counts + 31) // 32)
    return np.concatenate([pt_counts, pt_off_in[:-1], 32 * slice_off[:-1], cam_counts, cam_off, slice_off]).astype(
        np.int64)


def build_batch_layout(cam_counts: np.ndarray, pt_counts: np.ndarray, camera_index: torch.Tensor,
                       point_index: torch.Tensor, observations: torch.Tensor, *, ints: torch.Tensor | None = None,
                       obs_counts: np.ndarray | None = None, track_stats: list | None = None) -> BatchLayout:
    """``camera_index`` / ``point_index`` are global (problem offsets added). Points are
    sorted by track length (descending, stable in point id) within their problem, and
    each problem is padded to whole slices of 32. Device work on the current stream.

    ``ints``: batch_ints(cam_counts, pt_counts) already on the device (else copied here).
    ``track_stats``: each problem's (most observations of one point, duplicate flag) with
    ``obs_counts``; the slot count is then taken from the host bound
    sum_p (32 max_track_p + no_p) (slice s >= 1 of a problem is no longer than the mean
    track of slice s - 1, so a problem's slices hold at most 32 max_track + no slots) and
    the layout is built with no device-to-host read; without them, one read (the slot
    count and the duplicate flag)."""
    dev = camera_index.device
    B = len(cam_counts)
    ci = camera_index.to(torch.int64)
    pi = point_index.to(torch.int64)
    no = int(ci.numel())
    NP = int(pt_counts.sum())
    NC = int(cam_counts.sum())
    S = int(((pt_counts + 31) // 32).sum())
    i64 = dict(dtype=torch.int64, device=dev)
    if ints is None:
        ints = torch.from_numpy(batch_ints(cam_counts, pt_counts)).to(dev)
    pt_counts_d, start_in, q_base, cam_counts_d, cam_off_d, slice_off_d = torch.split(
        ints, [B, B, B, B, B + 1, B + 1])
    point_problem = torch.repeat_interleave(torch.arange(B, device=dev), pt_counts_d, output_size=NP)
    counts = torch.zeros(NP, **i64)
    if no:
        counts.index_add_(0, pi, torch.ones(no, **i64))
    # grouped by problem, then by track length descending, stable in point id
    order = torch.argsort(point_problem * (1 << 32) + ((1 << 31) - 1 - counts), stable=True)
    pos = torch.arange(NP, device=dev) - start_in[point_problem[order]]
    q_of_sorted = q_base[point_problem[order]] + pos
    q_of_point = torch.empty(NP, **i64)
    q_of_point[order] = q_of_sorted
    lane_point = torch.full((32 * S,), -1, **i64)
    lane_point[q_of_sorted] = order
    counts_q = torch.zeros(32 * S, **i64)
    counts_q[q_of_sorted] = counts[order]
    slice_len = counts_q.view(S, 32).amax(dim=1) if S else counts_q[:0]
    csum = torch.cumsum(slice_len, 0)
    slice_base = 32 * (csum - slice_len)
    if track_stats is not None and obs_counts is not None:
        num_slots = int(sum(32 * t[0] for t in track_stats) + int(np.sum(obs_counts)))
        has_dup = any(bool(t[1]) for t in track_stats)
    else:
        dup = torch.zeros((), **i64)
        if no > 1:
            pk = torch.sort(pi * max(NC, 1) + ci).values
            dup = (pk[1:] == pk[:-1]).any().to(torch.int64)
        info = torch.stack([csum[-1] if S else torch.zeros((), **i64), dup]).cpu()
        num_slots = 32 * int(info[0])
        has_dup = bool(info[1])
    if no:
        obs_sorted = torch.argsort(pi, stable=True)
        pstart = torch.cumsum(counts, 0) - counts
        rank = torch.empty(no, **i64)
        rank[obs_sorted] = torch.arange(no, device=dev) - pstart[pi[obs_sorted]]
        q = q_of_point[pi]
        slot = slice_base[q // 32] + 32 * rank + (q % 32)
    else:
        q = torch.zeros(0, **i64)
        slot = q
    cam_problem = torch.repeat_interleave(torch.arange(B, device=dev), cam_counts_d, output_size=NC)
    local_cam = ci - cam_off_d[:-1][cam_problem[ci]] if no else ci
    slot_cam = torch.full((max(num_slots, 1),), -1, dtype=torch.int32, device=dev)
    slot_obs = torch.zeros((max(num_slots, 1), 2), dtype=torch.float64, device=dev)
    if no:
        slot_cam[slot] = local_cam.to(torch.int32)
        slot_obs[slot] = observations.to(torch.float64)
    perm = torch.argsort(ci * max(num_slots, 1) + slot)
    cam_entries = torch.stack([slot[perm], q[perm]], dim=1).to(torch.int32).contiguous() if no else \
        torch.zeros((1, 2), dtype=torch.int32, device=dev)
    cam_counts_t = torch.zeros(NC, **i64)
    if no:
        cam_counts_t.index_add_(0, ci, torch.ones(no, **i64))
    cam_offsets = torch.zeros(NC + 1, **i64)
    cam_offsets[1:] = torch.cumsum(cam_counts_t, 0)
    return BatchLayout(
        num_problems=B, cam_off=cam_off_d.to(torch.int32), slice_off=slice_off_d.to(torch.int32),
        slice_base=slice_base.to(torch.int32).contiguous(), slice_len=slice_len.to(torch.int32).contiguous(),
        slot_cam=slot_cam, slot_obs=slot_obs, cam_offsets=cam_offsets.to(torch.int32).contiguous(),
        cam_entries=cam_entries, lane_point=lane_point, num_slots=num_slots, has_duplicate_cameras=has_dup,
        max_cameras=int(cam_counts.max()) if B else 0, num_slices=S)


def _check_options(options: SolverOptions) -> None:
    options.validate()
    if options.minimizer_type is not MinimizerType.TRUST_REGION or \
            options.trust_region_strategy_type is not TrustRegionStrategyType.LEVENBERG_MARQUARDT:
        raise NotImplementedError("batched solves run Levenberg-Marquardt trust-region steps only")
    if options.linear_solver_type is not LinearSolverType.ITERATIVE_SCHUR:
        raise NotImplementedError("batched solves use ITERATIVE_SCHUR")
    if options.preconditioner_type not in _PRECOND or \
            options.preconditioner_type is PreconditionerType.SCHUR_POWER_SERIES_EXPANSION:
        raise NotImplementedError(f"batched solves support IDENTITY, JACOBI and SCHUR_JACOBI, not "
                                  f"{options.preconditioner_type.value}")
    if options.use_nonmonotonic_steps:
        raise NotImplementedError("batched solves take monotonic steps only")
    if options.callbacks:
        raise NotImplementedError("batched solves run without per-iteration callbacks")
    if options.use_inner_iterations or options.check_gradients or options.use_spse_initialization:
        raise NotImplementedError("inner iterations, gradient checks and SPSE are not part of batched solves")


class BatchSolver:
    """Device state of one batch; ``launch()`` enqueues the persistent kernel once."""

    def __init__(self, problems: list[BundleAdjustmentProblem], options: SolverOptions, *, precision: str = "mixed",
                 max_refinements: int = 1, stream: torch.cuda.Stream | None = None):
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        _check_options(options)
        if not problems:
            raise ValueError("empty batch")
        for i, p in enumerate(problems):
            if p.num_cameras == 0 or p.num_observations == 0:
                raise ValueError(f"problem {i} of the batch has no cameras or no observations")
        self.lib = _lib.load()
        self.problems = problems
        self.options = options
        self.precision = precision
        dev = problems[0].cameras.device
        if dev.type != "cuda":
            raise NotImplementedError("batched solves run on CUDA tensors only")
        self.device = dev
        loss_spec = device_loss(problems[0].loss)
        for p in problems[1:]:
            if device_loss(p.loss) != loss_spec:
                raise ValueError("all problems of a batch must use the same loss function")
        self.loss_spec = loss_spec
        cam_counts = np.array([p.num_cameras for p in problems], dtype=np.int64)
        pt_counts = np.array([p.num_points for p in problems], dtype=np.int64)
        cam_off = np.concatenate([[0], np.cumsum(cam_counts)])
        pt_off = np.concatenate([[0], np.cumsum(pt_counts)])
        self.cam_off_np, self.pt_off_np = cam_off, pt_off
        # global indices: each problem's indices plus its offsets, in a few batch-wide
        # operations; every per-problem integer goes up in one asynchronous copy from
        # pinned memory, so the host does not wait for the stream
        nb = len(problems)
        obs_counts = np.array([p.num_observations for p in problems], dtype=np.int64)
        host = torch.from_numpy(np.concatenate([cam_off[:-1], pt_off[:-1], obs_counts,
                                                batch_ints(cam_counts, pt_counts)])).pin_memory()
        dv = host.to(dev, non_blocking=True)
        offs, ints = dv[:3 * nb], dv[3 * nb:]
        per_obs = torch.repeat_interleave(torch.arange(nb, device=dev), offs[2 * nb:],
                                          output_size=int(obs_counts.sum()))
        ci = torch.cat([p.camera_index for p in problems]).to(dev, torch.int64) + offs[:nb][per_obs]
        pi = torch.cat([p.point_index for p in problems]).to(dev, torch.int64) + offs[nb:2 * nb][per_obs]
        obs = torch.cat([p.observations for p in problems]).to(dev, torch.float64)
        stats = [p.track_stats for p in problems]
        L = build_batch_layout(cam_counts, pt_counts, ci, pi, obs, ints=ints, obs_counts=obs_counts,
                               track_stats=None if any(t is None for t in stats) else stats)
        self.layout = L
        S = L.num_slices
        NQ = 32 * S
        NC = int(cam_off[-1])
        f64 = dict(dtype=torch.float64, device=dev)
        jt = torch.float32 if precision == "mixed" else torch.float64
        self.cameras = torch.cat([p.cameras for p in problems]).to(**f64).contiguous()
        # lanes -> input points; padding lanes (-1) read a zero row appended at the end
        NPin = int(pt_off[-1])
        self.lane_src = torch.where(L.lane_point >= 0, L.lane_point, torch.full_like(L.lane_point, NPin))
        pts_in = torch.cat([p.points for p in problems] + [problems[0].points.new_zeros((1, 3))]).to(**f64)
        self.points = pts_in.index_select(0, self.lane_src).contiguous()
        if all(p.camera_constant is None for p in problems):
            cam_const = torch.zeros(NC, dtype=torch.bool, device=dev)
        else:
            cam_const = torch.cat([(p.camera_constant if p.camera_constant is not None else
                                    torch.zeros(p.num_cameras, dtype=torch.bool, device=dev)).to(dev)
                                   for p in problems])
        if all(p.point_constant is None for p in problems):
            pc_in = torch.zeros(NPin + 1, dtype=torch.bool, device=dev)
            pc_in[NPin] = True  # padding lanes are constant
        else:
            pc_in = torch.cat([(p.point_constant if p.point_constant is not None else
                                torch.zeros(p.num_points, dtype=torch.bool, device=dev)).to(dev) for p in problems]
                              + [torch.ones(1, dtype=torch.bool, device=dev)])  # padding lanes are constant
        self.cam_const = cam_const.to(torch.uint8).contiguous()
        self.pt_const = pc_in.index_select(0, self.lane_src).to(torch.uint8).contiguous()
        self.cand_cameras = torch.empty_like(self.cameras)
        self.cand_points = torch.empty_like(self.points)
        slots = max(L.num_slots, 1)
        # padding slots keep zero Jacobians (the product walks them); every other buffer
        # is written by the kernel before it is read
        self.jac = torch.zeros((slots, 24), dtype=jt, device=dev)
        self.res = torch.empty((slots, 2), **f64)
        self.point_raw = torch.empty((NQ, 9), **f64)
        self.winv = torch.empty((NQ, 6), dtype=jt, device=dev)
        self.winv_ga = torch.empty((NQ, 3), **f64)
        self.step_points = torch.empty((NQ, 3), **f64)
        self.cam_diag = torch.empty((NC, 9), **f64)
        self.precond = torch.empty((NC, 81), dtype=torch.float64, device=dev)  # float64 in both precisions
        self.rhs = torch.empty((NC, 9), **f64)
        self.step_cameras = torch.empty((NC, 9), **f64)
        self.cam_acc = torch.empty((NC, 72), **f64)
        self.frames = torch.empty((NC, 24), **f64)
        self.pcg = torch.empty((8, 9 * NC), **f64)
        self.max_trace = options.max_num_iterations + 1
        self.result = torch.empty((len(problems), _lib.BATCH_RESULT), **f64)
        self.trace = torch.empty((len(problems), self.max_trace, _lib.BATCH_TRACE), **f64)
        self.queue = torch.zeros(1, dtype=torch.int32, device=dev)
        self.stream = stream
        self.struct = self._struct(max_refinements)

    def _struct(self, max_refinements: int) -> _lib.BatchStruct:
        L, o = self.layout, self.options
        s = _lib.BatchStruct()
        s.num_problems = L.num_problems
        s.precision = _lib.FP32 if self.precision == "mixed" else _lib.FP64
        s.max_cameras = L.max_cameras
        s.has_duplicate_cameras = int(L.has_duplicate_cameras)
        for k, v in self.loss_spec.items():
            setattr(s, k, v)
        s.max_num_iterations = o.max_num_iterations
        s.min_linear_solver_iterations = o.min_linear_solver_iterations
        s.max_linear_solver_iterations = o.max_linear_solver_iterations
        s.preconditioner = _PRECOND[o.preconditioner_type]
        s.jacobi_scaling = int(o.jacobi_scaling)
        s.max_consecutive_invalid_steps = o.max_num_consecutive_invalid_steps
        s.max_refinements = max_refinements
        s.max_trace = self.max_trace
        s.function_tolerance = o.function_tolerance
        s.gradient_tolerance = o.gradient_tolerance
        s.parameter_tolerance = o.parameter_tolerance
        s.min_relative_decrease = o.min_relative_decrease
        s.initial_radius = o.initial_trust_region_radius
        s.max_radius = o.max_trust_region_radius
        s.min_radius = o.min_trust_region_radius
        s.min_lm_diagonal = o.min_lm_diagonal
        s.max_lm_diagonal = o.max_lm_diagonal
        s.eta = o.eta
        for name in ("cam_off", "slice_off", "slice_base", "slice_len", "slot_cam", "slot_obs", "cam_offsets",
                     "cam_entries"):
            setattr(s, name, getattr(L, name).data_ptr())
        for name in ("cam_const", "pt_const", "cameras", "points", "cand_cameras", "cand_points", "jac", "res",
                     "point_raw", "winv", "winv_ga", "step_points", "cam_diag", "precond", "rhs", "step_cameras",
                     "cam_acc", "frames", "pcg", "result", "trace", "queue"):
            setattr(s, name, getattr(self, name).data_ptr())
        return s

    def _stream_handle(self) -> int:
        st = self.stream if self.stream is not None else torch.cuda.current_stream(self.device)
        return st.cuda_stream

    def launch(self, threads_per_cta: int = 0, ctas_per_sm: int = 0, cluster_size: int = 1) -> None:
        """Enqueue the solve (asynchronous on the stream); ``cluster_size`` CTAs per problem."""
        with torch.cuda.device(self.device):
            self.queue.zero_()
            rc = self.lib.ceres_b200_batch_solve(ctypes.byref(self.struct), int(threads_per_cta), int(ctas_per_sm),
                                                 int(cluster_size), self._stream_handle())
        _lib.check(rc, "ceres_b200_batch_solve")

    def write_back(self) -> None:
        """Solved parameters into each problem's tensors."""
        pts = torch.empty((int(self.pt_off_np[-1]) + 1, 3), dtype=torch.float64, device=self.device)
        pts.index_copy_(0, self.lane_src, self.points)  # padding lanes land in the extra last row
        with torch.no_grad():
            for i, p in enumerate(self.problems):
                p.cameras.copy_(self.cameras[self.cam_off_np[i]:self.cam_off_np[i + 1]])
                p.points.copy_(pts[self.pt_off_np[i]:self.pt_off_np[i + 1]])

    def fetch(self) -> tuple[np.ndarray, np.ndarray]:
        """The per-problem results and iteration records, copied to the host."""
        return self.result.cpu().numpy(), self.trace.cpu().numpy()

    def summaries(self) -> list[SolverSummary]:
        res, tr = self.fetch()
        return [self.summary_of(i, res, tr) for i in range(len(self.problems))]

    def summary_of(self, i: int, res: np.ndarray, tr: np.ndarray) -> SolverSummary:
        """Problem i's SolverSummary from the fetched arrays."""
        return summary_from_arrays(self.problems[i], self.options, self.precision, self.max_trace, res[i], tr[i], i)


def summary_from_arrays(p: BundleAdjustmentProblem, options: SolverOptions, precision: str, max_trace: int,
                        r: np.ndarray, trace: np.ndarray, i: int = 0) -> SolverSummary:
    """A batched problem's SolverSummary from its result row and iteration records."""
    s = _new_summary(options)
    s.num_parameter_blocks = p.num_cameras + p.num_points
    s.num_parameters = 9 * p.num_cameras + 3 * p.num_points
    ncc = int(p.camera_constant.sum()) if p.camera_constant is not None else 0
    npc = int(p.point_constant.sum()) if p.point_constant is not None else 0
    s.num_effective_parameters = 9 * (p.num_cameras - ncc) + 3 * (p.num_points - npc)
    s.num_residual_blocks = p.num_observations
    s.num_residuals = 2 * p.num_observations
    s.initial_cost = float(r[_lib.BR_INITIAL_COST])
    s.final_cost = float(r[_lib.BR_FINAL_COST])
    s.termination_type = _TERMS[int(r[_lib.BR_TERMINATION])]
    s.message = _lib.MESSAGES[int(r[_lib.BR_MESSAGE])]
    if s.num_effective_parameters == 0:
        s.termination_type = TerminationType.CONVERGENCE
        s.message = "No active parameters."
    s.num_successful_steps = int(r[_lib.BR_SUCCESSFUL])
    s.num_unsuccessful_steps = int(r[_lib.BR_UNSUCCESSFUL])
    s.num_jacobian_evaluations = int(r[_lib.BR_JACOBIAN_EVALS])
    s.num_residual_evaluations = int(r[_lib.BR_RESIDUAL_EVALS])
    s.num_linear_solves = int(r[_lib.BR_LINEAR_SOLVES])
    s.precision = precision
    n = min(int(r[_lib.BR_RECORDS]), max_trace)
    for k in range(n):
        t = trace[k]
        flags = int(t[_lib.BT_FLAGS])
        s.iterations.append(IterationSummary(
            iteration=k, step_is_valid=bool(flags & 1), step_is_successful=bool(flags & 2),
            step_is_nonmonotonic=bool(flags & 4), cost=float(t[_lib.BT_COST]),
            cost_change=float(t[_lib.BT_COST_CHANGE]), gradient_max_norm=float(t[_lib.BT_GMAX]),
            gradient_norm=float(t[_lib.BT_GNORM]), step_norm=float(t[_lib.BT_STEP_NORM]),
            relative_decrease=float(t[_lib.BT_RHO]), trust_region_radius=float(t[_lib.BT_RADIUS]),
            eta=options.eta, linear_solver_iterations=int(t[_lib.BT_LINEAR_ITERATIONS])))
    if int(r[_lib.BR_ERROR]):
        raise _lib.NativeLibraryError(f"batched solve of problem {i}: device error bits {int(r[_lib.BR_ERROR])}")
    return s


# CTA shapes (threads per CTA, resident CTAs per SM) the library is compiled for; the
# CTAs per SM set the register cap (255 registers at one 256-thread CTA, 128 at the
# others), trading register spills for problems in flight per SM.
SHAPES = ((128, 1), (128, 4), (256, 1), (256, 2), (512, 1))
_TUNED: dict = {}


def _size_class(problems: list[BundleAdjustmentProblem]) -> tuple[int, int]:
    """Power-of-two buckets of the largest camera count and the mean observation count."""
    nc = max(p.num_cameras for p in problems)
    no = sum(p.num_observations for p in problems) / len(problems)
    return (int(nc).bit_length(), int(no).bit_length())


def autotune(options: SolverOptions, problems: list[BundleAdjustmentProblem], *, precision: str = "mixed",
             sample: int = 296, shapes=SHAPES, repeats: int = 1) -> tuple[int, int]:
    """Pick the CTA shape for batches like ``problems``: each shape solves the same
    sample (the first ``sample`` problems; the problems themselves are not changed)
    once to warm up and ``repeats`` times timed with CUDA events; the fastest wins.
    The choice is cached per (precision, size class)."""
    key = (precision, _size_class(problems))
    if key in _TUNED:
        return _TUNED[key]
    sub = problems[:sample]
    best, best_ms = None, float("inf")
    for shape in shapes:
        times = []
        for r in range(repeats + 1):
            solver = BatchSolver(sub, options, precision=precision)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record()
            solver.launch(*shape)
            ev1.record()
            torch.cuda.synchronize(solver.device)
            if r:
                times.append(ev0.elapsed_time(ev1))
        ms = min(times)
        if ms < best_ms:
            best, best_ms = shape, ms
    _TUNED[key] = best
    return best


def solve_batch(options: SolverOptions, problems: list[BundleAdjustmentProblem], *, precision: str = "mixed",
                max_refinements: int = 1, threads_per_cta: int = 0, ctas_per_sm: int = 0, cluster_size: int = 1,
                tune: bool = False) -> list[SolverSummary]:
    """Solve every problem (in place) in one persistent launch; one SolverSummary each.
    ``cluster_size`` CTAs (one thread-block cluster) work on each problem. ``tune``
    picks the CTA shape with ``autotune`` (cached) unless one is given."""
    start = time.perf_counter()
    if tune and threads_per_cta == 0:
        threads_per_cta, ctas_per_sm = autotune(options, problems, precision=precision)
    solver = BatchSolver(problems, options, precision=precision, max_refinements=max_refinements)
    prep = time.perf_counter() - start
    solver.launch(threads_per_cta, ctas_per_sm, cluster_size)
    torch.cuda.synchronize(solver.device)
    solver.write_back()
    summaries = solver.summaries()
    total = time.perf_counter() - start
    for s in summaries:
        s.preprocessor_time_in_seconds = prep
        s.total_time_in_seconds = total
        s.minimizer_time_in_seconds = total - prep
    return summaries
