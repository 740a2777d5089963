"""Autotuner for the single-problem kernels.

Two launch-shape knobs of the LM iteration are picked by timing them on the problem
itself: whether the evaluator writes the camera-major copy of the Jacobian store
(the camera-side passes then stream records instead of gathering them by slot) and
the length of the camera work items of the PCG's camera pass (how a camera's
observations are cut into warp-sized units of work). Each candidate runs one LM
iteration's kernels on the problem — evaluation with Jacobian, point and camera
assembly, a 10-iteration PCG, the step — timed with CUDA events on the engine's
stream; the estimate of an LM iteration is 0.75 evaluations + one assembly + 2 PCG
iterations + one step (the mix of the configuration-2 solves). The default (copy for
the mixed path only, 256-entry items) is kept unless a candidate's estimate is more
than 3% lower. The winner is cached per (precision, log2 observations, log2 cameras),
so a process tunes each size class once.

The camera-major copy does not change any result (the same record values are read in
the same order); the item length changes how the camera pass's sums are grouped, so
two item lengths give results that differ by rounding (each is reproducible).
The batched path has its own tuner (``batch.autotune``, CTA shapes).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import torch

ITEM_SIZES = (128, 256, 512, 1024)
PCG_ITERATIONS = 10
MARGIN = 0.03  # a candidate replaces the default only when its estimate is this much lower
_CACHE: dict[tuple, "TunedConfig"] = {}


@dataclass
class TunedConfig:
    camera_copy: bool
    item_size: int
    estimate_ms: float
    timings: dict = field(default_factory=dict)   # (copy, item) -> per-kernel ms and the estimate

    def as_dict(self) -> dict:
        return {"camera_copy": self.camera_copy, "item_size": self.item_size, "estimate_ms_per_lm_iteration":
                self.estimate_ms, "candidates": {f"copy={c},item={i}": t for (c, i), t in self.timings.items()}}


def size_class(precision: str, num_observations: int, num_cameras: int) -> tuple:
    return (precision, int(round(math.log2(max(num_observations, 1)))), int(round(math.log2(max(num_cameras, 1)))))


def cached(precision: str, num_observations: int, num_cameras: int) -> TunedConfig | None:
    return _CACHE.get(size_class(precision, num_observations, num_cameras))


def clear_cache() -> None:
    _CACHE.clear()


def _time(eng, fn, reps: int = 2) -> float:
    stream = torch.cuda.current_stream(eng.device)
    fn()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(reps):
        fn()
    e.record(stream)
    e.synchronize()
    return s.elapsed_time(e) / reps


def tune(cameras, points, observations, camera_index, point_index, *, loss=None, camera_constant=None,
         point_constant=None, precision: str = "mixed", options=None, item_sizes=ITEM_SIZES) -> TunedConfig:
    """Time every candidate on this problem and cache the fastest for its size class."""
    from . import _lib
    from .engine import BAEngine
    from .types import SolverOptions

    key = size_class(precision, int(observations.shape[0]), int(cameras.shape[0]))
    if key in _CACHE:
        return _CACHE[key]
    opts = options or SolverOptions()
    radius = float(opts.initial_trust_region_radius)
    timings = {}
    layout = None
    for copy in (True, False):
        eng = BAEngine(cameras, points, observations, camera_index, point_index, loss=loss,
                       camera_constant=camera_constant, point_constant=point_constant, precision=precision,
                       layout=layout, camera_copy=copy)
        layout = eng.layout  # one layout for both; items are re-cut per candidate below
        for item in item_sizes:
            eng.retile_items(item)
            t_eval = _time(eng, lambda: eng.evaluate(True))
            t_asm = _time(eng, lambda: eng.assemble(radius, opts, _lib.PRECOND_SCHUR_JACOBI))
            t_pcg = _time(eng, lambda: eng.pcg(_lib.PRECOND_SCHUR_JACOBI, PCG_ITERATIONS, PCG_ITERATIONS, 0.0, 0))
            t_step = _time(eng, lambda: eng.step())
            est = 0.75 * t_eval + t_asm + 2.0 * t_pcg / PCG_ITERATIONS + t_step
            timings[(copy, item)] = {"evaluate": t_eval, "assemble": t_asm, "pcg_iteration": t_pcg / PCG_ITERATIONS,
                                     "step": t_step, "estimate": est}
        eng.read_stats()
        del eng
    (copy, item), best = min(timings.items(), key=lambda kv: kv[1]["estimate"])
    # keep the default unless a candidate beats it clearly: the item length changes the
    # grouping of the camera pass's sums, hence the rounding and the LM trajectory, so a
    # choice that flips between runs on timing noise would make runs differ
    default = (precision == "mixed", _lib.CAM_ITEM)
    if default in timings and timings[default]["estimate"] <= (1.0 + MARGIN) * best["estimate"]:
        (copy, item), best = default, timings[default]
    cfg = TunedConfig(camera_copy=copy, item_size=item, estimate_ms=best["estimate"], timings=timings)
    _CACHE[key] = cfg
    return cfg
