"""The single-problem autotuner's choice (autotune.tune) on the CPU, with the engine and
the CUDA-event timer replaced by fakes that return set timings per candidate:

* the estimate of an LM iteration is 0.75 evaluations + one assembly + 2 PCG
  iterations + one step;
* the default (camera-major copy for the mixed path only, 256-entry items) is kept
  unless a candidate's estimate is more than MARGIN lower;
* the choice is cached per (precision, log2 observations, log2 cameras).
"""
from __future__ import annotations

from types import SimpleNamespace

import pytest
import torch

from ceres_torch_cuda_b200 import autotune as AT
from ceres_torch_cuda_b200 import engine as E


def _install(monkeypatch, table):
    """table[(copy, item)] = (evaluate, assemble, pcg for 10 iterations, step) in ms."""
    state = {}

    class FakeEngine:
        def __init__(self, *a, camera_copy=None, layout=None, **kw):
            self.copy = camera_copy
            self.layout = layout or SimpleNamespace()
            state["engine"] = self

        def retile_items(self, item):
            self.item = item

        def evaluate(self, jac):
            state["op"] = 0

        def assemble(self, *a, **kw):
            state["op"] = 1

        def pcg(self, *a, **kw):
            state["op"] = 2

        def step(self):
            state["op"] = 3

        def read_stats(self):
            return None

    def fake_time(eng, fn, reps=2):
        fn()
        return table[(eng.copy, eng.item)][state["op"]]

    monkeypatch.setattr(E, "BAEngine", FakeEngine)
    monkeypatch.setattr(AT, "_time", fake_time)
    AT.clear_cache()


def _args(no=1000, nc=20):
    return (torch.zeros((nc, 9)), torch.zeros((10, 3)), torch.zeros((no, 2)), torch.zeros(no, dtype=torch.long),
            torch.zeros(no, dtype=torch.long))


def _table(base=(0.5, 0.4, 2.8, 0.3)):
    return {(c, i): base for c in (True, False) for i in AT.ITEM_SIZES}


def test_estimate_formula_and_default_kept_within_margin(monkeypatch):
    t = _table()
    # a candidate 2% faster than the default: inside the margin, the default stays
    t[(False, 512)] = (0.5, 0.4, 2.8 * 0.95, 0.3)
    _install(monkeypatch, t)
    cfg = AT.tune(*_args(), precision="mixed")
    assert (cfg.camera_copy, cfg.item_size) == (True, 256)
    expected = 0.75 * 0.5 + 0.4 + 2 * 2.8 / AT.PCG_ITERATIONS + 0.3
    assert cfg.estimate_ms == pytest.approx(expected)
    assert cfg.timings[(False, 512)]["estimate"] < cfg.timings[(True, 256)]["estimate"]
    assert cfg.timings[(True, 256)]["estimate"] <= (1 + AT.MARGIN) * cfg.timings[(False, 512)]["estimate"]


def test_clearly_faster_candidate_wins_and_is_cached(monkeypatch):
    t = _table()
    t[(False, 1024)] = (0.3, 0.3, 2.0, 0.25)
    _install(monkeypatch, t)
    cfg = AT.tune(*_args(), precision="fp64")
    assert (cfg.camera_copy, cfg.item_size) == (False, 1024)
    assert AT.cached("fp64", 1000, 20) is cfg
    # same size class (log2 of the counts rounds the same): no new timing
    t[(False, 1024)] = (9.0, 9.0, 90.0, 9.0)
    assert AT.tune(*_args(no=1100, nc=21), precision="fp64") is cfg
    assert AT.cached("mixed", 1000, 20) is None


def test_float64_default_is_without_the_copy(monkeypatch):
    _install(monkeypatch, _table())
    cfg = AT.tune(*_args(), precision="fp64")
    assert (cfg.camera_copy, cfg.item_size) == (False, 256)
