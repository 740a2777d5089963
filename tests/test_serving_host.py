"""The serving loop's host logic on the CPU (serving.BAServer), with the batched solver,
the streams and the events replaced by fakes that record what the server asks of them:

* a launch waits for ``min_batch`` requests or for the oldest to have waited
  ``batch_window_s``;
* the oldest waiting request sets the cluster size; requests of that size class join it
  in arrival order up to ``max_batch``, the others keep their place in the queue, and
  only the first SCAN_FACTOR * max_batch waiting requests are looked at;
* a request whose footprint does not fit next to the batches in flight waits (the
  order is kept), and completed batches give their footprint back;
* at most ``max_inflight`` batches run, each on a stream no other running batch uses;
* a completed batch hands every request its result row and a completion time.
"""
from __future__ import annotations

import contextlib
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from ceres_torch_cuda_b200 import serving as SV


class _FakeSolver:
    launched: list = []

    def __init__(self, problems, options, *, precision, stream):
        self.problems, self.options, self.precision, self.stream = problems, options, precision, stream
        self.max_trace = 3
        self.written = False

    def launch(self, threads, ctas, cluster):
        self.shape = (threads, ctas, cluster)
        _FakeSolver.launched.append(self)

    def write_back(self):
        self.written = True

    def fetch(self):
        n = len(self.problems)
        return np.arange(n, dtype=np.float64)[:, None] * np.ones((1, 4)), np.zeros((n, self.max_trace, 2))


class _FakeEvent:
    def __init__(self):
        self.done = False

    def record(self, stream):
        self.stream = stream

    def query(self):
        return self.done


@pytest.fixture
def fakes(monkeypatch):
    _FakeSolver.launched = []
    events = []

    def make_event():
        e = _FakeEvent()
        events.append(e)
        return e

    monkeypatch.setattr(SV, "BatchSolver", _FakeSolver)
    monkeypatch.setattr(SV, "_stream_pool", lambda device, count: [SimpleNamespace(k=i) for i in range(count)])
    monkeypatch.setattr(torch.cuda, "stream", lambda s: contextlib.nullcontext())
    monkeypatch.setattr(torch.cuda, "Event", make_event)
    return events


def _req(no, nc=10, npts=100):
    return SimpleNamespace(num_observations=no, num_cameras=nc, num_points=npts)


def _server(**kw):
    base = dict(options=None, precision="mixed", memory_budget=10**12, device=torch.device("cpu"), max_inflight=4,
                max_batch=3, min_batch=2, batch_window_s=10.0, size_classes=((1000, 4), (None, 8)))
    base.update(kw)
    return SV.BAServer(**base)


def test_launch_waits_for_min_batch_or_the_window(fakes):
    s = _server()
    s.submit(_req(500), arrival=0.0 + 1e9)  # arrived "now" as far as the window is concerned
    s.step()
    assert s.launches == 0
    s.submit(_req(500), arrival=1e9)
    s.step()
    assert s.launches == 1 and len(_FakeSolver.launched[0].problems) == 2
    s2 = _server(batch_window_s=0.0)  # a zero window launches a lone request at once
    s2.submit(_req(500))
    s2.step()
    assert s2.launches == 1


def test_size_classes_and_arrival_order(fakes):
    s = _server(min_batch=1, batch_window_s=0.0)
    small = [_req(100 + i) for i in range(4)]
    big = [_req(5000 + i) for i in range(2)]
    order = [small[0], big[0], small[1], small[2], big[1], small[3]]
    for r in order:
        s.submit(r)
    s.step()
    shapes = [(sv.shape[2], [p.num_observations for p in sv.problems]) for sv in _FakeSolver.launched]
    # the oldest (small) sets cluster 4 and takes the next two smalls; then the oldest
    # waiting (big[0]) sets cluster 8 with big[1]; then the last small alone
    assert shapes == [(4, [100, 101, 102]), (8, [5000, 5001]), (4, [103])]
    streams = [id(sv.stream) for sv in _FakeSolver.launched]
    assert len(set(streams)) == 3


def test_admission_scans_a_bounded_prefix(fakes):
    s = _server(min_batch=1, batch_window_s=0.0, max_batch=2, max_inflight=1)
    first = _req(100)
    s.submit(first)
    bigs = [_req(5000 + i) for i in range(SV.SCAN_FACTOR * 2 + 3)]
    for r in bigs:
        s.submit(r)
    late_small = _req(101)
    s.submit(late_small)  # beyond the scanned prefix: not pulled forward
    s.step()
    assert [p.num_observations for p in _FakeSolver.launched[0].problems] == [100]
    assert list(s._waiting)[0].problem is bigs[0] and list(s._waiting)[-1].problem is late_small


def test_memory_budget_and_completion(fakes):
    probe = SV.footprint_bytes(_req(500), "mixed")
    s = _server(min_batch=1, batch_window_s=0.0, memory_budget=2 * probe + 1, max_batch=1)
    reqs = [s.submit(_req(500)) for _ in range(3)]
    s.step()
    assert s.launches == 2 and s._in_use == 2 * probe  # the third does not fit yet
    assert s.peak_bytes <= s.memory_budget
    fakes[0].done = True  # the first batch completes
    s.step()
    assert reqs[0].done is not None and reqs[0].latency >= 0
    assert _FakeSolver.launched[0].written
    assert reqs[0]._result[3][0] == 0.0  # its row of the batch's results
    assert s.launches == 3 and s._in_use == 2 * probe
    with pytest.raises(ValueError, match="above the server budget"):
        s.submit(_req(10**7, nc=500, npts=10**6))


def test_inflight_cap_and_distinct_streams(fakes):
    s = _server(min_batch=1, batch_window_s=0.0, max_batch=1, max_inflight=2)
    for _ in range(5):
        s.submit(_req(200))
    s.step()
    assert s.launches == 2 and len(s._flights) == 2
    assert id(s._flights[0].stream) != id(s._flights[1].stream)
    fakes[1].done = True
    s.step()
    assert s.launches == 3
    running = [id(f.stream) for f in s._flights]
    assert len(running) == len(set(running)) == 2


def test_footprint_covers_the_host_slot_bound():
    """A request with host track statistics is laid out with 32 max_track + no slots; its
    footprint counts at least that many."""
    long_track = SimpleNamespace(num_observations=6000, num_cameras=10, num_points=1000, track_stats=(5000, False))
    plain = SimpleNamespace(num_observations=6000, num_cameras=10, num_points=1000)
    per_slot = 24 * 4 + 16 + 16 + 4
    assert SV.footprint_bytes(long_track, "mixed") - SV.footprint_bytes(plain, "mixed") == \
        per_slot * (32 * 5000 + 6000 - (int(6000 * 1.15) + 256))
