"""ceres_b200_ba_evaluate_noalloc gives the same evaluation as ceres_b200_ba_evaluate.

The no-allocation entry point is for callers that cannot call cudaMalloc (their
device memory belongs to another allocator, or their runtime allows no
allocation after start-up) and so cannot provide the scratch buffer the regular
entry point reduces its cost partials into. This test calls both through the C
ABI on the same device-resident problem, twice in a row, and requires the same
cost, residuals and Jacobians within the float64 tolerance of the other GPU tests
(1e-12 relative). Residuals and Jacobians are per-observation values and agree to
the bit; the cost sums are folded in different orders (this entry folds per-CTA
partials of fixed slice sets, the regular one per-slice partials in slice order),
so the two costs agree to rounding only. It lives in its own file so that pytest
collects it last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _engine(precision):
    import ceres_torch_cuda_b200 as tc
    from ceres_torch_cuda_b200 import synthetic as S

    d = S.make_small_ba(12, 3000, 5, seed=21, loss=("cauchy", 2.0))
    t = lambda a, dt=torch.float64: torch.as_tensor(a).to("cuda", dt)  # noqa: E731
    return tc.BAEngine(t(d.cameras), t(d.points), t(d.observations), t(d.camera_index, torch.int64),
                       t(d.point_index, torch.int64), loss=tc.CauchyLoss(2.0), precision=precision)


def _call(eng, name, with_jacobian=1):
    from ceres_torch_cuda_b200 import _lib

    fn = getattr(eng.lib, name)
    with torch.cuda.device(eng.device):
        rc = fn(ctypes.byref(eng.struct), with_jacobian, eng._stream())
    assert rc == _lib.OK, (name, rc)
    st = eng.read_stats()
    r, jc, jp = (x.cpu().numpy().copy() for x in eng.slot_view())
    return st[0], r, jc, jp, eng.point_raw.cpu().numpy().copy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_evaluation_matches_regular_entry_point(precision):
    eng = _engine(precision)
    for _ in range(2):  # two calls in a row: the shared static scratch keeps the last call's contents
        ref = _call(eng, "ceres_b200_ba_evaluate")
        got = _call(eng, "ceres_b200_ba_evaluate_noalloc")
        np.testing.assert_allclose(got[0], ref[0], rtol=1e-12)
        for a, b in zip(got[1:], ref[1:]):
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=0.0)
    # the residual-only form as well
    ref = _call(eng, "ceres_b200_ba_evaluate", 0)
    got = _call(eng, "ceres_b200_ba_evaluate_noalloc", 0)
    np.testing.assert_allclose(got[0], ref[0], rtol=1e-12)
    np.testing.assert_allclose(got[1], ref[1], rtol=1e-12, atol=0.0)


def test_noalloc_evaluation_needs_no_scratch_buffer():
    eng = _engine("fp64")
    ref = _call(eng, "ceres_b200_ba_evaluate")
    eng.struct.scratch = None  # the no-allocation form does not read it
    eng.struct.scratch_bytes = 0
    for _ in range(2):
        got = _call(eng, "ceres_b200_ba_evaluate_noalloc")
        np.testing.assert_allclose(got[0], ref[0], rtol=1e-12)
        np.testing.assert_allclose(got[2], ref[2], rtol=1e-12, atol=0.0)
