"""The camera reduction's warp reduce-scatter of its 72 sums (warp_reduce_scatter72 in
csrc/ba_kernels.cu), restated lane by lane in numpy.

At xor distances 16, 8, 4, 2, 1 each lane keeps one half of its values (the upper half
when its bit is set) and adds the partner's copy of that half; the 9 values left after
distance 4 are padded to 10, the 5 after distance 2 to 6. The kernel then writes lane
l's value k to index 36 b4 + 18 b3 + 9 b2 + 5 b1 + 3 b0 + k when 3 b0 + k < 5 and
5 b1 + 3 b0 + k < 9. Checked here: every index is written exactly once, and each sum
equals the shuffle-tree warp sum (v += shfl_xor(v, o) for o = 16 .. 1) bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest


def _warp_sum_tree(x: np.ndarray) -> np.ndarray:
    """x [32 lanes, n]: every lane's result of v += shfl_xor(v, o), o = 16, 8, 4, 2, 1."""
    v = x.copy()
    lanes = np.arange(32)
    for o in (16, 8, 4, 2, 1):
        v = v + v[lanes ^ o]
    return v


def _reduce_scatter72(x: np.ndarray) -> np.ndarray:
    """x [32, 72] -> [32, 3]: the kernel's recursive halving, lane by lane."""
    v = np.zeros((32, 72))
    v[:, :72] = x
    lanes = np.arange(32)
    for o, h in ((16, 36), (8, 18), (4, 9), (2, 5), (1, 3)):
        if o == 2:
            v[:, 9] = 0.0   # 9 values padded to 10
        if o == 1:
            v[:, 5] = 0.0   # 5 values padded to 6
        hi = (lanes & o) != 0
        keep = np.where(hi[:, None], v[:, h:2 * h], v[:, :h])
        send = np.where(hi[:, None], v[:, :h], v[:, h:2 * h])
        v[:, :h] = keep + send[lanes ^ o]
    return v[:, :3]


@pytest.mark.parametrize("seed", range(4))
def test_reduce_scatter_writes_every_sum_once_equal_to_the_warp_sum(seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((32, 72)) * 10.0 ** rng.integers(-3, 4, size=(32, 72))
    out = _reduce_scatter72(x)
    ref = _warp_sum_tree(x)[0]
    got = np.full(72, np.nan)
    writes = np.zeros(72, dtype=int)
    for lane in range(32):
        base = 36 * ((lane >> 4) & 1) + 18 * ((lane >> 3) & 1) + 9 * ((lane >> 2) & 1)
        l0, s0 = 5 * ((lane >> 1) & 1), 3 * (lane & 1)
        for k in range(3):
            if s0 + k < 5 and l0 + s0 + k < 9:
                idx = base + l0 + s0 + k
                got[idx] = out[lane, k]
                writes[idx] += 1
    assert (writes == 1).all()
    assert np.array_equal(got, ref)  # same pairwise tree, so the same bits
