"""Point bucketing of the observation store (host logic, CPU tensors).

The sliced store must hold every observation exactly once, group a point's
observations in input order, and its camera-major list must give back, per
camera, exactly the sorted visible-point tuples the reference computes in
``_schur_visibility_from_residual_blocks`` (solver.py:744-785) - checked
bit-exactly against fixtures produced by the reference.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from ceres_torch_cuda_b200 import synthetic as S
from ceres_torch_cuda_b200.engine import build_layout
from tests import _golden as G


def _layout(ci, pi, obs, nc, npts):
    return build_layout(torch.as_tensor(ci), torch.as_tensor(pi), torch.as_tensor(obs), nc, npts)


def _check_invariants(L, ci, pi, obs, nc, npts):
    slot = L.slot_of_obs.numpy()
    assert len(np.unique(slot)) == len(slot)
    assert (L.slot_cam.numpy()[slot] == ci).all()
    np.testing.assert_array_equal(L.slot_obs.numpy()[slot], obs)
    base = L.slice_base.numpy()
    q = (slot % 32) + 32 * (np.searchsorted(base, slot, side="right") - 1)
    assert (L.lane_point.numpy()[q] == pi).all()
    sl = L.slice_len.numpy()
    assert (np.diff(sl) <= 0).all(), "slices sorted by track length"
    assert L.num_slots == 32 * int(sl.sum())
    # a point's observations sit in increasing k in input order
    for p in np.unique(pi)[:50]:
        idx = np.flatnonzero(pi == p)
        assert (np.diff(slot[idx]) > 0).all()
    ent = L.cam_entries.numpy()
    off = L.cam_offsets.numpy()
    # camera-major positions: the inverse of the entries' slot column, -1 on padding
    pos = L.slot_pos.numpy()
    if len(ent):
        np.testing.assert_array_equal(pos[ent[:, 0]], np.arange(len(ent)))
    assert (pos >= 0).sum() == len(ent)
    # camera work items cover each camera's entries in order, in runs of at most CAM_ITEM
    from ceres_torch_cuda_b200 import _lib

    items, ci_off = L.items.numpy(), L.cam_items.numpy()
    for c in range(nc):
        firsts = items[ci_off[c]:ci_off[c + 1]]
        assert (firsts[:, 0] == c).all()
        np.testing.assert_array_equal(firsts[:, 1], np.arange(off[c], off[c + 1], _lib.CAM_ITEM))
    assert L.max_camera_obs == (int(np.diff(off).max()) if nc else 0)
    assert off[-1] == len(ci)
    for c in range(nc):
        e = ent[off[c]:off[c + 1]]
        assert (np.diff(e[:, 0]) > 0).all()
        assert (L.slot_cam.numpy()[e[:, 0]] == c).all()


@pytest.mark.parametrize("name", G.BA_CASES + G.BIG_CASES)
def test_layout_visibility_is_bit_exact_with_reference(name):
    d = G.load(name)
    nc, npts = d["cameras"].shape[0], d["points"].shape[0]
    L = _layout(d["camera_index"], d["point_index"], d["observations"], nc, npts)
    _check_invariants(L, d["camera_index"], d["point_index"], d["observations"], nc, npts)
    if int(d["num_eliminate"]) == 0:
        return
    const = set(d["meta"]["constant_cameras"])
    ent = L.cam_entries.numpy()
    off = L.cam_offsets.numpy()
    # camera-major positions: the inverse of the entries' slot column, -1 on padding
    pos = L.slot_pos.numpy()
    if len(ent):
        np.testing.assert_array_equal(pos[ent[:, 0]], np.arange(len(ent)))
    assert (pos >= 0).sum() == len(ent)
    # camera work items cover each camera's entries in order, in runs of at most CAM_ITEM
    from ceres_torch_cuda_b200 import _lib

    items, ci_off = L.items.numpy(), L.cam_items.numpy()
    for c in range(nc):
        firsts = items[ci_off[c]:ci_off[c + 1]]
        assert (firsts[:, 0] == c).all()
        np.testing.assert_array_equal(firsts[:, 1], np.arange(off[c], off[c + 1], _lib.CAM_ITEM))
    assert L.max_camera_obs == (int(np.diff(off).max()) if nc else 0)
    lane_point = L.lane_point.numpy()
    vis = [np.unique(lane_point[ent[off[c]:off[c + 1], 1]]) for c in range(nc) if c not in const]
    np.testing.assert_array_equal(np.concatenate(vis), d["visibility_flat"])
    np.testing.assert_array_equal([len(v) for v in vis], d["visibility_len"])


def test_layout_edge_cases():
    # unobserved points, a point with one observation, duplicate camera in a track
    ci = np.array([0, 1, 1, 2, 0, 0])
    pi = np.array([0, 0, 3, 3, 5, 5])
    obs = np.arange(12, dtype=np.float64).reshape(6, 2)
    L = _layout(ci, pi, obs, 3, 40)
    _check_invariants(L, ci, pi, obs, 3, 40)
    assert L.has_duplicate_cameras
    assert L.num_slices == 2
    # no observations at all
    L0 = _layout(np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros((0, 2)), 2, 5)
    assert L0.num_slots == 0 and int(L0.cam_offsets[-1]) == 0


def test_layout_of_a_ragged_problem():
    d = S.ba_config(1, scale=0.01)
    L = _layout(d.camera_index, d.point_index, d.observations, d.num_cameras, d.num_points)
    _check_invariants(L, d.camera_index, d.point_index, d.observations, d.num_cameras, d.num_points)
    # padding overhead of the sliced store stays small with length-sorted slices
    assert L.num_slots <= 1.3 * d.num_observations


@pytest.mark.parametrize("item_size", [1, 32, 128, 256, 1024])
def test_camera_work_items_of_any_length(item_size):
    """The autotuner's item lengths: every camera's entries are cut into consecutive
    runs of ``item_size`` (the last one shorter), in order, none empty."""
    d = S.make_ring_ba(40, 900, seed=3)
    L = build_layout(torch.as_tensor(d.camera_index), torch.as_tensor(d.point_index),
                     torch.as_tensor(d.observations), 40, 900, item_size)
    items, ci_off, off = L.items.numpy(), L.cam_items.numpy(), L.cam_offsets.numpy()
    assert ci_off[-1] == sum(-(-(off[c + 1] - off[c]) // item_size) for c in range(40))
    for c in range(40):
        firsts = items[ci_off[c]:ci_off[c + 1]]
        assert (firsts[:, 0] == c).all()
        np.testing.assert_array_equal(firsts[:, 1], np.arange(off[c], off[c + 1], item_size))
