"""Device-resident bundle-adjustment state and the Levenberg-Marquardt driver.

``BAEngine`` owns every device buffer of one problem (allocated with torch),
builds the sliced-ELL observation store on the GPU, and drives the C-ABI
kernels. ``run_lm`` is the trust-region loop of ceres-torch's
``_trust_region_solve`` (solver.py:35-357) with the same decisions, counters
and termination messages; the only host/device traffic per LM iteration is one
read of a 256-byte control block (two on accepted steps).
"""
from __future__ import annotations

import ctypes
import math
import os
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .losses import device_loss
from .types import (CallbackReturnType, IterationSummary, LinearSolverType, LoggingType, PreconditionerType,
                    SolverOptions, SolverSummary, TerminationType, TrustRegionStrategyType)

_PRECOND = {
    PreconditionerType.IDENTITY: _lib.PRECOND_IDENTITY,
    PreconditionerType.JACOBI: _lib.PRECOND_JACOBI,
    PreconditionerType.SCHUR_JACOBI: _lib.PRECOND_SCHUR_JACOBI,
    PreconditionerType.SCHUR_POWER_SERIES_EXPANSION: _lib.PRECOND_SCHUR_POWER_SERIES,
    PreconditionerType.CLUSTER_JACOBI: _lib.PRECOND_CLUSTER,
    PreconditionerType.CLUSTER_TRIDIAGONAL: _lib.PRECOND_CLUSTER,
}
_CLUSTER_MAX_DIM = 16384  # 9 x cameras of the largest component (the sweep's 32-bit element index)
SCHUR_ORDER_MAX = 1 << 24  # contributions of the ordered explicit S (12 B each); longer lists sum with atomics

PRECISIONS = ("fp64", "mixed")


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


@dataclass
class Layout:
    """Sliced-ELL observation store (see include/ceres_b200.h)."""

    num_slices: int
    num_slots: int
    max_slice_len: int
    has_duplicate_cameras: bool
    slice_base: torch.Tensor      # int32 [S]
    slice_len: torch.Tensor       # int32 [S]
    slot_cam: torch.Tensor        # int32 [slots]
    slot_obs: torch.Tensor        # float64 [slots, 2]
    slot_of_obs: torch.Tensor     # int64 [no]  slot of each input observation
    cam_offsets: torch.Tensor     # int32 [nc+1]
    cam_entries: torch.Tensor     # int32 [no, 2]  (slot, q)
    lane_point: torch.Tensor      # int64 [32 S]  original point id of each lane, -1 padding
    point_order: torch.Tensor     # int64 [np]   q -> point id for q < np
    slot_pos: torch.Tensor        # int32 [slots] camera-major position of the slot, -1 padding
    cam_items: torch.Tensor       # int32 [nc+1] first camera work item of each camera
    items: torch.Tensor           # int32 [items, 2] (camera, first entry)
    max_camera_obs: int = 0


def build_layout(camera_index: torch.Tensor, point_index: torch.Tensor, observations: torch.Tensor,
                 num_cameras: int, num_points: int, item_size: int | None = None) -> Layout:
    """Bucket observations by point (stable in observation order) into slices of
    32 points sorted by track length, and list them per camera. GPU torch ops."""
    dev = camera_index.device
    no = int(camera_index.numel())
    ci = camera_index.to(torch.int64)
    pi = point_index.to(torch.int64)
    counts = torch.bincount(pi, minlength=num_points) if no else torch.zeros(num_points, dtype=torch.int64, device=dev)
    order = torch.argsort(-counts, stable=True)
    num_slices = (num_points + 31) // 32
    np_pad = 32 * num_slices
    lane_point = torch.full((np_pad,), -1, dtype=torch.int64, device=dev)
    lane_point[:num_points] = order
    counts_q = torch.zeros(np_pad, dtype=torch.int64, device=dev)
    counts_q[:num_points] = counts[order]
    slice_len = counts_q.view(num_slices, 32).amax(dim=1) if num_slices else counts_q[:0]
    csum = torch.cumsum(slice_len, 0)
    slice_base = 32 * (csum - slice_len)
    num_slots = int(32 * int(csum[-1])) if num_slices else 0
    inv_order = torch.empty(num_points, dtype=torch.int64, device=dev)
    inv_order[order] = torch.arange(num_points, device=dev)
    if no:
        obs_sorted = torch.argsort(pi, stable=True)
        pstart = torch.cumsum(counts, 0) - counts
        rank = torch.empty(no, dtype=torch.int64, device=dev)
        rank[obs_sorted] = torch.arange(no, device=dev) - pstart[pi[obs_sorted]]
        q = inv_order[pi]
        slot = slice_base[q // 32] + 32 * rank + (q % 32)
    else:
        q = torch.zeros(0, dtype=torch.int64, device=dev)
        slot = q
    slot_cam = torch.full((max(num_slots, 1),), -1, dtype=torch.int32, device=dev)
    slot_obs = torch.zeros((max(num_slots, 1), 2), dtype=torch.float64, device=dev)
    if no:
        slot_cam[slot] = ci.to(torch.int32)
        slot_obs[slot] = observations.to(torch.float64)
    key = ci * max(num_slots, 1) + slot
    perm = torch.argsort(key)
    cam_entries = torch.stack([slot[perm], q[perm]], dim=1).to(torch.int32).contiguous()
    cam_counts = torch.bincount(ci, minlength=num_cameras) if no else torch.zeros(num_cameras, dtype=torch.int64,
                                                                                    device=dev)
    cam_offsets = torch.zeros(num_cameras + 1, dtype=torch.int64, device=dev)
    cam_offsets[1:] = torch.cumsum(cam_counts, 0)
    has_dup = False
    if no:
        pk = torch.sort(pi * max(num_cameras, 1) + ci).values
        has_dup = bool((pk[1:] == pk[:-1]).any()) if no > 1 else False
    slot_pos, cam_items, items, max_cam = camera_items(cam_entries if no else cam_entries[:0], cam_counts, num_slots,
                                                       item_size)
    return Layout(
        num_slices=num_slices, num_slots=num_slots,
        max_slice_len=int(slice_len.max()) if num_slices else 0,
        has_duplicate_cameras=has_dup,
        slice_base=slice_base.to(torch.int32).contiguous(), slice_len=slice_len.to(torch.int32).contiguous(),
        slot_cam=slot_cam, slot_obs=slot_obs, slot_of_obs=slot,
        cam_offsets=cam_offsets.to(torch.int32), cam_entries=cam_entries if no else torch.zeros((1, 2), dtype=torch.int32, device=dev),
        lane_point=lane_point, point_order=order, slot_pos=slot_pos, cam_items=cam_items, items=items,
        max_camera_obs=max_cam,
    )


def schur_contributions(L: Layout, nc: int, cam_const: torch.Tensor, pt_const: torch.Tensor, np_pad: int,
                        limit: int = SCHUR_ORDER_MAX):
    """The fixed summation order of the explicit reduced camera matrix: for every active
    camera, each of its observations with itself and every ordered pair of its
    observations of one active point (the diagonal block); for every two active cameras
    a < b, each pair of their observations of one active point; grouped by block and
    sorted by (point, slot i, slot j). Returns (blocks [B, 2] int32, block_start [B + 1]
    int64, contributions [C, 3] int32 (slot i, slot j, point lane), B), or None when the
    list's bound (the observations plus twice the pairs of observations of one point)
    exceeds ``limit``. Torch ops on the layout's device."""
    dev = L.cam_offsets.device
    i64 = dict(dtype=torch.int64, device=dev)
    no = int(L.cam_offsets[-1]) if nc else 0
    ents = L.cam_entries[:no].to(torch.int64)                     # (slot, q), sorted by (camera, slot)
    cam = torch.repeat_interleave(torch.arange(nc, **i64), (L.cam_offsets[1:] - L.cam_offsets[:-1]).to(torch.int64))
    act = cam_const.to(dev)[cam] == 0
    slot, q, cam = ents[act, 0], ents[act, 1], cam[act]
    # the observations of active points, grouped by point (a stable sort keeps (camera, slot))
    sel = torch.nonzero(pt_const.to(dev)[q] == 0).flatten()
    sel = sel[torch.sort(q[sel], stable=True).indices]
    ps, pq, pc = slot[sel], q[sel], cam[sel]
    n = int(pq.numel())
    idx = torch.arange(n, **i64)
    if n:
        start = torch.ones(n, dtype=torch.bool, device=dev)
        start[1:] = pq[1:] != pq[:-1]
        grp = torch.cumsum(start.to(torch.int64), 0) - 1
        later = (torch.cumsum(torch.bincount(grp), 0) - 1)[grp] - idx  # observations after this one at its point
    else:
        later = idx
    total = int(later.sum()) if n else 0
    if int(slot.numel()) + 2 * total > limit:
        return None
    i = torch.repeat_interleave(idx, later)
    j = i + 1 + torch.arange(total, **i64) - (torch.cumsum(later, 0) - later)[i]
    ca, cb = pc[i], pc[j]
    cross = ca != cb
    dup = ~cross
    lo, hi = torch.minimum(ca, cb), torch.maximum(ca, cb)
    swap = ca > cb
    # rows (block key, q, slot i, slot j): self pairs of every observation, the cross pairs
    # oriented a < b, the same-camera pairs in both orders
    blk = torch.cat([cam * nc + cam, (lo * nc + hi)[cross], (ca * nc + ca)[dup], (ca * nc + ca)[dup]])
    qq = torch.cat([q, pq[i][cross], pq[i][dup], pq[i][dup]])
    si = torch.cat([slot, torch.where(swap, ps[j], ps[i])[cross], ps[i][dup], ps[j][dup]])
    sj = torch.cat([slot, torch.where(swap, ps[i], ps[j])[cross], ps[j][dup], ps[i][dup]])
    o = torch.sort(si * max(L.num_slots, 1) + sj, stable=True).indices
    o = o[torch.sort((blk * max(np_pad, 1) + qq)[o], stable=True).indices]
    blk, qq, si, sj = blk[o], qq[o], si[o], sj[o]
    uniq, cnt = torch.unique_consecutive(blk, return_counts=True)
    blocks = torch.stack([uniq // max(nc, 1), uniq % max(nc, 1)], dim=1).to(torch.int32).contiguous()
    bstart = torch.zeros(int(uniq.numel()) + 1, **i64)
    bstart[1:] = torch.cumsum(cnt, 0)
    contrib = torch.stack([si, sj, qq], dim=1).to(torch.int32).contiguous()
    pad = torch.zeros(3, dtype=torch.int32, device=dev)  # non-null pointers for an empty list
    return (blocks if blocks.numel() else pad, bstart, contrib if contrib.numel() else pad, int(uniq.numel()))


def camera_items(cam_entries: torch.Tensor, cam_counts: torch.Tensor, num_slots: int, item_size: int | None = None):
    """The camera-major position of every slot (inverse of cam_entries' slot column,
    -1 for padding) and the camera work items: each camera's entries cut into runs of
    ``item_size`` (default CAM_ITEM, include/ceres_b200.h). Returns (slot_pos, cam_items,
    items, largest camera entry count)."""
    item = int(item_size or _lib.CAM_ITEM)
    if item < 1:
        raise ValueError("item_size must be positive")
    dev = cam_counts.device
    no = int(cam_entries.shape[0])
    nc = int(cam_counts.numel())
    slot_pos = torch.full((max(num_slots, 1),), -1, dtype=torch.int32, device=dev)
    if no:
        slot_pos[cam_entries[:, 0].long()] = torch.arange(no, dtype=torch.int32, device=dev)
    per_cam = (cam_counts + item - 1) // item
    cam_items = torch.zeros(nc + 1, dtype=torch.int64, device=dev)
    cam_items[1:] = torch.cumsum(per_cam, 0)
    n_items = int(cam_items[-1]) if nc else 0
    if n_items:
        item_cam = torch.repeat_interleave(torch.arange(nc, device=dev), per_cam)
        start = torch.cumsum(cam_counts, 0) - cam_counts
        first = start[item_cam] + item * (torch.arange(n_items, device=dev) - cam_items[item_cam])
        items = torch.stack([item_cam, first], dim=1).to(torch.int32).contiguous()
    else:
        items = torch.zeros((1, 2), dtype=torch.int32, device=dev)
    max_cam = int(cam_counts.max()) if nc else 0
    return slot_pos, cam_items.to(torch.int32).contiguous(), items, max_cam


class BAEngine:
    """All device state of one bundle-adjustment problem."""

    def __init__(self, cameras: torch.Tensor, points: torch.Tensor, observations: torch.Tensor,
                 camera_index: torch.Tensor, point_index: torch.Tensor, *, loss=None,
                 camera_constant: torch.Tensor | None = None, point_constant: torch.Tensor | None = None,
                 precision: str = "fp64", layout: Layout | None = None, camera_copy: bool | None = None,
                 item_size: int | None = None):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {PRECISIONS}")
        if cameras.device.type != "cuda":
            raise _lib.NativeLibraryError("the bundle-adjustment engine needs CUDA tensors")
        self.lib = _lib.load()
        self.device = cameras.device
        dev = self.device
        self.precision = precision
        self.nc = int(cameras.shape[0])
        self.np = int(points.shape[0])
        self.no = int(observations.shape[0])
        if cameras.shape[1:] != (9,) or points.shape[1:] != (3,) or observations.shape[1:] != (2,):
            raise ValueError("expected cameras [nc,9], points [np,3], observations [no,2]")
        if camera_index.numel() != self.no or point_index.numel() != self.no:
            raise ValueError("camera_index and point_index need one entry per observation")
        if self.no:
            cmin, cmax = int(camera_index.min()), int(camera_index.max())
            pmin, pmax = int(point_index.min()), int(point_index.max())
            if cmin < 0 or cmax >= self.nc or pmin < 0 or pmax >= self.np:
                raise ValueError("camera_index / point_index out of range")
        if not torch.isfinite(observations).all():
            raise ValueError("observations must be finite")
        self.layout = layout or build_layout(camera_index.to(dev), point_index.to(dev), observations.to(dev),
                                             self.nc, self.np, item_size)
        self.item_size = int(item_size or _lib.CAM_ITEM)
        self._index = (camera_index, point_index, point_constant)
        self._schur_order = None
        self.clusters: ClusterPlan | None = None
        L = self.layout
        self.np_pad = 32 * L.num_slices
        T = torch.float32 if precision == "mixed" else torch.float64
        self.T = T
        f64 = dict(dtype=torch.float64, device=dev)
        cc = torch.zeros(self.nc, dtype=torch.uint8, device=dev)
        if camera_constant is not None:
            cc = camera_constant.to(dev).to(torch.uint8).contiguous()
        pc = torch.ones(max(self.np_pad, 1), dtype=torch.uint8, device=dev)
        if self.np:
            src = torch.zeros(self.np, dtype=torch.uint8, device=dev) if point_constant is None else \
                point_constant.to(dev).to(torch.uint8)
            pc[:self.np] = src[L.point_order]
        self.cam_const = cc
        self.pt_const = pc
        nslot = max(L.num_slots, 1)
        npq = max(self.np_pad, 1)
        ncq = max(self.nc, 1)
        self.cameras = torch.zeros((ncq, 9), **f64)
        self.cand_cameras = torch.zeros((ncq, 9), **f64)
        self.best_cameras = torch.zeros((ncq, 9), **f64)
        self.points = torch.zeros((npq, 3), **f64)
        self.cand_points = torch.zeros((npq, 3), **f64)
        self.best_points = torch.zeros((npq, 3), **f64)
        self.jac = torch.zeros((nslot, 24), dtype=T, device=dev)
        # camera-major copy of the Jacobian store: the camera-side passes stream it instead of
        # gathering records by slot. It pays for itself with 96-byte float32 records (6.0M
        # observations: 1.68 against 1.80 ms per LM iteration) but not with 192-byte float64
        # records, whose second copy costs the evaluator more (0.85 against 0.44 ms) than the
        # streaming saves (2.53 against 2.41 ms per LM iteration), so by default only the
        # mixed path keeps it. CERES_B200_CAMERA_COPY=1/0 overrides the default.
        env = os.environ.get("CERES_B200_CAMERA_COPY")
        if camera_copy is None:
            camera_copy = (env != "0") if env is not None else precision == "mixed"
        self.camera_copy = bool(camera_copy)
        self.cm_jac = torch.zeros((max(self.no, 1), 24), dtype=T, device=dev) if self.camera_copy else None
        self.res = torch.zeros((nslot, 2), **f64)
        self.point_raw = torch.zeros((npq, 9), **f64)
        self.winv = torch.zeros((npq, 6), dtype=T, device=dev)
        self.winv_ga = torch.zeros((npq, 3), **f64)
        self.step_points = torch.zeros((npq, 3), **f64)
        self.cam_diag = torch.zeros((ncq, 9), **f64)
        # float64 in both precisions: an inverted 9x9 block of an ill-conditioned camera
        # rounded to float32 preconditions worse (more PCG iterations per solve)
        self.precond = torch.zeros((ncq, 81), **f64)
        self.rhs = torch.zeros((ncq, 9), **f64)
        self.step_cameras = torch.zeros((ncq, 9), **f64)
        self.pcg_vec = {k: torch.zeros(9 * ncq, **f64) for k in ("x", "r", "z", "ap")}
        self.pcg_vec["p"] = torch.zeros(2 * 9 * ncq, **f64)
        self.ctl = torch.zeros(_lib.CTL_BYTES, dtype=torch.uint8, device=dev)
        self.ctl_host = torch.zeros(_lib.CTL_BYTES, dtype=torch.uint8, pin_memory=True)
        self.dense_work: torch.Tensor | None = None
        self.struct = _lib.BAStruct()
        s = self.struct
        s.num_cameras, s.num_observations, s.num_points = self.nc, self.no, self.np_pad
        s.num_slices, s.num_slots, s.max_slice_len = L.num_slices, L.num_slots, L.max_slice_len
        s.precision = _lib.FP32 if precision == "mixed" else _lib.FP64
        s.has_duplicate_cameras = int(L.has_duplicate_cameras)
        for k, v in device_loss(loss).items():
            setattr(s, k, v)
        s.slice_base, s.slice_len = _ptr(L.slice_base), _ptr(L.slice_len)
        s.slot_cam, s.slot_obs = _ptr(L.slot_cam), _ptr(L.slot_obs)
        s.cam_offsets, s.cam_entries = _ptr(L.cam_offsets), _ptr(L.cam_entries)
        s.cam_const, s.pt_const = _ptr(self.cam_const), _ptr(self.pt_const)
        s.jac, s.res = _ptr(self.jac), _ptr(self.res)
        s.slot_pos, s.cm_jac = _ptr(L.slot_pos), _ptr(self.cm_jac)
        s.cam_items, s.items = _ptr(L.cam_items), _ptr(L.items)
        s.num_items, s.max_camera_obs = int(L.cam_items[-1]) if self.nc else 0, int(L.max_camera_obs)
        s.point_raw = _ptr(self.point_raw)
        s.winv, s.winv_ga, s.step_points = _ptr(self.winv), _ptr(self.winv_ga), _ptr(self.step_points)
        s.cam_diag, s.precond, s.rhs, s.step_cameras = (_ptr(self.cam_diag), _ptr(self.precond), _ptr(self.rhs),
                                                        _ptr(self.step_cameras))
        s.pcg_x, s.pcg_r, s.pcg_z = _ptr(self.pcg_vec["x"]), _ptr(self.pcg_vec["r"]), _ptr(self.pcg_vec["z"])
        s.pcg_p, s.pcg_ap = _ptr(self.pcg_vec["p"]), _ptr(self.pcg_vec["ap"])
        s.counters = self.ctl.data_ptr() + _lib.CTL_COUNTERS
        s.stats = self.ctl.data_ptr()
        self._bind_params()
        nbytes = ctypes.c_int64(0)
        with torch.cuda.device(dev):
            _lib.check(self.lib.ceres_b200_scratch_bytes(ctypes.byref(s), ctypes.byref(nbytes)), "scratch size")
        self.scratch = torch.zeros(int(nbytes.value), dtype=torch.uint8, device=dev)
        s.scratch, s.scratch_bytes = self.scratch.data_ptr(), int(nbytes.value)
        self.set_parameters(cameras, points)

    # ---------------------------------------------------------------- parameters
    def _bind_params(self):
        s = self.struct
        s.cameras, s.points = _ptr(self.cameras), _ptr(self.points)
        s.cand_cameras, s.cand_points = _ptr(self.cand_cameras), _ptr(self.cand_points)

    def set_parameters(self, cameras: torch.Tensor, points: torch.Tensor) -> None:
        if self.nc:
            self.cameras[: self.nc].copy_(cameras.to(self.device, torch.float64))
        if self.np:
            self.points[: self.np].copy_(points.to(self.device, torch.float64)[self.layout.point_order])

    def get_parameters(self, which: str = "current") -> tuple[torch.Tensor, torch.Tensor]:
        cams = {"current": self.cameras, "candidate": self.cand_cameras, "best": self.best_cameras}[which]
        pts_q = {"current": self.points, "candidate": self.cand_points, "best": self.best_points}[which]
        pts = torch.empty((self.np, 3), dtype=torch.float64, device=self.device)
        if self.np:
            pts[self.layout.point_order] = pts_q[: self.np]
        return cams[: self.nc].clone(), pts

    def accept(self) -> None:
        """The candidate becomes the current state (pointer swap)."""
        self.cameras, self.cand_cameras = self.cand_cameras, self.cameras
        self.points, self.cand_points = self.cand_points, self.points
        self._bind_params()

    def save_best(self) -> None:
        self.best_cameras.copy_(self.cameras)
        self.best_points.copy_(self.points)

    def restore_best(self) -> None:
        self.cameras.copy_(self.best_cameras)
        self.points.copy_(self.best_points)

    # ---------------------------------------------------------------- kernels
    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    def enable_profiling(self) -> dict:
        """Record CUDA events around every library call (no extra synchronisation);
        ``profile_report()`` sums the device time per entry point."""
        self._events = []
        return self._events

    def profile_report(self) -> dict:
        torch.cuda.current_stream(self.device).synchronize()
        out: dict = {}
        for name, a, b in getattr(self, "_events", []):
            ms = a.elapsed_time(b)
            t = out.setdefault(name, [0, 0.0])
            t[0] += 1
            t[1] += ms
        return {k: {"calls": v[0], "ms": v[1]} for k, v in out.items()}

    def _call(self, name: str, *args) -> None:
        fn = getattr(self.lib, name)
        events = getattr(self, "_events", None)
        if events is not None:
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
        with torch.cuda.device(self.device):
            _lib.check(fn(ctypes.byref(self.struct), *args, self._stream()), name)
        if events is not None:
            b.record()
            events.append((name, a, b))

    def evaluate(self, with_jacobian: bool = True) -> None:
        self._call("ceres_b200_ba_evaluate", int(with_jacobian))

    def assemble(self, radius: float, options: SolverOptions, precond: int, spse_base: bool = False) -> None:
        flags = _lib.PRECOND_FLAG_SPSE_BASE if spse_base else 0
        self._call("ceres_b200_ba_point_assemble", float(radius), float(options.min_lm_diagonal),
                   float(options.max_lm_diagonal), int(options.jacobi_scaling))
        self._call("ceres_b200_ba_camera_assemble", float(radius), float(options.min_lm_diagonal),
                   float(options.max_lm_diagonal), int(options.jacobi_scaling), int(precond) | flags)
        if precond == _lib.PRECOND_CLUSTER:
            if self.clusters is None:
                raise RuntimeError("setup_clusters() first")
            self._call("ceres_b200_ba_cluster_factor", ctypes.byref(self.clusters.struct))

    def retile_items(self, item_size: int) -> None:
        """Cut the cameras' entries into work items of ``item_size`` entries (the
        camera pass's unit of work; the autotuner's knob) and resize the scratch."""
        L = self.layout
        cam_counts = (L.cam_offsets[1:] - L.cam_offsets[:-1]).to(torch.int64)
        ents = L.cam_entries if self.no else L.cam_entries[:0]
        _, L.cam_items, L.items, _ = camera_items(ents, cam_counts, L.num_slots, item_size)
        self.item_size = int(item_size)
        s = self.struct
        s.cam_items, s.items = _ptr(L.cam_items), _ptr(L.items)
        s.num_items = int(L.cam_items[-1]) if self.nc else 0
        nbytes = ctypes.c_int64(0)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.ceres_b200_scratch_bytes(ctypes.byref(s), ctypes.byref(nbytes)), "scratch size")
        if int(nbytes.value) > self.scratch.numel():
            self.scratch = torch.zeros(int(nbytes.value), dtype=torch.uint8, device=self.device)
        s.scratch, s.scratch_bytes = self.scratch.data_ptr(), int(self.scratch.numel())

    def setup_clusters(self, tridiagonal: bool, clustering: str = "CANONICAL_VIEWS") -> bool:
        """Cluster the active cameras by visibility (linear.py:953-990) and allocate the
        preconditioner's storage. False when the reference would not use the clusters:
        fewer than two active cameras, or no camera sees an active point (it then uses
        SCHUR_JACOBI's blocks, linear.py:498-528)."""
        self.clusters = ClusterPlan.build(self, tridiagonal, clustering)
        return self.clusters is not None

    def cluster_flags(self) -> np.ndarray:
        return self.clusters.flags.cpu().numpy().view(np.uint32).copy()

    def pcg(self, precond: int, min_iterations: int, max_iterations: int, tolerance: float,
            max_refinements: int = 0, spse_terms: int = 0, spse_tolerance: float = 0.0,
            spse_init: bool = False) -> None:
        """PCG on the reduced camera system. With the SCHUR_POWER_SERIES preconditioner
        or ``spse_init`` the series options apply (``spse_terms`` = max_num_spse_iterations);
        ``spse_init`` needs the SPSE base blocks from ``assemble(..., spse_base=True)``
        unless the preconditioner is the power series itself."""
        if precond == _lib.PRECOND_CLUSTER:
            self._call("ceres_b200_ba_pcg_cluster", ctypes.byref(self.clusters.struct), int(min_iterations),
                       int(max_iterations), float(tolerance), int(max_refinements))
        elif precond == _lib.PRECOND_SCHUR_POWER_SERIES or spse_init:
            self._call("ceres_b200_ba_pcg_spse", int(precond), int(min_iterations), int(max_iterations),
                       float(tolerance), int(max_refinements), int(spse_terms), float(spse_tolerance), int(bool(spse_init)))
        else:
            self._call("ceres_b200_ba_pcg", int(precond), int(min_iterations), int(max_iterations), float(tolerance),
                       int(max_refinements))

    def ensure_schur_order(self) -> bool:
        """Give the explicit-S paths (dense_schur_solve, schur_matrix) the fixed summation
        order of ``schur_contributions`` (built once per problem); returns whether it is in
        place (a list longer than SCHUR_ORDER_MAX is not built and the atomic summation
        stays)."""
        if self._schur_order is None:
            order = schur_contributions(self.layout, self.nc, self.cam_const[:self.nc], self.pt_const, self.np_pad)
            self._schur_order = order or ()
            if order:
                st = self.struct
                st.schur_blocks, st.schur_block_start, st.schur_contrib = (_ptr(t) for t in order[:3])
                st.num_schur_blocks = int(order[3])
        return bool(self._schur_order)

    def schur_matrix(self, ordered: bool = True) -> torch.Tensor:
        """The explicit reduced camera matrix [9 nc, 9 nc] (float64) of the last assembly,
        damping included; ``ordered``: in the fixed summation order where the list fits."""
        if ordered:
            self.ensure_schur_order()
        n = 9 * self.nc
        S = torch.empty((max(n, 1), max(n, 1)), dtype=torch.float64, device=self.device)
        kept = self.struct.schur_blocks
        if not ordered:
            self.struct.schur_blocks = None
        try:
            self._call("ceres_b200_ba_schur_matrix", S.data_ptr())
        finally:
            self.struct.schur_blocks = kept
        return S

    def dense_solve(self) -> None:
        if self.nc == 0:
            return
        self.ensure_schur_order()
        if self.dense_work is None:
            nbytes = ctypes.c_int64(0)
            _lib.check(self.lib.ceres_b200_dense_schur_bytes(ctypes.byref(self.struct), ctypes.byref(nbytes)),
                       "dense work size")
            self.dense_work = torch.empty(max(int(nbytes.value) // 8, 1), dtype=torch.float64, device=self.device)
        self._call("ceres_b200_ba_dense_schur_solve", self.dense_work.data_ptr())

    def schur_matvec(self, x: torch.Tensor) -> torch.Tensor:
        x = x.to(self.device, torch.float64).contiguous()
        y = torch.zeros(9 * self.nc, dtype=torch.float64, device=self.device)
        self._call("ceres_b200_ba_schur_matvec", x.data_ptr(), y.data_ptr())
        return y

    def step(self) -> None:
        self._call("ceres_b200_ba_step")

    def read_stats(self) -> np.ndarray:
        self.ctl_host.copy_(self.ctl, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        raw = self.ctl_host.numpy()
        stats = np.frombuffer(raw, dtype=np.float64, count=_lib.NSTATS).copy()
        err = int(stats[_lib.STAT_ERROR])
        if err & _lib.DEVERR_LOSS:
            raise ValueError("Loss function has rho'' > 0 but rho' <= 0")
        if err & _lib.DEVERR_BARRIER:
            raise _lib.NativeLibraryError("a grid barrier of the cooperative PCG timed out")
        if err & _lib.DEVERR_NOT_PD:
            raise _lib.NativeLibraryError("the reduced camera matrix is not positive definite")
        return stats

    # ---------------------------------------------------------------- views for tests
    def slot_view(self):
        """(residuals [no,2], Jc [no,2,9], Jp [no,2,3]) in input observation order."""
        slots = self.layout.slot_of_obs
        r = self.res[slots]
        J = self.jac[slots].to(torch.float64)
        return r, J[:, :18].reshape(-1, 2, 9), J[:, 18:].reshape(-1, 2, 3)


class ClusterPlan:
    """Device arrays of the visibility-cluster preconditioner of one engine
    (ceres_b200_clusters_t): the kept camera block pairs, the components they link, the
    cameras' point lists by point lane, and the storage of the component inverses."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @classmethod
    def build(cls, eng: "BAEngine", tridiagonal: bool, clustering: str) -> "ClusterPlan | None":
        from . import clustering as C

        dev = eng.device
        active = np.flatnonzero(eng.cam_const[:eng.nc].cpu().numpy() == 0)
        if active.size < 2:
            return None
        ci_t, pi_t, pconst = eng._index
        ci = ci_t.detach().cpu().numpy().astype(np.int64)
        pi = pi_t.detach().cpu().numpy().astype(np.int64)
        col = np.full(eng.nc, -1, dtype=np.int64)
        col[active] = np.arange(active.size)
        keep = col[ci] >= 0
        if pconst is not None:
            keep &= ~pconst.detach().cpu().numpy().astype(bool)[pi]
        if not keep.any():
            return None
        incidence = C.incidence_from_observations(active.size, col[ci[keep]], pi[keep])
        st = C.cluster_structure(tridiagonal=tridiagonal, clustering=clustering, incidence=incidence)
        comps = st.components()
        dims = np.array([9 * g.size for g in comps], dtype=np.int64)
        if int(dims.max()) > _CLUSTER_MAX_DIM:
            raise NotImplementedError(
                f"a visibility-cluster component of {int(dims.max()) // 9} cameras: the GPU preconditioner "
                f"inverts components of up to {_CLUSTER_MAX_DIM // 9} cameras")
        member = st.membership
        pairs = []
        cam_comp = np.full(eng.nc, -1, dtype=np.int32)
        cam_pos = np.zeros(eng.nc, dtype=np.int32)
        cam_cluster = np.full(eng.nc, -1, dtype=np.int32)
        cam_cluster[active] = member
        for k, g in enumerate(comps):
            cams = active[g]
            cam_comp[cams] = k
            cam_pos[cams] = np.arange(g.size)
            kg = member[g]
            same = kg[:, None] == kg[None, :]
            nb = st.neighbors[kg]                                   # [m][2]
            linked = (nb[:, None, :] == kg[None, :, None]).any(axis=2)
            a, b = np.nonzero(np.triu(same | linked))
            pairs.append(np.stack([cams[a], cams[b]], axis=1))
        pairs = np.concatenate(pairs).astype(np.int32)
        comp_cams = np.concatenate([active[g] for g in comps]).astype(np.int32)
        comp_cam_off = np.concatenate([[0], np.cumsum([g.size for g in comps])]).astype(np.int32)
        comp_base = np.concatenate([[0], np.cumsum(dims * dims)]).astype(np.int64)
        comp_piv = np.concatenate([[0], np.cumsum(64 * dims + 32 * 32)]).astype(np.int64)  # P, W, A11^-1
        # every camera's observations by point lane (the pair kernel looks points up)
        L = eng.layout
        ents = L.cam_entries[:eng.no].to(torch.int64)
        counts = (L.cam_offsets[1:] - L.cam_offsets[:-1]).to(torch.int64)
        owner = torch.repeat_interleave(torch.arange(eng.nc, device=dev), counts)
        order = torch.argsort(owner * max(eng.np_pad, 1) + ents[:, 1], stable=True)
        entries = ents[order].to(torch.int32).contiguous() if eng.no else L.cam_entries
        t = lambda a: torch.as_tensor(a).to(dev).contiguous()  # noqa: E731
        plan = cls(structure=st, components=comps, pairs=t(pairs), entries=entries, cam_comp=t(cam_comp),
                   cam_pos=t(cam_pos), cam_cluster=t(cam_cluster), comp_cams=t(comp_cams),
                   comp_cam_off=t(comp_cam_off), comp_base=t(comp_base), comp_piv=t(comp_piv),
                   inv=torch.zeros(int(comp_base[-1]), dtype=torch.float64, device=dev),
                   piv=torch.zeros(int(comp_piv[-1]), dtype=torch.float64, device=dev),
                   flags=torch.zeros(8, dtype=torch.int32, device=dev), tridiagonal=bool(tridiagonal))
        s = _lib.ClusterStruct()
        s.num_components, s.num_pairs = len(comps), int(pairs.shape[0])
        s.max_dim, s.tridiagonal, s.num_elements = int(dims.max()), int(bool(tridiagonal)), int(comp_base[-1])
        for name in ("pairs", "entries", "cam_comp", "cam_pos", "cam_cluster", "comp_cams", "comp_cam_off",
                     "comp_base", "comp_piv", "inv", "piv", "flags"):
            setattr(s, name, _ptr(getattr(plan, name)))
        plan.struct = s
        return plan

    def matrices(self) -> list[torch.Tensor]:
        """The component inverses (views into the storage), after cluster_factor."""
        base = self.comp_base.cpu().numpy()
        return [self.inv[int(base[k]):int(base[k + 1])].view(9 * g.size, 9 * g.size)
                for k, g in enumerate(self.components)]


# ======================================================================================
# Levenberg-Marquardt (solver.py:35-357 for the LM strategy)
# ======================================================================================
class _StepEvaluator:
    """solver.py:823-861: relative and historical step quality."""

    def __init__(self, initial_cost: float, max_nonmonotonic: int):
        self.max_nonmonotonic = max(0, int(max_nonmonotonic))
        self.minimum_cost = self.current_cost = self.reference_cost = self.candidate_cost = initial_cost
        self.acc_reference = 0.0
        self.acc_candidate = 0.0
        self.nonmonotonic = 0

    def step_quality(self, cost: float, model_change: float) -> float:
        if model_change <= 0.0:
            return float("-inf")
        relative = (self.current_cost - cost) / model_change
        historical = (self.reference_cost - cost) / (self.acc_reference + model_change)
        return max(relative, historical)

    def step_accepted(self, cost: float, model_change: float) -> None:
        self.current_cost = cost
        self.acc_candidate += model_change
        self.acc_reference += model_change
        if cost < self.minimum_cost:
            self.minimum_cost = cost
            self.nonmonotonic = 0
            self.candidate_cost = cost
            self.acc_candidate = 0.0
        else:
            self.nonmonotonic += 1
            if cost > self.candidate_cost:
                self.candidate_cost = cost
                self.acc_candidate = 0.0
        if self.nonmonotonic == self.max_nonmonotonic:
            self.reference_cost = self.candidate_cost
            self.acc_reference = self.acc_candidate


class _LMRadius:
    """solver.py:805-820."""

    def __init__(self, radius: float, max_radius: float):
        self.radius = radius
        self.max_radius = max_radius
        self.decrease_factor = 2.0

    def accepted(self, quality: float) -> float:
        self.radius = min(self.max_radius, self.radius / max(1.0 / 3.0, 1.0 - (2.0 * quality - 1.0) ** 3))
        self.decrease_factor = 2.0
        return self.radius

    def rejected(self) -> float:
        self.radius = self.radius / self.decrease_factor
        self.decrease_factor *= 2.0
        return self.radius


@dataclass
class LMResult:
    summary: SolverSummary
    time_to_tolerance: float | None = None


def _log(options: SolverOptions, it: IterationSummary) -> None:
    if not options.minimizer_progress_to_stdout or options.logging_type is LoggingType.SILENT:
        return
    print(f"{it.iteration:4d}: f:{it.cost: .6e} d:{it.cost_change: .3e} g:{it.gradient_max_norm: .3e} "
          f"h:{it.step_norm: .3e} rho:{it.relative_decrease: .3e} mu:{it.trust_region_radius: .3e}")


def linear_solver_kind(options: SolverOptions) -> str:
    lst = options.linear_solver_type
    if lst in (LinearSolverType.DENSE_SCHUR, LinearSolverType.SPARSE_SCHUR):
        return "dense"
    if lst is LinearSolverType.ITERATIVE_SCHUR:
        if options.preconditioner_type not in _PRECOND:
            raise NotImplementedError(
                f"ITERATIVE_SCHUR with {options.preconditioner_type.value} is not implemented on the GPU path "
                "(IDENTITY, JACOBI, SCHUR_JACOBI, SCHUR_POWER_SERIES_EXPANSION, CLUSTER_JACOBI and "
                "CLUSTER_TRIDIAGONAL are)")
        return "iterative"
    raise NotImplementedError(f"{lst.value} is not a Schur solver; the GPU path implements DENSE_SCHUR, "
                              "SPARSE_SCHUR and ITERATIVE_SCHUR")


def run_lm(engine: BAEngine, options: SolverOptions, summary: SolverSummary, *, start: float,
           num_active_columns: int, max_refinements: int = 1, target_cost: float | None = None,
           stop_at_target: bool = False, on_state=None) -> LMResult:
    """The trust-region loop. ``summary`` arrives with the preprocessing fields set.

    ``target_cost``: when given, the wall time at which the best cost first
    drops to or below it is returned as ``time_to_tolerance``; with
    ``stop_at_target`` the solve ends there (USER_SUCCESS, "Target cost reached.").
    ``on_state(engine, which)``: copies device parameters to the caller's
    tensors (used for callbacks that look at the parameters).
    """
    kind = linear_solver_kind(options)
    precond = _PRECOND.get(options.preconditioner_type, _lib.PRECOND_SCHUR_JACOBI)
    if precond == _lib.PRECOND_CLUSTER:
        # the visibility clusters of the active cameras (linear.py:498-521); without them the
        # reference uses the SCHUR_JACOBI blocks
        tri = options.preconditioner_type is PreconditionerType.CLUSTER_TRIDIAGONAL
        if kind != "iterative" or not engine.setup_clusters(tri, options.visibility_clustering_type.name):
            precond = _lib.PRECOND_SCHUR_JACOBI
    spse_init = kind == "iterative" and bool(options.use_spse_initialization)
    spse_base = spse_init and precond != _lib.PRECOND_SCHUR_POWER_SERIES
    refinements = max_refinements if engine.precision == "mixed" else 0
    lm = _LMRadius(options.initial_trust_region_radius, options.max_trust_region_radius)
    radius = lm.radius
    consecutive_invalid = 0
    previous_cost: float | None = None
    minimizer_start = time.perf_counter()
    ttt: float | None = None

    t0 = time.perf_counter()
    engine.evaluate(True)
    engine.assemble(radius, options, precond, spse_base)
    st = engine.read_stats()
    eval_time = time.perf_counter() - t0
    summary.jacobian_evaluation_time_in_seconds += eval_time
    cost = float(st[_lib.STAT_COST])
    gmax = max(st[_lib.STAT_GMAX_P], st[_lib.STAT_GMAX_C])
    gnorm = math.sqrt(st[_lib.STAT_GSQ_P] + st[_lib.STAT_GSQ_C])
    summary.initial_cost = cost
    summary.final_cost = cost
    best_cost = cost
    engine.save_best()
    best_is_current = True
    if target_cost is not None and best_cost <= target_cost:
        ttt = time.perf_counter() - start
    evaluator = _StepEvaluator(cost, options.max_consecutive_nonmonotonic_steps if options.use_nonmonotonic_steps else 0)
    need_assemble = False
    terminated = False
    # After an accepted step the evaluation and assembly at the new point are launched
    # without waiting for their statistics: the next PCG and step are queued behind them
    # and one read after the step brings both (their statistics slots are disjoint). The
    # gradient test of the new point then runs before anything of the next iteration is
    # used, so the iterations, counters and terminations are those of the unpipelined
    # loop; a solve that stops there has launched one PCG and step for nothing.
    pending_eval = False

    def take_evaluation(st) -> bool:
        """The new point's cost and gradient from ``st``; True when its gradient test ends
        the solve (solver.py:1165-1175)."""
        nonlocal cost, gmax, gnorm, pending_eval, terminated
        pending_eval = False
        cost = float(st[_lib.STAT_COST])
        gmax = max(st[_lib.STAT_GMAX_P], st[_lib.STAT_GMAX_C])
        gnorm = math.sqrt(st[_lib.STAT_GSQ_P] + st[_lib.STAT_GSQ_C])
        if gmax <= options.gradient_tolerance:
            summary.termination_type = TerminationType.CONVERGENCE
            summary.message = "Gradient tolerance reached."
            summary.final_cost = cost
            terminated = True
            return True
        return False

    def finalize() -> LMResult:
        if summary.minimizer_time_in_seconds == 0.0:
            summary.minimizer_time_in_seconds = time.perf_counter() - minimizer_start
        post = time.perf_counter()
        if not best_is_current:
            engine.restore_best()
        summary.final_cost = best_cost
        summary.postprocessor_time_in_seconds += time.perf_counter() - post
        summary.total_time_in_seconds = time.perf_counter() - start
        return LMResult(summary, ttt)

    if num_active_columns == 0:
        summary.termination_type = TerminationType.CONVERGENCE
        summary.message = "No active parameters."
        return finalize()

    for iteration in range(options.max_num_iterations + 1):
        it_start = time.perf_counter()
        jac_time = 0.0
        if need_assemble:
            t0 = time.perf_counter()
            engine.assemble(radius, options, precond, spse_base)
            need_assemble = False
            jac_time = time.perf_counter() - t0
        summary.num_jacobian_evaluations += 1
        it = IterationSummary(iteration=iteration, step_is_valid=True, step_is_successful=True, cost=cost,
                              gradient_norm=gnorm, gradient_max_norm=gmax, trust_region_radius=radius,
                              eta=options.eta, jacobian_evaluation_time_in_seconds=jac_time)
        if iteration == 0:
            it.iteration_time_in_seconds = time.perf_counter() - it_start
            it.cumulative_time_in_seconds = time.perf_counter() - start
            summary.iterations.append(it)
            _log(options, it)
            if gmax <= options.gradient_tolerance:
                summary.termination_type = TerminationType.CONVERGENCE
                summary.message = "Gradient tolerance reached."
                summary.final_cost = cost
                terminated = True
                break
            if options.max_num_iterations == 0:
                summary.termination_type = TerminationType.NO_CONVERGENCE
                summary.message = "Maximum iterations reached."
                summary.final_cost = cost
                terminated = True
                break
            continue

        lin_start = time.perf_counter()
        if kind == "dense":
            engine.dense_solve()
            lin_iters = 1
        else:
            engine.pcg(precond, options.min_linear_solver_iterations, options.max_linear_solver_iterations,
                       options.eta, refinements, options.max_num_spse_iterations, options.spse_tolerance, spse_init)
        engine.step()
        st = engine.read_stats()
        if pending_eval:
            if take_evaluation(st):
                summary.num_jacobian_evaluations -= 1  # this iteration never started
                break
            it.cost, it.gradient_norm, it.gradient_max_norm = cost, gnorm, gmax
        lin_time = time.perf_counter() - lin_start
        if kind != "dense":
            lin_iters = int(st[_lib.STAT_PCG_ITERS]) if engine.nc else 1
        summary.num_linear_solves += 1
        summary.linear_solver_time_in_seconds += lin_time

        if st[_lib.STAT_NONFINITE] > 0:
            consecutive_invalid += 1
            radius = lm.rejected()
            need_assemble = True
            it.step_is_valid = False
            it.step_is_successful = False
            it.linear_solver_iterations = lin_iters
            it.linear_solver_time_in_seconds = lin_time
            it.step_solver_time_in_seconds = lin_time
            it.trust_region_radius = radius
            it.iteration_time_in_seconds = time.perf_counter() - it_start
            it.cumulative_time_in_seconds = time.perf_counter() - start
            summary.num_unsuccessful_steps += 1
            if consecutive_invalid >= options.max_num_consecutive_invalid_steps:
                summary.termination_type = TerminationType.FAILURE
                summary.message = "Too many invalid trust-region steps."
                terminated = True
                break
            summary.iterations.append(it)
            _log(options, it)
            continue

        summary.num_residual_evaluations += 1
        candidate_cost = float(st[_lib.STAT_CAND_COST])
        model_decrease = max(float(st[_lib.STAT_MODEL]), 0.0)
        step_is_valid = model_decrease > 0.0
        rho = evaluator.step_quality(candidate_cost, model_decrease) if step_is_valid else 0.0
        accepted = step_is_valid and rho > options.min_relative_decrease
        step_norm = math.sqrt(st[_lib.STAT_STEP_SQ_P] + st[_lib.STAT_STEP_SQ_C])
        it.step_norm = step_norm
        it.cost_change = cost - candidate_cost
        it.relative_decrease = float(rho)
        it.step_is_valid = step_is_valid
        it.linear_solver_iterations = lin_iters
        it.linear_solver_time_in_seconds = lin_time
        it.step_solver_time_in_seconds = lin_time
        it.iteration_time_in_seconds = time.perf_counter() - it_start
        it.cumulative_time_in_seconds = time.perf_counter() - start

        if accepted:
            consecutive_invalid = 0
            summary.num_successful_steps += 1
            evaluator.step_accepted(candidate_cost, model_decrease)
            engine.accept()
            if candidate_cost < best_cost:
                best_cost = candidate_cost
                best_is_current = True
                if options.use_nonmonotonic_steps:
                    engine.save_best()
                it.step_is_nonmonotonic = False
            else:
                if best_is_current and options.use_nonmonotonic_steps:
                    pass  # best buffers already hold the best state
                best_is_current = False
                it.step_is_nonmonotonic = candidate_cost > best_cost
            reached = target_cost is not None and ttt is None and best_cost <= target_cost
            if reached:
                ttt = time.perf_counter() - start
            summary.final_cost = best_cost
            radius = lm.accepted(rho)
            it.trust_region_radius = radius
            it.step_is_successful = True
            if reached and stop_at_target:
                summary.iterations.append(it)
                summary.termination_type = TerminationType.USER_SUCCESS
                summary.message = "Target cost reached."
                return finalize()
        else:
            summary.num_unsuccessful_steps += 1
            radius = lm.rejected()
            it.trust_region_radius = radius
            it.step_is_successful = False
            need_assemble = True

        summary.iterations.append(it)
        _log(options, it)
        if options.callbacks:
            if on_state is not None and options.update_state_every_iteration:
                on_state(engine, "best" if (options.use_nonmonotonic_steps and not best_is_current) else "current")
            stop = None
            for callback in options.callbacks:
                result = callback(it)
                if result is CallbackReturnType.SOLVER_ABORT:
                    summary.termination_type = TerminationType.USER_FAILURE
                    summary.message = "User callback aborted."
                    stop = True
                    break
                if result is CallbackReturnType.SOLVER_TERMINATE_SUCCESSFULLY:
                    summary.termination_type = TerminationType.USER_SUCCESS
                    summary.message = "User callback terminated successfully."
                    stop = True
                    break
            if stop:
                return finalize()

        if accepted:
            state_norm = math.sqrt(st[_lib.STAT_CAND_STATE_SQ_P] + st[_lib.STAT_CAND_STATE_SQ_C])
            if step_norm <= options.parameter_tolerance * (state_norm + options.parameter_tolerance):
                summary.termination_type = TerminationType.CONVERGENCE
                summary.message = "Parameter tolerance reached."
                terminated = True
                break
            if previous_cost is not None and abs(previous_cost - candidate_cost) <= \
                    options.function_tolerance * max(previous_cost, 1.0):
                summary.termination_type = TerminationType.CONVERGENCE
                summary.message = "Function tolerance reached."
                terminated = True
                break
            previous_cost = candidate_cost
            t0 = time.perf_counter()
            engine.evaluate(True)
            engine.assemble(radius, options, precond, spse_base)
            summary.jacobian_evaluation_time_in_seconds += time.perf_counter() - t0  # launch time
            summary.num_jacobian_evaluations += 1
            pending_eval = True
        stopping = radius <= options.min_trust_region_radius or \
            time.perf_counter() - start >= options.max_solver_time_in_seconds
        if pending_eval and (stopping or iteration == options.max_num_iterations):
            # the new point's gradient test comes first, as in the unpipelined loop
            if take_evaluation(engine.read_stats()):
                break
        if radius <= options.min_trust_region_radius:
            summary.termination_type = TerminationType.CONVERGENCE
            summary.message = "Minimum trust-region radius reached."
            terminated = True
            break
        if time.perf_counter() - start >= options.max_solver_time_in_seconds:
            summary.termination_type = TerminationType.NO_CONVERGENCE
            summary.message = "Maximum solver time reached."
            terminated = True
            break
    if not terminated:
        summary.termination_type = TerminationType.NO_CONVERGENCE
        summary.message = "Maximum iterations reached."
    return finalize()
