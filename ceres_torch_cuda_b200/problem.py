"""Problem modelling API with ceres-torch's names (problem.py:43-572) for the
bundle-adjustment path, plus a tensor-level constructor.

Two ways to describe a bundle-adjustment problem:

* ``Problem`` with one residual block per observation, each a
  ``SnavelyReprojectionError`` over a 9-parameter camera block and a 3-parameter
  point block, points in ordering group 0 (as in ceres-torch's
  ``examples/simple_bundle_adjuster.py:82-112``);
* ``BundleAdjustmentProblem`` holding the whole problem as tensors
  (cameras [nc,9], points [np,3], observations [no,2], camera/point index
  [no]), which needs no Python object per observation.

``solve`` turns either into the device-resident form; results are written back
into the caller's parameter tensors.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from .losses import LossFunction, as_loss, device_loss


# ------------------------------------------------------------------------------------
# Cost functions
# ------------------------------------------------------------------------------------
class CostFunction:
    parameter_block_sizes: Optional[list[int]] = None
    num_residuals: Optional[int] = None

    def residuals(self, *parameters: torch.Tensor) -> torch.Tensor:
        raise NotImplementedError

    def __call__(self, *parameters: torch.Tensor) -> torch.Tensor:
        return self.residuals(*parameters)


def _rotate(aa: torch.Tensor, X: torch.Tensor) -> torch.Tensor:
    """Angle-axis rotation through a unit quaternion (rotation.py:104-110, :211-222)."""
    theta = torch.linalg.norm(aa, dim=-1, keepdim=True)
    eps = torch.finfo(aa.dtype).eps
    small = theta <= eps
    k = torch.where(small, 0.5 - theta * theta / 48.0, torch.sin(0.5 * theta) / torch.where(small, 1.0, theta))
    q = torch.cat([torch.cos(0.5 * theta), k * aa], dim=-1)
    q = q / torch.linalg.norm(q, dim=-1, keepdim=True).clamp_min(torch.finfo(aa.dtype).tiny)
    u = q[..., 1:]
    uv = 2.0 * torch.linalg.cross(u, X, dim=-1)
    return X + q[..., :1] * uv + torch.linalg.cross(u, uv, dim=-1)


def snavely_project(camera: torch.Tensor, point: torch.Tensor) -> torch.Tensor:
    """Pixel of ``point`` in ``camera`` (9 params: angle-axis, translation, f, k1, k2),
    batched over leading dimensions; the formula of simple_bundle_adjuster.py:73-79."""
    p = _rotate(camera[..., 0:3], point) + camera[..., 3:6]
    xp = -p[..., 0] / p[..., 2]
    yp = -p[..., 1] / p[..., 2]
    r2 = xp * xp + yp * yp
    d = 1.0 + r2 * (camera[..., 7] + camera[..., 8] * r2)
    fd = camera[..., 6] * d
    return torch.stack([fd * xp, fd * yp], dim=-1)


class SnavelyReprojectionError(CostFunction):
    """Residual ``snavely_project(camera, point) - observation`` (2 residuals,
    parameter blocks [camera 9, point 3]). The solver recognises this class and
    evaluates it (with its Jacobian and the robust corrector) on the GPU."""

    parameter_block_sizes = [9, 3]
    num_residuals = 2

    def __init__(self, observed_x: float | torch.Tensor, observed_y: float | None = None) -> None:
        if observed_y is None:
            obs = torch.as_tensor(observed_x, dtype=torch.float64).reshape(-1)
            self.observed = (float(obs[0]), float(obs[1]))
        else:
            self.observed = (float(observed_x), float(observed_y))

    @classmethod
    def Create(cls, observed_x: float, observed_y: float) -> "SnavelyReprojectionError":  # noqa: N802
        return cls(observed_x, observed_y)

    def residuals(self, camera: torch.Tensor, point: torch.Tensor) -> torch.Tensor:
        obs = torch.tensor(self.observed, dtype=camera.dtype, device=camera.device)
        return snavely_project(camera.reshape(9), point.reshape(3)) - obs


# ------------------------------------------------------------------------------------
# Parameter / residual blocks and the Problem
# ------------------------------------------------------------------------------------
@dataclass(eq=False)
class ParameterBlock:
    tensor: torch.Tensor
    constant: bool = False
    name: Optional[str] = None
    ordering_group: Optional[int] = None
    lower_bound: Optional[torch.Tensor] = None
    upper_bound: Optional[torch.Tensor] = None

    def __post_init__(self) -> None:
        if not isinstance(self.tensor, torch.Tensor):
            raise TypeError("ParameterBlock tensor must be a torch.Tensor")

    @property
    def size(self) -> int:
        return self.tensor.numel()

    @property
    def tangent_size(self) -> int:
        return 0 if self.constant else self.size

    @property
    def dtype(self) -> torch.dtype:
        return self.tensor.dtype

    @property
    def device(self) -> torch.device:
        return self.tensor.device


@dataclass(eq=False)
class ResidualBlock:
    cost_function: CostFunction
    loss_function: Optional[LossFunction]
    parameter_blocks: list[ParameterBlock]
    name: Optional[str] = None


@dataclass
class ProblemOptions:
    enable_fast_removal: bool = False
    disable_all_safety_checks: bool = False
    evaluation_callback: object = None


class Problem:
    def __init__(self, options: Optional[ProblemOptions] = None) -> None:
        self.options = options or ProblemOptions()
        self.parameter_blocks: list[ParameterBlock] = []
        self.residual_blocks: list[ResidualBlock] = []
        self._by_id: dict[int, ParameterBlock] = {}

    # -- parameter blocks
    def add_parameter_block(self, values: torch.Tensor, size: Optional[int] = None, manifold=None, *,
                            name: Optional[str] = None) -> ParameterBlock:
        if manifold is not None:
            raise NotImplementedError("only Euclidean parameter blocks are supported on the bundle-adjustment path")
        if size is not None and values.numel() != size:
            raise ValueError(f"Expected parameter block size {size}, got {values.numel()}")
        block = self._by_id.get(id(values))
        if block is None:
            block = ParameterBlock(values, name=name)
            self.parameter_blocks.append(block)
            self._by_id[id(values)] = block
        elif name is not None:
            block.name = name
        return block

    AddParameterBlock = add_parameter_block

    def _block(self, value) -> ParameterBlock:
        if isinstance(value, ParameterBlock):
            return value
        block = self._by_id.get(id(value))
        return block if block is not None else self.add_parameter_block(value)

    def _require(self, value) -> ParameterBlock:
        if isinstance(value, ParameterBlock):
            if value not in self.parameter_blocks:
                raise KeyError("Parameter block is not part of this problem")
            return value
        block = self._by_id.get(id(value))
        if block is None:
            raise KeyError("Parameter block is not part of this problem")
        return block

    def add_residual_block(self, cost_function: CostFunction, loss_function: Optional[LossFunction],
                           parameter_blocks: Sequence, *, name: Optional[str] = None) -> ResidualBlock:
        if not isinstance(cost_function, CostFunction):
            raise TypeError("cost_function must be a CostFunction (SnavelyReprojectionError on this path)")
        blocks = [self._block(p) for p in parameter_blocks]
        if cost_function.parameter_block_sizes is not None:
            expected = list(cost_function.parameter_block_sizes)
            got = [b.size for b in blocks]
            if expected != got:
                raise ValueError(f"Cost function parameter sizes {expected} do not match blocks {got}")
        rb = ResidualBlock(cost_function, loss_function, blocks, name=name)
        self.residual_blocks.append(rb)
        return rb

    AddResidualBlock = add_residual_block

    def remove_residual_block(self, residual_block: ResidualBlock) -> None:
        self.residual_blocks.remove(residual_block)

    RemoveResidualBlock = remove_residual_block

    def set_parameter_block_constant(self, block) -> None:
        self._block(block).constant = True

    SetParameterBlockConstant = set_parameter_block_constant

    def set_parameter_block_variable(self, block) -> None:
        self._block(block).constant = False

    SetParameterBlockVariable = set_parameter_block_variable

    def is_parameter_block_constant(self, block) -> bool:
        return self._block(block).constant

    IsParameterBlockConstant = is_parameter_block_constant

    def set_parameter_block_ordering_group(self, block, group: Optional[int]) -> None:
        self._block(block).ordering_group = group

    SetParameterBlockOrderingGroup = set_parameter_block_ordering_group

    def get_parameter_block_ordering_group(self, block) -> Optional[int]:
        return self._require(block).ordering_group

    GetParameterBlockOrderingGroup = get_parameter_block_ordering_group

    def has_parameter_block(self, block) -> bool:
        if isinstance(block, ParameterBlock):
            return block in self.parameter_blocks
        return id(block) in self._by_id

    HasParameterBlock = has_parameter_block

    def num_parameter_blocks(self) -> int:
        return len(self.parameter_blocks)

    NumParameterBlocks = num_parameter_blocks

    def num_parameters(self) -> int:
        return sum(b.size for b in self.parameter_blocks)

    NumParameters = num_parameters

    def num_effective_parameters(self) -> int:
        return sum(b.tangent_size for b in self.parameter_blocks)

    NumEffectiveParameters = num_effective_parameters

    def num_residual_blocks(self) -> int:
        return len(self.residual_blocks)

    NumResidualBlocks = num_residual_blocks

    def num_residuals(self) -> int:
        return sum(int(rb.cost_function.num_residuals or 0) for rb in self.residual_blocks)

    NumResiduals = num_residuals

    def get_parameter_blocks(self) -> list[ParameterBlock]:
        return list(self.parameter_blocks)

    GetParameterBlocks = get_parameter_blocks

    def get_residual_blocks(self) -> list[ResidualBlock]:
        return list(self.residual_blocks)

    GetResidualBlocks = get_residual_blocks

    def parameter_block_size(self, block) -> int:
        return self._require(block).size

    ParameterBlockSize = parameter_block_size


# ------------------------------------------------------------------------------------
# Tensor-level problem
# ------------------------------------------------------------------------------------
@dataclass
class BundleAdjustmentProblem:
    """A whole bundle-adjustment problem as tensors.

    ``cameras`` [nc, 9] and ``points`` [np, 3] are updated in place by ``solve``.
    ``camera_constant`` / ``point_constant`` are optional bool masks.
    """

    cameras: torch.Tensor
    points: torch.Tensor
    observations: torch.Tensor
    camera_index: torch.Tensor
    point_index: torch.Tensor
    loss: Optional[LossFunction] = None
    camera_constant: Optional[torch.Tensor] = None
    point_constant: Optional[torch.Tensor] = None
    _engine_cache: dict = field(default_factory=dict, repr=False)
    _track_stats: Optional[tuple] = field(default=None, repr=False)

    @classmethod
    def from_arrays(cls, cameras, points, observations, camera_index, point_index, *, loss=None,
                    device: str | torch.device = "cuda", camera_constant=None, point_constant=None,
                    track_stats: bool = False):
        """``track_stats``: also record, from the host indices, the most observations of
        one point and whether a camera observes a point twice (about 0.1 ms for 5k
        observations), so that a batch of such problems is laid out without a
        device-to-host read (worth it for the many small batches of a server)."""
        def t(x, dt):
            return torch.as_tensor(x).to(device=device, dtype=dt).contiguous()
        prob = cls(t(cameras, torch.float64), t(points, torch.float64), t(observations, torch.float64),
                   t(camera_index, torch.int64), t(point_index, torch.int64), loss,
                   None if camera_constant is None else t(camera_constant, torch.bool),
                   None if point_constant is None else t(point_constant, torch.bool))
        if track_stats:
            ci = np.asarray(camera_index.cpu() if isinstance(camera_index, torch.Tensor) else camera_index,
                            dtype=np.int64).reshape(-1)
            pi = np.asarray(point_index.cpu() if isinstance(point_index, torch.Tensor) else point_index,
                            dtype=np.int64).reshape(-1)
            if ci.size == pi.size:
                prob._set_track_stats(ci, pi)
        return prob

    def _set_track_stats(self, ci: np.ndarray, pi: np.ndarray) -> None:
        """Record, from the host copy of the indices, the most observations of one point
        and whether a camera observes a point more than once, tied to the index tensors'
        version counters (an in-place change of either drops them)."""
        no, npts, nc = ci.size, self.num_points, self.num_cameras
        if no == 0 or pi.min() < 0 or pi.max() >= npts or ci.min() < 0 or ci.max() >= nc:
            return
        max_track = int(np.bincount(pi, minlength=npts).max())
        key = np.sort(pi * max(nc, 1) + ci)
        dup = bool(no > 1 and (key[1:] == key[:-1]).any())
        self._track_stats = (max_track, dup, self.camera_index._version, self.point_index._version)

    @property
    def track_stats(self) -> Optional[tuple[int, bool]]:
        """(most observations of one point, whether a camera observes a point twice), when
        recorded from host indices and the index tensors are unchanged since; else None."""
        st = self._track_stats
        if st is None or st[2] != self.camera_index._version or st[3] != self.point_index._version:
            return None
        return st[0], st[1]

    @classmethod
    def from_bal_text(cls, text: str, *, loss=None, device: str | torch.device = "cuda"):
        """Parse the BAL format (BALProblem.from_text, examples/simple_bundle_adjuster.py:33-70):
        "nc np no", no lines "camera point x y", 9 nc camera values, 3 np point values,
        whitespace separated. Vectorised (one numpy conversion of all values) instead of
        one Python object per observation."""
        tokens = text.split()
        if len(tokens) < 3:
            raise ValueError("BAL input is missing its header")
        nc, npts, no = (int(t) for t in tokens[:3])
        expected = 3 + 4 * no + 9 * nc + 3 * npts
        if len(tokens) > expected:
            raise ValueError("BAL input contains trailing values")
        if len(tokens) < expected:
            raise ValueError("BAL input is truncated")
        vals = np.array(tokens[3:], dtype=np.float64)
        obs_block = vals[:4 * no].reshape(no, 4)
        ci, pi = obs_block[:, 0], obs_block[:, 1]
        if not (np.all(ci == np.round(ci)) and np.all(pi == np.round(pi))):
            raise ValueError("BAL camera and point indices must be integers")
        cameras = vals[4 * no:4 * no + 9 * nc].reshape(nc, 9)
        points = vals[4 * no + 9 * nc:].reshape(npts, 3)
        return cls.from_arrays(cameras, points, obs_block[:, 2:4], ci.astype(np.int64), pi.astype(np.int64),
                               loss=loss, device=device)

    @classmethod
    def from_bal_file(cls, path, *, loss=None, device: str | torch.device = "cuda"):
        from pathlib import Path
        return cls.from_bal_text(Path(path).read_text(), loss=loss, device=device)

    @property
    def num_cameras(self) -> int:
        return int(self.cameras.shape[0])

    @property
    def num_points(self) -> int:
        return int(self.points.shape[0])

    @property
    def num_observations(self) -> int:
        return int(self.observations.shape[0])


@dataclass
class ExtractedBA:
    """A ``Problem`` recognised as bundle adjustment, as flat tensors."""

    cameras: torch.Tensor
    points: torch.Tensor
    observations: torch.Tensor
    camera_index: torch.Tensor
    point_index: torch.Tensor
    loss: Optional[LossFunction]
    camera_constant: torch.Tensor
    point_constant: torch.Tensor
    camera_blocks: list
    point_blocks: list


def snavely_cost(cost_function) -> "SnavelyReprojectionError | None":
    """The SnavelyReprojectionError behind a residual block's cost function: the object
    itself, or the one ceres-torch's Problem wrapped when it was added there
    (``CallableCostFunction(functor)``, problem.py:167-168 / costs.py:50-62)."""
    if isinstance(cost_function, SnavelyReprojectionError):
        return cost_function
    inner = getattr(cost_function, "functor", None)
    return inner if isinstance(inner, SnavelyReprojectionError) else None


def extract_bundle_adjustment(problem: Problem) -> ExtractedBA:
    """Recognise ``problem`` as Snavely bundle adjustment or raise NotImplementedError."""
    if not problem.residual_blocks:
        raise NotImplementedError("the problem has no residual blocks")
    cam_of: dict[int, int] = {}
    pt_of: dict[int, int] = {}
    cam_blocks: list[ParameterBlock] = []
    pt_blocks: list[ParameterBlock] = []
    ci: list[int] = []
    pi: list[int] = []
    obs: list[tuple[float, float]] = []
    loss0 = problem.residual_blocks[0].loss_function
    spec0 = device_loss(loss0)
    for rb in problem.residual_blocks:
        cost = snavely_cost(rb.cost_function)
        if cost is None or len(rb.parameter_blocks) != 2:
            raise NotImplementedError(
                "the GPU path solves bundle-adjustment problems whose residual blocks are all "
                f"SnavelyReprojectionError; found {type(rb.cost_function).__name__}")
        if rb.loss_function is not loss0 and device_loss(rb.loss_function) != spec0:
            raise NotImplementedError("all residual blocks must share one loss function on the GPU path")
        cb, pb = rb.parameter_blocks
        k = cam_of.get(id(cb))
        if k is None:
            k = cam_of[id(cb)] = -1
        ci.append(id(cb))
        pi.append(id(pb))
        if id(pb) not in pt_of:
            pt_of[id(pb)] = -1
        obs.append(cost.observed)
    # camera / point numbering follows the problem's parameter-block order
    for b in problem.parameter_blocks:
        if id(b) in cam_of:
            cam_of[id(b)] = len(cam_blocks)
            cam_blocks.append(b)
        elif id(b) in pt_of:
            pt_of[id(b)] = len(pt_blocks)
            pt_blocks.append(b)
    if set(cam_of) & set(pt_of):
        raise NotImplementedError("a parameter block is used both as a camera and as a point")
    groups_p = {b.ordering_group for b in pt_blocks}
    groups_c = {b.ordering_group for b in cam_blocks}
    if any(g is not None for g in groups_p | groups_c):
        gp = [g for g in groups_p if g is not None]
        gc = [g if g is not None else float("inf") for g in groups_c]
        if len(gp) != len(groups_p) or (gc and max(gp) >= min(gc)):
            raise NotImplementedError("points must be in the first ordering group (the eliminated one) and "
                                      "cameras in later groups")
    dev = cam_blocks[0].tensor.device
    cameras = torch.stack([b.tensor.detach().reshape(9) for b in cam_blocks]).to(dev, torch.float64)
    points = torch.stack([b.tensor.detach().reshape(3) for b in pt_blocks]).to(dev, torch.float64)
    return ExtractedBA(
        cameras=cameras,
        points=points,
        observations=torch.tensor(obs, dtype=torch.float64, device=dev),
        camera_index=torch.tensor([cam_of[i] for i in ci], dtype=torch.int64, device=dev),
        point_index=torch.tensor([pt_of[i] for i in pi], dtype=torch.int64, device=dev),
        loss=as_loss(loss0),
        camera_constant=torch.tensor([b.constant for b in cam_blocks], dtype=torch.bool, device=dev),
        point_constant=torch.tensor([b.constant for b in pt_blocks], dtype=torch.bool, device=dev),
        camera_blocks=cam_blocks,
        point_blocks=pt_blocks,
    )


def write_back(blocks: list[ParameterBlock], values: torch.Tensor) -> None:
    """Copy rows of ``values`` into the block tensors (one batched copy when the
    blocks are consecutive rows of one base tensor)."""
    if not blocks:
        return
    with torch.no_grad():
        t0 = blocks[0].tensor
        n = t0.numel()
        base = t0._base if t0._base is not None else None
        if base is not None and base.is_contiguous() and base.numel() >= len(blocks) * n:
            start = t0.storage_offset()
            ok = all(b.tensor._base is base and b.tensor.is_contiguous() and b.tensor.storage_offset() == start + i * n
                     for i, b in enumerate(blocks))
            if ok:
                flat = base.reshape(-1)
                off = start - base.storage_offset()
                flat[off: off + len(blocks) * n].copy_(values.reshape(-1).to(flat.dtype))
                return
        for b, v in zip(blocks, values):
            b.tensor.reshape(-1).copy_(v.to(b.tensor.dtype))
