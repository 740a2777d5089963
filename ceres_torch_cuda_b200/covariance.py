"""Post-solve covariance of a bundle-adjustment problem through the Schur system, with
ceres-torch's ``Covariance`` interface (covariance.py:13-445: the same options,
summary fields, block API and failure message).

ceres-torch forms the dense Jacobian and takes its SVD (or QR). Here the covariance of
the tangent space, (J^T J)^-1 with points eliminated first, comes from the reduced
camera system on the GPU:

* camera blocks:       S^-1, with S = U - F^T W^-1 F the undamped Schur complement
                       (``ceres_b200_ba_schur_matrix`` after the point and camera
                       assembly at radius +inf; ``ceres_b200_dense_spd_inverse``: Cholesky
                       and one CTA per column of the inverse);
* camera-point blocks: -S^-1 F_q^T W_q^-1;
* point blocks:        W_q^-1 delta_qp + W_q^-1 F_q S^-1 F_p^T W_p^-1,

where W_q = J_q^T J_q is point q's 3x3 block and F_q the coupling of point q with the
cameras that see it (summed over its observations). This is exactly (J^T J)^-1 when J
has full column rank; a rank-deficient Jacobian (a free gauge, for instance) makes S
singular, and the computation reports the reference's failure ("Jacobian is rank
deficient."). Pseudo-inverses (null_space_rank != 0) are not offered on the GPU path.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Optional, Sequence

import torch

from . import _lib
from .engine import BAEngine
from .problem import extract_bundle_adjustment
from .types import CovarianceAlgorithmType, SparseLinearAlgebraLibraryType


@dataclass
class CovarianceOptions:
    sparse_linear_algebra_library_type: SparseLinearAlgebraLibraryType = SparseLinearAlgebraLibraryType.NO_SPARSE
    algorithm_type: CovarianceAlgorithmType = CovarianceAlgorithmType.DENSE_SVD
    column_pivot_threshold: float = -1.0
    min_reciprocal_condition_number: float = 1e-14
    null_space_rank: int = 0
    num_threads: int = 1
    apply_loss_function: bool = True

    def validate(self) -> None:
        for ok, message in ((self.column_pivot_threshold >= -1.0, "column_pivot_threshold must be >= -1"),
                            (self.min_reciprocal_condition_number >= 0.0,
                             "min_reciprocal_condition_number must be >= 0"),
                            (self.null_space_rank >= -1, "null_space_rank must be >= -1"),
                            (self.num_threads > 0, "num_threads must be > 0")):
            if not ok:
                raise ValueError(message)


@dataclass
class CovarianceSummary:
    algorithm_type: CovarianceAlgorithmType
    success: bool = False
    message: str = "Covariance.compute was not called."
    rank: int = 0
    nullity: int = 0
    num_rows: int = 0
    num_columns: int = 0
    num_requested_blocks: int = 0
    num_computed_blocks: int = 0
    ambient_dimension: int = 0
    tangent_dimension: int = 0
    max_singular_value: float = 0.0
    min_retained_singular_value: float = 0.0
    reciprocal_condition_number: float = 0.0
    requested_null_space_rank: int = 0

    def BriefReport(self) -> str:  # noqa: N802 - ceres-torch API name
        return (f"ceres-torch Covariance Report: Algorithm: {self.algorithm_type.value}, Rank: {self.rank}, "
                f"Nullity: {self.nullity}, Success: {self.success}")


class Covariance:
    """``Covariance(options).compute(blocks, problem)`` for bundle-adjustment problems
    (residual blocks all SnavelyReprojectionError; this package's or ceres-torch's
    Problem) on CUDA tensors."""

    def __init__(self, options: Optional[CovarianceOptions] = None) -> None:
        self.options = options or CovarianceOptions()
        self.summary = CovarianceSummary(algorithm_type=self.options.algorithm_type,
                                         requested_null_space_rank=self.options.null_space_rank)
        self._problem = None
        self._blocks: set = set()
        self._where: dict = {}
        self._cov_c: Optional[torch.Tensor] = None
        self._winv: Optional[torch.Tensor] = None
        self._point_index: Optional[torch.Tensor] = None
        self._F: dict = {}
        self._engine: Optional[BAEngine] = None

    # ------------------------------------------------------------------ compute
    def compute(self, covariance_blocks, problem) -> bool:
        self.options.validate()
        if self.options.null_space_rank != 0:
            raise NotImplementedError("the GPU covariance inverts the reduced camera matrix; null_space_rank must be 0")
        self.summary = CovarianceSummary(algorithm_type=self.options.algorithm_type,
                                         requested_null_space_rank=self.options.null_space_rank)
        self._problem = problem
        self._cov_c = None
        if not covariance_blocks:
            self._blocks = set()
            self.summary.success = True
            self.summary.message = "No covariance blocks requested."
            self.summary.ambient_dimension = problem.num_parameters()
            self.summary.tangent_dimension = problem.num_effective_parameters()
            return True
        ex = extract_bundle_adjustment(problem)
        if ex.cameras.device.type != "cuda":
            raise NotImplementedError("the covariance runs on CUDA tensors only")
        pairs = self._normalize(covariance_blocks)
        self._blocks = {(id(a), id(b)) for a, b in pairs} | {(id(b), id(a)) for a, b in pairs}
        self._where = {id(b): ("camera", i) for i, b in enumerate(ex.camera_blocks)}
        self._where.update({id(b): ("point", i) for i, b in enumerate(ex.point_blocks)})
        eng = BAEngine(ex.cameras, ex.points, ex.observations, ex.camera_index, ex.point_index,
                       loss=ex.loss if self.options.apply_loss_function else None,
                       camera_constant=ex.camera_constant, point_constant=ex.point_constant, precision="fp64")
        self._engine = eng
        self._point_index = ex.point_index.to(eng.device)
        self._F = {}
        nc, n_active = eng.nc, problem.num_effective_parameters()
        self.summary.num_requested_blocks = len(pairs)
        self.summary.num_computed_blocks = len(self._blocks)
        self.summary.ambient_dimension = problem.num_parameters()
        self.summary.tangent_dimension = n_active
        self.summary.num_rows = 2 * eng.no
        self.summary.num_columns = n_active
        # undamped point and camera assembly: radius +inf gives D = 0
        eng.evaluate(True)
        eng._call("ceres_b200_ba_point_assemble", math.inf, 0.0, 0.0, 0)
        eng._call("ceres_b200_ba_camera_assemble", math.inf, 0.0, 0.0, 0, _lib.PRECOND_IDENTITY)
        n = 9 * nc
        S = eng.schur_matrix()
        S0 = S.clone()
        inv = torch.empty_like(S)
        flags = torch.zeros(4, dtype=torch.int32, device=eng.device)
        if n:
            with torch.cuda.device(eng.device):
                _lib.check(eng.lib.ceres_b200_dense_spd_inverse(S.data_ptr(), inv.data_ptr(), ctypes.c_int64(n),
                                                                 flags.data_ptr(), eng._stream()),
                           "covariance inverse")
        not_pd = bool(int(flags[3]) & _lib.DEVERR_NOT_PD)
        winv = eng.winv[: eng.np].to(torch.float64)
        # a point block W_q that is singular (an unobserved or degenerate point) also
        # makes J rank deficient: its inverse comes out non-finite or zero
        free_pt = eng.pt_const[: eng.np] == 0
        pt_sing = bool((free_pt & (~torch.isfinite(winv).all(dim=1) | (winv[:, 0] <= 0))).any()) if eng.np else False
        if not_pd or pt_sing or not torch.isfinite(inv[:n, :n]).all():
            # the nullity of J^T J is that of S when every point block is positive
            # definite: eigenvalues of S below 1e-12 of the largest count as null
            null = 0
            if n:
                ev = torch.linalg.eigvalsh(S0[:n, :n])
                null = int((ev <= 1e-12 * ev.max().clamp_min(0)).sum())
            self.summary.rank = max(0, n_active - max(null, 1))
            self.summary.nullity = n_active - self.summary.rank
            self.summary.message = "Jacobian is rank deficient."
            return False
        cc = inv[:n, :n].clone()
        const = ex.camera_constant.to(eng.device)
        if bool(const.any()):
            mask = const.repeat_interleave(9)
            cc[mask, :] = 0.0
            cc[:, mask] = 0.0
        self._cov_c = cc
        self._winv = winv
        self.summary.rank = n_active
        self.summary.nullity = 0
        self.summary.success = True
        self.summary.message = "Computed covariance with the Schur complement."
        return True

    Compute = compute

    # ------------------------------------------------------------------ blocks
    def _point_terms(self, q: int):
        """(W_q^-1 [3, 3], F_q [3, 9 nc]) of original point q."""
        if q in self._F:
            return self._F[q]
        eng = self._engine
        L = eng.layout
        sorted_q = int(torch.nonzero(L.point_order == q)[0, 0])
        w = self._winv[sorted_q]
        W = torch.stack([torch.stack([w[0], w[1], w[2]]), torch.stack([w[1], w[3], w[4]]),
                         torch.stack([w[2], w[4], w[5]])])
        obs = torch.nonzero(self._point_index == q).flatten()
        slots = L.slot_of_obs[obs]
        J = eng.jac[slots].to(torch.float64)
        Jc = J[:, :18].reshape(-1, 2, 9)
        Jp = J[:, 18:].reshape(-1, 2, 3)
        cams = L.slot_cam[slots].long().tolist()
        F = torch.zeros((3, 9 * eng.nc), dtype=torch.float64, device=eng.device)
        blocks = torch.einsum("kri,krj->kij", Jp, Jc)  # [k, 3, 9]
        for k, c in enumerate(cams):
            F[:, 9 * c:9 * c + 9] += blocks[k]
        self._F[q] = (W, F)
        return self._F[q]

    def _tangent_block(self, a, b) -> torch.Tensor:
        if self._problem is None or self._cov_c is None:
            raise RuntimeError("Covariance.compute must be called first")
        pa, pb = self._require(a), self._require(b)
        if (id(pa), id(pb)) not in self._blocks:
            raise KeyError("Requested covariance block was not computed")
        ka, ia = self._where[id(pa)]
        kb, ib = self._where[id(pb)]
        if pa.constant or pb.constant:
            return torch.zeros((0 if pa.constant else pa.size, 0 if pb.constant else pb.size), dtype=torch.float64,
                               device=self._cov_c.device)
        C = self._cov_c
        if ka == "camera" and kb == "camera":
            return C[9 * ia:9 * ia + 9, 9 * ib:9 * ib + 9].clone()
        if ka == "point" and kb == "camera":
            return self._tangent_block(b, a).T.contiguous()
        if ka == "camera" and kb == "point":
            W, F = self._point_terms(ib)
            return -(C[9 * ia:9 * ia + 9, :] @ F.T) @ W
        Wa, Fa = self._point_terms(ia)
        Wb, Fb = self._point_terms(ib)
        out = Wa @ Fa @ C @ Fb.T @ Wb
        if ia == ib:
            out = out + Wa
        return out

    def get_covariance_block(self, a, b, out: torch.Tensor | None = None) -> torch.Tensor:
        pa, pb = self._require(a), self._require(b)
        blk = self._tangent_block(a, b)
        if blk.numel() == 0:
            blk = torch.zeros((pa.size, pb.size), dtype=torch.float64, device=blk.device)
        return _copy_to_output(blk, out)

    def get_covariance_block_in_tangent_space(self, a, b, out: torch.Tensor | None = None) -> torch.Tensor:
        return _copy_to_output(self._tangent_block(a, b), out)

    def get_covariance_matrix(self, parameter_blocks: Sequence, out: torch.Tensor | None = None) -> torch.Tensor:
        rows = [torch.cat([self.get_covariance_block(a, b) for b in parameter_blocks], dim=1) for a in parameter_blocks]
        return _copy_to_output(torch.cat(rows, dim=0), out)

    def get_covariance_matrix_in_tangent_space(self, parameter_blocks: Sequence,
                                               out: torch.Tensor | None = None) -> torch.Tensor:
        rows = [torch.cat([self.get_covariance_block_in_tangent_space(a, b) for b in parameter_blocks], dim=1)
                for a in parameter_blocks]
        return _copy_to_output(torch.cat(rows, dim=0), out)

    GetCovarianceBlock = get_covariance_block
    GetCovarianceBlockInTangentSpace = get_covariance_block_in_tangent_space
    GetCovarianceMatrix = get_covariance_matrix
    GetCovarianceMatrixInTangentSpace = get_covariance_matrix_in_tangent_space

    def has_covariance_block(self, a, b) -> bool:
        if self._problem is None:
            return False
        try:
            return (id(self._require(a)), id(self._require(b))) in self._blocks
        except KeyError:
            return False

    HasCovarianceBlock = has_covariance_block

    def rank(self) -> int:
        return self.summary.rank

    def nullity(self) -> int:
        return self.summary.nullity

    def reciprocal_condition_number(self) -> float:
        return self.summary.reciprocal_condition_number

    Rank = rank
    Nullity = nullity
    ReciprocalConditionNumber = reciprocal_condition_number

    # ------------------------------------------------------------------ helpers
    def _require(self, value):
        """The problem's parameter block for ``value`` (a block or its tensor)."""
        for b in self._problem.parameter_blocks:
            if b is value or getattr(b, "tensor", None) is value:
                return b
        raise KeyError("parameter block is not part of the problem")

    def _normalize(self, covariance_blocks) -> list:
        first = covariance_blocks[0]
        if isinstance(first, tuple):
            pairs = [(self._require(a), self._require(b)) for a, b in covariance_blocks]
            seen = set()
            for a, b in pairs:
                key = frozenset((id(a), id(b)))
                if key in seen:
                    raise ValueError("covariance_blocks cannot contain duplicate block pairs")
                seen.add(key)
            return pairs
        params = [self._require(p) for p in covariance_blocks]
        if len({id(p) for p in params}) != len(params):
            raise ValueError("parameter_blocks cannot contain duplicates")
        return [(a, b) for a in params for b in params]


def _copy_to_output(value: torch.Tensor, out: torch.Tensor | None) -> torch.Tensor:
    if out is None:
        return value
    if out.numel() != value.numel():
        raise ValueError("Output tensor has the wrong number of elements")
    out.reshape(-1).copy_(value.reshape(-1).to(dtype=out.dtype, device=out.device))
    return out


__all__ = ["Covariance", "CovarianceOptions", "CovarianceSummary"]
