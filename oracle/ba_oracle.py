"""CPU oracle: a float64 numpy restatement of ceres-torch's Schur bundle-adjustment path.

TEST INFRASTRUCTURE ONLY. This module is the checker that the CUDA path is
compared against; the product never imports it. Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm may
load it.

What it restates, function by function (reference paths are relative to the
ceres-torch project root):

* ``angle_axis_rotate_point``   rotation.py:104-110 (angle-axis -> quaternion, with the
  theta<=eps branch k = 0.5 - theta^2/48), rotation.py:68-69 (normalize), rotation.py:211-214
  (unit-quaternion rotate) and rotation.py:221-222.
* ``snavely_residuals``         examples/simple_bundle_adjuster.py:73-79 (and the residual
  ``snavely_reprojection(camera, point) - observation`` built at :105).
* Jacobians                     costs.py:31-44 differentiates that formula with autograd; the
  oracle carries forward-mode tangents through the same operation sequence (``_Dual``), so it is
  the same derivative, including the quaternion normalisation.
* ``LOSSES``                    losses.py:21-133 (Trivial, Huber, SoftLOne, Cauchy, Arctan,
  Tolerant, Tukey, Scaled, Composed).
* ``robustify``                 losses.py:158-193 (Ceres corrector: sqrt(rho') scaling, Triggs
  rank-1 term only when s>0 and rho''>0).
* ``evaluate``                  problem.py:377-413 / :486-520 (cost = sum 0.5 rho, corrected
  residuals and Jacobian, gradient J^T r).
* ``jacobi_damping``            linear.py:539-551.
* Schur system                  linear.py:794-839 (H = J^T J + diag(d), S = Hbb - Hba Haa^-1 Hab,
  rhs = gb - Hba Haa^-1 ga) written block-sparsely: Haa is block diagonal (3x3 per point) in BA.
* ``schur_solve_dense``         linear.py:667-699 (exact solve of S).
* ``iterative_schur``           linear.py:702-776 with the PCG of linear.py:1216-1256 and the
  preconditioners of linear.py:462-536 / :1156-1182 (SCHUR_JACOBI = Cholesky of each retained
  block of S; JACOBI = clamped diagonal; IDENTITY; SCHUR_POWER_SERIES_EXPANSION = the series
  of linear.py:59-67 on the SCHUR_JACOBI factors of Hbb, linear.py:482-497) and the SPSE initial
  point of linear.py:745-756.
* cluster preconditioners      linear.py:498-521 and :1032-1085 (S kept on the visibility cluster
  block pairs, Cholesky, the halved retry of CLUSTER_TRIDIAGONAL, the general-solve fallback of
  :1366-1370), with the clustering of linear.py:842-1028 (visibility graph, SINGLE_LINKAGE,
  CANONICAL_VIEWS, cluster graph, degree-2 maximum spanning forest) restated loop for loop.
* ``solve``                     solver.py:35-357 (trust-region LM), with :798-802 (model
  decrease), :805-820 (LM radius), :823-861 (step evaluator), :1165-1175 (convergence tests),
  :661-676 (restore best state), :714-785 (parameter order, num_eliminate, visibility).

Parity of this restatement is pinned against the reference itself by
``tests/golden/make_golden.py`` (fixtures generated by running ceres-torch) and
``tests/test_oracle_golden.py``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

EPS64 = float(np.finfo(np.float64).eps)
TINY64 = float(np.finfo(np.float64).tiny)


# --------------------------------------------------------------------------------------
# Forward-mode tangents
# --------------------------------------------------------------------------------------
class _Dual:
    """Value ``v`` [n] with tangents ``d`` [n, k]; just enough algebra for the projection."""

    __slots__ = ("v", "d")

    def __init__(self, v, d):
        self.v = v
        self.d = d

    def __add__(self, o):
        if isinstance(o, _Dual):
            return _Dual(self.v + o.v, self.d + o.d)
        return _Dual(self.v + o, self.d)

    __radd__ = __add__

    def __sub__(self, o):
        if isinstance(o, _Dual):
            return _Dual(self.v - o.v, self.d - o.d)
        return _Dual(self.v - o, self.d)

    def __rsub__(self, o):
        return _Dual(o - self.v, -self.d)

    def __neg__(self):
        return _Dual(-self.v, -self.d)

    def __mul__(self, o):
        if isinstance(o, _Dual):
            return _Dual(self.v * o.v, self.d * o.v[:, None] + o.d * self.v[:, None])
        return _Dual(self.v * o, self.d * o)

    __rmul__ = __mul__

    def __truediv__(self, o):
        if isinstance(o, _Dual):
            q = self.v / o.v
            return _Dual(q, (self.d - o.d * q[:, None]) / o.v[:, None])
        return _Dual(self.v / o, self.d / o)


def _dsqrt(a: _Dual) -> _Dual:
    v = np.sqrt(a.v)
    safe = np.where(v > 0.0, 2.0 * v, 1.0)
    d = np.where((v > 0.0)[:, None], a.d / safe[:, None], 0.0)
    return _Dual(v, d)


def _dsin(a: _Dual) -> _Dual:
    return _Dual(np.sin(a.v), a.d * np.cos(a.v)[:, None])


def _dcos(a: _Dual) -> _Dual:
    return _Dual(np.cos(a.v), -a.d * np.sin(a.v)[:, None])


def _dwhere(mask, a: _Dual, b: _Dual) -> _Dual:
    return _Dual(np.where(mask, a.v, b.v), np.where(mask[:, None], a.d, b.d))


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _snavely(cam: list, X: list, with_tangents: bool):
    """rotation.py:104-110,68-69,211-214 + simple_bundle_adjuster.py:73-79, one op at a time."""
    aa = cam[0:3]
    theta = _dsqrt(aa[0] * aa[0] + aa[1] * aa[1] + aa[2] * aa[2])  # torch.linalg.norm
    half = theta * 0.5
    small = theta.v <= EPS64
    one = _Dual(np.ones_like(theta.v), np.zeros_like(theta.d))
    safe_theta = _dwhere(small, one, theta)
    k = _dwhere(small, 0.5 - theta * theta / 48.0, _dsin(half) / safe_theta)
    q = [_dcos(half), k * aa[0], k * aa[1], k * aa[2]]
    qn = _dsqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    qn = _dwhere(qn.v < TINY64, _Dual(np.full_like(qn.v, TINY64), np.zeros_like(qn.d)), qn)
    q = [c / qn for c in q]
    u = q[1:4]
    c1 = _cross(u, X)
    uv = [c * 2.0 for c in c1]
    c2 = _cross(u, uv)
    rp = [X[i] + q[0] * uv[i] + c2[i] for i in range(3)]
    p = [rp[i] + cam[3 + i] for i in range(3)]
    xp = -p[0] / p[2]
    yp = -p[1] / p[2]
    r2 = xp * xp + yp * yp
    distortion = 1.0 + r2 * (cam[7] + cam[8] * r2)
    fd = cam[6] * distortion
    return fd * xp, fd * yp


def snavely_residuals_and_jacobians(cameras, points, obs, ci, pi, *, jacobians=True):
    """Raw (uncorrected) residuals [no,2] and Jacobians Jc [no,2,9], Jp [no,2,3]."""
    cam = cameras[ci]
    X = points[pi]
    n = cam.shape[0]
    k = 12 if jacobians else 0
    eye = np.eye(12)
    cd = [_Dual(cam[:, j].copy(), np.broadcast_to(eye[j, :k], (n, k)).copy()) for j in range(9)]
    xd = [_Dual(X[:, j].copy(), np.broadcast_to(eye[9 + j, :k], (n, k)).copy()) for j in range(3)]
    u, v = _snavely(cd, xd, jacobians)
    r = np.stack([u.v - obs[:, 0], v.v - obs[:, 1]], axis=1)
    if not jacobians:
        return r, None, None
    J = np.stack([u.d, v.d], axis=1)  # [n, 2, 12]
    return r, np.ascontiguousarray(J[:, :, :9]), np.ascontiguousarray(J[:, :, 9:])


def angle_axis_rotate_point(aa: np.ndarray, X: np.ndarray) -> np.ndarray:
    """rotation.py:221-222 for row-aligned arrays."""
    n = aa.shape[0]
    z = np.zeros((n, 0))
    aad = [_Dual(aa[:, j].copy(), z) for j in range(3)]
    theta = _dsqrt(aad[0] * aad[0] + aad[1] * aad[1] + aad[2] * aad[2])
    half = theta * 0.5
    small = theta.v <= EPS64
    safe = np.where(small, 1.0, theta.v)
    kk = np.where(small, 0.5 - theta.v * theta.v / 48.0, np.sin(half.v) / safe)
    q = np.stack([np.cos(half.v), kk * aa[:, 0], kk * aa[:, 1], kk * aa[:, 2]], axis=1)
    q = q / np.maximum(np.linalg.norm(q, axis=1, keepdims=True), TINY64)
    u = q[:, 1:]
    uv = 2.0 * np.cross(u, X)
    return X + q[:, :1] * uv + np.cross(u, uv)


# --------------------------------------------------------------------------------------
# Losses (losses.py:21-133) and the corrector (losses.py:158-193)
# --------------------------------------------------------------------------------------
def loss_rho(spec: tuple, s: np.ndarray):
    """Returns (rho0, rho1, rho2) for a loss spec tuple, elementwise over ``s``."""
    kind = spec[0]
    if kind == "trivial":
        return s.copy(), np.ones_like(s), np.zeros_like(s)
    if kind == "huber":
        a = float(spec[1])
        b = a * a
        mask = s <= b
        sq = np.sqrt(np.maximum(s, TINY64))
        with np.errstate(divide="ignore", invalid="ignore"):
            rho0 = np.where(mask, s, 2.0 * a * sq - b)
            rho1 = np.where(mask, 1.0, a / sq)
            rho2 = np.where(mask, 0.0, -0.5 * a / (sq * s))
        return rho0, rho1, rho2
    if kind == "softlone":
        b = float(spec[1]) ** 2
        z = 1.0 + s / b
        sz = np.sqrt(z)
        return 2.0 * b * (sz - 1.0), 1.0 / sz, -0.5 / (b * z * sz)
    if kind == "cauchy":
        b = float(spec[1]) ** 2
        z = 1.0 + s / b
        return b * np.log(z), 1.0 / z, -1.0 / (b * z * z)
    if kind == "arctan":
        a = float(spec[1])
        z = s / a
        den = 1.0 + z * z
        return a * np.arctan(z), 1.0 / den, -2.0 * z / (a * den * den)
    if kind == "tolerant":
        a, b = float(spec[1]), float(spec[2])
        z = (s - a) / b
        c = b * np.logaddexp(0.0, -a / b)
        rho1 = 1.0 / (1.0 + np.exp(-z))
        return b * np.logaddexp(0.0, z) - c, rho1, rho1 * (1.0 - rho1) / b
    if kind == "tukey":
        a2 = float(spec[1]) ** 2
        z = s / a2
        inner = 1.0 - z
        mask = s <= a2
        return (np.where(mask, (a2 / 3.0) * (1.0 - inner ** 3), a2 / 3.0),
                np.where(mask, inner ** 2, 0.0),
                np.where(mask, -2.0 * inner / a2, 0.0))
    if kind == "scaled":
        base = spec[1] if spec[1] is not None else ("trivial",)
        r0, r1, r2 = loss_rho(base, s)
        sc = float(spec[2])
        return sc * r0, sc * r1, sc * r2
    if kind == "composed":
        g0, g1, g2 = loss_rho(spec[2], s)
        f0, f1, f2 = loss_rho(spec[1], g0)
        return f0, f1 * g1, f2 * g1 * g1 + f1 * g2
    raise ValueError(f"unknown loss {spec!r}")


def robustify(spec, r, Jc=None, Jp=None):
    """losses.py:158-193 per residual block of size 2. Returns (cost_i, r', Jc', Jp')."""
    s = np.sum(r * r, axis=1)
    rho0, rho1, rho2 = loss_rho(spec, s)
    sqrt_rho1 = np.sqrt(np.maximum(rho1, 0.0))
    scale = sqrt_rho1.copy()
    alpha_s = np.zeros_like(s)
    corr = (s > 0.0) & (rho2 > 0.0)
    if np.any(corr):
        if np.any(rho1[corr] <= 0.0):
            raise ValueError("Loss function has rho'' > 0 but rho' <= 0")
        disc = 1.0 + 2.0 * s[corr] * rho2[corr] / rho1[corr]
        alpha = 1.0 - np.sqrt(disc)
        scale[corr] = sqrt_rho1[corr] / (1.0 - alpha)
        alpha_s[corr] = alpha / s[corr]
    r2 = scale[:, None] * r
    if Jc is None:
        return 0.5 * rho0, r2, None, None
    out = []
    for J in (Jc, Jp):
        rTj = np.einsum("ni,nij->nj", r, J)
        Jn = sqrt_rho1[:, None, None] * (J - alpha_s[:, None, None] * r[:, :, None] * rTj[:, None, :])
        out.append(Jn)
    return 0.5 * rho0, r2, out[0], out[1]


# --------------------------------------------------------------------------------------
# Problem structure
# --------------------------------------------------------------------------------------
@dataclass
class OracleProblem:
    cameras: np.ndarray
    points: np.ndarray
    observations: np.ndarray
    camera_index: np.ndarray
    point_index: np.ndarray
    loss: tuple = ("trivial",)
    camera_constant: np.ndarray | None = None
    point_constant: np.ndarray | None = None

    def __post_init__(self):
        self.cameras = np.array(self.cameras, dtype=np.float64)
        self.points = np.array(self.points, dtype=np.float64)
        self.observations = np.asarray(self.observations, dtype=np.float64)
        self.camera_index = np.asarray(self.camera_index, dtype=np.int64)
        self.point_index = np.asarray(self.point_index, dtype=np.int64)
        nc, npt = self.cameras.shape[0], self.points.shape[0]
        if self.camera_constant is None:
            self.camera_constant = np.zeros(nc, dtype=bool)
        if self.point_constant is None:
            self.point_constant = np.zeros(npt, dtype=bool)
        self.active_cams = np.flatnonzero(~self.camera_constant)
        self.active_pts = np.flatnonzero(~self.point_constant)
        self.cam_col = np.full(nc, -1, dtype=np.int64)
        self.cam_col[self.active_cams] = np.arange(self.active_cams.size)
        self.pt_col = np.full(npt, -1, dtype=np.int64)
        self.pt_col[self.active_pts] = np.arange(self.active_pts.size)


@dataclass
class Evaluation:
    cost: float
    r: np.ndarray
    Jc: np.ndarray | None = None
    Jp: np.ndarray | None = None


def evaluate(prob: OracleProblem, cameras, points, *, jacobians=True) -> Evaluation:
    """problem.py:377-413: cost = sum_i 0.5 rho_i; corrected residuals and Jacobians."""
    r, Jc, Jp = snavely_residuals_and_jacobians(cameras, points, prob.observations, prob.camera_index,
                                                 prob.point_index, jacobians=jacobians)
    cost_i, r2, Jc2, Jp2 = robustify(prob.loss, r, Jc, Jp)
    if jacobians:
        Jc2 = Jc2 * (~prob.camera_constant[prob.camera_index])[:, None, None]
        Jp2 = Jp2 * (~prob.point_constant[prob.point_index])[:, None, None]
    return Evaluation(float(np.sum(cost_i)), r2, Jc2, Jp2)


def jacobi_damping(col_sq: np.ndarray, radius: float, min_diag: float, max_diag: float, jacobi_scaling=True):
    """linear.py:539-551."""
    diag = col_sq if jacobi_scaling else np.ones_like(col_sq)
    return np.clip(diag, min_diag, max_diag) / max(radius, EPS64)


def _segment_sum(values: np.ndarray, keys: np.ndarray, n: int) -> np.ndarray:
    out = np.zeros((n,) + values.shape[1:])
    np.add.at(out, keys, values)
    return out


@dataclass
class SchurSystem:
    """Block-sparse pieces of linear.py:794-839 for BA (points eliminated)."""

    Winv: np.ndarray        # [np_a, 3, 3]  Haa^-1 blocks
    Fi: np.ndarray          # [no, 3, 9]    Jp_i^T Jc_i (Hab row blocks per observation)
    U: np.ndarray           # [nc_a, 9, 9]  Hbb diagonal blocks (incl. damping)
    ga: np.ndarray          # [np_a, 3]
    gb: np.ndarray          # [nc_a, 9]
    Winv_ga: np.ndarray     # [np_a, 3]
    rhs: np.ndarray         # [nc_a, 9]
    pt: np.ndarray          # [no] active point column per obs (-1 constant)
    cam: np.ndarray         # [no] active camera column per obs (-1 constant)
    n_cam: int
    n_pt: int


def build_schur(prob: OracleProblem, ev: Evaluation, damping_p: np.ndarray, damping_c: np.ndarray) -> SchurSystem:
    pt = prob.pt_col[prob.point_index]
    cam = prob.cam_col[prob.camera_index]
    n_pt, n_cam = prob.active_pts.size, prob.active_cams.size
    b = -ev.r
    vp = pt >= 0
    vc = cam >= 0
    W = _segment_sum(np.einsum("nri,nrj->nij", ev.Jp[vp], ev.Jp[vp]), pt[vp], n_pt)
    W[:, [0, 1, 2], [0, 1, 2]] += damping_p.reshape(n_pt, 3)
    U = _segment_sum(np.einsum("nri,nrj->nij", ev.Jc[vc], ev.Jc[vc]), cam[vc], n_cam)
    U[:, np.arange(9), np.arange(9)] += damping_c.reshape(n_cam, 9)
    ga = _segment_sum(np.einsum("nri,nr->ni", ev.Jp[vp], b[vp]), pt[vp], n_pt)
    gb = _segment_sum(np.einsum("nri,nr->ni", ev.Jc[vc], b[vc]), cam[vc], n_cam)
    Winv = np.linalg.inv(W) if n_pt else np.zeros((0, 3, 3))
    Winv_ga = np.einsum("nij,nj->ni", Winv, ga)
    Fi = np.einsum("nri,nrj->nij", ev.Jp, ev.Jc)
    both = vp & vc
    contrib = np.einsum("nij,ni->nj", Fi[both], Winv_ga[pt[both]])
    rhs = gb - _segment_sum(contrib, cam[both], n_cam)
    return SchurSystem(Winv, Fi, U, ga, gb, Winv_ga, rhs, pt, cam, n_cam, n_pt)


def schur_matvec(sys: SchurSystem, x: np.ndarray) -> np.ndarray:
    """S x = Hbb x - Hba Haa^-1 Hab x, streamed per observation (x: [nc_a, 9])."""
    y = np.einsum("nij,nj->ni", sys.U, x)
    both = (sys.pt >= 0) & (sys.cam >= 0)
    pt, cam, F = sys.pt[both], sys.cam[both], sys.Fi[both]
    t = _segment_sum(np.einsum("nij,nj->ni", F, x[cam]), pt, sys.n_pt)
    s = np.einsum("nij,nj->ni", sys.Winv, t)
    y -= _segment_sum(np.einsum("nij,ni->nj", F, s[pt]), cam, sys.n_cam)
    return y


def schur_eliminated_matvec(sys: SchurSystem, x: np.ndarray) -> np.ndarray:
    """E x = Hba Haa^-1 Hab x (the term S subtracts from Hbb; linear.py:809), x: [nc_a, 9]."""
    both = (sys.pt >= 0) & (sys.cam >= 0)
    pt, cam, F = sys.pt[both], sys.cam[both], sys.Fi[both]
    t = _segment_sum(np.einsum("nij,nj->ni", F, x[cam]), pt, sys.n_pt)
    s = np.einsum("nij,nj->ni", sys.Winv, t)
    return _segment_sum(np.einsum("nij,ni->nj", F, s[pt]), cam, sys.n_cam)


def schur_dense(sys: SchurSystem) -> np.ndarray:
    """Explicit S [9 nc_a, 9 nc_a] (small problems only)."""
    n = sys.n_cam
    S = np.zeros((n, 9, n, 9))
    S[np.arange(n), :, np.arange(n), :] = sys.U
    both = (sys.pt >= 0) & (sys.cam >= 0)
    idx = np.flatnonzero(both)
    order = idx[np.argsort(sys.pt[idx], kind="stable")]
    pts = sys.pt[order]
    bounds = np.flatnonzero(np.diff(pts)) + 1
    for grp in np.split(order, bounds):
        if grp.size == 0:
            continue
        p = sys.pt[grp[0]]
        G = sys.Fi[grp]                              # [L, 3, 9]
        WG = np.einsum("ij,ljk->lik", sys.Winv[p], G)  # [L, 3, 9]
        blk = np.einsum("lia,mib->lamb", G, WG)      # [L, 9, L, 9]
        cams = sys.cam[grp]
        for a in range(grp.size):
            for b_ in range(grp.size):
                S[cams[a], :, cams[b_], :] -= blk[a, :, b_, :]
    return S.reshape(9 * n, 9 * n)


def schur_diag_blocks(sys: SchurSystem) -> np.ndarray:
    """Retained 9x9 diagonal blocks of S (the SCHUR_JACOBI blocks), duplicates of a
    camera inside one track summed before the W^-1 product."""
    both = (sys.pt >= 0) & (sys.cam >= 0)
    idx = np.flatnonzero(both)
    key = sys.pt[idx] * max(sys.n_cam, 1) + sys.cam[idx]
    uk, inv = np.unique(key, return_inverse=True)
    G = _segment_sum(sys.Fi[idx], inv, uk.size)       # [groups, 3, 9]
    gp = uk // max(sys.n_cam, 1)
    gc = uk % max(sys.n_cam, 1)
    blk = np.einsum("gia,gij,gjb->gab", G, sys.Winv[gp], G)
    D = sys.U.copy()
    np.subtract.at(D, gc, blk)
    return D


class _Preconditioner:
    """linear.py:462-536 / :1156-1182 / :53-79 for the retained camera blocks."""

    def __init__(self, kind: str, diag_blocks: np.ndarray):
        self.kind = kind
        if kind == "IDENTITY":
            return
        if kind == "SCHUR_JACOBI":
            self.factors = []
            for blk in diag_blocks:
                try:
                    self.factors.append((np.linalg.cholesky(blk), True))
                except np.linalg.LinAlgError:
                    self.factors.append((blk, False))
            return
        # JACOBI and the other diagonal fallbacks: 1 / clamp(diag(S), eps)
        d = np.einsum("nii->ni", diag_blocks)
        self.dinv = 1.0 / np.maximum(d, EPS64)

    def apply(self, r: np.ndarray) -> np.ndarray:
        if self.kind == "IDENTITY":
            return r.copy()
        if self.kind == "SCHUR_JACOBI":
            z = np.empty_like(r)
            for c, (f, chol) in enumerate(self.factors):
                if chol:
                    y = np.linalg.solve(f, r[c])
                    z[c] = np.linalg.solve(f.T, y)
                else:
                    try:
                        z[c] = np.linalg.solve(f, r[c])
                    except np.linalg.LinAlgError:
                        z[c] = np.linalg.lstsq(f, r[c], rcond=None)[0]
            return z
        return self.dinv * r


class _ClusterPreconditioner:
    """linear.py:1032-1085 and :53-59: S kept on the cluster block pairs, Cholesky-
    factored; CLUSTER_TRIDIAGONAL whose kept matrix is not positive definite halves the
    blocks between different clusters and tries again; a matrix that still fails is
    solved as a general square system (linear.py:1366-1370)."""

    def __init__(self, S: np.ndarray, st: "OracleClusterStructure", tridiagonal: bool):
        n = S.shape[0] // 9
        member = np.asarray(st.membership)
        keep = np.zeros((n, n), dtype=bool)
        for a, b in st.block_pairs:
            keep[a, b] = keep[b, a] = True
        mask = np.kron(keep, np.ones((9, 9), dtype=bool))
        M = np.where(mask, S, 0.0)
        self.factor, self.chol = self._factor(M)
        if not self.chol and tridiagonal:
            cross = np.kron(keep & (member[:, None] != member[None, :]), np.ones((9, 9), dtype=bool))
            scaled = np.where(cross, 0.5 * M, M)
            f, ok = self._factor(scaled)
            self.factor, self.chol = (f, True) if ok else (scaled, False)

    @staticmethod
    def _factor(M):
        try:
            return np.linalg.cholesky(M), True
        except np.linalg.LinAlgError:
            return M, False

    def apply(self, r: np.ndarray) -> np.ndarray:
        v = r.reshape(-1)
        if self.chol:
            y = np.linalg.solve(self.factor, v)
            return np.linalg.solve(self.factor.T, y).reshape(r.shape)
        try:
            return np.linalg.solve(self.factor, v).reshape(r.shape)
        except np.linalg.LinAlgError:
            return np.linalg.lstsq(self.factor, v, rcond=None)[0].reshape(r.shape)


class _PowerSeries:
    """SCHUR_POWER_SERIES_EXPANSION (linear.py:482-497, applied at :59-67):
    z = sum_i (B E)^i B r with B the SCHUR_JACOBI factors of the damped Hbb blocks and
    E = Hba Haa^-1 Hab; term i >= 1 is added while its norm is above
    tolerance * max(|partial sum|, 1), at most ``max_terms`` terms in all."""

    kind = "SCHUR_POWER_SERIES_EXPANSION"

    def __init__(self, sys: SchurSystem, max_terms: int, tolerance: float):
        self.base = _Preconditioner("SCHUR_JACOBI", sys.U)
        self.sys = sys
        self.max_terms = max_terms
        self.tolerance = tolerance

    def apply(self, r: np.ndarray) -> np.ndarray:
        result = self.base.apply(r)
        term = result
        for _ in range(max(0, self.max_terms - 1)):
            term = self.base.apply(schur_eliminated_matvec(self.sys, term))
            if np.linalg.norm(term) <= self.tolerance * max(float(np.linalg.norm(result)), 1.0):
                break
            result = result + term
        return result


def pcg(matvec, rhs: np.ndarray, prec, *, min_iterations=0, max_iterations=500,
        tolerance=0.1, eps=EPS64, initial_x: np.ndarray | None = None):
    """linear.py:1216-1256."""
    x = np.zeros_like(rhs) if initial_x is None else initial_x.copy()
    r = rhs.copy() if initial_x is None else rhs - matvec(x)
    z = prec.apply(r)
    p = z.copy()
    rz_old = float(np.sum(r * z))
    rhs_norm = max(float(np.linalg.norm(rhs)), eps)
    if min_iterations <= 0 and np.linalg.norm(r) <= tolerance * rhs_norm:
        return x, 0, True
    iterations = 0
    success = False
    for k in range(max_iterations):
        Ap = matvec(p)
        denom = float(np.sum(p * Ap))
        if abs(denom) <= eps:
            success = bool(np.linalg.norm(r) <= tolerance * rhs_norm)
            break
        alpha = rz_old / denom
        x = x + alpha * p
        r = r - alpha * Ap
        iterations = k + 1
        if iterations >= min_iterations and np.linalg.norm(r) <= tolerance * rhs_norm:
            success = True
            break
        z = prec.apply(r)
        rz_new = float(np.sum(r * z))
        if abs(rz_old) <= eps:
            break
        beta = rz_new / rz_old
        p = z + beta * p
        rz_old = rz_new
    return x, iterations, success


def back_substitute(sys: SchurSystem, xb: np.ndarray) -> np.ndarray:
    """xa = Haa^-1 ga - Haa^-1 Hab xb (linear.py:698 / :766)."""
    both = (sys.pt >= 0) & (sys.cam >= 0)
    t = _segment_sum(np.einsum("nij,nj->ni", sys.Fi[both], xb[sys.cam[both]]), sys.pt[both], sys.n_pt)
    return sys.Winv_ga - np.einsum("nij,nj->ni", sys.Winv, t)


def solve_step(prob, ev, radius, opts, *, explicit_limit=1800):
    """Damping (solver.py:135-141) + the Schur linear solve for one LM iteration.

    Returns (step_points [np_a,3], step_cams [nc_a,9], linear iterations)."""
    pt = prob.pt_col[prob.point_index]
    cam = prob.cam_col[prob.camera_index]
    col_p = _segment_sum(np.sum(ev.Jp[pt >= 0] ** 2, axis=1), pt[pt >= 0], prob.active_pts.size)
    col_c = _segment_sum(np.sum(ev.Jc[cam >= 0] ** 2, axis=1), cam[cam >= 0], prob.active_cams.size)
    dp = jacobi_damping(col_p, radius, opts.min_lm_diagonal, opts.max_lm_diagonal, opts.jacobi_scaling)
    dc = jacobi_damping(col_c, radius, opts.min_lm_diagonal, opts.max_lm_diagonal, opts.jacobi_scaling)
    sys = build_schur(prob, ev, dp, dc)
    if sys.n_cam == 0:
        return sys.Winv_ga, np.zeros((0, 9)), 1
    if opts.linear_solver_type in ("DENSE_SCHUR", "SPARSE_SCHUR"):
        S = schur_dense(sys)
        try:
            xb = np.linalg.solve(S, sys.rhs.reshape(-1))
        except np.linalg.LinAlgError:
            xb = np.linalg.lstsq(S, sys.rhs.reshape(-1), rcond=None)[0]
        xb = xb.reshape(-1, 9)
        its = 1
    else:
        if 9 * sys.n_cam <= explicit_limit:
            S = schur_dense(sys)
            mv = lambda v: (S @ v.reshape(-1)).reshape(-1, 9)  # noqa: E731
        else:
            mv = lambda v: schur_matvec(sys, v)  # noqa: E731
        if opts.preconditioner_type == "SCHUR_POWER_SERIES_EXPANSION":
            prec = _PowerSeries(sys, opts.max_num_spse_iterations, opts.spse_tolerance)
        elif (opts.preconditioner_type in ("CLUSTER_JACOBI", "CLUSTER_TRIDIAGONAL") and sys.n_cam > 1
              and schur_visibility(prob) is not None):
            # linear.py:498-521: the visibility clusters of the retained (camera) blocks
            st = cluster_structure(schur_visibility(prob), tridiagonal=opts.preconditioner_type == "CLUSTER_TRIDIAGONAL",
                                   clustering=opts.visibility_clustering_type)
            prec = _ClusterPreconditioner(schur_dense(sys), st, opts.preconditioner_type == "CLUSTER_TRIDIAGONAL")
        else:
            prec = _Preconditioner(opts.preconditioner_type, schur_diag_blocks(sys))
        x0 = None
        if opts.use_spse_initialization:
            x0 = _PowerSeries(sys, opts.max_num_spse_iterations, opts.spse_tolerance).apply(sys.rhs)
        xb, its, _ = pcg(mv, sys.rhs, prec, min_iterations=opts.min_linear_solver_iterations,
                         max_iterations=opts.max_linear_solver_iterations, tolerance=opts.eta, initial_x=x0)
    xa = back_substitute(sys, xb)
    return xa, xb, its


# --------------------------------------------------------------------------------------
# LM driver (solver.py:35-357)
# --------------------------------------------------------------------------------------
@dataclass
class OracleOptions:
    linear_solver_type: str = "ITERATIVE_SCHUR"
    preconditioner_type: str = "SCHUR_JACOBI"
    max_num_iterations: int = 50
    initial_trust_region_radius: float = 1e4
    max_trust_region_radius: float = 1e16
    min_trust_region_radius: float = 1e-32
    min_relative_decrease: float = 1e-3
    min_lm_diagonal: float = 1e-6
    max_lm_diagonal: float = 1e32
    max_num_consecutive_invalid_steps: int = 5
    function_tolerance: float = 1e-6
    gradient_tolerance: float = 1e-10
    parameter_tolerance: float = 1e-8
    min_linear_solver_iterations: int = 0
    max_linear_solver_iterations: int = 500
    eta: float = 0.1
    jacobi_scaling: bool = True
    use_nonmonotonic_steps: bool = False
    max_consecutive_nonmonotonic_steps: int = 5
    explicit_schur_limit: int = 1800  # PCG on an explicit S up to this many camera columns
    max_num_spse_iterations: int = 5
    spse_tolerance: float = 0.1
    use_spse_initialization: bool = False
    visibility_clustering_type: str = "CANONICAL_VIEWS"


@dataclass
class OracleIteration:
    iteration: int
    cost: float
    cost_change: float = 0.0
    gradient_max_norm: float = 0.0
    gradient_norm: float = 0.0
    step_norm: float = 0.0
    relative_decrease: float = 0.0
    trust_region_radius: float = 0.0
    linear_solver_iterations: int = 0
    step_is_valid: bool = True
    step_is_successful: bool = True


@dataclass
class OracleResult:
    initial_cost: float
    final_cost: float
    termination: str
    message: str
    iterations: list = field(default_factory=list)
    cameras: np.ndarray | None = None
    points: np.ndarray | None = None
    num_successful_steps: int = 0
    num_unsuccessful_steps: int = 0


class StepEvaluator:
    """solver.py:823-861."""

    def __init__(self, initial_cost, max_nonmono):
        self.max_nonmono = max(0, int(max_nonmono))
        self.minimum_cost = self.current_cost = self.reference_cost = self.candidate_cost = initial_cost
        self.acc_ref = 0.0
        self.acc_cand = 0.0
        self.n_nonmono = 0

    def step_quality(self, cost, model_change):
        if model_change <= 0.0:
            return float("-inf")
        rel = (self.current_cost - cost) / model_change
        hist = (self.reference_cost - cost) / (self.acc_ref + model_change)
        return max(rel, hist)

    def step_accepted(self, cost, model_change):
        self.current_cost = cost
        self.acc_cand += model_change
        self.acc_ref += model_change
        if self.current_cost < self.minimum_cost:
            self.minimum_cost = self.current_cost
            self.n_nonmono = 0
            self.candidate_cost = self.current_cost
            self.acc_cand = 0.0
        else:
            self.n_nonmono += 1
            if self.current_cost > self.candidate_cost:
                self.candidate_cost = self.current_cost
                self.acc_cand = 0.0
        if self.n_nonmono == self.max_nonmono:
            self.reference_cost = self.candidate_cost
            self.acc_ref = self.acc_cand


def _gradient(prob, ev):
    pt = prob.pt_col[prob.point_index]
    cam = prob.cam_col[prob.camera_index]
    gp = _segment_sum(np.einsum("nri,nr->ni", ev.Jp[pt >= 0], ev.r[pt >= 0]), pt[pt >= 0], prob.active_pts.size)
    gc = _segment_sum(np.einsum("nri,nr->ni", ev.Jc[cam >= 0], ev.r[cam >= 0]), cam[cam >= 0], prob.active_cams.size)
    return np.concatenate([gp.reshape(-1), gc.reshape(-1)])


def solve(prob: OracleProblem, opts: OracleOptions | None = None) -> OracleResult:
    """solver.py:35-357 for the LM strategy, no bounds, no inner iterations."""
    opts = opts or OracleOptions()
    cams = prob.cameras.copy()
    pts = prob.points.copy()
    radius = opts.initial_trust_region_radius
    decrease_factor = 2.0
    consecutive_invalid = 0
    previous_cost = None
    ev = evaluate(prob, cams, pts)
    res = OracleResult(ev.cost, ev.cost, "FAILURE", "")
    best_cost = ev.cost
    best = (cams.copy(), pts.copy())
    se = StepEvaluator(ev.cost, opts.max_consecutive_nonmonotonic_steps if opts.use_nonmonotonic_steps else 0)
    if prob.active_pts.size + prob.active_cams.size == 0:
        res.termination, res.message = "CONVERGENCE", "No active parameters."
        res.cameras, res.points = cams, pts
        return res
    ncols = 3 * prob.active_pts.size + 9 * prob.active_cams.size
    terminated = False
    for iteration in range(opts.max_num_iterations + 1):
        cost = ev.cost
        g = _gradient(prob, ev)
        gmax = float(np.max(np.abs(g))) if g.size else 0.0
        it = OracleIteration(iteration, cost, gradient_max_norm=gmax, gradient_norm=float(np.linalg.norm(g)),
                             trust_region_radius=radius)
        if iteration == 0:
            res.iterations.append(it)
            if gmax <= opts.gradient_tolerance:
                res.termination, res.message = "CONVERGENCE", "Gradient tolerance reached."
                res.final_cost = cost
                terminated = True
                break
            if opts.max_num_iterations == 0:
                res.termination, res.message = "NO_CONVERGENCE", "Maximum iterations reached."
                res.final_cost = cost
                terminated = True
                break
            continue
        if ncols == 0:
            res.termination, res.message = "CONVERGENCE", "No active parameters."
            terminated = True
            break
        xa, xb, its = solve_step(prob, ev, radius, opts, explicit_limit=opts.explicit_schur_limit)
        step = np.concatenate([xa.reshape(-1), xb.reshape(-1)])
        if not np.all(np.isfinite(step)):
            consecutive_invalid += 1
            radius = radius / decrease_factor
            decrease_factor *= 2.0
            it.step_is_valid = it.step_is_successful = False
            it.linear_solver_iterations = its
            it.trust_region_radius = radius
            res.num_unsuccessful_steps += 1
            if consecutive_invalid >= opts.max_num_consecutive_invalid_steps:
                res.termination, res.message = "FAILURE", "Too many invalid trust-region steps."
                terminated = True
                break
            res.iterations.append(it)
            continue
        new_cams = cams.copy()
        new_pts = pts.copy()
        new_pts[prob.active_pts] += xa
        new_cams[prob.active_cams] += xb
        cand = evaluate(prob, new_cams, new_pts, jacobians=False)
        # model decrease: 0.5|r|^2 - 0.5|r + J step|^2 (solver.py:798-802)
        pt = prob.pt_col[prob.point_index]
        cam = prob.cam_col[prob.camera_index]
        Jd = np.zeros_like(ev.r)
        m = pt >= 0
        Jd[m] += np.einsum("nij,nj->ni", ev.Jp[m], xa[pt[m]])
        m = cam >= 0
        Jd[m] += np.einsum("nij,nj->ni", ev.Jc[m], xb[cam[m]])
        before = 0.5 * float(np.dot(ev.r.reshape(-1), ev.r.reshape(-1)))
        after_r = (ev.r + Jd).reshape(-1)
        model_decrease = max(before - 0.5 * float(np.dot(after_r, after_r)), 0.0)
        step_is_valid = model_decrease > 0.0
        rho = se.step_quality(cand.cost, model_decrease) if step_is_valid else 0.0
        accepted = step_is_valid and rho > opts.min_relative_decrease
        it.step_norm = float(np.linalg.norm(step))
        it.cost_change = cost - cand.cost
        it.relative_decrease = float(rho)
        it.step_is_valid = step_is_valid
        it.linear_solver_iterations = its
        if accepted:
            consecutive_invalid = 0
            res.num_successful_steps += 1
            se.step_accepted(cand.cost, model_decrease)
            cams, pts = new_cams, new_pts
            if cand.cost < best_cost:
                best_cost = cand.cost
                best = (cams.copy(), pts.copy())
            res.final_cost = best_cost
            denom = max(1.0 / 3.0, 1.0 - (2.0 * rho - 1.0) ** 3)
            radius = min(opts.max_trust_region_radius, radius / denom)
            decrease_factor = 2.0
            it.trust_region_radius = radius
            it.step_is_successful = True
        else:
            res.num_unsuccessful_steps += 1
            radius = radius / decrease_factor
            decrease_factor *= 2.0
            it.trust_region_radius = radius
            it.step_is_successful = False
        res.iterations.append(it)
        if accepted:
            state_norm = math.sqrt(float(np.sum(cams * cams)) + float(np.sum(pts * pts)))
            if it.step_norm <= opts.parameter_tolerance * (state_norm + opts.parameter_tolerance):
                res.termination, res.message = "CONVERGENCE", "Parameter tolerance reached."
                terminated = True
                break
            if previous_cost is not None and abs(previous_cost - cand.cost) <= opts.function_tolerance * max(previous_cost, 1.0):
                res.termination, res.message = "CONVERGENCE", "Function tolerance reached."
                terminated = True
                break
            previous_cost = cand.cost
            ev = evaluate(prob, cams, pts)
            g2 = _gradient(prob, ev)
            if g2.size and float(np.max(np.abs(g2))) <= opts.gradient_tolerance:
                res.termination, res.message = "CONVERGENCE", "Gradient tolerance reached."
                res.final_cost = ev.cost
                terminated = True
                break
        if radius <= opts.min_trust_region_radius:
            res.termination, res.message = "CONVERGENCE", "Minimum trust-region radius reached."
            terminated = True
            break
    if not terminated:
        res.termination, res.message = "NO_CONVERGENCE", "Maximum iterations reached."
    if res.termination == "FAILURE" and res.message == "":
        res.message = "Solver failed."
    # solver.py:661-676: restore the best state, final cost = best cost
    res.cameras, res.points = best
    res.final_cost = best_cost
    return res


def schur_visibility(prob: OracleProblem):
    """solver.py:744-785: per active camera, the sorted tuple of active points it sees."""
    sets = [set() for _ in range(prob.active_cams.size)]
    pt = prob.pt_col[prob.point_index]
    cam = prob.cam_col[prob.camera_index]
    for p, c in zip(pt.tolist(), cam.tolist()):
        if p >= 0 and c >= 0:
            sets[c].add(p)
    if not any(sets):
        return None
    return tuple(tuple(sorted(s)) for s in sets)


# --------------------------------------------------------------------------------------
# Covariance (covariance.py:86-445, DENSE_SVD path)
# --------------------------------------------------------------------------------------
@dataclass
class OracleCovariance:
    success: bool
    message: str
    rank: int
    nullity: int
    tangent: np.ndarray          # [n, n] covariance of the active tangent columns
    cam_col: np.ndarray          # camera -> first column (-1 constant)
    pt_col: np.ndarray           # point -> first column (-1 constant)

    def block(self, kind_a: str, a: int, kind_b: str, b: int) -> np.ndarray:
        """Ambient covariance block (Euclidean blocks: the tangent block; constant blocks:
        zeros), as get_covariance_block (covariance.py:270-282) returns it."""
        sa = self._slice(kind_a, a)
        sb = self._slice(kind_b, b)
        na, nb = (9 if kind_a == "camera" else 3), (9 if kind_b == "camera" else 3)
        if sa is None or sb is None:
            return np.zeros((na, nb))
        return self.tangent[sa, sb].copy()

    def _slice(self, kind: str, i: int):
        c = (self.cam_col if kind == "camera" else self.pt_col)[i]
        if c < 0:
            return None
        return slice(c, c + (9 if kind == "camera" else 3))


def covariance(prob: OracleProblem, cameras, points, *, apply_loss: bool = True, null_space_rank: int = 0,
               min_reciprocal_condition_number: float = 1e-14) -> OracleCovariance:
    """covariance.py:139-246: the dense Jacobian of the active blocks (corrected by the
    loss when apply_loss, covariance.py:122-125), its SVD, singular values above
    20 (m + n) eps s_max kept (:414-417), the retained spectrum checked against
    min_reciprocal_condition_number (:216-224), covariance V diag(1/s^2) V^T (:202-203);
    a rank-deficient Jacobian with null_space_rank 0 is a failure (:206-214)."""
    if apply_loss:
        ev = evaluate(prob, cameras, points)
        Jc, Jp = ev.Jc, ev.Jp
    else:
        _, Jc, Jp = snavely_residuals_and_jacobians(cameras, points, prob.observations, prob.camera_index,
                                                     prob.point_index)
        Jc = Jc * (~prob.camera_constant[prob.camera_index])[:, None, None]
        Jp = Jp * (~prob.point_constant[prob.point_index])[:, None, None]
    nca, npa = prob.active_cams.size, prob.active_pts.size
    n = 9 * nca + 3 * npa
    cam_col = np.where(prob.cam_col >= 0, 9 * prob.cam_col, -1)
    pt_col = np.where(prob.pt_col >= 0, 9 * nca + 3 * prob.pt_col, -1)
    no = prob.observations.shape[0]
    J = np.zeros((2 * no, n))
    for o in range(no):
        c, q = prob.camera_index[o], prob.point_index[o]
        if cam_col[c] >= 0:
            J[2 * o:2 * o + 2, cam_col[c]:cam_col[c] + 9] = Jc[o]
        if pt_col[q] >= 0:
            J[2 * o:2 * o + 2, pt_col[q]:pt_col[q] + 3] = Jp[o]
    _, S, Vh = np.linalg.svd(J, full_matrices=False)
    threshold = 20.0 * (J.shape[0] + J.shape[1]) * EPS64 * S.max()
    keep = S > threshold
    ratios = (S / max(S.max(), TINY64)) ** 2
    if null_space_rank == -1:
        keep &= ratios >= min_reciprocal_condition_number
    elif null_space_rank > 0:
        keep = keep.copy()
        keep[-null_space_rank:] = False
    inv_s2 = np.where(keep, 1.0 / np.where(keep, S * S, 1.0), 0.0)
    tangent = (Vh.T * inv_s2) @ Vh
    rank = int(keep.sum())
    success, message = True, "Computed covariance with dense SVD."
    if null_space_rank == 0 and rank < J.shape[1]:
        success, message = False, "Jacobian is rank deficient."
    elif np.any(ratios[keep] < min_reciprocal_condition_number):
        success, message = False, "Retained covariance spectrum is below min_reciprocal_condition_number."
    return OracleCovariance(success, message, rank, max(0, J.shape[1] - rank), tangent, cam_col, pt_col)


# --------------------------------------------------------------------------------------
# Visibility clustering (linear.py:842-1153), a loop-for-loop restatement
# --------------------------------------------------------------------------------------
def _norm_vis(visibility):
    out = []
    for pts in visibility:
        st = set()
        for p in pts:
            p = int(p)
            if p < 0:
                raise ValueError("visibility point ids must be non-negative")
            st.add(p)
        out.append(frozenset(st))
    return tuple(out)


def visibility_graph(visibility) -> dict:
    """linear.py:842-862."""
    vis = _norm_vis(visibility)
    cams_of: dict = {}
    for c, pts in enumerate(vis):
        for p in pts:
            cams_of.setdefault(p, []).append(c)
    counts: dict = {}
    for cams in cams_of.values():
        cams = sorted(cams)
        for i, a in enumerate(cams):
            for b in cams[i + 1:]:
                counts[(a, b)] = counts.get((a, b), 0) + 1
    edges = {(c, c): 1.0 for c in range(len(vis))}
    for (a, b), k in counts.items():
        denom = math.sqrt(float(len(vis[a]) * len(vis[b])))
        if denom > 0.0:
            edges[(a, b)] = float(k) / denom
    return dict(sorted(edges.items()))


def _flatten_membership(membership: dict, n: int) -> tuple:
    """linear.py:1108-1118."""
    index: dict = {}
    out = []
    for v in range(n):
        key = membership.get(v, -1)
        if key < 0:
            key = v
        if key not in index:
            index[key] = len(index)
        out.append(index[key])
    return tuple(out)


def _find(parent: dict, v: int) -> int:
    root = v
    while parent[root] != root:
        root = parent[root]
    while parent[v] != v:
        parent[v], v = root, parent[v]
    return root


def single_linkage_clustering(visibility, min_similarity: float = 0.9) -> tuple:
    """linear.py:865-893."""
    graph = visibility_graph(visibility)
    n = len(_norm_vis(visibility))
    parent = {v: v for v in range(n)}
    for (a, b), w in graph.items():
        if a >= b or w < min_similarity:
            continue
        ra, rb = _find(parent, a), _find(parent, b)
        if ra == rb:
            continue
        if ra < rb:
            parent[rb] = ra
        else:
            parent[ra] = rb
    return _flatten_membership({v: _find(parent, v) for v in range(n)}, n)


def canonical_views_clustering(visibility, min_views=3, size_penalty_weight=3.0, similarity_penalty_weight=0.0,
                               view_score_weight=0.0) -> tuple:
    """linear.py:896-950."""
    graph = visibility_graph(visibility)
    n = len(_norm_vis(visibility))

    def nbrs(v):
        out = set()
        for a, b in graph:
            if a == v:
                out.add(b)
            if b == v:
                out.add(a)
        return sorted(out)

    def w(a, b):
        return graph.get((a, b) if a <= b else (b, a), 0.0)

    valid = set(range(n))
    centers: list = []
    center_of: dict = {}
    sim_of: dict = {}
    while valid:
        best_diff = -float("inf")
        best_view = min(valid)
        for cand in sorted(valid):
            diff = view_score_weight
            for nb in nbrs(cand):
                old = sim_of.get(nb, 0.0)
                new = w(nb, cand)
                if new > old:
                    diff += new - old
            diff -= size_penalty_weight
            for c in centers:
                diff -= similarity_penalty_weight * w(c, cand)
            if diff > best_diff:
                best_diff, best_view = diff, cand
        if best_diff <= 0.0 and len(centers) >= min_views:
            break
        centers.append(best_view)
        valid.remove(best_view)
        for nb in nbrs(best_view):
            old = sim_of.get(nb, 0.0)
            new = w(nb, best_view)
            if new > old:
                center_of[nb] = best_view
                sim_of[nb] = new
    idx = {c: i for i, c in enumerate(centers)}
    return _flatten_membership({v: idx[center_of[v]] if v in center_of else -1 for v in range(n)}, n)


def degree2_forest(num_vertices: int, weighted_edges: dict) -> tuple:
    """linear.py:993-1028."""
    parent = {v: v for v in range(num_vertices)}
    degree = {v: 0 for v in range(num_vertices)}
    edges = []
    for (a, b), wt in weighted_edges.items():
        if a == b:
            continue
        edges.append((float(wt), (a, b) if a < b else (b, a)))
    forest = []
    for _, (a, b) in sorted(edges, reverse=True):
        if degree[a] == 2 or degree[b] == 2:
            continue
        ra, rb = _find(parent, a), _find(parent, b)
        if ra == rb:
            continue
        forest.append((a, b))
        degree[a] += 1
        degree[b] += 1
        if rb < ra:
            ra, rb = rb, ra
        parent[rb] = ra
    return tuple(sorted(forest))


@dataclass(frozen=True)
class OracleClusterStructure:
    membership: tuple
    num_clusters: int
    cluster_pairs: tuple
    block_pairs: tuple


def cluster_structure(visibility, *, tridiagonal: bool, clustering: str = "CANONICAL_VIEWS") -> OracleClusterStructure:
    """linear.py:953-990 with the cluster graph of linear.py:1121-1134."""
    vis = _norm_vis(visibility)
    if clustering == "SINGLE_LINKAGE":
        membership = single_linkage_clustering(vis)
    elif clustering == "CANONICAL_VIEWS":
        membership = canonical_views_clustering(vis)
    else:
        raise ValueError(f"Unknown visibility clustering type: {clustering}")
    k = max(membership) + 1 if membership else 0
    pairs = {(i, i) for i in range(k)}
    if tridiagonal and k > 1:
        seen = [set() for _ in range(k)]
        for c, pts in enumerate(vis):
            seen[membership[c]].update(pts)
        cg = {}
        for a in range(k):
            for b in range(a + 1, k):
                m = len(seen[a] & seen[b])
                if m:
                    cg[(a, b)] = float(m)
        pairs.update(degree2_forest(k, dict(sorted(cg.items()))))
    blocks = []
    for a in range(len(membership)):
        for b in range(a, len(membership)):
            if tuple(sorted((membership[a], membership[b]))) in pairs:
                blocks.append((a, b))
    return OracleClusterStructure(membership, k, tuple(sorted(pairs)), tuple(blocks))
