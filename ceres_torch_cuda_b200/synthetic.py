"""Seeded synthetic bundle-adjustment problems.

Every problem is drawn from one ``numpy.random.Generator(PCG64(seed))`` so the
same seed gives the same bytes on any machine. The camera is the 9-parameter
Snavely model used by the reference's BAL example
(``examples/simple_bundle_adjuster.py:73-79``): angle-axis rotation (3),
translation (3), focal length, radial distortion k1, k2. A point is 3 floats.

Generated observations are ordered by point (all observations of point 0,
then point 1, ...), and within a point by camera draw order. The residual
blocks a ``Problem`` is built from follow this order.

The projection used to synthesise pixels is the reference's own formula,
restated in numpy float64:

    p  = R(aa) X + t          (R from the angle-axis via a unit quaternion)
    xp = -p0 / p2,  yp = -p1 / p2
    d  = 1 + r2 (k1 + k2 r2),  r2 = xp^2 + yp^2
    uv = f d (xp, yp)
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "BAData",
    "project",
    "make_uniform_ba",
    "make_ring_ba",
    "make_small_ba",
    "make_batched_instances",
    "make_serving_requests",
    "ba_config",
]


@dataclass
class BAData:
    """A bundle-adjustment instance as flat arrays (float64 / int64)."""

    cameras: np.ndarray          # [nc, 9] initial guess
    points: np.ndarray           # [np, 3] initial guess
    observations: np.ndarray     # [no, 2] pixels
    camera_index: np.ndarray     # [no] int64
    point_index: np.ndarray      # [no] int64
    true_cameras: np.ndarray     # [nc, 9]
    true_points: np.ndarray      # [np, 3]
    loss: tuple = ("trivial",)   # ("trivial",) | ("huber", a) | ("cauchy", a)
    description: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def num_cameras(self) -> int:
        return int(self.cameras.shape[0])

    @property
    def num_points(self) -> int:
        return int(self.points.shape[0])

    @property
    def num_observations(self) -> int:
        return int(self.observations.shape[0])


def _rotate(aa: np.ndarray, X: np.ndarray) -> np.ndarray:
    """Angle-axis rotation through a unit quaternion (vectorised over rows)."""
    theta = np.linalg.norm(aa, axis=-1, keepdims=True)
    half = 0.5 * theta
    small = theta <= np.finfo(np.float64).eps
    safe = np.where(small, 1.0, theta)
    k = np.where(small, 0.5 - theta * theta / 48.0, np.sin(half) / safe)
    q = np.concatenate([np.cos(half), k * aa], axis=-1)
    q = q / np.maximum(np.linalg.norm(q, axis=-1, keepdims=True), np.finfo(np.float64).tiny)
    w = q[..., :1]
    u = q[..., 1:]
    uv = 2.0 * np.cross(u, X)
    return X + w * uv + np.cross(u, uv)


def project(cameras: np.ndarray, points: np.ndarray) -> np.ndarray:
    """Snavely projection of ``points[i]`` by ``cameras[i]`` (row-aligned)."""
    p = _rotate(cameras[:, 0:3], points) + cameras[:, 3:6]
    xp = -p[:, 0] / p[:, 2]
    yp = -p[:, 1] / p[:, 2]
    r2 = xp * xp + yp * yp
    d = 1.0 + r2 * (cameras[:, 7] + cameras[:, 8] * r2)
    return np.stack([cameras[:, 6] * d * xp, cameras[:, 6] * d * yp], axis=1)


def _distinct_cameras(rng: np.random.Generator, track: np.ndarray, nc: int) -> tuple[np.ndarray, np.ndarray]:
    """For point j draw ``track[j]`` distinct cameras uniformly from ``nc``.

    Returns (camera_index, point_index), ordered by point. Vectorised by
    drawing, per point, the first ``track[j]`` entries of a random
    permutation when tracks are dense, or by rejection of duplicates when
    ``track << nc``.
    """
    npts = track.shape[0]
    total = int(track.sum())
    point_index = np.repeat(np.arange(npts, dtype=np.int64), track)
    if nc <= 64:
        keys = rng.random((npts, nc))
        order = np.argsort(keys, axis=1)
        starts = np.concatenate([[0], np.cumsum(track)[:-1]])
        within = np.arange(total) - np.repeat(starts, track)
        cam = order[point_index, within].astype(np.int64)
        return cam, point_index
    cam = rng.integers(0, nc, size=total, dtype=np.int64)
    # Redraw duplicates within a point until every track is distinct.
    starts = np.concatenate([[0], np.cumsum(track)[:-1]])
    for _ in range(1000):
        key = point_index * nc + cam
        order = np.argsort(key, kind="stable")
        sk = key[order]
        dup_sorted = np.zeros(total, dtype=bool)
        dup_sorted[1:] = sk[1:] == sk[:-1]
        if not dup_sorted.any():
            break
        dup = np.zeros(total, dtype=bool)
        dup[order[dup_sorted]] = True
        cam[dup] = rng.integers(0, nc, size=int(dup.sum()), dtype=np.int64)
    else:  # pragma: no cover - 1000 rounds never needed for nc > 64
        raise RuntimeError("could not draw distinct cameras")
    del starts
    return cam, point_index


def _perturb(rng, true_cameras, true_points, rot_sigma=0.02, trans_sigma=0.1, point_sigma=0.1):
    cams = true_cameras.copy()
    cams[:, 0:3] += rng.normal(0.0, rot_sigma, size=(cams.shape[0], 3))
    cams[:, 3:6] += rng.normal(0.0, trans_sigma, size=(cams.shape[0], 3))
    pts = true_points + rng.normal(0.0, point_sigma, size=true_points.shape)
    return cams, pts


def _standard_cameras(rng, nc, focal=500.0):
    cams = np.zeros((nc, 9))
    cams[:, 0:3] = rng.normal(0.0, 0.1, size=(nc, 3))
    cams[:, 3:6] = rng.normal(0.0, 1.0, size=(nc, 3)) + np.array([0.0, 0.0, 8.0])
    cams[:, 6] = focal
    cams[:, 7:9] = rng.normal(0.0, 1e-3, size=(nc, 2))
    return cams


def _finish(rng, true_cams, true_pts, cam, pt, loss, description, outlier_fraction=0.0, meta=None):
    obs = project(true_cams[cam], true_pts[pt]) + rng.normal(0.0, 1.0, size=(cam.shape[0], 2))
    if outlier_fraction > 0.0:
        mask = rng.random(cam.shape[0]) < outlier_fraction
        obs[mask] = rng.uniform(0.0, 1000.0, size=(int(mask.sum()), 2))
    cams0, pts0 = _perturb(rng, true_cams, true_pts)
    return BAData(
        cameras=cams0,
        points=pts0,
        observations=obs,
        camera_index=cam,
        point_index=pt,
        true_cameras=true_cams,
        true_points=true_pts,
        loss=loss,
        description=description,
        meta=dict(meta or {}),
    )


def make_uniform_ba(
    num_cameras: int,
    num_points: int,
    track: int | str = 4,
    *,
    seed: int = 0,
    loss: tuple = ("trivial",),
    outlier_fraction: float = 0.0,
    description: str = "",
) -> BAData:
    """Cameras around (0,0,8), points uniform in [-1,1]^3.

    ``track`` is an int (every point seen by that many distinct cameras) or
    ``"poisson6"`` (Poisson(6)+2 capped at the camera count).
    """
    rng = np.random.default_rng(seed)
    true_cams = _standard_cameras(rng, num_cameras)
    true_pts = rng.uniform(-1.0, 1.0, size=(num_points, 3))
    if isinstance(track, str):
        if track != "poisson6":
            raise ValueError(f"unknown track model {track!r}")
        lengths = np.minimum(rng.poisson(6.0, size=num_points) + 2, num_cameras).astype(np.int64)
    else:
        lengths = np.full(num_points, min(int(track), num_cameras), dtype=np.int64)
    cam, pt = _distinct_cameras(rng, lengths, num_cameras)
    return _finish(rng, true_cams, true_pts, cam, pt, loss, description or f"uniform nc={num_cameras} np={num_points}",
                   outlier_fraction=outlier_fraction, meta={"seed": seed})


def make_ring_ba(
    num_cameras: int,
    num_points: int,
    *,
    seed: int = 0,
    loss: tuple = ("cauchy", 2.0),
    max_track: int = 100,
    p: float = 0.2,
    description: str = "",
) -> BAData:
    """Cameras on a ring of radius 10 looking at the origin; points in [-3,3]^3.

    Camera i has angle-axis (0, 2*pi*i/nc, 0) + N(0, 0.01^2) and translation
    (0, 0, 10) + N(0, 0.1^2), so the origin sits 10 units along the optical
    axis of every camera. Track length is Geometric(p) on {0, 1, ...} plus 2,
    capped at ``min(max_track, num_cameras)`` (mean 1/p + 1).
    """
    rng = np.random.default_rng(seed)
    true_cams = np.zeros((num_cameras, 9))
    phi = 2.0 * np.pi * np.arange(num_cameras) / num_cameras
    true_cams[:, 1] = phi
    true_cams[:, 0:3] += rng.normal(0.0, 0.01, size=(num_cameras, 3))
    true_cams[:, 3:6] = np.array([0.0, 0.0, 10.0]) + rng.normal(0.0, 0.1, size=(num_cameras, 3))
    true_cams[:, 6] = 500.0
    true_cams[:, 7:9] = rng.normal(0.0, 1e-3, size=(num_cameras, 2))
    true_pts = rng.uniform(-3.0, 3.0, size=(num_points, 3))
    lengths = np.minimum(rng.geometric(p, size=num_points) + 1, min(max_track, num_cameras)).astype(np.int64)
    cam, pt = _distinct_cameras(rng, lengths, num_cameras)
    return _finish(rng, true_cams, true_pts, cam, pt, loss, description or f"ring nc={num_cameras} np={num_points}",
                   meta={"seed": seed})


def make_sequence_ba(num_cameras: int, num_points: int, window: int, *, seed: int = 0, loss=("trivial",),
                     closed: bool = False) -> BAData:
    """A capture sequence: the ring cameras of ``make_ring_ba``, and each point seen by
    ``window`` consecutive cameras from a uniform start (wrapping round the ring when
    ``closed``), so that the camera visibility graph is banded and the visibility
    clusters are runs of neighbouring cameras."""
    rng = np.random.default_rng(seed)
    window = min(int(window), num_cameras)
    true_cams = np.zeros((num_cameras, 9))
    true_cams[:, 1] = 2.0 * np.pi * np.arange(num_cameras) / num_cameras
    true_cams[:, 0:3] += rng.normal(0.0, 0.01, size=(num_cameras, 3))
    true_cams[:, 3:6] = np.array([0.0, 0.0, 10.0]) + rng.normal(0.0, 0.1, size=(num_cameras, 3))
    true_cams[:, 6] = 500.0
    true_cams[:, 7:9] = rng.normal(0.0, 1e-3, size=(num_cameras, 2))
    true_pts = rng.uniform(-3.0, 3.0, size=(num_points, 3))
    span = num_cameras if closed else num_cameras - window + 1
    start = rng.integers(0, span, size=num_points)
    cam = ((start[:, None] + np.arange(window)[None, :]) % num_cameras).reshape(-1).astype(np.int64)
    pt = np.repeat(np.arange(num_points, dtype=np.int64), window)
    return _finish(rng, true_cams, true_pts, cam, pt, loss, f"sequence nc={num_cameras} np={num_points} w={window}",
                   meta={"seed": seed})


def make_small_ba(num_cameras: int, num_points: int, track: int, *, seed: int = 0, loss=("trivial",),
                  outlier_fraction: float = 0.0) -> BAData:
    """Small instance with the configuration-0 camera/point model (tests, fixtures)."""
    return make_uniform_ba(num_cameras, num_points, track, seed=seed, loss=loss,
                           outlier_fraction=outlier_fraction)


def make_batched_instances(count: int, *, seed: int = 0, max_points: int = 2000) -> list[BAData]:
    """Independent instances: nc ~ U{3..32}, np ~ U{50..max_points}, track ~ U{3..8} capped at nc."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nc = int(rng.integers(3, 33))
        npts = int(rng.integers(50, max_points + 1))
        sub = np.random.default_rng([seed, i])
        true_cams = _standard_cameras(sub, nc)
        true_pts = sub.uniform(-1.0, 1.0, size=(npts, 3))
        lengths = np.minimum(sub.integers(3, 9, size=npts), nc).astype(np.int64)
        cam, pt = _distinct_cameras(sub, lengths, nc)
        out.append(_finish(sub, true_cams, true_pts, cam, pt, ("trivial",), f"batched[{i}] nc={nc} np={npts}"))
    return out


def make_serving_requests(count: int, *, seed: int = 0, rate_hz: float = 1000.0, max_cameras: int = 500,
                          points_per_camera: int = 250) -> tuple[np.ndarray, list[BAData]]:
    """Poisson arrivals; nc = clip(lognormal(ln 20, 0.8), 3, max_cameras), np = points_per_camera*nc,
    track ~ Poisson(4)+2 capped at nc. Returns (arrival_times_s, problems)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, size=count)
    arrivals = np.cumsum(gaps) - gaps[0]
    problems = []
    for i in range(count):
        nc = int(np.clip(np.round(rng.lognormal(np.log(20.0), 0.8)), 3, max_cameras))
        npts = points_per_camera * nc
        sub = np.random.default_rng([seed, 7, i])
        true_cams = _standard_cameras(sub, nc)
        true_pts = sub.uniform(-1.0, 1.0, size=(npts, 3))
        lengths = np.minimum(sub.poisson(4.0, size=npts) + 2, nc).astype(np.int64)
        cam, pt = _distinct_cameras(sub, lengths, nc)
        problems.append(_finish(sub, true_cams, true_pts, cam, pt, ("trivial",), f"request[{i}] nc={nc}"))
    return arrivals, problems


def ba_config(index: int, *, scale: float = 1.0, seed: int | None = None) -> BAData:
    """The five benchmark configurations; ``scale`` < 1 shrinks point counts
    (and camera counts for the ring) with the same distributions."""
    if index == 0:
        return make_uniform_ba(16, max(1, int(2000 * scale)), 4, seed=100 if seed is None else seed,
                               description="config0 nc=16 np=2000 track=4 trivial DENSE_SCHUR")
    if index == 1:
        return make_uniform_ba(max(3, int(200 * min(1.0, scale * 10))), max(1, int(50_000 * scale)), "poisson6",
                               seed=101 if seed is None else seed, loss=("huber", 1.0), outlier_fraction=0.05,
                               description="config1 nc=200 np=50000 track=Poisson(6)+2 huber(1) 5% outliers")
    if index == 2:
        return make_ring_ba(max(3, int(1500 * min(1.0, scale * 10))), max(1, int(1_000_000 * scale)),
                            seed=102 if seed is None else seed,
                            description="config2 ring nc=1500 np=1000000 track=Geometric(0.2)+2<=100 cauchy(2)")
    raise ValueError("configurations 3 and 4 are collections; use make_batched_instances / make_serving_requests")
