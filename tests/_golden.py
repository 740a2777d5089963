"""Helpers that load the golden fixtures produced by ``tests/golden/make_golden.py``."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"

BA_CASES = [
    "ba_small_iterative",
    "ba_small_dense",
    "ba_small_sparse",
    "ba_huber_outliers",
    "ba_cauchy",
    "ba_const_camera_jacobi",
    "ba_fixed_cameras",
    "ba_spse",
    "ba_spse_cauchy",
    "ba_spse_init",
    "ba_cluster_jacobi",
    "ba_cluster_tridiagonal",
    "ba_cluster_single_linkage",
    "ba_cluster_uniform",
]
BIG_CASES = ["config0_dense", "config1_small", "config2_small"]


def available(name: str) -> bool:
    return (GOLDEN / f"{name}.npz").exists()


def load(name: str) -> dict:
    z = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    out = {k: z[k] for k in z.files}
    out["meta"] = json.loads(str(out["meta"]))
    return out


def loss_spec(meta_loss) -> tuple:
    kind = meta_loss[0]
    return (kind,) + tuple(float(v) for v in meta_loss[1:])


def constant_mask(n: int, idx) -> np.ndarray:
    m = np.zeros(n, dtype=bool)
    m[list(idx)] = True
    return m
