"""The fixed summation order of the explicit reduced camera matrix (engine.schur_contributions).

The DENSE_SCHUR / SPARSE_SCHUR solve and the covariance's explicit S (the reference's
dense Schur route, linear.py:667-699) are summed in the order this list gives, so two
runs give the same bits. On the CPU:

* the list equals a brute-force enumeration over cameras, points and observations
  (self pairs, same-camera pairs of one point in both orders, cross-camera pairs
  oriented a < b; constant cameras and constant points as the reference treats them);
* summing the list with the kernel's arithmetic (-G_i W_q^-1 G_j^T, plus Jc^T Jc on self
  pairs, diagonal blocks from their upper triangle) gives Jc^T Jc - Jc^T Jp W^-1 Jp^T Jc
  of the dense Jacobian;
* an over-long list is refused (the atomic summation then stays).
"""
from __future__ import annotations

import itertools

import numpy as np
import pytest
import torch

from ceres_torch_cuda_b200 import engine as E
from ceres_torch_cuda_b200 import synthetic as S


def _case(nc, npt, k, seed, dup_every=0, const_cams=(), const_pts=()):
    d = S.make_small_ba(nc, npt, k, seed=seed)
    ci, pi = d.camera_index.astype(np.int64), d.point_index.astype(np.int64)
    if dup_every:
        rep = np.arange(0, ci.size, dup_every)
        ci, pi = np.concatenate([ci, ci[rep]]), np.concatenate([pi, pi[rep]])
    obs = np.zeros((ci.size, 2))
    L = E.build_layout(torch.as_tensor(ci), torch.as_tensor(pi), torch.as_tensor(obs), nc, npt)
    np_pad = 32 * L.num_slices
    cam_const = torch.zeros(nc, dtype=torch.uint8)
    cam_const[list(const_cams)] = 1
    pt_const = torch.ones(max(np_pad, 1), dtype=torch.uint8)
    pt_const[:npt] = 0
    q_of = torch.empty(npt, dtype=torch.int64)
    q_of[L.point_order] = torch.arange(npt)
    for p in const_pts:
        pt_const[q_of[p]] = 1
    return L, nc, cam_const, pt_const, np_pad


def _brute(L, nc, cam_const, pt_const):
    ents = L.cam_entries.numpy()
    off = L.cam_offsets.numpy()
    rows = {}
    for a in range(nc):
        if cam_const[a]:
            continue
        obs_a = [tuple(e) for e in ents[off[a]:off[a + 1]]]
        for s, q in obs_a:
            rows.setdefault((a, a), []).append((q, s, s))
        for (s1, q1), (s2, q2) in itertools.permutations(obs_a, 2):
            if q1 == q2 and not pt_const[q1]:
                rows[(a, a)].append((q1, s1, s2))
        for b in range(a + 1, nc):
            if cam_const[b]:
                continue
            for (s1, q1), (s2, q2) in itertools.product(obs_a, [tuple(e) for e in ents[off[b]:off[b + 1]]]):
                if q1 == q2 and not pt_const[q1]:
                    rows.setdefault((a, b), []).append((q1, s1, s2))
    blocks = sorted(rows)
    return blocks, [sorted(rows[k]) for k in blocks]


CASES = [
    dict(nc=6, npt=40, k=3, seed=1),
    dict(nc=9, npt=70, k=4, seed=2, dup_every=5),
    dict(nc=8, npt=50, k=3, seed=3, const_cams=(0, 5), const_pts=(1, 7, 8)),
    dict(nc=7, npt=33, k=7, seed=4, dup_every=3, const_cams=(2,), const_pts=(0,)),
]


@pytest.mark.parametrize("case", CASES)
def test_list_equals_brute_force_enumeration(case):
    L, nc, cc, pc, np_pad = _case(**case)
    blocks, start, contrib, nb = E.schur_contributions(L, nc, cc, pc, np_pad)
    ref_blocks, ref_rows = _brute(L, nc, cc.numpy(), pc.numpy())
    assert nb == len(ref_blocks)
    assert [tuple(b) for b in blocks[:nb].tolist()] == ref_blocks
    c = contrib.numpy()
    st = start.numpy()
    for k, rows in enumerate(ref_rows):
        got = [(int(q), int(i), int(j)) for i, j, q in c[st[k]:st[k + 1]]]
        assert got == rows  # points ascending, then (slot i, slot j)


def _sum_list(L, nc, np_pad, jac, winv, order):
    blocks, start, contrib, nb = order
    S_ = np.zeros((9 * nc, 9 * nc))
    for k in range(nb):
        a, b = (int(x) for x in blocks[k])
        acc = np.zeros((9, 9))
        for i, j, q in contrib[int(start[k]):int(start[k + 1])].tolist():
            ra, rb = jac[i], jac[j]
            Ga = np.outer(ra[:9], ra[18:21]) + np.outer(ra[9:18], ra[21:24])
            Gb = np.outer(rb[:9], rb[18:21]) + np.outer(rb[9:18], rb[21:24])
            jj = np.outer(ra[:9], ra[:9]) + np.outer(ra[9:18], ra[9:18]) if i == j else 0.0
            acc += jj - Ga @ winv[q] @ Gb.T
        if a == b:
            acc = np.triu(acc) + np.triu(acc, 1).T
        S_[9 * a:9 * a + 9, 9 * b:9 * b + 9] = acc
        S_[9 * b:9 * b + 9, 9 * a:9 * a + 9] = acc.T
    return S_


@pytest.mark.parametrize("case", CASES)
def test_list_sums_to_the_reduced_camera_matrix(case):
    L, nc, cc, pc, np_pad = _case(**case)
    order = E.schur_contributions(L, nc, cc, pc, np_pad)
    rng = np.random.default_rng(case["seed"])
    nslot = max(L.num_slots, 1)
    jac = rng.standard_normal((nslot, 24))
    winv = np.zeros((max(np_pad, 1), 3, 3))
    for q in range(np_pad):
        if not pc[q]:
            m = rng.standard_normal((3, 3))
            winv[q] = np.linalg.inv(m @ m.T + 3 * np.eye(3))
    got = _sum_list(L, nc, np_pad, jac, winv, order)
    # dense restatement: J over (active cameras, points), W^-1 block diagonal
    slot_cam = L.slot_cam.numpy()
    Jc = np.zeros((2 * nslot, 9 * nc))
    Jp = np.zeros((2 * nslot, 3 * np_pad))
    for s in range(L.num_slots):
        c = slot_cam[s]
        if c < 0 or cc[c]:
            continue
        q = int(np.nonzero(L.cam_entries.numpy()[:, 0] == s)[0][0])
        q = int(L.cam_entries.numpy()[q, 1])
        Jc[2 * s, 9 * c:9 * c + 9], Jc[2 * s + 1, 9 * c:9 * c + 9] = jac[s, :9], jac[s, 9:18]
        if not pc[q]:
            Jp[2 * s, 3 * q:3 * q + 3], Jp[2 * s + 1, 3 * q:3 * q + 3] = jac[s, 18:21], jac[s, 21:24]
    Winv = np.zeros((3 * np_pad, 3 * np_pad))
    for q in range(np_pad):
        Winv[3 * q:3 * q + 3, 3 * q:3 * q + 3] = winv[q]
    ref = Jc.T @ Jc - Jc.T @ Jp @ Winv @ Jp.T @ Jc
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-11 * np.abs(ref).max())
    assert np.array_equal(got, got.T)  # the diagonal blocks are written from their upper triangle


def test_over_long_list_is_refused():
    L, nc, cc, pc, np_pad = _case(nc=6, npt=40, k=3, seed=1)
    full = E.schur_contributions(L, nc, cc, pc, np_pad)
    n = int(full[2].shape[0])
    # the bound counts every pair of observations at a point twice (an upper bound)
    assert E.schur_contributions(L, nc, cc, pc, np_pad, limit=2 * n) is not None
    assert E.schur_contributions(L, nc, cc, pc, np_pad, limit=n - 1) is None


def test_empty_problem():
    L, nc, cc, pc, np_pad = _case(nc=4, npt=10, k=2, seed=5, const_cams=(0, 1, 2, 3))
    blocks, start, contrib, nb = E.schur_contributions(L, nc, cc, pc, np_pad)
    assert nb == 0 and start.tolist() == [0]
