"""Visibility clustering of the CLUSTER_JACOBI / CLUSTER_TRIDIAGONAL preconditioners.

``tests/golden/clustering.npz`` holds the reference's own cluster structures
(``build_visibility_cluster_structure``, linear.py:953-990) for capture sequences,
uniform problems and edge cases (an empty camera, duplicate ids, identical views, one
camera, no shared points), both clustering types and both preconditioners. The
product's vectorised clustering (``ceres_torch_cuda_b200.clustering``) and the oracle's
loop restatement must both reproduce them exactly: memberships, cluster pairs and
kept block pairs are integer data, and the similarity weights are the same float64
operations.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from ceres_torch_cuda_b200 import clustering as C
from ceres_torch_cuda_b200 import synthetic as S
from oracle import ba_oracle as O
from tests import _golden as G


def _fixture():
    z = np.load(G.GOLDEN / "clustering.npz", allow_pickle=False)
    return json.loads(str(z["visibility"])), json.loads(str(z["results"]))


VIS, RESULTS = _fixture()


@pytest.mark.parametrize("key", sorted(RESULTS))
def test_product_clustering_matches_reference(key):
    case, pre, kind = key.split("|")
    ref = RESULTS[key]
    st = C.cluster_structure(VIS[case], tridiagonal=pre == "CLUSTER_TRIDIAGONAL", clustering=kind)
    assert tuple(st.membership.tolist()) == tuple(ref["membership"])
    assert st.num_clusters == ref["num_clusters"]
    assert [list(p) for p in st.cluster_pairs] == ref["cluster_pairs"]
    assert [list(p) for p in st.block_pairs()] == ref["block_pairs"]
    # the similarity graph: same edges, same float64 weights
    g = C.visibility_graph(C._incidence(VIS[case]))
    a, b = np.nonzero(np.triu(g.weights))
    got = [[int(x), int(y), float(g.weights[x, y])] for x, y in zip(a, b)]
    assert got == [[int(e[0]), int(e[1]), float(e[2])] for e in ref["camera_graph_edges"]]


@pytest.mark.parametrize("key", sorted(RESULTS))
def test_oracle_clustering_matches_reference(key):
    case, pre, kind = key.split("|")
    ref = RESULTS[key]
    st = O.cluster_structure(VIS[case], tridiagonal=pre == "CLUSTER_TRIDIAGONAL", clustering=kind)
    assert st.membership == tuple(ref["membership"])
    assert [list(p) for p in st.cluster_pairs] == ref["cluster_pairs"]
    assert [list(p) for p in st.block_pairs] == ref["block_pairs"]
    graph = O.visibility_graph(VIS[case])
    assert [[a, b, w] for (a, b), w in graph.items()] == [[int(e[0]), int(e[1]), float(e[2])]
                                                          for e in ref["camera_graph_edges"]]


@pytest.mark.parametrize("seed", range(6))
def test_product_clustering_matches_oracle_on_random_problems(seed):
    rng = np.random.default_rng(seed)
    nc = int(rng.integers(3, 40))
    if seed % 2:
        d = S.make_sequence_ba(nc, int(rng.integers(20, 400)), int(rng.integers(2, 5)), seed=seed,
                               closed=bool(seed % 3))
    else:
        d = S.make_small_ba(nc, int(rng.integers(10, 300)), int(rng.integers(2, min(nc, 6) + 1)), seed=seed)
    inc = C.incidence_from_observations(nc, d.camera_index, d.point_index)
    vis = [sorted(set(d.point_index[d.camera_index == c].tolist())) for c in range(nc)]
    for tri in (False, True):
        for kind in (C.CANONICAL_VIEWS, C.SINGLE_LINKAGE):
            a = O.cluster_structure(vis, tridiagonal=tri, clustering=kind)
            b = C.cluster_structure(tridiagonal=tri, clustering=kind, incidence=inc)
            assert tuple(b.membership.tolist()) == a.membership
            assert b.cluster_pairs == a.cluster_pairs
            assert b.block_pairs() == a.block_pairs


def test_components_partition_the_kept_pattern():
    d = S.make_sequence_ba(30, 600, 4, seed=8)
    inc = C.incidence_from_observations(30, d.camera_index, d.point_index)
    for tri in (False, True):
        st = C.cluster_structure(tridiagonal=tri, incidence=inc)
        comps = st.components()
        where = np.concatenate([np.full(g.size, k) for k, g in enumerate(comps)])[np.argsort(np.concatenate(comps))]
        assert sorted(np.concatenate(comps).tolist()) == list(range(30))
        for a, b in st.block_pairs():
            assert where[a] == where[b]  # no kept block crosses two components
        if not tri:  # CLUSTER_JACOBI: the components are the clusters
            assert len(comps) == st.num_clusters


def test_unknown_clustering_type_is_refused():
    with pytest.raises(ValueError, match="Unknown visibility clustering type"):
        C.cluster_structure([[0, 1], [1]], tridiagonal=False, clustering="NONE")
    with pytest.raises(ValueError, match="non-negative"):
        C.cluster_structure([[0, -1], [1]], tridiagonal=False)
