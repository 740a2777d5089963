"""Visibility clustering of the cameras for the CLUSTER_JACOBI and CLUSTER_TRIDIAGONAL
preconditioners of the reduced camera system (ceres-torch linear.py:842-1153).

Host-side graph logic, run once per problem: the camera similarity graph (shared
points over the geometric mean of the two cameras' point counts), a clustering
(CANONICAL_VIEWS greedy centre selection, or SINGLE_LINKAGE over edges of similarity
>= 0.9), the cluster graph (shared points between clusters) and the degree-2 maximum
spanning forest that links clusters for CLUSTER_TRIDIAGONAL. The preconditioner keeps
the camera blocks (a, b) whose cluster pair is a diagonal pair or a forest edge.

Every decision is the reference's: the same edge order, the same first-seen cluster
numbering, the same first-maximum tie break, and the canonical-view scores summed in
the reference's order (neighbours ascending, one addition at a time: numpy's
``add.accumulate`` adds sequentially, and the extra ``+ 0.0`` terms of non-neighbours
leave a float64 sum unchanged), so the memberships and kept pairs equal the
reference's bit for bit. The work is vectorised over cameras: sparse products for the
shared-point counts, dense similarity rows for the canonical-view scores.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

CANONICAL_VIEWS = "CANONICAL_VIEWS"
SINGLE_LINKAGE = "SINGLE_LINKAGE"


def _incidence(visibility: Sequence[Iterable[int]]):
    """cameras x points 0/1 matrix (CSR) of the distinct (camera, point) pairs."""
    import scipy.sparse as sp

    rows, cols = [], []
    for c, pts in enumerate(visibility):
        a = np.unique(np.fromiter((int(p) for p in pts), dtype=np.int64))
        if a.size and a[0] < 0:
            raise ValueError("visibility point ids must be non-negative")
        rows.append(np.full(a.size, c, dtype=np.int64))
        cols.append(a)
    n = len(rows)
    r = np.concatenate(rows) if rows else np.zeros(0, np.int64)
    c = np.concatenate(cols) if cols else np.zeros(0, np.int64)
    width = int(c.max()) + 1 if c.size else 0
    return sp.csr_matrix((np.ones(r.size, dtype=np.int64), (r, c)), shape=(n, width))


def incidence_from_observations(num_cameras: int, camera_index, point_index):
    """The incidence matrix of a bundle-adjustment problem, from its observation arrays."""
    import scipy.sparse as sp

    ci = np.asarray(camera_index, dtype=np.int64)
    pi = np.asarray(point_index, dtype=np.int64)
    width = int(pi.max()) + 1 if pi.size else 0
    m = sp.csr_matrix((np.ones(ci.size, dtype=np.int64), (ci, pi)), shape=(num_cameras, width))
    m.sum_duplicates()
    m.data[:] = 1
    return m


@dataclass(frozen=True)
class VisibilityGraph:
    """Similarity of camera pairs: a dense symmetric matrix (1 on the diagonal, 0 where
    two cameras share no point) and the number of points each camera sees."""
    weights: np.ndarray
    counts: np.ndarray


def visibility_graph(incidence) -> VisibilityGraph:
    """linear.py:842-862: w(a, b) = shared(a, b) / sqrt(n_a n_b) for a != b sharing a point."""
    n = incidence.shape[0]
    counts = np.asarray(incidence.sum(axis=1)).ravel().astype(np.int64)
    shared = (incidence @ incidence.T).tocoo()
    W = np.zeros((n, n), dtype=np.float64)
    a, b, s = shared.row, shared.col, shared.data
    keep = (a != b) & (s > 0)
    a, b, s = a[keep], b[keep], s[keep]
    denom = np.sqrt((counts[a] * counts[b]).astype(np.float64))
    ok = denom > 0.0
    W[a[ok], b[ok]] = s[ok].astype(np.float64) / denom[ok]
    W[np.arange(n), np.arange(n)] = 1.0
    return VisibilityGraph(W, counts)


def _flatten(keys: Sequence[int]) -> np.ndarray:
    """Cluster ids in order of first appearance over the cameras; a camera without a
    cluster (key -1) keys on its own id (linear.py:1108-1118)."""
    index: dict[int, int] = {}
    out = np.empty(len(keys), dtype=np.int64)
    for v, key in enumerate(keys):
        key = int(key)
        if key < 0:
            key = v
        out[v] = index.setdefault(key, len(index))
    return out


class _UnionFind:
    def __init__(self, n: int):
        self.parent = list(range(n))

    def find(self, v: int) -> int:
        root = v
        while self.parent[root] != root:
            root = self.parent[root]
        while self.parent[v] != v:
            self.parent[v], v = root, self.parent[v]
        return root

    def union(self, a: int, b: int) -> bool:
        """Join the sets of a and b (the larger root joins the smaller); False when they
        are one set already."""
        ra, rb = self.find(a), self.find(b)
        if ra == rb:
            return False
        if ra < rb:
            self.parent[rb] = ra
        else:
            self.parent[ra] = rb
        return True


def single_linkage(graph: VisibilityGraph, min_similarity: float = 0.9) -> np.ndarray:
    """linear.py:865-893: union of the cameras joined by an edge of similarity >= the
    minimum, edges in ascending (a, b) order."""
    W = graph.weights
    n = W.shape[0]
    a, b = np.nonzero(np.triu(W, 1) >= min_similarity)  # row-major: ascending (a, b)
    uf = _UnionFind(n)
    for x, y in zip(a.tolist(), b.tolist()):
        uf.union(x, y)
    return _flatten([uf.find(v) for v in range(n)])


def canonical_views(graph: VisibilityGraph, min_views: int = 3, size_penalty_weight: float = 3.0,
                    similarity_penalty_weight: float = 0.0, view_score_weight: float = 0.0) -> np.ndarray:
    """linear.py:896-950: greedy canonical-view selection; each view joins the centre
    most similar to it."""
    W = graph.weights
    n = W.shape[0]
    valid = np.ones(n, dtype=bool)
    best_sim = np.zeros(n, dtype=np.float64)
    best_center = np.full(n, -1, dtype=np.int64)
    centers: list[int] = []
    while valid.any():
        cand = np.flatnonzero(valid)
        Wc = W[:, cand]                                   # rows: neighbour, ascending
        gain = np.where(Wc > best_sim[:, None], Wc - best_sim[:, None], 0.0)
        diff = np.add.accumulate(np.vstack([np.full((1, cand.size), view_score_weight), gain]), axis=0)[-1]
        diff = diff - size_penalty_weight
        for c in centers:
            diff = diff - similarity_penalty_weight * W[c, cand]
        k = int(np.argmax(diff))                          # first maximum in ascending order
        if diff[k] <= 0.0 and len(centers) >= min_views:
            break
        view = int(cand[k])
        centers.append(view)
        valid[view] = False
        w = W[:, view]
        better = w > best_sim
        best_center[better] = view
        best_sim[better] = w[better]
    index = {c: i for i, c in enumerate(centers)}
    return _flatten([index[int(c)] if c >= 0 else -1 for c in best_center])


def cluster_graph(incidence, membership: np.ndarray, num_clusters: int) -> np.ndarray:
    """linear.py:1121-1134: points seen by both clusters, a dense k x k count matrix."""
    import scipy.sparse as sp

    n = incidence.shape[0]
    M = sp.csr_matrix((np.ones(n, dtype=np.int64), (membership, np.arange(n))), shape=(num_clusters, n))
    seen = (M @ incidence)
    seen.data[:] = 1
    shared = (seen @ seen.T).toarray()
    np.fill_diagonal(shared, 0)
    return shared


def degree2_forest(num_vertices: int, shared: np.ndarray) -> list[tuple[int, int]]:
    """linear.py:993-1028: maximum spanning forest of vertex degree <= 2; edges by
    descending weight, then descending (a, b)."""
    a, b = np.nonzero(np.triu(shared, 1))
    w = shared[a, b].astype(np.float64)
    order = np.lexsort((-b, -a, -w))
    uf = _UnionFind(num_vertices)
    degree = np.zeros(num_vertices, dtype=np.int64)
    forest = []
    for x, y in zip(a[order].tolist(), b[order].tolist()):
        if degree[x] == 2 or degree[y] == 2:
            continue
        if not uf.union(x, y):
            continue
        forest.append((x, y))
        degree[x] += 1
        degree[y] += 1
        if len(forest) == num_vertices - 1:
            break
    return sorted(forest)


@dataclass(frozen=True)
class ClusterStructure:
    membership: np.ndarray                 # camera (retained block) -> cluster
    num_clusters: int
    cluster_pairs: tuple[tuple[int, int], ...]
    neighbors: np.ndarray = field(repr=False)  # [k][2] forest neighbours of each cluster, -1 for none

    def kept(self, a: int, b: int) -> bool:
        ka, kb = int(self.membership[a]), int(self.membership[b])
        return ka == kb or kb in self.neighbors[ka]

    def block_pairs(self) -> tuple[tuple[int, int], ...]:
        """(b1, b2), b1 <= b2: the camera blocks the preconditioner keeps, in the
        reference's order (linear.py:974-979)."""
        n = self.membership.size
        out = []
        for a in range(n):
            for b in range(a, n):
                if self.kept(a, b):
                    out.append((a, b))
        return tuple(out)

    def components(self) -> list[np.ndarray]:
        """The connected groups of cameras of the kept pattern (clusters joined by forest
        edges), ascending camera ids each, ordered by their smallest camera: the kept
        matrix is block diagonal over them."""
        uf = _UnionFind(self.num_clusters)
        for a, b in self.cluster_pairs:
            uf.union(a, b)
        root = np.array([uf.find(int(k)) for k in self.membership], dtype=np.int64)
        groups: dict[int, list[int]] = {}
        for cam, r in enumerate(root.tolist()):
            groups.setdefault(r, []).append(cam)
        return [np.asarray(g, dtype=np.int64) for g in sorted(groups.values(), key=lambda g: g[0])]


def cluster_structure(visibility=None, *, tridiagonal: bool, clustering: str = CANONICAL_VIEWS,
                      incidence=None) -> ClusterStructure:
    """linear.py:953-990 (build_visibility_cluster_structure). ``visibility``: per
    camera, the points it sees; or ``incidence`` (incidence_from_observations)."""
    if incidence is None:
        incidence = _incidence(visibility)
    graph = visibility_graph(incidence)
    if clustering == SINGLE_LINKAGE:
        membership = single_linkage(graph)
    elif clustering == CANONICAL_VIEWS:
        membership = canonical_views(graph)
    else:
        raise ValueError(f"Unknown visibility clustering type: {clustering}")
    k = int(membership.max()) + 1 if membership.size else 0
    pairs = {(i, i) for i in range(k)}
    neighbors = np.full((k, 2), -1, dtype=np.int64)
    if tridiagonal and k > 1:
        forest = degree2_forest(k, cluster_graph(incidence, membership, k))
        for a, b in forest:
            pairs.add((a, b))
            neighbors[a, int(neighbors[a, 0] >= 0)] = b
            neighbors[b, int(neighbors[b, 0] >= 0)] = a
    return ClusterStructure(membership, k, tuple(sorted(pairs)), neighbors)
