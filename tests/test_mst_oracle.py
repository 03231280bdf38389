"""The KD-tree / Borůvka MST oracle pinned to the reference's golden intermediates.

medium_800's fixtures hold what Python EVoC computed on its final node
embedding when building the cluster layers (build_cluster_layers,
src/clustering.rs:28-110): the KD-tree's index order (leaf size 40), the core
distances (squared distance to the 5th neighbour, self included in the query)
and the Borůvka MST edges (tests/fixtures/medium_800/intermediates/
py_*.npy; src/np_argsort.rs:286-300 reads the edges).
"""
import os

import numpy as np

from oracle import mst

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _z():
    return np.load(os.path.join(GOLDEN, "lp_medium_800.npz"))


def test_kdtree_index_order_medium_800():
    z = _z()
    t = mst.build_kdtree(z["embedding"], 40)
    assert np.array_equal(t["idx_array"], z["py_kdtree_idx_array"])
    # every node's points lie inside its bounds; children split the parent's range
    for node in range(len(t["idx_start"])):
        s, e = t["idx_start"][node], t["idx_end"][node]
        pts = z["embedding"][t["idx_array"][s:e]]
        assert (pts >= t["lo"][node]).all() and (pts <= t["hi"][node]).all()


def test_core_distances_and_mst_edges_medium_800():
    z = _z()
    edges, core, idx = mst.boruvka_mst(z["embedding"], min_samples=5)
    assert np.array_equal(idx, z["py_kdtree_idx_array"])
    assert np.abs(core - z["py_core_distances"]).max() <= 1e-7
    want = z["py_boruvka_edges"]
    assert edges.shape == want.shape == (799, 3)
    # same edges, found in the same order, distances within f32 rounding
    assert np.array_equal(edges[:, :2], want[:, :2])
    assert np.abs(edges[:, 2] - want[:, 2]).max() <= 1e-6


def test_mst_spans_and_is_minimal_on_random_points():
    """On random low-dimensional points: n - 1 edges joining every point, and a total weight no
    larger than Prim's algorithm gives for the same mutual-reachability distances."""
    rng = np.random.default_rng(3)
    x = rng.normal(size=(300, 5)).astype(np.float32)
    edges, core, _ = mst.boruvka_mst(x, min_samples=5)
    assert edges.shape == (299, 3)
    parent = list(range(300))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for a, b, _ in edges:
        parent[find(int(a))] = find(int(b))
    assert len({find(i) for i in range(300)}) == 1
    d2 = ((x[:, None, :].astype(np.float64) - x[None, :, :]) ** 2).sum(-1)
    mr = np.sqrt(np.maximum(np.maximum(d2, core[:, None]), core[None, :]))
    inside = np.zeros(300, bool)
    inside[0] = True
    best = mr[0].copy()
    total = 0.0
    for _ in range(299):
        best[inside] = np.inf
        j = int(np.argmin(best))
        total += best[j]
        inside[j] = True
        best = np.minimum(best, mr[j])
    assert abs(edges[:, 2].astype(np.float64).sum() - total) <= 1e-4 * total
