"""The GPU Borůvka MST and core distances against the oracle (src/kdtree.rs, src/boruvka.rs).

The MST of a point set under mutual-reachability distance is unique up to
edges of equal weight: every MST has the same sorted weights.  So the GPU's
(non-reproducible mode) edges must span the points, their sorted weights must
equal the oracle's (reproducible Borůvka, itself pinned to the reference's
golden MST) within f32 rounding, and each edge's weight must be the mutual
reachability distance of its two points.  Core distances come from the same
f32 arithmetic as the reference's rdist and are compared within 1e-7.
"""
import numpy as np
import pytest

import evoc
from oracle import mst

pytestmark = pytest.mark.gpu


def _check(x, edges, core, min_samples, oracle_edges=None, oracle_core=None):
    n = len(x)
    assert edges.shape == (n - 1, 3)
    parent = list(range(n))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    a = edges[:, 0].astype(np.int64)
    b = edges[:, 1].astype(np.int64)
    for u, v in zip(a, b):
        ru, rv = find(int(u)), find(int(v))
        assert ru != rv, "cycle"
        parent[ru] = rv
    x64 = x.astype(np.float64)
    d2 = ((x64[a] - x64[b]) ** 2).sum(1)
    mr = np.sqrt(np.maximum(np.maximum(d2, core[a]), core[b]))
    assert np.abs(mr - edges[:, 2]).max() <= 1e-5 * max(1.0, float(mr.max()))
    if oracle_edges is not None:
        gw = np.sort(edges[:, 2].astype(np.float64))
        ow = np.sort(oracle_edges[:, 2].astype(np.float64))
        assert np.abs(gw - ow).max() <= 1e-6 * max(1.0, float(ow.max())), np.abs(gw - ow).max()
        assert abs(gw.sum() - ow.sum()) <= 1e-6 * ow.sum() + 1e-6
    if oracle_core is not None:
        assert np.abs(core - oracle_core).max() <= 1e-7 * max(1.0, float(oracle_core.max()))


def test_medium_800_golden_embedding():
    import os

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "lp_medium_800.npz"))
    x = z["embedding"].astype(np.float32)
    edges, core = evoc.parallel_boruvka(x, 5, return_core=True)
    _check(x, edges, core, 5, z["py_boruvka_edges"], z["py_core_distances"])


@pytest.mark.parametrize("n,dim,min_samples,seed", [(2, 3, 1, 0), (7, 2, 3, 1), (300, 5, 5, 2), (1000, 4, 5, 3),
                                                    (2500, 15, 10, 4), (4000, 7, 0, 5), (3000, 32, 5, 6),
                                                    (5000, 9, 1, 7)])
def test_random_points_against_oracle(n, dim, min_samples, seed):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(6, dim)) * 4
    x = (c[rng.integers(0, 6, n)] + rng.normal(size=(n, dim))).astype(np.float32)
    edges, core = evoc.parallel_boruvka(x, min_samples, return_core=True)
    oe, oc, _ = mst.boruvka_mst(x, min_samples=min_samples)
    _check(x, edges, core, min_samples, oe, oc)


def test_duplicates_and_grid_ties():
    """Many equal distances (a lattice with repeated points): only the weights are unique."""
    g = np.stack(np.meshgrid(np.arange(12), np.arange(12), np.arange(6)), -1).reshape(-1, 3).astype(np.float32)
    x = np.concatenate([g, g[:200]])  # 200 exact duplicates
    edges, core = evoc.parallel_boruvka(x, 5, return_core=True)
    oe, oc, _ = mst.boruvka_mst(x, min_samples=5)
    _check(x, edges, core, 5, oe, oc)


def test_large_clustered_embedding_weights_match_oracle():
    rng = np.random.default_rng(11)
    n, dim = 100_000, 7
    c = rng.normal(size=(40, dim)) * 3
    x = (c[rng.integers(0, 40, n)] + 0.5 * rng.normal(size=(n, dim))).astype(np.float32)
    edges, core = evoc.parallel_boruvka(x, 5, return_core=True)
    oe, oc, _ = mst.boruvka_mst(x, min_samples=5)
    _check(x, edges, core, 5, oe, oc)


def test_errors():
    with pytest.raises(evoc.EmptyData):
        evoc.parallel_boruvka(np.zeros((0, 3), np.float32))
    with pytest.raises(evoc.BackendError):
        evoc.parallel_boruvka(np.zeros((4, 3), np.float32), min_samples=5)  # n must exceed min_samples
    with pytest.raises(evoc.BackendError):
        evoc.parallel_boruvka(np.zeros((100, 40), np.float32))  # dim > 32
