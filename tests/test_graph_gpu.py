"""Fuzzy-graph epilogue on the GPU against the reference goldens and the oracle.

  smooth_knn_dist vs sigmas_py / rhos_py (tests/graph_parity.rs:28-62, <= 1e-6)
  fuzzy union of the golden kNN vs graph_csr: identical indptr/indices, data
      within 1e-6 (tests/graph_parity.rs:64-90, tests/parity.rs:191-232)
  the oracle on other inputs: identical pattern, weights within 1e-5 relative
"""
import numpy as np
import pytest

import evoc
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_smooth_knn_dist_matches_python(golden):
    z = golden["medium_800"]
    s, r = evoc.smooth_knn_dist(z["nn_dists"], 15.0)
    assert np.abs(s - z["sigmas_py"]).max() < 1e-6
    assert np.abs(r - z["rhos_py"]).max() < 1e-6


@pytest.mark.parametrize("name", ["medium_800", "large_2000"])
def test_fuzzy_graph_matches_golden_csr(golden, name):
    z = golden[name]
    ip, ix, dv, _, _ = evoc.neighbor_graph_csr(15.0, z["nn_inds"], z["nn_dists"])
    assert np.array_equal(ip, z["graph_csr_indptr"])
    assert np.array_equal(ix, z["graph_csr_indices"])
    assert np.abs(dv - z["graph_csr_data"]).max() <= 1e-6


def _compare_with_oracle(ind, dst, kf, symmetrize=True):
    ip, ix, dv, s, r = evoc.neighbor_graph_csr(kf, ind, dst, symmetrize)
    oip, oix, odv, os_, or_ = O.fuzzy_graph(ind, dst, kf, symmetrize)
    assert np.array_equal(ip, oip)
    assert np.array_equal(ix, oix)
    assert np.all(np.abs(dv - odv) <= 1e-5 * np.maximum(np.abs(odv), 1e-30))
    assert np.abs(s - os_).max() <= 1e-6 * max(1.0, np.abs(os_).max())
    assert np.array_equal(r, or_)


def test_fuzzy_graph_on_gpu_knn_output():
    from evoc import synthetic

    x = synthetic.blobs(n_per=300, centres=10, dim=64, seed=5)
    ind, dst = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=15, form="fp32"))
    _compare_with_oracle(ind, dst, 15.0)
    _compare_with_oracle(ind, dst, 15.0, symmetrize=False)


def test_fuzzy_graph_duplicate_rows_use_global_mean():
    # rows whose distances are all zero have rho == 0 and take the floor from
    # the mean of all distances (ndarray's f32 mean)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((600, 24)).astype(np.float32)
    x[100:140] = x[99]
    ind, dst = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=20, form="fp32"))
    assert np.any(np.all(dst == 0.0, axis=1))
    _compare_with_oracle(ind, dst, 20.0)


def test_fuzzy_graph_int8_and_binary_knn():
    rng = np.random.default_rng(8)
    xi = np.clip(np.round(127 * rng.standard_normal((500, 32)) / 6), -127, 127).astype(np.int8)
    ind, dst = evoc.knn_graph(xi, evoc.KnnGraphOptions(n_neighbors=12, form="exact_int"))
    _compare_with_oracle(ind, dst, 12.0)
    xb = np.packbits(rng.random((500, 256)) < 0.2, axis=1)
    ind, dst = evoc.knn_graph(xb, evoc.KnnGraphOptions(n_neighbors=12, form="exact_int"))
    _compare_with_oracle(ind, dst, 12.0)


def test_fuzzy_graph_hub_columns():
    # Hub rows that are neighbours of thousands of rows: the transpose's column
    # buckets take the warp sort (small), the block sort (3,000 entries) and
    # the single-thread fallback (> 8,192 entries).
    n, k = 12000, 10
    rng = np.random.default_rng(12)
    ind = np.empty((n, k), np.int32)
    for i in range(n):
        row = [i, 0]
        if i < 3000:
            row.append(1)
        while len(row) < k:
            c = int(rng.integers(2, n))
            if c != i and c not in row:
                row.append(c)
        ind[i] = row[:k]
    ind[0, 1] = 5  # row 0 cannot list itself twice
    dst = np.sort(rng.random((n, k)).astype(np.float32) * 2.0, axis=1)
    dst[:, 0] = 0.0
    _compare_with_oracle(ind, dst, 10.0)


def test_fuzzy_graph_large_k():
    # k = 150 (no k limit, as smooth_knn_dist has none): rows keep their
    # membership entries in column order in place
    from evoc import synthetic

    x = synthetic.blobs(n_per=100, centres=8, dim=32, seed=9)
    ind, dst = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=150, form="fp32"))
    assert ind.shape == (800, 150)
    _compare_with_oracle(ind, dst, 150.0)
    _compare_with_oracle(ind, dst, 150.0, symmetrize=False)
