"""Tensor-core forms on the GPU (tcgen05), through the C ABI.

  bf16_rerank (f32 input): BF16 scan keeps 2k candidates, FP32 rerank from the
      original rows.  Against the goldens it must meet the reference's parity
      rules (tests/parity.rs:34-68); against the oracle recall@k >= 0.99 and
      every reported distance within 1e-6 of the oracle's for the same pair.
  exact_int (i8 input): int8 dot products with s32 accumulation; indices and
      distances bit-exact to the oracle's exact selection
      (src/nndescent/int8.rs:15-21, src/knn.rs:173-176).
"""
import numpy as np
import pytest

import evoc
from conftest import FIXTURES, assert_knn_parity
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def bf16(k, **kw):
    return evoc.KnnGraphOptions(n_neighbors=k, form="bf16_rerank", **kw)


def exact_int(k, **kw):
    return evoc.KnnGraphOptions(n_neighbors=k, form="exact_int", **kw)


@pytest.mark.parametrize("name", FIXTURES)
def test_bf16_rerank_matches_golden(golden, name):
    z = golden[name]
    rng = np.random.RandomState(int(z["seed"]))
    ind, dst = evoc.knn_graph(z["data"], bf16(15, deterministic=True), rng)
    assert_knn_parity(ind, dst, z["nn_inds"], z["nn_dists"])
    assert np.array_equal(rng.get_state()[1], z["rng_after_knn_key"])
    assert np.all(ind[:, 0] == np.arange(len(ind)))


def _recall_and_dist_check(x, k, ind, raw):
    """Recall against the oracle's exact selection, and every reported raw
    dissimilarity within 1e-6 of the FP64 value for that pair."""
    xn = O.prepare_float(x)
    kk = max(1, min(k, len(x) - 1))
    ei, er = O.exact_knn(xn, kk)
    hits = 0
    x64 = xn.astype(np.float64)
    for r in range(len(x)):
        hits += len(set(ind[r].tolist()) & set(ei[r].tolist()))
        dots = x64[ind[r]] @ x64[r]
        want = np.where(dots > 0, -dots, 1.17549435e-38)
        want[ind[r] == r] = -1.0
        err = np.abs(raw[r].astype(np.float64) - want)
        assert err.max() <= 1e-6, (r, err.max())
    return hits / ei.size


@pytest.mark.parametrize("n,d,k", [(2, 3, 1), (5, 64, 10), (129, 33, 15), (300, 128, 30), (1000, 100, 15),
                                   (513, 770, 20), (2000, 256, 64)])
def test_bf16_rerank_random_shapes(n, d, k):
    rng = np.random.default_rng(n + 7 * d)
    c = rng.standard_normal((6, d))
    x = (c[rng.integers(0, 6, n)] + 0.25 * rng.standard_normal((n, d))).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    ind, dst, raw = evoc.knn_graph(x, bf16(k), None, return_raw=True)
    rec = _recall_and_dist_check(x, k, ind, raw)
    assert rec >= 0.99, rec
    assert np.all(np.diff(raw, axis=1) >= -1e-6)


def test_bf16_rerank_blobs_2k_128_recall_one():
    from evoc import synthetic

    x = synthetic.blobs_2k_128()
    ind, dst, raw = evoc.knn_graph(x, bf16(15), None, return_raw=True)
    assert _recall_and_dist_check(x, 15, ind, raw) == 1.0


def test_bf16_rerank_locality_path_matches_fp32_form():
    # n >= 65536 takes the pivot-ordered rerank; compare with the FP32 form.
    from evoc import synthetic

    x = synthetic.zipf_f32(n=70000, dim=64, clusters=50, seed=3)
    ia, da = evoc.knn_graph(x, bf16(15))
    ib, db = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=15, form="fp32"))
    rec = np.mean([len(set(ia[r]) & set(ib[r])) / 15 for r in range(0, len(x), 7)])
    assert rec >= 0.99, rec
    same = ia == ib
    assert np.all(np.abs(da[same] - db[same]) <= 1e-6)


def _int8_data(n, d, seed, clusters=8, scale=127):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((clusters, d))
    x = c[rng.integers(0, clusters, n)] + 0.3 * rng.standard_normal((n, d))
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return np.clip(np.round(scale * x), -127, 127).astype(np.int8)


@pytest.mark.parametrize("n,d,k", [(2, 3, 1), (7, 16, 10), (129, 33, 15), (300, 128, 30), (1000, 384, 15),
                                   (600, 1000, 12), (700, 130, 64)])
def test_int8_exact_bit_exact(n, d, k):
    x = _int8_data(n, d, n + d)
    ind, dst, raw = evoc.knn_graph(x, exact_int(k), None, return_raw=True)
    kk = max(1, min(k, n - 1))
    ei, er = O.exact_knn(x, kk)
    ed = O.transform(O.DT_I8, er)
    assert np.array_equal(ind, ei)
    assert np.array_equal(raw.view(np.uint32), er.view(np.uint32))
    assert np.array_equal(dst.view(np.uint32), ed.view(np.uint32))


def test_int8_heavy_ties_and_duplicates():
    rng = np.random.default_rng(9)
    x = rng.integers(-2, 3, (500, 24)).astype(np.int8)  # tiny value range -> many equal dots
    x[100:120] = x[99]
    x[7] = 0
    ind, dst, raw = evoc.knn_graph(x, exact_int(20), None, return_raw=True)
    ei, er = O.exact_knn(x, 20)
    assert np.array_equal(ind, ei)
    assert np.array_equal(raw.view(np.uint32), er.view(np.uint32))


def test_int8_rng_contract_and_errors():
    x = _int8_data(50, 16, 1)
    rng = np.random.RandomState(3)
    evoc.knn_graph(x, exact_int(5, deterministic=True), rng)
    ref = np.random.RandomState(3)
    for _ in range(15):
        ref.randint(-(2**31) + 1, 2**31 - 2)
    assert rng.randint(0, 1 << 30) == ref.randint(0, 1 << 30)
    with pytest.raises(evoc.InvalidNeighbors):
        evoc.knn_graph(x, exact_int(0))
