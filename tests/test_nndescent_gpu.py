"""GPU NN-descent form (EVOC_FORM_NNDESCENT), checked by recall.

The reference's kNN is NN-descent (src/nndescent/*.rs); the GPU form is an
NN-descent too, so it is held to recall@k against exact neighbours (FP64 for
f32, the oracle's exact integer selection for i8 / binary), reported next to
the reference NN-descent's own recall (the oracle's restatement) on the same
data.  Distances it reports must be the true dissimilarities of the pairs
(f32: within 1e-6 of FP64 after the FP32 rerank; integer forms: bit-exact).
"""
import numpy as np
import pytest

import evoc
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def nnd(k, **kw):
    return evoc.KnnGraphOptions(n_neighbors=k, form="nndescent", **kw)


def _recall(ind, truth):
    return np.mean([len(set(ind[r]) & set(truth[r])) / truth.shape[1] for r in range(len(ind))])


def test_nndescent_f32_recall_and_exact_distances():
    from evoc import synthetic

    x = synthetic.blobs(n_per=600, centres=10, dim=64, noise=0.3, seed=9)
    k = 15
    ind, dst, raw = evoc.knn_graph(x, nnd(k), np.random.RandomState(3), return_raw=True)
    ei, er = O.exact_knn(x, k)
    rec = _recall(ind, ei)
    ref_ind, _ = O.knn_graph(x, k, O.RandomState(3), deterministic=False, n_threads=4)
    ref_rec = _recall(ref_ind, ei)
    print(f"GPU NN-descent recall {rec:.4f}, reference NN-descent recall {ref_rec:.4f}")
    assert rec >= 0.95 and rec >= ref_rec - 0.02
    x64 = x.astype(np.float64)
    dots = np.einsum("rkd,rd->rk", x64[ind], x64)
    want = np.where(dots > 0, -dots, 1.17549435e-38)
    want[ind == np.arange(len(x))[:, None]] = -1.0
    assert np.abs(raw - want).max() <= 1e-6
    assert np.all(ind[:, 0] == np.arange(len(x)))


def test_nndescent_deterministic():
    from evoc import synthetic

    x = synthetic.blobs(n_per=300, centres=8, dim=48, seed=2)
    a = evoc.knn_graph(x, nnd(10), np.random.RandomState(5))
    b = evoc.knn_graph(x, nnd(10), np.random.RandomState(5))
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def _int8(n, d, seed):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((12, d))
    v = c[rng.integers(0, 12, n)] + 0.3 * rng.standard_normal((n, d))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return np.clip(np.round(127 * v), -127, 127).astype(np.int8)


def test_nndescent_int8_recall_exact_values():
    x = _int8(4000, 96, 1)
    k = 12
    ind, dst, raw = evoc.knn_graph(x, nnd(k), np.random.RandomState(1), return_raw=True)
    ei, er = O.exact_knn(x, k)
    hits = np.mean([np.sum(raw[r] <= er[r][-1]) / k for r in range(len(x))])
    assert hits >= 0.95
    for r in range(0, len(x), 97):
        for j in range(k):
            c = ind[r, j]
            want = -1.0 if c == r else O.distance(x, r, c)
            assert raw[r, j] == np.float32(want)


def test_nndescent_binary_recall_exact_values():
    rng = np.random.default_rng(4)
    P = rng.random((20, 512)) < 0.1
    rows = P[rng.integers(0, 20, 3000)] ^ (rng.random((3000, 512)) < 0.05)
    x = np.packbits(rows, axis=1)
    k = 10
    ind, dst, raw = evoc.knn_graph(x, nnd(k), np.random.RandomState(2), return_raw=True)
    ei, er = O.exact_knn(x, k)
    hits = np.mean([np.sum(raw[r] <= er[r][-1]) / k for r in range(len(x))])
    assert hits >= 0.9
    for r in range(0, len(x), 89):
        for j in range(k):
            c = ind[r, j]
            want = -1.0 if c == r else O.distance(x, r, c)
            assert raw[r, j] == np.float32(want)


@pytest.mark.parametrize("k", [40, 64])
def test_nndescent_k_above_32(k):
    """Lists of up to 64 neighbours (two keys per lane)."""
    from evoc import synthetic

    x = synthetic.blobs(n_per=500, centres=8, dim=48, noise=0.3, seed=4)
    ind, dst, raw = evoc.knn_graph(x, nnd(k), np.random.RandomState(3), return_raw=True)
    ei, er = O.exact_knn(x, k)
    rec = _recall(ind, ei)
    assert rec >= 0.95, rec
    assert np.all(ind[:, 0] == np.arange(len(x)))
    assert np.all(np.diff(raw, axis=1) >= -1e-6)
    assert all(len(set(r)) == k for r in ind)  # no index twice in a row


def test_nndescent_options_max_candidates_and_delta_improv():
    """max_candidates bounds the sampled candidates (fewer candidates: recall can only drop a little,
    never the exactness of reported pairs); a large delta_improv stops after fewer iterations."""
    from evoc import _lib, synthetic

    x = synthetic.blobs(n_per=400, centres=10, dim=32, noise=0.3, seed=6)
    ei, _ = O.exact_knn(x, 15)
    ctx = _lib.context(0)
    a, _ = evoc.knn_graph(x, nnd(15, max_candidates=4), np.random.RandomState(1))
    b, _ = evoc.knn_graph(x, nnd(15), np.random.RandomState(1))
    assert _recall(b, ei) >= 0.95 and _recall(a, ei) >= 0.5
    ctx.profile(True)  # stage records count the iterations
    evoc.knn_graph(x, nnd(15, delta=0.0, delta_improv=0.0, n_iters=8), np.random.RandomState(1))
    full = [nm for nm, _ in ctx.stages()].count("nnd_iteration")
    evoc.knn_graph(x, nnd(15, delta=0.0, delta_improv=0.5, n_iters=8), np.random.RandomState(1))
    early = [nm for nm, _ in ctx.stages()].count("nnd_iteration")
    # delta_improv = 0.5: the second iteration's sum moves by far less than half, so it stops there
    assert early == 2 and full > early, (full, early)


def test_nndescent_rejects_unsupported():
    x = np.random.default_rng(0).standard_normal((100, 16)).astype(np.float32)
    with pytest.raises(evoc.BackendError):
        evoc.knn_graph(x, nnd(5, row_begin=0, row_end=50))


def test_nndescent_large_k_takes_the_exact_form():
    # above k = 64 the NN-descent request is built by the dtype's exact form
    rng = np.random.default_rng(3)
    x = rng.standard_normal((400, 24)).astype(np.float32)
    a = evoc.knn_graph(x, nnd(80), np.random.RandomState(0))
    b = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=80, form="half_rerank"))
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    xi = np.clip(np.round(40 * rng.standard_normal((300, 32))), -127, 127).astype(np.int8)
    a = evoc.knn_graph(xi, nnd(70), np.random.RandomState(0))
    b = evoc.knn_graph(xi, evoc.KnnGraphOptions(n_neighbors=70, form="exact_int"))
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_nndescent_f32_recall_at_60k_rows():
    """A larger graph (60,000 rows of 40 overlapping clusters, k = 20): recall against the exact
    graph (the FP32 form, itself held to the oracle) above a floor, and on the first 10,000 rows at
    least the reference NN-descent's there (the oracle's restatement), less 0.02."""
    rng = np.random.default_rng(17)
    d, k = 48, 20
    c = rng.standard_normal((40, d))
    x = (c[rng.integers(0, 40, 60000)] + 0.6 * rng.standard_normal((60000, d))).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    ind, _ = evoc.knn_graph(x, nnd(k), np.random.RandomState(4))
    ei, _ = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=k, form="fp32"))
    rec = _recall(ind, ei)
    xs = x[:10000]
    ref_ind, _ = O.knn_graph(xs, k, O.RandomState(4), deterministic=False, n_threads=8)
    es, _ = O.exact_knn(xs, k)
    ref_rec = _recall(ref_ind, es)
    sub, _ = evoc.knn_graph(xs, nnd(k), np.random.RandomState(4))
    print(f"GPU NN-descent recall {rec:.4f} (60,000 rows), {_recall(sub, es):.4f} (10,000); "
          f"reference {ref_rec:.4f} (10,000)")
    assert rec >= 0.8 and _recall(sub, es) >= ref_rec - 0.02
