"""The 16-bit tensor-core form's per-row certificate (rerank.cu) and its rescans.

On tight clusters the scan's rounding is larger than the gaps between
neighbours, so oversampling 2k candidates alone silently drops true
neighbours (checked below with the BF16 operands and the certificate off, the
form as it stood before).  With the certificate every row is either proven to
hold its k nearest among the candidates (within the 1e-6 tie tolerance of the
exact FP32 form) or rescanned -- with 256 candidates, then exactly in FP32 --
so the result must equal the exact neighbour sets up to ties within 1e-6.
"""
import numpy as np
import pytest

import evoc
from evoc import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def tight_clusters(n, d, clusters, sigma, seed):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((clusters, d))
    x = c[rng.integers(0, clusters, n)] + sigma * rng.standard_normal((n, d))
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return x.astype(np.float32)


def misses_beyond_ties(x, ind, k, tol=1e-6):
    """Entries of the exact k nearest (FP64, self first) missing from `ind` whose dissimilarity is
    more than `tol` better than the k-th, plus reported keys more than `tol` worse than the k-th."""
    x64 = O.prepare_float(x).astype(np.float64)
    n = len(x)
    bad = 0
    for r0 in range(0, n, 512):
        r1 = min(n, r0 + 512)
        s = x64[r0:r1] @ x64.T
        raw = np.where(s > 0, -s, 1.17549435e-38)
        raw[np.arange(r1 - r0), np.arange(r0, r1)] = -1.0
        part = np.argpartition(raw, k - 1, axis=1)[:, :k]
        kth = np.take_along_axis(raw, part, 1).max(axis=1)
        for i in range(r1 - r0):
            got = ind[r0 + i]
            want = set(part[i].tolist())
            for j in want - set(got.tolist()):
                bad += raw[i, j] < kth[i] - tol
            bad += int(np.sum(raw[i, got] > kth[i] + tol))
    return int(bad)


def half(k, **kw):
    return evoc.KnnGraphOptions(n_neighbors=k, form="bf16_rerank", **kw)


@pytest.mark.parametrize("sigma", [0.01, 0.03])
def test_tight_clusters_fail_without_certificate_and_pass_with_it(sigma):
    n, d, k = 3000, 128, 15
    x = tight_clusters(n, d, 10, sigma, 1)
    ind_old, _ = evoc.knn_graph(x, half(k, scan_type="bf16", certify=False))
    assert misses_beyond_ties(x, ind_old, k) > n * k // 100  # the uncertified BF16 form loses neighbours
    ctx = _lib.context(0)
    for scan in ("fp16", "bf16"):
        ind, dst, raw = evoc.knn_graph(x, half(k, scan_type=scan), return_raw=True)
        counts = ctx.certify_counts()
        assert counts["checked"] == n and counts["second_pass"] > 0, counts
        assert misses_beyond_ties(x, ind, k) == 0, (scan, counts)
        assert np.all(ind[:, 0] == np.arange(n))
        assert np.all(np.diff(raw, axis=1) >= -1e-6)


def test_certificate_matches_oracle_exact_selection():
    """Certified rows and rescanned rows together against the oracle's exact FP32 selection."""
    n, d, k = 2000, 64, 10
    x = tight_clusters(n, d, 8, 0.02, 4)
    ind, dst, raw = evoc.knn_graph(x, half(k), return_raw=True)
    ei, er = O.exact_knn(O.prepare_float(x), k)
    same = ind == ei
    # a differing entry is a tie: within 1e-6 of the oracle's value at that position
    assert np.all(np.abs(raw[~same].astype(np.float64) - er[~same].astype(np.float64)) <= 1e-6)
    assert np.all(np.abs(raw.astype(np.float64) - er.astype(np.float64)) <= 1e-6)


def test_benign_clusters_certify_without_rescans():
    """Well-separated data: nearly every row is proven at the first pass (a broken bound would send
    every row to the rescans and still pass the exactness tests)."""
    rng = np.random.default_rng(3)
    n, d, k = 4000, 256, 15
    c = rng.standard_normal((6, d))
    x = (c[rng.integers(0, 6, n)] + 0.25 * rng.standard_normal((n, d))).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    evoc.knn_graph(x, half(k))
    counts = _lib.context(0).certify_counts()
    assert counts["checked"] == n
    assert counts["second_pass"] <= n // 20, counts


def test_all_keys_candidates_is_certified_and_row_slices():
    x = tight_clusters(50, 32, 2, 0.01, 2)
    ind, _ = evoc.knn_graph(x, half(30))  # C = min(60, n) = n: every key is a candidate
    assert _lib.context(0).certify_counts()["second_pass"] == 0
    assert misses_beyond_ties(x, ind, 30) == 0
    y = tight_clusters(3000, 96, 10, 0.01, 5)
    full, _ = evoc.knn_graph(y, half(12))
    part, _ = evoc.knn_graph(y, half(12, row_begin=700, row_end=2300))
    assert _lib.context(0).certify_counts()["checked"] == 1600
    # rescanned rows of a slice land in the slice's own output rows
    assert misses_beyond_ties(y, full, 12) == 0
    diff = part != full[700:2300]
    x64 = y.astype(np.float64)
    for r, c in zip(*np.nonzero(diff)):
        a = x64[700 + r] @ x64[part[r, c]]
        b = x64[700 + r] @ x64[full[700 + r, c]]
        assert abs(a - b) <= 1e-6


def test_batch_rescans_match_single_calls():
    xs = [tight_clusters(n, d, 6, 0.01, s) for n, d, s in ((1500, 64, 1), (700, 128, 2), (2500, 96, 3))]
    opts = half(15)
    got = evoc.knn_graph_batch(xs, opts)
    assert _lib.context(0).certify_counts()["second_pass"] > 0
    for x, (bi, bd) in zip(xs, got):
        si, sd = evoc.knn_graph(x, opts)
        assert np.array_equal(bi, si)
        assert np.array_equal(bd.view(np.uint32), sd.view(np.uint32))


def test_half_form_beyond_256_candidates_is_exact():
    # oversample * k > 256 (k = 150): every row takes the exact FP32 scan
    rng = np.random.default_rng(21)
    x = rng.standard_normal((700, 40)).astype(np.float32)
    a = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=150, form="half_rerank"))
    b = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=150, form="fp32"))
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_few_failed_rows_take_the_split_exact_pass():
    """A few rows fail (planted near-duplicate groups in benign data): they go straight to the exact
    FP32 pass with the keys split over the SMs, and match the oracle's exact selection."""
    rng = np.random.default_rng(9)
    n, d, k = 12000, 64, 15
    c = rng.standard_normal((6, d))
    x = (c[rng.integers(0, 6, n)] + 0.25 * rng.standard_normal((n, d))).astype(np.float32)
    for t in range(6):
        base = x[t * 1000]
        x[t * 1000 + 1:t * 1000 + 25] = base + 1e-4 * rng.standard_normal((24, d)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    ind, dst, raw = evoc.knn_graph(x, half(k), return_raw=True)
    counts = _lib.context(0).certify_counts()
    assert 0 < counts["second_pass"] <= 1000 and counts["exact_rescan"] == counts["second_pass"], counts
    ei, er = O.exact_knn(O.prepare_float(x), k)
    same = ind == ei
    assert np.all(np.abs(raw[~same].astype(np.float64) - er[~same].astype(np.float64)) <= 1e-6)
    assert np.all(np.abs(raw.astype(np.float64) - er.astype(np.float64)) <= 1e-6)
