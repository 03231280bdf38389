"""Binary (UInt8 / Binary) exact form on the GPU: popcount Jaccard, bit-exact.

The dissimilarity is the reference's -(inter/union) with f32 division and 0.0
for an empty union (src/nndescent/uint8.rs:21-35); the transform is
-log2 in f64 (src/knn.rs:178-187), so self comes out as -0.0.  Indices, raw
bits and transformed-distance bits must equal the oracle's exact selection.
"""
import numpy as np
import pytest

import evoc
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def opts(k, **kw):
    return evoc.KnnGraphOptions(n_neighbors=k, form="exact_int", **kw)


def _bits(n, nbytes, seed, protos=6, p_on=0.1, p_flip=0.05):
    rng = np.random.default_rng(seed)
    P = rng.random((protos, nbytes * 8)) < p_on
    rows = P[rng.integers(0, protos, n)] ^ (rng.random((n, nbytes * 8)) < p_flip)
    return np.packbits(rows, axis=1)


def _check(x, k):
    ind, dst, raw = evoc.knn_graph(x, opts(k), None, return_raw=True)
    kk = max(1, min(k, len(x) - 1))
    ei, er = O.exact_knn(x, kk)
    ed = O.transform(O.DT_U8, er)
    assert np.array_equal(ind, ei)
    assert np.array_equal(raw.view(np.uint32), er.view(np.uint32))
    assert np.array_equal(dst.view(np.uint32), ed.view(np.uint32))
    return ind, dst


@pytest.mark.parametrize("n,nbytes,k", [(2, 1, 1), (9, 3, 10), (129, 16, 15), (300, 33, 20), (1000, 128, 15),
                                        (700, 64, 64), (257, 200, 7)])
def test_jaccard_bit_exact(n, nbytes, k):
    ind, dst = _check(_bits(n, nbytes, n + nbytes), k)
    # every row holds itself; rows at Jaccard 1 (self and exact duplicates,
    # ordered by index) carry -0.0 = -log2(1.0)
    assert all(r in ind[r] for r in range(n))
    assert np.all(np.signbit(dst[ind == np.arange(n)[:, None]]))


def test_jaccard_zero_rows_duplicates_and_ties():
    x = _bits(400, 16, 11)
    x[5] = 0
    x[6] = 0          # two empty rows: union 0 -> raw +0.0 between them
    x[40:60] = x[39]  # duplicates: Jaccard 1 ties broken by index
    x[100] = 0xFF
    _check(x, 25)


def test_jaccard_row_slice():
    x = _bits(900, 32, 5)
    full_i, full_d = evoc.knn_graph(x, opts(12))
    si, sd = evoc.knn_graph(x, opts(12, row_begin=300, row_end=650))
    assert np.array_equal(si, full_i[300:650])
    assert np.array_equal(sd.view(np.uint32), full_d[300:650].view(np.uint32))
