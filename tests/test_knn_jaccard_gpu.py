"""Binary (UInt8 / Binary) exact forms on the GPU, bit-exact.

Two forms: `exact_int` expands the bits to 0/1 int8 rows and counts the
intersections on the tensor cores (tcgen05 kind::i8, s32 accumulation);
`popcount` runs AND + popcount over the packed words on the SIMT cores.
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


FORMS = ("exact_int", "popcount")


def opts(k, form="exact_int", **kw):
    return evoc.KnnGraphOptions(n_neighbors=k, form=form, **kw)


def _bits(n, nbytes, seed, protos=6, p_on=0.1, p_flip=0.05):
    rng = np.random.default_rng(seed)
    P = rng.random((protos, nbytes * 8)) < p_on
    rows = P[rng.integers(0, protos, n)] ^ (rng.random((n, nbytes * 8)) < p_flip)
    return np.packbits(rows, axis=1)


def _check(x, k, form):
    ind, dst, raw = evoc.knn_graph(x, opts(k, form), None, return_raw=True)
    kk = max(1, min(k, len(x) - 1))
    ei, er = O.exact_knn(x, kk)
    ed = O.transform(O.DT_U8, er)
    assert np.array_equal(ind, ei)
    assert np.array_equal(raw.view(np.uint32), er.view(np.uint32))
    assert np.array_equal(dst.view(np.uint32), ed.view(np.uint32))
    return ind, dst


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("n,nbytes,k", [(2, 1, 1), (9, 3, 10), (129, 16, 15), (300, 33, 20), (1000, 128, 15),
                                        (700, 64, 64), (257, 200, 7), (3000, 128, 15)])
def test_jaccard_bit_exact(n, nbytes, k, form):
    ind, dst = _check(_bits(n, nbytes, n + nbytes), k, form)
    # every row holds itself; rows at Jaccard 1 (self and exact duplicates,
    # ordered by index) carry -0.0 = -log2(1.0)
    assert all(r in ind[r] for r in range(n))
    assert np.all(np.signbit(dst[ind == np.arange(n)[:, None]]))


@pytest.mark.parametrize("form", FORMS)
def test_jaccard_zero_rows_duplicates_and_ties(form):
    x = _bits(400, 16, 11)
    x[5] = 0
    x[6] = 0          # two empty rows: union 0 -> raw +0.0 between them
    x[40:60] = x[39]  # duplicates: Jaccard 1 ties broken by index
    x[100] = 0xFF
    _check(x, 25, form)


@pytest.mark.parametrize("form", FORMS)
def test_jaccard_sparse_rows(form):
    # few bits per row: many equal small Jaccard values and empty intersections
    rng = np.random.default_rng(4)
    x = np.packbits(rng.random((600, 256)) < 0.01, axis=1)
    _check(x, 20, form)


def test_jaccard_forms_agree():
    x = _bits(2500, 96, 21, protos=40)
    a = evoc.knn_graph(x, opts(15, "exact_int"))
    b = evoc.knn_graph(x, opts(15, "popcount"))
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


@pytest.mark.parametrize("form", FORMS)
def test_jaccard_row_slice(form):
    x = _bits(900, 32, 5)
    full_i, full_d = evoc.knn_graph(x, opts(12, form))
    si, sd = evoc.knn_graph(x, opts(12, form, row_begin=300, row_end=650))
    assert np.array_equal(si, full_i[300:650])
    assert np.array_equal(sd.view(np.uint32), full_d[300:650].view(np.uint32))
