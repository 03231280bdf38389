"""The reference's integer brute-force branch (src/knn.rs:189-281,418-421) on the GPU.

With n <= brute_force_max_n, i8 and u8 data skip NN-descent: every row's k
nearest (self excluded) come out in the reference's max-heap order, so the
raw heap arrays, the indices and the transformed distances must equal the
oracle's brute_force_knn bit for bit -- which is also what lets the Cuda
backend honour strict_precision for these calls.
"""
import numpy as np
import pytest

import evoc
from evoc import backend as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _i8(n, d, seed, clusters=6):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((clusters, d))
    x = c[rng.integers(0, clusters, n)] + 0.4 * rng.standard_normal((n, d))
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return np.clip(np.round(127 * x), -127, 127).astype(np.int8)


def _u8(n, nbytes, seed, protos=8):
    rng = np.random.default_rng(seed)
    P = rng.random((protos, nbytes * 8)) < 0.15
    rows = P[rng.integers(0, protos, n)] ^ (rng.random((n, nbytes * 8)) < 0.05)
    return np.packbits(rows, axis=1)


@pytest.mark.parametrize("kind,n,d,k", [("i8", 2, 3, 1), ("i8", 300, 40, 15), ("i8", 1500, 130, 31),
                                        ("i8", 700, 384, 64), ("u8", 2, 4, 1), ("u8", 500, 16, 15),
                                        ("u8", 1200, 128, 30), ("u8", 257, 3, 7)])
def test_brute_force_heap_order_bit_exact(kind, n, d, k):
    x = _i8(n, d, n + d) if kind == "i8" else _u8(n, d, n + d)
    opts = evoc.KnnGraphOptions(n_neighbors=k, brute_force_max_n=n)
    rng = np.random.RandomState(5)
    ind, dst, raw = evoc.knn_graph(x, opts, rng, return_raw=True)
    oi, orr = O.brute_force_knn(x, k)
    dt = O.DT_I8 if kind == "i8" else O.DT_U8
    assert np.array_equal(ind, oi)
    assert np.array_equal(raw.view(np.uint32), orr.view(np.uint32))
    assert np.array_equal(dst.view(np.uint32), O.transform(dt, orr).view(np.uint32))
    assert np.all(ind != np.arange(len(x))[:, None])  # self excluded
    # only randint3_for_tau is drawn: the brute-force branch builds no forest (src/knn.rs:416-421)
    ref = np.random.RandomState(5)
    for _ in range(3):
        ref.randint(-(2**31) + 1, 2**31 - 2)
    assert np.array_equal(rng.get_state()[1], ref.get_state()[1]) and rng.get_state()[2] == ref.get_state()[2]


def test_brute_force_ties_and_duplicates_keep_the_reference_heap():
    rng = np.random.default_rng(11)
    x = rng.integers(-2, 3, (400, 24)).astype(np.int8)  # tiny value range -> many equal dots
    x[50:70] = x[49]
    x[3] = 0
    ind, dst, raw = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=20, brute_force_max_n=10**6),
                                   return_raw=True)
    oi, orr = O.brute_force_knn(x, 20)
    assert np.array_equal(ind, oi) and np.array_equal(raw.view(np.uint32), orr.view(np.uint32))
    xu = np.zeros((64, 8), np.uint8)  # empty rows: union 0 -> 0.0
    xu[10:20, 0] = 0xF0
    ind, dst, raw = evoc.knn_graph(xu, evoc.KnnGraphOptions(n_neighbors=9, brute_force_max_n=64), return_raw=True)
    oi, orr = O.brute_force_knn(xu, 9)
    assert np.array_equal(ind, oi) and np.array_equal(raw.view(np.uint32), orr.view(np.uint32))


def test_brute_force_row_slice_and_strict_backend():
    x = _i8(900, 64, 3)
    opts = evoc.KnnGraphOptions(n_neighbors=12, brute_force_max_n=900)
    full, fd = evoc.knn_graph(x, opts)
    part, pd = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=12, brute_force_max_n=900, row_begin=100,
                                                      row_end=613))
    assert np.array_equal(part, full[100:613]) and np.array_equal(pd.view(np.uint32), fd[100:613].view(np.uint32))
    be = B.make_backend(B.ComputeBackend.Cuda)
    si, sd = be.knn_graph(x, opts, np.random.RandomState(1), strict_precision=True)
    oi, orr = O.brute_force_knn(x, 12)
    assert np.array_equal(si, oi) and np.array_equal(sd.view(np.uint32), O.transform(O.DT_I8, orr).view(np.uint32))
    # above brute_force_max_n the exact GPU search runs unless strict_precision is asked for
    small = evoc.KnnGraphOptions(n_neighbors=12, brute_force_max_n=899)
    with pytest.raises(B.StrictPrecisionUnavailable):
        be.knn_graph(x, small, np.random.RandomState(1), strict_precision=True)
    ei, _ = be.knn_graph(x, small, np.random.RandomState(1), strict_precision=False)
    assert np.array_equal(ei, O.exact_knn(x, 12)[0])
