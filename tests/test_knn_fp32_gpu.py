"""Plain FP32 exact form on the GPU, through the C ABI, against the golden
fixtures and the oracle.

Tolerances are the reference's own (tests/parity.rs:34-68): distances within
1e-6 absolute; an index may differ only where the two distances agree within
1e-6 (a tie); tie swaps are bounded.
"""
import numpy as np
import pytest

import evoc
from conftest import FIXTURES, assert_knn_parity
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def opts(k, **kw):
    return evoc.KnnGraphOptions(n_neighbors=k, form="fp32", **kw)


@pytest.mark.parametrize("name", FIXTURES)
def test_fp32_matches_golden(golden, name):
    z = golden[name]
    rng = np.random.RandomState(int(z["seed"]))
    ind, dst = evoc.knn_graph(z["data"], opts(15, deterministic=True), rng)
    assert_knn_parity(ind, dst, z["nn_inds"], z["nn_dists"])
    # the caller's RNG advanced exactly as the CPU path advances it
    key = rng.get_state()[1]
    assert np.array_equal(key, z["rng_after_knn_key"])
    assert rng.get_state()[2] == int(z["rng_after_knn_pos"])
    # self at column 0 with +0.0 (find_duplicates relies on it, src/cluster_util.rs:431-449)
    assert np.all(ind[:, 0] == np.arange(len(ind)))
    assert np.all(dst[:, 0] == 0.0) and not np.any(np.signbit(dst[:, 0]))


def _check_against_oracle(x, k, max_tie_frac=0.01):
    """Neighbour sets equal to the oracle's except for ties within 1e-6 cosine,
    and every reported raw dissimilarity within 1e-6 of the FP64 value for
    that pair.  (Two FP32 summation orders differ by a few 1e-7 in the dot,
    which the -log2 transform can stretch past 1e-6, so distances are held to
    FP64 truth rather than to another FP32 ordering.)"""
    ind, dst, raw = evoc.knn_graph(x, opts(k), None, return_raw=True)
    xn = O.prepare_float(x)
    kk = max(1, min(k, len(x) - 1))
    ei, er = O.exact_knn(xn, kk)
    assert ind.shape == ei.shape
    x64 = xn.astype(np.float64)
    dots = np.einsum("rkd,rd->rk", x64[ind], x64)
    want = np.where(dots > 0, -dots, 1.17549435e-38)
    want[ind == np.arange(len(x))[:, None]] = -1.0
    assert np.abs(raw - want).max() <= 1e-6
    # index disagreements only where the oracle's raw values tie within 1e-6
    diff = ind != ei
    assert np.all(np.abs(raw[diff] - er[diff]) <= 1e-6)
    assert diff.sum() <= max(8, max_tie_frac * ind.size), diff.sum()
    assert np.array_equal(dst, transform_f32(raw))
    # raw is -dot, or f32::MIN_POSITIVE when the dot is <= 0 (src/fast_cosine.rs:40-44)
    assert raw.max() <= np.float32(1.17549435e-38)
    assert np.all(np.diff(raw, axis=1) >= -1e-6)
    return ind, dst


def transform_f32(raw):
    return O.transform(O.DT_F32, raw)


@pytest.mark.parametrize("n,d,k", [(2, 3, 1), (3, 5, 10), (17, 16, 4), (129, 33, 15), (300, 128, 30),
                                   (777, 100, 64), (1000, 7, 15)])
def test_fp32_random_shapes(n, d, k):
    rng = np.random.default_rng(n * 1000 + d)
    c = rng.standard_normal((5, d))
    x = (c[rng.integers(0, 5, n)] + 0.2 * rng.standard_normal((n, d))).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    _check_against_oracle(x, k)


def test_fp32_blobs_2k_128():
    from evoc import synthetic

    x = synthetic.blobs_2k_128()
    ind, dst = _check_against_oracle(x, 15)
    assert np.all(ind[:, 0] == np.arange(len(x)))


def test_fp32_unnormalised_rows_are_renormalised():
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((400, 24)) * 3.0).astype(np.float32)
    _check_against_oracle(x, 12)


def test_fp32_zero_and_duplicate_rows():
    rng = np.random.default_rng(6)
    x = rng.standard_normal((200, 32)).astype(np.float32)
    x[10] = 0.0
    x[20] = x[21] = x[22]
    x[50:60] = x[49]
    _check_against_oracle(x, 15, max_tie_frac=0.05)


def test_fp32_single_row():
    x = np.ones((1, 8), np.float32)
    ind, dst = evoc.knn_graph(x, opts(5))
    assert ind.shape == (1, 1) and ind[0, 0] == 0 and dst[0, 0] == 0.0


def test_errors_mirror_knnerror():
    with pytest.raises(evoc.InvalidNeighbors):
        evoc.knn_graph(np.ones((4, 4), np.float32), opts(0))
    with pytest.raises(evoc.EmptyData):
        evoc.knn_graph(np.ones((0, 4), np.float32), opts(3))


def test_device_pointer_entry():
    import torch

    rng = np.random.default_rng(7)
    x = rng.standard_normal((500, 64)).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    xt = torch.from_numpy(x).cuda()
    oi = torch.empty((500, 10), dtype=torch.int32, device="cuda")
    od = torch.empty((500, 10), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    k = evoc.knn_graph_device(xt.data_ptr(), 0, 500, 64, 10, oi.data_ptr(), od.data_ptr(), opts(10))
    assert k == 10
    hi, hd = evoc.knn_graph(x, opts(10))
    assert np.array_equal(oi.cpu().numpy(), hi) and np.array_equal(od.cpu().numpy(), hd)


@pytest.mark.parametrize("r0,r1", [(100, 612), (301, 777), (0, 1000), (996, 1000), (3, 4)])
def test_fp32_row_slices_match_full_graph(r0, r1):
    """Row slices give the full graph's rows bit for bit.  Slices starting at a
    multiple of 4 take the k-major kernel, the others the row-major one; both
    sum each dot in coordinate order, so their FP32 results agree exactly."""
    rng = np.random.default_rng(11)
    x = rng.standard_normal((1000, 100)).astype(np.float32)
    fi, fd = evoc.knn_graph(x, opts(15))
    si, sd = evoc.knn_graph(x, opts(15, row_begin=r0, row_end=r1))
    assert np.array_equal(si, fi[r0:r1]) and np.array_equal(sd, fd[r0:r1])
