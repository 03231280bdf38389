"""The oracle, pinned against the reference's own golden vectors and KATs.

Everything here runs on the CPU.  The oracle (oracle/evoc_oracle.c) is the
checker the GPU tests trust, so it is held to the same fixtures and rules the
evoc-rs test suite uses (tests/parity.rs, tests/graph_parity.rs,
tests/parity_intermediates.rs, src/numpy_rng.rs:232-252,
src/fast_cosine.rs:65-86).
"""
import os

import numpy as np
import pytest

from conftest import FIXTURES, assert_knn_parity, knn_parity_counts
from oracle import oracle as O


@pytest.fixture(scope="module", autouse=True)
def _oracle_built():
    O.build()
    O.use_reference_cosine(True)
    yield
    O.use_reference_cosine(False)


def test_mt19937_seed42_kat():
    # src/numpy_rng.rs:232-252 (matches_numpy_seed_42)
    r = O.RandomState(42)
    lo, hi = -(2**31) + 1, 2**31 - 2
    assert [r.randint(lo, hi) for _ in range(3)] == [-538846105, 1273642420, 1935803229]
    assert [r.randint(lo, hi) for _ in range(5)] == [-1359637233, 996406379, 1201263688, 423734973, 415968277]
    n = [r.normal() for _ in range(3)]
    assert abs(n[0] - (-0.23415337472333597)) < 1e-12
    assert abs(n[1] - (-0.23413695694918055)) < 1e-12
    assert abs(n[2] - 1.5792128155073915) < 1e-12


def test_numpy_randomstate_is_the_same_generator():
    # The host mirror uses numpy.random.RandomState directly as the rng.
    r1 = O.RandomState(1234)
    r2 = np.random.RandomState(1234)
    lo, hi = -(2**31) + 1, 2**31 - 2
    for _ in range(700):  # crosses one MT19937 regeneration
        assert r1.randint(lo, hi) == int(r2.randint(lo, hi))


def test_cosine_sentinel_kats():
    # src/fast_cosine.rs:65-86
    a = np.array([[1.0, 0.0], [0.5, 0.8660254], [-1.0, 0.0]], np.float32)
    assert abs(O.distance(a, 0, 1, strict=True) + 0.5) < 1e-6
    assert O.distance(a, 0, 2, strict=True) == np.float32(1.17549435e-38)
    assert O.distance(a, 0, 2, strict=False) == np.float32(1.17549435e-38)


@pytest.mark.skipif(not os.path.exists(O.REF_COS_PATH), reason="reference fast_cosine.c not built here")
def test_restated_fastmath_cosine_matches_reference_binary():
    rng = np.random.default_rng(0)
    for dim in (1, 3, 16, 32, 33, 64, 128, 768):
        x = rng.standard_normal((64, dim)).astype(np.float32)
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        O.use_reference_cosine(True)
        ref = [O.distance(x, 0, j, strict=True) for j in range(64)]
        O.use_reference_cosine(False)
        mine = [O.distance(x, 0, j, strict=True) for j in range(64)]
        O.use_reference_cosine(True)
        assert np.array_equal(np.array(ref, np.float32), np.array(mine, np.float32)), dim


@pytest.mark.parametrize("name", FIXTURES)
def test_nndescent_deterministic_matches_golden(golden, name):
    # tests/parity.rs:134-189 (parity_knn_medium_800 / large_2000 rules) and
    # tests/parity_intermediates.rs:655-687 (RNG state after knn_graph).
    z = golden[name]
    rng = O.RandomState(int(z["seed"]))
    ind, dst = O.knn_graph(z["data"], 15, rng, deterministic=True)
    assert_knn_parity(ind, dst, z["nn_inds"], z["nn_dists"])
    assert np.array_equal(rng.key, z["rng_after_knn_key"])
    assert rng.pos == int(z["rng_after_knn_pos"]) == 15


@pytest.mark.parametrize("name", FIXTURES)
def test_exact_selector_matches_golden(golden, name):
    # The GPU contract (self at column 0, k-1 nearest) reproduces the goldens.
    z = golden[name]
    ind, raw = O.exact_knn(z["data"], 15)
    dst = O.transform(O.DT_F32, raw)
    assert_knn_parity(ind, dst, z["nn_inds"], z["nn_dists"])
    assert np.all(ind[:, 0] == np.arange(len(ind)))
    assert np.all(dst[:, 0] == 0.0) and not np.any(np.signbit(dst[:, 0]))


def test_raw_distances_non_positive(golden):
    # src/knn.rs:456-520 (pre_transform_distances_are_negative)
    z = golden["medium_800"]
    _, _, raw, _ = O.knn_graph(z["data"], 15, O.RandomState(42), deterministic=True, return_raw=True)
    assert raw.max() <= 0.0


def test_smooth_knn_dist_matches_python(golden):
    # tests/graph_parity.rs:28-62
    z = golden["medium_800"]
    s, r = O.smooth_knn_dist(z["nn_dists"], 15.0)
    assert np.abs(s - z["sigmas_py"]).max() < 1e-6
    assert np.abs(r - z["rhos_py"]).max() < 1e-6


@pytest.mark.parametrize("name", ["medium_800", "large_2000"])
def test_fuzzy_graph_from_golden_knn_matches(golden, name):
    # tests/graph_parity.rs:64-90 and the pattern half of tests/parity.rs:191-232
    z = golden[name]
    ip, ix, dv, _, _ = O.fuzzy_graph(z["nn_inds"], z["nn_dists"], 15.0)
    assert np.array_equal(ip, z["graph_csr_indptr"])
    assert np.array_equal(ix, z["graph_csr_indices"])
    assert np.abs(dv - z["graph_csr_data"]).max() <= 1e-6


def test_fuzzy_graph_coo_golden_small(golden):
    z = golden["small_200"]
    ip, ix, dv, _, _ = O.fuzzy_graph(z["nn_inds"], z["nn_dists"], 15.0)
    rows = np.repeat(np.arange(len(ip) - 1), np.diff(ip))
    got = dict(zip(zip(rows.tolist(), ix.tolist()), dv.tolist()))
    exp = dict(zip(zip(z["graph_coo_rows"].tolist(), z["graph_coo_cols"].tolist()), z["graph_coo_data"].tolist()))
    assert got.keys() == exp.keys()
    assert max(abs(got[k] - exp[k]) for k in got) <= 1e-6


def test_transforms_kats():
    raw = np.array([-1.0, -0.5, 0.0, -0.0, 1e-38, -2.0], np.float32)
    f = O.transform(O.DT_F32, raw)
    assert f[0] == 0.0 and not np.signbit(f[0])
    assert f[1] == np.float32(1.0)
    assert f[2] == 0.0 and f[3] == 0.0 and f[4] == 0.0 and f[5] == 0.0
    i = O.transform(O.DT_I8, np.array([-4.0, 0.0, -1.0, 3.0], np.float32))
    assert list(i) == [0.25, 0.0, 1.0, 0.0]
    u = O.transform(O.DT_U8, np.array([-1.0, -0.5, 0.0, -0.0], np.float32))
    # self (raw -1.0) transforms to -0.0 for u8 (src/knn.rs:178-187)
    assert u[0] == 0.0 and np.signbit(u[0])
    assert u[1] == np.float32(1.0)
    assert u[2] == 0.0 and u[3] == 0.0


def _int8_data(n, d, seed):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((8, d))
    x = c[rng.integers(0, 8, n)] + 0.3 * rng.standard_normal((n, d))
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return np.clip(np.round(127 * x), -127, 127).astype(np.int8)


def _binary_data(n, nbytes, seed):
    rng = np.random.default_rng(seed)
    protos = rng.random((6, nbytes * 8)) < 0.1
    rows = protos[rng.integers(0, 6, n)] ^ (rng.random((n, nbytes * 8)) < 0.05)
    return np.packbits(rows, axis=1)


@pytest.mark.parametrize("kind", ["i8", "u8"])
def test_integer_exact_selector_agrees_with_brute_force(kind):
    # brute_force_knn (src/knn.rs:189-281) excludes self and returns heap order;
    # the exact selector offers self with raw -1.0.  Outside self, with ties
    # broken by index, the two must agree on every row's raw distances.
    x = _int8_data(300, 40, 1) if kind == "i8" else _binary_data(300, 16, 2)
    k = 10
    bi, br = O.brute_force_knn(x, k)
    ei, er = O.exact_knn(x, k + 1)
    for r in range(len(x)):
        b = np.sort(br[r])
        e = np.array([er[r][j] for j in range(k + 1) if ei[r][j] != r][:k], np.float32)
        assert np.array_equal(b, np.sort(e)), r


@pytest.mark.parametrize("kind", ["i8", "u8"])
def test_integer_nndescent_recall(kind):
    # NN-descent (int8.rs:575-678 / uint8.rs:563-666) vs the exact selector.
    x = _int8_data(1500, 48, 3) if kind == "i8" else _binary_data(1500, 32, 4)
    ind, _, raw, _ = O.knn_graph(x, 10, O.RandomState(5), deterministic=True, return_raw=True)
    ei, er = O.exact_knn(x, 10)
    # recall measured on raw values (ties make index sets ambiguous)
    hits = 0
    for r in range(len(x)):
        kth = er[r][-1]
        hits += int(np.sum(raw[r] <= kth))
    assert hits / ind.size > 0.95
