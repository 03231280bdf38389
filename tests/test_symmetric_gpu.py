"""The symmetric 16-bit scan (tc_scan.cu symmetric mode + sym.cu) on the GPU.

A self-join's score matrix is symmetric, so the symmetric scan multiplies
each pair of rows once and routes the scores for the later row through
per-row mailboxes, filtered by thresholds from a sampled pre-scan.  Its
candidates are the plain scan's, so the whole graph (indices and distance
bits, tolerance 0) must equal the one built with the symmetric scan off, and
the exact neighbour sets up to ties within 1e-6.  Rows whose mailbox
overflows are failed by the certificate and rescanned: on data made of a few
rows repeated thousands of times every mailbox overflows, and the graph must
still equal the plain path's.
"""
import numpy as np
import pytest

import evoc
from evoc import _lib

from test_certify_gpu import misses_beyond_ties, tight_clusters

pytestmark = pytest.mark.gpu


def _half(k):
    return evoc.KnnGraphOptions(n_neighbors=k, form="bf16_rerank")


def _both(x, k):
    """The graph with the symmetric scan forced on, its statistics, and the graph with it off."""
    ctx = _lib.context(0)
    try:
        ctx.set_symmetric_scan(1)
        ind_s, dst_s = evoc.knn_graph(x, _half(k))
        stats = ctx.symmetric_stats()
        cert = ctx.certify_counts()
        ctx.set_symmetric_scan(-1)
        ind_p, dst_p = evoc.knn_graph(x, _half(k))
        assert ctx.symmetric_stats()["sample_rows"] == 0
    finally:
        ctx.set_symmetric_scan(0)  # off again (the default)
    return ind_s, dst_s, stats, cert, ind_p, dst_p


@pytest.mark.parametrize("n,d,k", [(20000, 128, 15), (33333, 768, 30), (4099, 64, 10)])
def test_symmetric_equals_plain_scan(n, d, k):
    x = tight_clusters(n, d, 40, 0.3, n + d)
    ind_s, dst_s, stats, cert, ind_p, dst_p = _both(x, k)
    assert stats["sample_rows"] == n // 16 and stats["mailbox_cap"] > 0
    assert stats["overflowed"] == 0, stats
    assert 0 < stats["max_offers"] <= stats["mailbox_cap"]
    assert cert["checked"] == n
    assert np.array_equal(ind_s, ind_p)
    assert np.array_equal(dst_s.view(np.uint32), dst_p.view(np.uint32))
    assert np.all(ind_s[:, 0] == np.arange(n))
    if n <= 20000:
        assert misses_beyond_ties(x, ind_s, k) == 0


def test_symmetric_tight_clusters_are_exact():
    """Rounding larger than the gaps between neighbours: rows fail the certificate and are
    rescanned after the symmetric scan as after the plain one."""
    n, d, k = 12000, 128, 15
    x = tight_clusters(n, d, 10, 0.01, 5)
    ind_s, dst_s, stats, cert, ind_p, dst_p = _both(x, k)
    assert stats["sample_rows"] > 0
    assert cert["second_pass"] > 0
    assert np.array_equal(ind_s, ind_p)
    assert np.array_equal(dst_s.view(np.uint32), dst_p.view(np.uint32))
    assert misses_beyond_ties(x, ind_s, k) == 0


def test_overflowing_mailboxes_are_rescanned():
    """Four rows repeated 4,000 times each: a row's duplicates tie with its self value, so every
    earlier duplicate reaches the row's mailbox; beyond the capacity the row overflows, the
    certificate fails it and the rescans build its neighbours."""
    rng = np.random.default_rng(9)
    base = rng.standard_normal((4, 64)).astype(np.float32)
    x = np.repeat(base, 4000, axis=0)
    x = x[rng.permutation(len(x))]
    ind_s, dst_s, stats, cert, ind_p, dst_p = _both(x, 15)
    assert stats["overflowed"] > 0 and stats["max_offers"] > stats["mailbox_cap"]
    assert np.array_equal(ind_s, ind_p)
    assert np.array_equal(dst_s.view(np.uint32), dst_p.view(np.uint32))


def test_setting_is_per_context_and_off_by_default():
    ctx = _lib.context(0)
    x = tight_clusters(5000, 32, 5, 0.3, 3)
    evoc.knn_graph(x, _half(10))
    assert ctx.symmetric_stats()["sample_rows"] == 0  # off by default
    ctx.set_symmetric_scan(6000)  # above these 5,000 rows
    evoc.knn_graph(x, _half(10))
    assert ctx.symmetric_stats()["sample_rows"] == 0
    ctx.set_symmetric_scan(5000)
    evoc.knn_graph(x, _half(10))
    assert ctx.symmetric_stats()["sample_rows"] == 5000 // 16
    ctx.set_symmetric_scan(-5)  # off
    evoc.knn_graph(x, _half(10))
    assert ctx.symmetric_stats()["sample_rows"] == 0
    ctx.set_symmetric_scan(0)
