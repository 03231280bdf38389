"""GPU label propagation / node embedding against the oracle (and the golden vectors).

Partitions and node embeddings are compared bit for bit with the oracle on the
same graph and the same NumPy RNG state, and the RNG must end in the same
state.  The full label_propagation_init ends in a PCA of fewer than 64 rows
(f64; the oracle uses NumPy's SVD, the GPU a Jacobi eigen-decomposition), so
it is compared within the reference's own init tolerance, 1e-4
(tests/parity_intermediates.rs:127), and against the golden init_embedding.
"""
import os

import numpy as np
import pytest

import evoc
from oracle import label_prop as L

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _lp(name):
    return np.load(os.path.join(GOLDEN, f"lp_{name}.npz"))


def _main(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def _graph(name):
    z = _lp(name)
    if "graph_csr_indptr" in z.files:
        return L.Csr.make(z["graph_csr_indptr"], z["graph_csr_indices"], z["graph_csr_data"], z["graph_csr_shape"])
    m = _main(name)
    r, c, d = m["graph_coo_rows"], m["graph_coo_cols"], m["graph_coo_data"]
    n = int(m["graph_coo_shape"][0])
    o = np.lexsort((c, r))
    indptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=indptr[1:])
    return L.Csr.make(indptr, c[o], d[o], (n, n))


def _tuple(g):
    return (g.indptr, g.indices, g.data, g.shape[0])


def _np_state(z, tag):
    rs = np.random.RandomState(0)
    rs.set_state(("MT19937", z[f"rng_{tag}_key"].astype(np.uint32), int(z[f"rng_{tag}_pos"]),
                  int(z[f"rng_{tag}_has_gauss"]), float(z[f"rng_{tag}_gauss"])))
    return rs


def _oracle_rng(rs):
    _, key, pos, hg, g = rs.get_state()
    return L.mt_from_state(key, pos, hg, g)


def _same_state(rs, orng):
    _, key, pos, _, _ = rs.get_state()
    return np.array_equal(key, orng.key) and int(pos) == orng.pos


def _approx(n):
    return int(np.clip(8 * np.sqrt(n), 256, 16384))


@pytest.fixture(scope="module")
def blob_graph():
    """A 12,000-vertex fuzzy graph (GPU kNN + fuzzy union) and its data, built once."""
    rng = np.random.default_rng(21)
    c = rng.normal(size=(40, 48))
    x = (c[rng.integers(0, 40, 12000)] + 0.35 * rng.normal(size=(12000, 48))).astype(np.float32)
    ind, dst = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=15, form="fp32"))
    indptr, indices, data, _, _ = evoc.neighbor_graph_csr(15.0, ind, dst)
    return L.Csr.make(indptr, indices, data, (len(x), len(x))), x


@pytest.mark.parametrize("name", ["medium_800", "large_2000"])
def test_label_prop_loop_matches_oracle_and_golden(name):
    z = _lp(name)
    g = _graph(name)
    rs = _np_state(z, "after_knn")
    orng = _oracle_rng(rs)
    part = evoc.label_prop_loop(_tuple(g), rs, 20, _approx(g.shape[0]))
    want = L.label_prop_loop(g, orng, 20, _approx(g.shape[0]))
    assert np.array_equal(part, want) and np.array_equal(part, z["partition"])
    assert _same_state(rs, orng)


def test_label_prop_loop_larger_graph(blob_graph):
    g, _ = blob_graph
    for seed, approx in ((3, 876), (4, 40), (5, 5000)):
        rs = np.random.RandomState(seed)
        orng = _oracle_rng(rs)
        part = evoc.label_prop_loop(_tuple(g), rs, 20, approx)
        want = L.label_prop_loop(g, orng, 20, approx)
        assert np.array_equal(part, want), (seed, approx, int((part != want).sum()))
        assert _same_state(rs, orng)


def test_label_prop_loop_few_iterations_leaves_outliers(blob_graph):
    """With one sweep most rows are still unlabelled: the outlier walk (64-pop limit, random
    fallback label, labels set earlier in the pass visible) decides them."""
    g, _ = blob_graph
    rs = np.random.RandomState(9)
    orng = _oracle_rng(rs)
    part = evoc.label_prop_loop(_tuple(g), rs, 1, 64)
    want = L.label_prop_loop(g, orng, 1, 64)
    assert np.array_equal(part, want)


@pytest.mark.parametrize("name", ["small_200", "medium_800", "large_2000"])
def test_node_embedding_bit_exact(name):
    z = _lp(name)
    g = _graph(name)
    rs = _np_state(z, "after_init")
    orng = _oracle_rng(rs)
    emb = evoc.node_embedding(_tuple(g), 4, 50, z["init_embedding"], 0.1, 1.0, 0.5, rs)
    want = L.node_embedding(g, 4, 50, z["init_embedding"], 0.1, 1.0, 0.5, orng)
    assert np.array_equal(emb.view(np.uint32), want.view(np.uint32))
    assert _same_state(rs, orng)
    assert np.abs(emb - z["embedding"]).max() <= (3.6e-4 if name == "medium_800" else 2e-3)


def test_node_embedding_random_init_and_wide(blob_graph):
    """Initial embedding drawn from the RNG (normal(0.25)), 15 components, more than 8 blocks per
    epoch on a 12,000-vertex graph."""
    g, _ = blob_graph
    rs = np.random.RandomState(77)
    orng = _oracle_rng(rs)
    emb = evoc.node_embedding(_tuple(g), 15, 12, None, 0.1, 1.0, 0.5, rs)
    want = L.node_embedding(g, 15, 12, None, 0.1, 1.0, 0.5, orng)
    assert np.array_equal(emb.view(np.uint32), want.view(np.uint32))
    assert _same_state(rs, orng)


@pytest.mark.parametrize("name", ["small_200", "medium_800", "large_2000"])
def test_label_propagation_init_matches_oracle_and_golden(name):
    z = _lp(name)
    g = _graph(name)
    data = _main(name)["data"]
    rs = _np_state(z, "after_knn")
    orng = _oracle_rng(rs)
    init = evoc.label_propagation_init(_tuple(g), 20, 50, _approx(g.shape[0]), 4, 0.5, 0.1, 0.5, rs, data)
    want = L.label_propagation_init(g, 20, 50, _approx(g.shape[0]), 4, 0.5, 0.1, 0.5, orng, data)
    assert np.abs(init - want).max() <= 1e-4
    assert np.abs(init - z["init_embedding"]).max() <= 1e-4
    assert _same_state(rs, orng)


def test_label_propagation_init_larger_graph(blob_graph):
    g, x = blob_graph
    rs = np.random.RandomState(5)
    orng = _oracle_rng(rs)
    init = evoc.label_propagation_init(_tuple(g), 20, 30, _approx(g.shape[0]), 7, 0.5, 0.1, 0.5, rs, x)
    want = L.label_propagation_init(g, 20, 30, _approx(g.shape[0]), 7, 0.5, 0.1, 0.5, orng, x)
    assert init.shape == (len(x), 7)
    assert np.abs(init - want).max() <= 1e-4
    assert _same_state(rs, orng)


def test_errors_are_reported_not_faulted(blob_graph):
    g, _ = blob_graph
    with pytest.raises(evoc.BackendError):  # PCA base init needs the data (LabelPropError::PcaRequiresData)
        evoc.label_propagation_init(_tuple(g), 20, 5, 300, 4, 0.5, 0.1, 0.5, np.random.RandomState(1), None)
    bad = g.indices.copy()
    bad[7] = g.shape[0]  # a column outside the graph is caught before any kernel reads through it
    with pytest.raises(evoc.BackendError):
        evoc.label_prop_loop((g.indptr, bad, g.data, g.shape[0]), np.random.RandomState(1), 3, 100)
    with pytest.raises(evoc.EmptyData):
        evoc.node_embedding((np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0, np.float32), 0), 4, 5)


def _hub_graph(n=6000, hubs=5, hub_deg=2500, seed=3):
    """Symmetric random graph with a few rows of thousands of edges (above the one-CTA-per-row
    threshold of the embedding kernel), weights in (0, 1]."""
    rng = np.random.default_rng(seed)
    r = rng.integers(0, n, 8 * n)
    c = rng.integers(0, n, 8 * n)
    for h in range(hubs):
        t = rng.choice(n, hub_deg, replace=False)
        r = np.concatenate([r, np.full(hub_deg, h)])
        c = np.concatenate([c, t])
    keep = r != c
    r, c = r[keep], c[keep]
    key = np.unique(np.minimum(r, c).astype(np.int64) * n + np.maximum(r, c))
    a, b = key // n, key % n
    w = rng.uniform(0.05, 1.0, len(key)).astype(np.float32)
    rr = np.concatenate([a, b])
    cc = np.concatenate([b, a])
    ww = np.concatenate([w, w])
    o = np.lexsort((cc, rr))
    indptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rr, minlength=n), out=indptr[1:])
    return L.Csr.make(indptr, cc[o].astype(np.int32), ww[o], (n, n))


@pytest.mark.parametrize("nsr,ncomp", [(1.0, 4), (5.0, 7), (5.0, 20)])
def test_node_embedding_hub_rows_and_many_negative_samples(nsr, ncomp):
    """Rows of ~2500 edges take the one-CTA-per-row path; a negative-sample rate of 5 gives edges
    more negative samples than either kernel stages at once (their samples are then computed in
    order by the accumulating warp)."""
    g = _hub_graph()
    assert np.diff(g.indptr).max() > 2000
    rs = np.random.RandomState(11)
    orng = _oracle_rng(rs)
    emb = evoc.node_embedding(_tuple(g), ncomp, 6, None, 0.1, nsr, 0.5, rs)
    want = L.node_embedding(g, ncomp, 6, None, 0.1, nsr, 0.5, orng)
    assert np.array_equal(emb.view(np.uint32), want.view(np.uint32))
    assert _same_state(rs, orng)


def test_label_prop_and_init_on_hub_rows():
    """Hub rows see more distinct labels / parts than a warp's shared-memory table holds: the
    overflow passes (direct key index in global memory) must give the same votes and expander
    rows as the oracle."""
    g = _hub_graph(n=6000, hubs=6, hub_deg=3000, seed=5)
    for seed, approx in ((2, 1500), (3, 400)):
        rs = np.random.RandomState(seed)
        orng = _oracle_rng(rs)
        part = evoc.label_prop_loop(_tuple(g), rs, 20, approx)
        want = L.label_prop_loop(g, orng, 20, approx)
        assert np.array_equal(part, want), (seed, approx)
    x = np.random.default_rng(4).normal(size=(g.shape[0], 24)).astype(np.float32)
    rs = np.random.RandomState(8)
    orng = _oracle_rng(rs)
    init = evoc.label_propagation_init(_tuple(g), 20, 20, 1500, 5, 0.5, 0.1, 0.5, rs, x)
    want = L.label_propagation_init(g, 20, 20, 1500, 5, 0.5, 0.1, 0.5, orng, x)
    assert np.abs(init - want).max() <= 1e-4
    assert _same_state(rs, orng)


def _knn_label_rate(emb, labels, k=10):
    """Fraction of each point's k nearest embedding neighbours sharing its cluster."""
    import torch

    e = torch.from_numpy(emb).double()
    lab = torch.from_numpy(labels)
    hits = 0
    for r0 in range(0, len(e), 2048):
        d = torch.cdist(e[r0:r0 + 2048], e)
        d[torch.arange(d.shape[0]), torch.arange(r0, r0 + d.shape[0])] = float("inf")
        nn = d.topk(k, largest=False).indices
        hits += (lab[nn] == lab[r0:r0 + d.shape[0], None]).sum().item()
    return hits / (len(e) * k)


def test_node_embedding_non_reproducible(blob_graph):
    """reproducible_flag = false: the reference's serial in-place epochs against the GPU's
    lock-free ones.  Same draws from the caller's RNG; embeddings agree in quality (cluster
    purity of embedding neighbourhoods), not bit for bit."""
    g, x = blob_graph
    labels = np.random.default_rng(21)
    labels.normal(size=(40, 48))
    labels = labels.integers(0, 40, 12000)
    init = evoc.label_propagation_init(_tuple(g), 20, 20, _approx(g.shape[0]), 4, 0.5, 0.1, 0.5,
                                       np.random.RandomState(2), x)
    rs = np.random.RandomState(12)
    orng = _oracle_rng(rs)
    emb = evoc.node_embedding(_tuple(g), 4, 40, init, 0.1, 1.0, 0.5, rs, reproducible_flag=False)
    want = L.node_embedding_serial(g, 4, 40, init, 0.1, 1.0, 0.5, orng)
    assert _same_state(rs, orng)
    assert np.isfinite(emb).all()
    got_rate, want_rate = _knn_label_rate(emb, labels), _knn_label_rate(want, labels)
    assert got_rate >= want_rate - 0.03 and got_rate > 0.8, (got_rate, want_rate)


def test_label_propagation_init_small_graph_and_wide_components():
    """Fewer than 64 vertices: the PCA base init directly; 20 components takes the 32-wide kernels."""
    rng = np.random.default_rng(6)
    x = rng.normal(size=(50, 12)).astype(np.float32)
    g = _hub_graph(n=50, hubs=1, hub_deg=30, seed=6)
    rs = np.random.RandomState(4)
    orng = _oracle_rng(rs)
    init = evoc.label_propagation_init(_tuple(g), 20, 10, 256, 5, 0.5, 0.1, 0.5, rs, x)
    want = L.label_propagation_init(g, 20, 10, 256, 5, 0.5, 0.1, 0.5, orng, x)
    assert np.abs(init - want).max() <= 1e-4
    assert _same_state(rs, orng)  # no draws below the threshold
    g2 = _hub_graph(n=3000, hubs=2, hub_deg=800, seed=9)
    x2 = rng.normal(size=(3000, 16)).astype(np.float32)
    rs = np.random.RandomState(5)
    orng = _oracle_rng(rs)
    init = evoc.label_propagation_init(_tuple(g2), 20, 10, 400, 20, 0.5, 0.1, 0.5, rs, x2)
    want = L.label_propagation_init(g2, 20, 10, 400, 20, 0.5, 0.1, 0.5, orng, x2)
    assert init.shape == (3000, 20) and np.abs(init - want).max() <= 1e-4
    assert _same_state(rs, orng)


def test_label_propagation_limits_are_errors():
    # 100,000 seeds on 300,000 vertices leave ~85,000 distinct parts: above the 65,536 the
    # reduction's sort keys hold (the reference's own call clamps approx_n_parts to 16,384)
    g = _hub_graph(n=300000, hubs=1, hub_deg=100, seed=2)
    x = np.zeros((300000, 4), np.float32)
    with pytest.raises(evoc.BackendError):
        evoc.label_propagation_init(_tuple(g), 20, 5, 100000, 4, 0.5, 0.1, 0.5, np.random.RandomState(1), x)
    with pytest.raises(evoc.BackendError):  # components above 32
        evoc.label_propagation_init(_tuple(g), 20, 5, 300, 40, 0.5, 0.1, 0.5, np.random.RandomState(1), x)


@pytest.mark.parametrize("base_init,upscaling,recursive", [
    ("pca", "jitter_expander", True),
    ("pca", "node_embedding", True),
    ("pca", "partition_expander", False),
    ("random", "partition_expander", True),
    ("spectral", "partition_expander", True),
    ("spectral", "jitter_expander", False),
])
def test_label_propagation_init_with_options_matches_oracle(blob_graph, base_init, upscaling, recursive):
    """label_propagation_init_with_options (src/label_prop.rs:497-674) against the oracle: the
    recursion, the base init of the < 64-vertex level, the upscaler's normal draws in the
    reference's order (the caller's RNG ends in the same state)."""
    g, x = blob_graph
    rs = np.random.RandomState(13)
    orng = _oracle_rng(rs)
    kw = dict(recursive_init=recursive, base_init=base_init, upscaling=upscaling)
    init = evoc.label_propagation_init(_tuple(g), 20, 20, _approx(g.shape[0]), 5, 0.5, 0.1, 0.5, rs, x, **kw)
    want = L.label_propagation_init(g, 20, 20, _approx(g.shape[0]), 5, 0.5, 0.1, 0.5, orng, x, **kw)
    assert init.shape == (len(x), 5)
    assert np.abs(init - want).max() <= 1e-4
    assert _same_state(rs, orng)


def test_small_graph_base_inits_match_oracle():
    """Below the threshold the base init is the result (src/label_prop.rs:513-515): random draws
    bit for bit; spectral within 1e-4; MDS within 5e-3 -- its first column belongs to the zero
    eigenvalue of the doubly centred matrix, f32 rounding noise in every implementation."""
    rng = np.random.default_rng(31)
    x = rng.normal(size=(40, 48)).astype(np.float32)
    g = _hub_graph(n=40, hubs=1, hub_deg=20, seed=8)
    for base, tol in (("random", 0.0), ("spectral", 1e-4), ("mds", 5e-3), ("pca", 1e-4)):
        rs = np.random.RandomState(3)
        orng = _oracle_rng(rs)
        got = evoc.label_propagation_init(_tuple(g), 20, 10, 256, 6, 0.5, 0.1, 0.5, rs, x, base_init=base)
        want = L.small_graph_init(x, 40, 6, base, orng)
        assert got.shape == (40, 6)
        assert np.abs(got - want).max() <= tol, (base, np.abs(got - want).max())
        assert _same_state(rs, orng)
    # the random init needs no data
    rs = np.random.RandomState(3)
    got = evoc.label_propagation_init(_tuple(g), 20, 10, 256, 6, 0.5, 0.1, 0.5, rs, None, base_init="random")
    assert np.allclose(np.linalg.norm(got, axis=1), 1.0, atol=1e-6)


def test_label_propagation_option_errors(blob_graph):
    g, x = blob_graph
    with pytest.raises(ValueError):
        evoc.label_propagation_init(_tuple(g), 20, 5, 300, 4, 0.5, 0.1, 0.5, np.random.RandomState(1), x,
                                    base_init="tsne")
    with pytest.raises(evoc.BackendError):  # eigen-decompositions are one block of at most 64 rows
        evoc.label_propagation_init(_tuple(g), 20, 5, 300, 4, 0.5, 0.1, 0.5, np.random.RandomState(1), x,
                                    base_init_threshold=200)
    with pytest.raises(evoc.BackendError):  # spectral needs the data (LabelPropError::PcaRequiresData)
        evoc.label_propagation_init(_tuple(g), 20, 5, 300, 4, 0.5, 0.1, 0.5, np.random.RandomState(1), None,
                                    base_init="spectral")
    # the random base init takes any threshold
    out = evoc.label_propagation_init(_tuple(g), 20, 5, 300, 4, 0.5, 0.1, 0.5, np.random.RandomState(1), None,
                                      base_init="random", base_init_threshold=500)
    assert out.shape == (len(x), 4) and np.all(np.isfinite(out))
