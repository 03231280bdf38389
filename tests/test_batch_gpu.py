"""Batches of small requests in one pass (evoc_gpu_knn_graph_batch), on the GPU.

A batch runs one persistent tensor-core launch over the work-list of every
request's query blocks, with the row kernels and the rerank reading their
per-request data from device tables, replayed from a CUDA graph.  Each
request's graph must be identical (indices and distance bits, tolerance 0) to
the one evoc_gpu_knn_graph builds for it alone: the forms are deterministic.
"""
import numpy as np
import pytest
import torch

import evoc
from evoc import _lib
from evoc.knn import BackendError

pytestmark = pytest.mark.gpu


def _f32(n, d, seed, clusters=6):
    r = np.random.default_rng(seed)
    c = r.normal(size=(clusters, d))
    x = c[r.integers(0, clusters, n)] + 0.3 * r.normal(size=(n, d))
    return (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)


def _i8(n, d, seed):
    return np.clip(np.round(127 * _f32(n, d, seed)), -127, 127).astype(np.int8)


SHAPES = [(1, 16), (2, 7), (5, 33), (129, 64), (700, 128), (2048, 384), (3001, 96), (257, 768), (4500, 48)]


def _check(datas, form, k):
    opts = evoc.KnnGraphOptions(n_neighbors=k, form=form)
    got = evoc.knn_graph_batch(datas, opts)
    for x, (ind, dst) in zip(datas, got):
        ei, ed = evoc.knn_graph(x, opts)
        assert ind.shape == ei.shape
        assert np.array_equal(ind, ei)
        assert np.array_equal(dst.view(np.uint32), ed.view(np.uint32))


@pytest.mark.parametrize("k", [1, 10, 15, 30])
def test_f32_batch_equals_single(k):
    _check([_f32(n, d, 11 * n + d) for n, d in SHAPES], "bf16_rerank", k)


@pytest.mark.parametrize("k", [1, 15, 64])
def test_i8_batch_equals_single(k):
    _check([_i8(n, d, 7 * n + d) for n, d in SHAPES], "exact_int", k)


def test_replayed_graph_serves_batches_of_any_size():
    # one context: the first batch captures the graph, later batches of other
    # sizes replay it (fixed table offsets)
    for rep, m in enumerate((3, 9, 1, 40)):
        datas = [_f32(200 + 37 * i, 64 + 16 * (i % 3), 100 * rep + i) for i in range(m)]
        _check(datas, "bf16_rerank", 15)


def test_without_graphs_matches(monkeypatch):
    monkeypatch.setenv("EVOC_NO_GRAPHS", "1")
    ctx = _lib.Context(0)  # reads the variable at creation
    datas = [_i8(n, d, n) for n, d in SHAPES[:6]]
    xs = [torch.from_numpy(x).cuda() for x in datas]
    oi = [torch.empty((len(x), max(1, min(15, len(x) - 1))), dtype=torch.int32, device="cuda") for x in datas]
    od = [torch.empty(t.shape, dtype=torch.float32, device="cuda") for t in oi]
    import ctypes as C

    torch.cuda.synchronize()  # uploads on torch's stream finish before the library's stream reads them
    m = len(datas)
    P = C.c_void_p
    o = _lib.default_opts()
    o.buffers_on_device = 1
    st = _lib.lib().evoc_gpu_knn_graph_batch(
        ctx.h, C.byref(o), _lib.DTYPE_I8, m, (P * m)(*[P(t.data_ptr()) for t in xs]),
        (C.c_int64 * m)(*[len(x) for x in datas]), (C.c_int64 * m)(*[x.shape[1] for x in datas]), 15,
        (P * m)(*[P(t.data_ptr()) for t in oi]), (P * m)(*[P(t.data_ptr()) for t in od]), None, None)
    assert st == _lib.EVOC_OK, ctx.last_error()
    for x, a, b in zip(datas, oi, od):
        ei, ed = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=15, form="exact_int"))
        assert np.array_equal(a.cpu().numpy(), ei) and np.array_equal(b.cpu().numpy(), ed)
    ctx.close()


def test_batch_errors():
    x = _f32(100, 16, 1)
    with pytest.raises(evoc.InvalidNeighbors):
        evoc.knn_graph_batch([x], evoc.KnnGraphOptions(n_neighbors=0))
    with pytest.raises(evoc.EmptyData):
        evoc.knn_graph_batch([x, np.zeros((0, 16), np.float32)], evoc.KnnGraphOptions(n_neighbors=5))
    with pytest.raises(BackendError) as e:  # 2k = 100 candidates exceed the batch's shared-memory heaps
        evoc.knn_graph_batch([x], evoc.KnnGraphOptions(n_neighbors=50, form="bf16_rerank"))
    assert e.value.status == _lib.EVOC_ERR_UNSUPPORTED
    with pytest.raises(BackendError) as e:
        evoc.knn_graph_batch([x], evoc.KnnGraphOptions(n_neighbors=5, form="fp32"))
    assert e.value.status == _lib.EVOC_ERR_UNSUPPORTED
