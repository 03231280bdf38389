"""Serving loop (evoc_gpu_server_*) on the GPU.

The headline property: each request's graph is the same alone and in the mix.
The forms are deterministic, so "the same" is bit-identical indices and
distances (tolerance 0) against a knn_graph call on the same rows made with no
other work on the device.  The other tests cover admission against the HBM
budget, overlap of running requests, cancellation, failure isolation,
completion reporting and the RNG draw contract.
"""
import time

import numpy as np
import pytest

import evoc
from evoc import _lib
from evoc.knn import BackendError
from evoc.serving import JobCancelled, Server

pytestmark = pytest.mark.gpu


def _f32(n, d, seed):
    r = np.random.default_rng(seed)
    c = r.normal(size=(8, d))
    x = c[r.integers(0, 8, n)] + 0.3 * r.normal(size=(n, d))
    return (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)


def _i8(n, d, seed):
    return np.clip(np.round(127 * _f32(n, d, seed)), -127, 127).astype(np.int8)


def _u8(n, nbytes, seed):
    r = np.random.default_rng(seed)
    protos = r.random((20, nbytes * 8)) < 0.1
    bits = protos[r.integers(0, 20, n)] ^ (r.random((n, nbytes * 8)) < 0.05)
    return np.packbits(bits, axis=1)


MIX = [
    ("bf16_rerank", lambda: _f32(3000, 128, 1), 15),
    ("fp32", lambda: _f32(1500, 96, 2), 15),
    ("exact_int", lambda: _i8(2500, 384, 3), 15),
    ("exact_int", lambda: _u8(2000, 128, 4), 15),
    ("bf16_rerank", lambda: _f32(777, 768, 5), 10),
    ("nndescent", lambda: _f32(4000, 64, 6), 15),
    ("bf16_rerank", lambda: _f32(5, 16, 7), 15),  # k clamps to n - 1
    ("exact_int", lambda: _i8(1, 32, 8), 15),  # a single row
]


def _opts(form, k):
    return evoc.KnnGraphOptions(n_neighbors=k, form=form, deterministic=True)


@pytest.fixture(scope="module")
def alone():
    """Each request's graph built with nothing else on the device."""
    out = []
    for form, make, k in MIX:
        x = make()
        ind, dst = evoc.knn_graph(x, _opts(form, k), np.random.RandomState(11))
        out.append((x, ind, dst))
    return out


@pytest.mark.parametrize("lanes,admission,small_lanes", [(1, "oldest", 0), (4, "oldest", 0), (4, "smallest", 0),
                                                         (4, "smallest", 2)])
def test_same_result_alone_and_in_the_mix(alone, lanes, admission, small_lanes):
    with Server(max_inflight=lanes, admission=admission, small_lanes=small_lanes) as srv:
        jobs = []
        for rep in range(2):  # every request twice, interleaved
            for (form, _, k), (x, _, _) in zip(MIX, alone):
                jobs.append(srv.submit(x, _opts(form, k), np.random.RandomState(11), borrow=rep == 1))
        for i, j in enumerate(jobs):
            ind, dst = srv.result(j)
            _, ei, ed = alone[i % len(MIX)]
            assert ind.shape == ei.shape
            assert np.array_equal(ind, ei), (i, MIX[i % len(MIX)][0])
            assert np.array_equal(dst.view(np.uint32), ed.view(np.uint32)), i
        st = srv.stats()
        assert st["completed"] == len(jobs) and st["failed"] == 0
        assert st["workspace_misses"] == 0, "a form allocated more than its buffer plan"
        assert st["bytes_in_use"] == st["workspace_bytes"] and st["peak_bytes"] <= st["budget_bytes"]


def test_small_requests_are_batched_with_identical_results():
    """Many small requests submitted together are built in multi-request
    batches; each graph equals the one built alone."""
    xs = [(_f32(300 + 53 * i, 32 + 16 * (i % 4), 90 + i) if i % 3 else _i8(400 + 31 * i, 128, 90 + i))
          for i in range(40)]
    forms = ["exact_int" if x.dtype == np.int8 else "bf16_rerank" for x in xs]
    want = [evoc.knn_graph(x, _opts(f, 15)) for x, f in zip(xs, forms)]
    with Server(max_inflight=2) as srv:
        jobs = [srv.submit(x, _opts(f, 15)) for x, f in zip(xs, forms)]
        got = [srv.result(j) for j in jobs]
        st = srv.stats()
    assert st["batches"] >= 1 and st["batched"] > st["batches"], st
    assert st["workspace_misses"] == 0
    for (gi, gd), (wi, wd) in zip(got, want):
        assert np.array_equal(gi, wi) and np.array_equal(gd.view(np.uint32), wd.view(np.uint32))


def test_requests_overlap_on_the_device():
    """With four lanes, requests submitted together run at the same time."""
    xs = [_f32(20000, 256, 20 + i) for i in range(8)]
    with Server(max_inflight=4) as srv:
        jobs = [srv.submit(x, _opts("bf16_rerank", 15)) for x in xs]
        for j in jobs:
            srv.wait(j)
        spans = sorted((srv.info(j)["admit_ns"], srv.info(j)["done_ns"]) for j in jobs)
        lanes = {srv.info(j)["lane"] for j in jobs}
        for j in jobs:
            srv.release(j)
    overlapping = sum(1 for a, b in zip(spans, spans[1:]) if b[0] < a[1])
    assert overlapping >= 1, spans
    assert len(lanes) > 1


def test_admission_respects_the_budget():
    """A budget that holds one request at a time serialises four lanes; the
    planned lane buffers match what the contexts really allocate."""
    x = _f32(30000, 256, 30)
    with Server(max_inflight=2) as probe:
        res_b, ws_b = probe.request_bytes(_lib.DTYPE_F32, 30000, 256, _opts("fp32", 15))
    assert res_b == 30000 * 256 * 4 + 30000 * 15 * 8 and ws_b > 30000 * 256 * 4
    with Server(max_inflight=4, budget_bytes=int(1.5 * (res_b + ws_b))) as srv:
        jobs = [srv.submit(x, _opts("fp32", 15)) for _ in range(4)]
        res = [srv.result(j, keep_resident=True) for j in jobs]
        spans = sorted((srv.info(j)["admit_ns"], srv.info(j)["done_ns"]) for j in jobs)
        for j in jobs:
            srv.release(j)
        st = srv.stats()
        assert st["peak_bytes"] <= st["budget_bytes"]
        assert st["completed"] == 4 and st["workspace_misses"] == 0
        assert st["bytes_in_use"] == st["workspace_bytes"]
    assert all(b[0] >= a[1] for a, b in zip(spans, spans[1:])), spans
    for ind, dst in res[1:]:
        assert np.array_equal(ind, res[0][0]) and np.array_equal(dst, res[0][1])
    with Server(max_inflight=2, budget_bytes=10_000_000) as srv:
        with pytest.raises(BackendError) as e:
            srv.submit(_f32(20000, 512, 31), _opts("bf16_rerank", 15))
        assert e.value.status == _lib.EVOC_ERR_OOM
        assert srv.stats()["rejected"] == 1


def test_cancel_pending_and_failure_isolation():
    with Server(max_inflight=1) as srv:
        big = srv.submit(_f32(40000, 256, 40), _opts("bf16_rerank", 15))
        pend = srv.submit(_f32(1000, 64, 41), _opts("bf16_rerank", 15))
        srv.cancel(pend)
        bad = srv.submit(_i8(500, 64, 42), _opts("fp32", 15))  # fp32 form is f32-only
        ok = srv.submit(_i8(500, 64, 42), _opts("exact_int", 15))
        with pytest.raises(JobCancelled):
            srv.result(pend)
        with pytest.raises(BackendError) as e:
            srv.result(bad)
        assert e.value.status == _lib.EVOC_ERR_UNSUPPORTED
        ind, _ = srv.result(ok)
        assert np.array_equal(ind, evoc.knn_graph(_i8(500, 64, 42), _opts("exact_int", 15))[0])
        srv.result(big)
        st = srv.stats()
        assert st["cancelled"] == 1 and st["failed"] == 1 and st["completed"] == 2


def test_wait_any_reports_each_job_once():
    with Server(max_inflight=3) as srv:
        jobs = {srv.submit(_f32(500 + 100 * i, 32, 50 + i), _opts("bf16_rerank", 10)) for i in range(12)}
        seen = []
        while len(seen) < len(jobs):
            got = srv.wait_any(timeout=60)
            assert got is not None
            jid, rc = got
            assert rc == _lib.EVOC_OK
            seen.append(jid)
        assert sorted(seen) == sorted(jobs)
        assert srv.wait_any(timeout=0.05) is None
        for j in jobs:
            srv.release(j)


def test_submit_keeps_the_rng_contract_and_errors():
    x = _f32(600, 48, 60)
    r1, r2 = np.random.RandomState(5), np.random.RandomState(5)
    a = evoc.knn_graph(x, _opts("nndescent", 15), r1)
    with Server(max_inflight=2) as srv:
        j = srv.submit(x, _opts("nndescent", 15), r2)
        b = srv.result(j)
        assert np.array_equal(r1.get_state()[1], r2.get_state()[1])
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        with pytest.raises(evoc.InvalidNeighbors):
            srv.submit(x, _opts("bf16_rerank", 0))
        with pytest.raises(evoc.EmptyData):
            srv.submit(np.zeros((0, 8), np.float32), _opts("bf16_rerank", 5))


def test_device_rows_and_resident_result():
    import torch

    x = _f32(2048, 128, 70)
    ind0, dst0 = evoc.knn_graph(x, _opts("bf16_rerank", 15))
    t = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()  # the upload runs on torch's stream; the lanes read on their own
    with Server(max_inflight=2) as srv:
        j = srv.submit_device(t.data_ptr(), _lib.DTYPE_F32, 2048, 128, _opts("bf16_rerank", 15), keep_alive=t)
        assert srv.wait(j, timeout=60) == _lib.EVOC_OK
        pi, pd, k = srv.result_device(j)
        assert pi and pd and k == 15
        ind, dst = srv.result(j, keep_resident=True)
        assert np.array_equal(ind, ind0) and np.array_equal(dst, dst0)
        ind2, _ = srv.result(j)  # second fetch, then released
        assert np.array_equal(ind2, ind0)
        st = srv.stats()
        assert st["bytes_in_use"] == st["workspace_bytes"]


def test_timing_fields_are_ordered():
    with Server(max_inflight=2) as srv:
        t0 = srv.now_ns()
        j = srv.submit(_f32(1000, 64, 80), _opts("bf16_rerank", 15))
        srv.wait(j)
        info = srv.info(j)
        assert t0 <= info["submit_ns"] <= info["admit_ns"] <= info["done_ns"] <= srv.now_ns()
        srv.release(j)
        time.sleep(0.01)
