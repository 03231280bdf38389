"""The tensor-core scan's bounded waits, run out on purpose, on the GPU.

A context's pipeline-wait limit is set far below the time its producer is made
to start late (evoc_gpu_set_wait_limit), so the MMA and epilogue roles give up
on their first wait: the call must end with EVOC_ERR_TIMEOUT (no trap, no
hang), the loads already issued drain under their own full-length limit, the
tensor memory is freed (a later scan on every SM allocates it again), and the
next call on the same context, with the default limit, gives the normal
result.
"""
import numpy as np
import pytest

import evoc
from evoc import _lib

pytestmark = pytest.mark.gpu


def _rows(n, d, seed, dtype=np.float32):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, d))
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    if dtype == np.int8:
        return np.clip(np.round(127 * x), -127, 127).astype(np.int8)
    return x.astype(np.float32)


@pytest.mark.parametrize("dtype,form", [(np.float32, "bf16_rerank"), (np.int8, "exact_int")])
def test_wait_that_runs_out_returns_timeout_and_context_recovers(dtype, form):
    x = _rows(4096, 128, 1, dtype)
    opts = evoc.KnnGraphOptions(n_neighbors=15, form=form, device=0)
    ctx = _lib.context(0)
    want_i, want_d = evoc.knn_graph(x, opts)
    ctx.set_wait_limit(50_000, 2_000_000)  # 50 us per wait; the producer starts after 2 ms
    try:
        for _ in range(2):  # twice: a failed call must leave nothing behind for the next failure either
            with pytest.raises(evoc.BackendError) as e:
                evoc.knn_graph(x, opts)
            assert e.value.status == _lib.EVOC_ERR_TIMEOUT, str(e.value)
            assert "timed out" in str(e.value)
    finally:
        ctx.set_wait_limit(0, 0)
    got_i, got_d = evoc.knn_graph(x, opts)
    assert np.array_equal(got_i, want_i) and np.array_equal(got_d.view(np.uint32), want_d.view(np.uint32))
    # a bigger scan on every SM after the timeouts: tensor memory was freed by the failed launches
    y = _rows(40_000, 256, 2, dtype)
    yi, _ = evoc.knn_graph(y, opts)
    assert yi.shape == (len(y), 15) and np.all(yi >= 0)
    if dtype == np.float32:
        assert np.all(yi[:, 0] == np.arange(len(y)))  # self first (raw -1.0; int8 ranks it last)


def test_wait_limit_arguments():
    ctx = _lib.context(0)
    with pytest.raises(ValueError):
        ctx.set_wait_limit(1000, 10**9)  # producer delay above 100 ms is refused
    ctx.set_wait_limit(0, 0)
