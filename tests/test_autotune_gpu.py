"""Autotuner of the tensor-core scan (evoc_gpu_autotune) on the GPU.

Every kernel variant must give the same graph, so a tuned context's results
equal the default context's bit for bit; the tuner writes a cache file that a
new context loads through EVOC_TUNE_CACHE.
"""
import numpy as np
import pytest

import evoc
from evoc import _lib

pytestmark = pytest.mark.gpu


def _f32(n, d, seed):
    r = np.random.default_rng(seed)
    x = r.normal(size=(8, d))[r.integers(0, 8, n)] + 0.3 * r.normal(size=(n, d))
    return (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)


@pytest.mark.parametrize("kind,form,dim", [("Float32", "bf16_rerank", 96), ("Int8", "exact_int", 128),
                                           ("UInt8", "exact_int", 64)])
def test_tuned_variants_keep_results(tmp_path, monkeypatch, kind, form, dim):
    n, k = 3000, 15
    if kind == "Float32":
        x = _f32(n, dim, 1)
    elif kind == "Int8":
        x = np.clip(np.round(127 * _f32(n, dim, 2)), -127, 127).astype(np.int8)
    else:
        x = np.packbits(np.random.default_rng(3).random((n, dim * 8)) < 0.1, axis=1)
    base = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=k, form=form))
    cache = tmp_path / "tune.txt"
    rep = evoc.autotune(kind, n, dim, k, form, str(cache))
    assert rep["chosen"] in rep["variants_ms"] and len(rep["variants_ms"]) >= 2
    assert cache.read_text().startswith("evoc-tune 1 ")
    # every feasible variant, forced one at a time through a fresh context's cache, gives the same graph
    for v in rep["variants_ms"]:
        line = cache.read_text().splitlines()[-1]
        forced = tmp_path / f"v{v}.txt"
        forced.write_text(line.rsplit("variant=", 1)[0] + f"variant={v} ms=0\n")
        monkeypatch.setenv("EVOC_TUNE_CACHE", str(forced))
        ctx = _lib.Context(0)
        try:
            import ctypes as C

            arr = np.ascontiguousarray(x)
            ind = np.empty((n, k), np.int32)
            dst = np.empty((n, k), np.float32)
            o = _lib.default_opts()
            o.form = _lib.FORM_NAMES[form]
            P = C.c_void_p
            code = {"Float32": 0, "Int8": 1, "UInt8": 2}[kind]
            st = _lib.lib().evoc_gpu_knn_graph(ctx.h, C.byref(o), code, arr.ctypes.data_as(P), n, dim, k, None,
                                              ind.ctypes.data_as(P), dst.ctypes.data_as(P), None)
            assert st == 0, ctx.last_error()
            assert np.array_equal(ind, base[0]) and np.array_equal(dst.view(np.uint32), base[1].view(np.uint32))
        finally:
            ctx.close()
        monkeypatch.delenv("EVOC_TUNE_CACHE")


def test_tune_load_and_errors(tmp_path):
    ctx = _lib.Context(0)
    try:
        assert _lib.lib().evoc_gpu_tune_load(ctx.h, str(tmp_path / "missing.txt").encode()) == -1
        p = tmp_path / "t.txt"
        p.write_text("junk\nevoc-tune 1 mode=1 keep=15 row_bytes=128 log2n=11 variant=2 ms=1.0\n")
        assert _lib.lib().evoc_gpu_tune_load(ctx.h, str(p).encode()) == 1
    finally:
        ctx.close()
    with pytest.raises(evoc.BackendError):
        evoc.autotune("Float32", 1000, 64, 15, "fp32")


def _forced_graph(tmp_path, monkeypatch, x, kind, form, k, variant, **opt):
    """The graph with the scan's kernel variant forced through a fresh context's tune cache."""
    import ctypes as C

    n, dim = x.shape
    mode = {"Float32": 0, "Int8": 1, "UInt8": 2}[kind]
    keep = k if form == "exact_int" else (5 * k + 1) // 2
    log2n = int(np.floor(np.log2(n)))
    forced = tmp_path / f"forced{variant}.txt"
    forced.write_text(f"evoc-tune 1 mode={mode} keep={keep} row_bytes={{rb}} log2n={log2n} variant={variant} ms=0\n")
    row_bytes = {"Float32": ((dim + 63) // 64) * 64 * 2, "Int8": ((dim + 127) // 128) * 128,
                 "UInt8": ((dim * 8 + 127) // 128) * 128}[kind]
    forced.write_text(forced.read_text().replace("{rb}", str(row_bytes)))
    monkeypatch.setenv("EVOC_TUNE_CACHE", str(forced))
    ctx = _lib.Context(0)
    try:
        arr = np.ascontiguousarray(x)
        r0, r1 = opt.get("row_begin", 0), opt.get("row_end", 0)
        m = (r1 - r0) if (r0 or r1) else n
        ind = np.empty((m, k), np.int32)
        dst = np.empty((m, k), np.float32)
        o = _lib.default_opts()
        o.form = _lib.FORM_NAMES[form]
        o.row_begin, o.row_end = r0, r1
        P = C.c_void_p
        st = _lib.lib().evoc_gpu_knn_graph(ctx.h, C.byref(o), {"Float32": 0, "Int8": 1, "UInt8": 2}[kind],
                                          arr.ctypes.data_as(P), n, dim, k, None, ind.ctypes.data_as(P),
                                          dst.ctypes.data_as(P), None)
        assert st == 0, ctx.last_error()
        return ind, dst
    finally:
        ctx.close()
        monkeypatch.delenv("EVOC_TUNE_CACHE")


@pytest.mark.parametrize("variant", [6, 7, 8, 9, 10, 11, 12, 13, 14])
@pytest.mark.parametrize("n", [2900, 300, 129])
def test_cta_pair_variants_match_single_cta(tmp_path, monkeypatch, variant, n):
    """The CTA-pair scans (cluster of two, M = 256 MMAs; variants 6-9) and the four-epilogue-group
    scans (10, 11) give the default graph bit for bit, with an odd number of query blocks (the last
    pair half empty), a single block, and a row slice starting mid-block."""
    x = _f32(n, 96, 7)
    base = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=15, form="bf16_rerank"))
    ind, dst = _forced_graph(tmp_path, monkeypatch, x, "Float32", "bf16_rerank", 15, variant)
    assert np.array_equal(ind, base[0]) and np.array_equal(dst.view(np.uint32), base[1].view(np.uint32))
    if n > 200:
        r0, r1 = 37, n - 11
        ind, dst = _forced_graph(tmp_path, monkeypatch, x, "Float32", "bf16_rerank", 15, variant, row_begin=r0,
                                 row_end=r1)
        assert np.array_equal(ind, base[0][r0:r1]) and np.array_equal(dst.view(np.uint32),
                                                                      base[1][r0:r1].view(np.uint32))
    xi = np.clip(np.round(127 * x), -127, 127).astype(np.int8)
    bi = evoc.knn_graph(xi, evoc.KnnGraphOptions(n_neighbors=15, form="exact_int"))
    ind, dst = _forced_graph(tmp_path, monkeypatch, xi, "Int8", "exact_int", 15, variant)
    assert np.array_equal(ind, bi[0]) and np.array_equal(dst.view(np.uint32), bi[1].view(np.uint32))
