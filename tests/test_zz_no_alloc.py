"""The entry point that allocates no device memory.

evoc_gpu_knn_f32_noalloc exists for callers that may not let a library call
cudaMalloc (a process whose memory pool owns the whole GPU, a latency-bound
loop that cannot take cudaMalloc's implicit synchronisation).  Its scratch is
a fixed array inside the library, shared by every call on the device, so this
test calls it twice in a row and checks both results against the regular
entry point (evoc_gpu_knn_graph, FP32 form) with the FP32 tolerance used by
the other tests.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import evoc
from evoc import _lib

pytestmark = pytest.mark.gpu


def _noalloc():
    L = _lib.lib()
    f = L.evoc_gpu_knn_f32_noalloc
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.POINTER(C.c_int32), C.c_char_p, C.c_int32]
    f.restype = C.c_int
    return f


def _rows(n, d, seed):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((7, d))
    x = (c[rng.integers(0, 7, n)] + 0.3 * rng.standard_normal((n, d))).astype(np.float32)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return x


def _run(f, xt, n, d, k, stream):
    import torch

    kk = max(1, min(k, n - 1))
    oi = torch.full((n, kk), -7, dtype=torch.int32, device="cuda")
    od = torch.full((n, kk), -7.0, dtype=torch.float32, device="cuda")
    kout = C.c_int32(0)
    err = C.create_string_buffer(256)
    rc = f(xt.data_ptr(), n, d, k, oi.data_ptr(), od.data_ptr(), stream, C.byref(kout), err, 256)
    assert rc == 0, err.value
    assert kout.value == kk
    return oi, od


def test_noalloc_matches_regular_entry_point_on_two_calls():
    import torch

    f = _noalloc()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    cases = [(3000, 64, 15, 1), (1500, 128, 40, 2)]
    outs = []
    data = []
    for n, d, k, seed in cases:  # two calls in a row, nothing in between
        x = _rows(n, d, seed)
        xt = torch.from_numpy(x).cuda()
        data.append(x)
        outs.append(_run(f, xt, n, d, k, stream))
    torch.cuda.synchronize()
    for (n, d, k, seed), x, (oi, od) in zip(cases, data, outs):
        ri, rd = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=k, form="fp32"))
        gi, gd = oi.cpu().numpy(), od.cpu().numpy()
        assert np.all(np.abs(gd - rd) <= 1e-6)
        diff = gi != ri
        assert np.all(np.abs(gd[diff] - rd[diff]) <= 1e-6)  # only tie swaps
        assert np.all(gi[:, 0] == np.arange(n))


def test_noalloc_matches_the_oracle():
    """Directly against the oracle's exact FP32 selection (not only through the regular entry point):
    indices equal except ties within 1e-6, raw values held to FP64 truth within 1e-6."""
    import torch

    from oracle import oracle as O

    f = _noalloc()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    n, d, k = 1200, 48, 12
    x = _rows(n, d, 9)
    oi, od = _run(f, torch.from_numpy(x).cuda(), n, d, k, stream)
    torch.cuda.synchronize()
    gi, gd = oi.cpu().numpy(), od.cpu().numpy()
    ei, er = O.exact_knn(x, k)
    x64 = x.astype(np.float64)
    dots = np.einsum("rkd,rd->rk", x64[gi], x64)
    want = np.where(dots > 0, -dots, 1.17549435e-38)  # FP64 raw of the pairs the GPU returned
    want[gi == np.arange(n)[:, None]] = -1.0
    diff = gi != ei
    assert np.all(np.abs(want[diff] - er[diff]) <= 1e-6)  # a differing entry ties the oracle's
    assert diff.sum() <= max(8, 0.01 * gi.size)
    assert np.allclose(gd, O.transform(O.DT_F32, want.astype(np.float32)), atol=1e-5)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    f = _noalloc()
    xt = torch.from_numpy(_rows(200, 32, 3)).cuda()
    oi = torch.empty((200, 100), dtype=torch.int32, device="cuda")
    od = torch.empty((200, 100), dtype=torch.float32, device="cuda")
    err = C.create_string_buffer(256)
    rc = f(xt.data_ptr(), 200, 32, 100, oi.data_ptr(), od.data_ptr(), None, None, err, 256)
    assert rc == _lib.EVOC_ERR_UNSUPPORTED
    assert b"at most 64" in err.value
    rc = f(xt.data_ptr(), 200, 20, 10, oi.data_ptr(), od.data_ptr(), None, None, err, 256)
    assert rc == _lib.EVOC_ERR_ARG
    rc = f(xt.data_ptr(), 200, (1 << 31) + 16, 10, oi.data_ptr(), od.data_ptr(), None, None, err, 256)
    assert rc == _lib.EVOC_ERR_ARG and b"int32" in err.value  # stride beyond the kernel's int range


def test_noalloc_k64_grid_capped_by_the_fixed_scratch():
    """k = 64 with more than 128 * 128 rows: the persistent grid is capped by what fits in the fixed
    array (128 CTAs), so every CTA reuses its candidate buffers over several query blocks.  Checked
    against an FP64 brute force on a sample of rows (sets equal up to ties within 1e-6)."""
    import torch

    f = _noalloc()
    n, d, k = 20_000, 64, 64
    x = _rows(n, d, 5)
    xt = torch.from_numpy(x).cuda()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    oi, od = _run(f, xt, n, d, k, stream)
    torch.cuda.synchronize()
    gi, gd = oi.cpu().numpy(), od.cpu().numpy()
    x64 = x.astype(np.float64)
    rows = np.arange(0, n, 97)
    for r in rows:
        dots = x64 @ x64[r]
        raw = np.where(dots > 0, -dots, 1.17549435e-38)
        raw[r] = -1.0
        order = np.lexsort((np.arange(n), raw))
        want = order[:k]
        kth = raw[want[-1]]
        got = gi[r]
        assert got[0] == r
        assert len(set(got)) == k
        # every returned key is within 1e-6 of the k-th, or among the exact k
        extra = set(got) - set(want)
        assert all(raw[j] <= kth + 1e-6 for j in extra), (r, extra)
        assert np.all(np.diff(gd[r]) >= -1e-6)
