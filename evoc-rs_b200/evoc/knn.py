"""kNN graph construction on the GPU: the host-side mirror of evoc-rs src/knn.rs.

Names, argument meaning and error behaviour follow the reference:
  EmbeddingData      src/knn.rs:16-30
  KnnError           src/knn.rs:32-41
  KnnGraphOptions    src/knn.rs:44-76
  knn_graph          src/knn.rs:345-359   (-> evoc_gpu_knn_graph)
  knn_graph_ref      src/knn.rs:365-375
The search itself runs in libevoc_gpu.so; this module only marshals arrays
and keeps the reference's RNG draw contract: knn_graph advances the caller's
NumPy RandomState by randint3_for_tau() (3 draws, src/numpy_rng.rs:204-212)
and, unless the integer brute-force branch applies, by the 3*n_trees forest
draws of make_forest (src/knn.rs:124-129), so code that consumes the RNG
afterwards sees the same state as with the CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib

INT32_MIN = -(2**31) + 1  # i32::MIN + 1, src/knn.rs:11
INT32_MAX = 2**31 - 2     # i32::MAX - 1, src/knn.rs:12


class KnnError(Exception):
    """Mirror of KnnError (src/knn.rs:32-41)."""


class EmptyData(KnnError):
    def __init__(self):
        super().__init__("empty embedding matrix")


class InvalidNeighbors(KnnError):
    def __init__(self):
        super().__init__("n_neighbors must be positive")


class BackendError(KnnError):
    """A failure inside the GPU backend (CUDA error, out of memory, unsupported form)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"evoc_gpu status {status}: {message}")
        self.status = status


class EmbeddingData:
    """Tagged embedding matrix (src/knn.rs:16-20): Float32, Int8 or UInt8 (alias Binary)."""

    __slots__ = ("kind", "array")

    def __init__(self, kind: str, array: np.ndarray):
        want = {"Float32": np.float32, "Int8": np.int8, "UInt8": np.uint8}[kind]
        array = np.asarray(array)
        if array.ndim != 2:
            raise ValueError("embedding must be a 2-D array")
        if array.dtype != want:
            raise TypeError(f"{kind} expects dtype {np.dtype(want)}, got {array.dtype}")
        self.kind = kind
        self.array = array

    @classmethod
    def Float32(cls, a):
        return cls("Float32", a)

    @classmethod
    def Int8(cls, a):
        return cls("Int8", a)

    @classmethod
    def UInt8(cls, a):
        return cls("UInt8", a)

    Binary = UInt8

    @classmethod
    def wrap(cls, a) -> "EmbeddingData":
        if isinstance(a, EmbeddingData):
            return a
        a = np.asarray(a)
        kind = {np.dtype(np.float32): "Float32", np.dtype(np.int8): "Int8", np.dtype(np.uint8): "UInt8"}.get(a.dtype)
        if kind is None:
            raise TypeError(f"unsupported embedding dtype {a.dtype}")
        return cls(kind, a)

    def nrows(self) -> int:
        return int(self.array.shape[0])

    @property
    def dtype_code(self) -> int:
        return {"Float32": _lib.DTYPE_F32, "Int8": _lib.DTYPE_I8, "UInt8": _lib.DTYPE_U8}[self.kind]


@dataclass
class KnnGraphOptions:
    """KnnGraphOptions (src/knn.rs:44-76) plus the GPU form selection."""

    n_neighbors: int = 30
    n_trees: Optional[int] = None
    leaf_size: Optional[int] = None
    max_candidates: Optional[int] = None
    max_rptree_depth: int = 200
    n_iters: Optional[int] = None
    delta: float = 0.001
    delta_improv: float = 0.001
    use_sorted_updates: bool = True
    brute_force_max_n: int = 0
    deterministic: bool = False
    # GPU-only fields
    form: str = "auto"          # auto | fp32 | bf16_rerank (= half_rerank) | exact_int | nndescent | popcount
    oversample: int = 0         # bf16_rerank: candidates per row = oversample * k (0: ceil(2.5 k))
    scan_type: str = "fp16"     # bf16_rerank: 16-bit operands of the tensor-core scan, fp16 | bf16
    certify: bool = True        # bf16_rerank: certify every row, rescan the rows that fail
    device: Optional[int] = None  # CUDA device; None = torch's current device when torch is loaded, else 0
    row_begin: int = 0          # exact forms: query rows [row_begin, row_end) only; 0,0 = all
    row_end: int = 0
    # RlxBackend::knn_graph's strict_precision (src/rlx_backend/mod.rs:133-144); knn_graph itself
    # (the crate's free function) has no such argument, so False here
    strict_precision: bool = False


def _n_trees(options: KnnGraphOptions) -> int:
    if options.n_trees is not None:
        return options.n_trees
    threads = 1 if options.deterministic else (os.cpu_count() or 1)
    return max(4, min(8, threads))


def _to_opts(options: KnnGraphOptions, on_device: bool = False) -> _lib.Opts:
    o = _lib.default_opts()
    o.form = _lib.FORM_NAMES[options.form]
    o.oversample = int(options.oversample)
    o.buffers_on_device = 1 if on_device else 0
    o.deterministic = 1 if options.deterministic else 0
    o.n_iters = int(options.n_iters or 0)
    o.max_candidates = int(options.max_candidates or 0)
    o.delta = float(options.delta)
    o.delta_improv = float(options.delta_improv)
    o.row_begin = int(options.row_begin)
    o.row_end = int(options.row_end)
    o.strict_precision = 1 if options.strict_precision else 0
    o.scan_type = _lib.SCAN_TYPES[options.scan_type]
    o.brute_force_max_n = int(options.brute_force_max_n)
    o.certify = 1 if options.certify else 0
    return o


def device_of(options: KnnGraphOptions) -> int:
    """The CUDA device a call runs on: options.device, else torch's current device (so a process
    that pinned its GPU with torch.cuda.set_device -- one rank per GPU -- computes there), else 0."""
    if options.device is not None:
        return int(options.device)
    import sys

    torch = sys.modules.get("torch")
    if torch is not None and torch.cuda.is_available() and torch.cuda.is_initialized():
        return int(torch.cuda.current_device())
    return 0


def _advance_rng(rng, data: EmbeddingData, options: KnnGraphOptions) -> np.ndarray:
    """The reference's draws: randint3_for_tau, then make_forest's 3*n_trees."""
    tau = np.array([rng.randint(INT32_MIN, INT32_MAX) for _ in range(3)], dtype=np.int64)
    n = data.nrows()
    brute = n <= options.brute_force_max_n and data.kind != "Float32"
    if not brute:
        for _ in range(3 * _n_trees(options)):
            rng.randint(INT32_MIN, INT32_MAX)
    return tau


def _raise_for(status: int, ctx: _lib.Context) -> None:
    if status == _lib.EVOC_OK:
        return
    if status == _lib.EVOC_ERR_EMPTY:
        raise EmptyData()
    if status == _lib.EVOC_ERR_K:
        raise InvalidNeighbors()
    raise BackendError(status, ctx.last_error())


def knn_graph(data, options: KnnGraphOptions, rng=None, *, return_raw: bool = False, out=None):
    """Build the kNN graph on the GPU.  Returns (indices int32 (m,k), distances f32 (m,k)) where m
    is n, or row_end - row_begin when a row slice is requested.  `out` may supply preallocated
    (indices, distances) arrays (e.g. pinned host memory)."""
    data = EmbeddingData.wrap(data)
    if options.n_neighbors <= 0:
        raise InvalidNeighbors()
    if data.nrows() == 0:
        raise EmptyData()
    if options.strict_precision and not (data.kind != "Float32" and data.nrows() <= options.brute_force_max_n):
        # refused before any RNG draw (the library refuses the same call with EVOC_ERR_UNSUPPORTED)
        raise BackendError(_lib.EVOC_ERR_UNSUPPORTED, "strict_precision: only i8/u8 data with n <= "
                           "brute_force_max_n (the reference's brute-force branch) is bit-identical to Strict")
    tau = _advance_rng(rng, data, options) if rng is not None else np.zeros(3, np.int64)
    arr = np.ascontiguousarray(data.array)
    n, dim = arr.shape
    k = max(1, min(options.n_neighbors, n - 1))
    m = (options.row_end - options.row_begin) if (options.row_begin or options.row_end) else n
    ctx = _lib.context(device_of(options))
    o = _to_opts(options)
    if out is not None:
        ind, dst = out
        assert ind.shape == (m, k) and ind.dtype == np.int32 and ind.flags.c_contiguous
        assert dst.shape == (m, k) and dst.dtype == np.float32 and dst.flags.c_contiguous
    else:
        ind = np.empty((m, k), np.int32)
        dst = np.empty((m, k), np.float32)
    raw = np.empty((m, k), np.float32) if return_raw else None
    kout = C.c_int32(0)
    P = C.c_void_p
    if return_raw:
        st = _lib.lib().evoc_gpu_knn_graph_raw(ctx.h, C.byref(o), data.dtype_code, arr.ctypes.data_as(P), n, dim,
                                              int(options.n_neighbors), tau.ctypes.data_as(P),
                                              ind.ctypes.data_as(P), dst.ctypes.data_as(P), raw.ctypes.data_as(P),
                                              C.byref(kout))
    else:
        st = _lib.lib().evoc_gpu_knn_graph(ctx.h, C.byref(o), data.dtype_code, arr.ctypes.data_as(P), n, dim,
                                          int(options.n_neighbors), tau.ctypes.data_as(P), ind.ctypes.data_as(P),
                                          dst.ctypes.data_as(P), C.byref(kout))
    _raise_for(st, ctx)
    assert kout.value == k
    return (ind, dst, raw) if return_raw else (ind, dst)


def knn_graph_ref(data, options: KnnGraphOptions, rng=None):
    """Same as knn_graph; the GPU path never takes ownership of the caller's array."""
    return knn_graph(data, options, rng)


def knn_graph_device(ptr: int, dtype_code: int, n: int, dim: int, k: int, out_idx_ptr: int, out_dist_ptr: int,
                     options: Optional[KnnGraphOptions] = None, tau: Optional[np.ndarray] = None,
                     out_raw_ptr: int = 0) -> int:
    """Device-pointer entry: all buffers live on the context's GPU (e.g. torch tensors)."""
    options = options or KnnGraphOptions(n_neighbors=k)
    ctx = _lib.context(device_of(options))
    o = _to_opts(options, on_device=True)
    tau = np.zeros(3, np.int64) if tau is None else np.ascontiguousarray(tau, np.int64)
    kout = C.c_int32(0)
    P = C.c_void_p
    st = _lib.lib().evoc_gpu_knn_graph_raw(ctx.h, C.byref(o), dtype_code, P(ptr), n, dim, k, tau.ctypes.data_as(P),
                                          P(out_idx_ptr), P(out_dist_ptr) if out_dist_ptr else None,
                                          P(out_raw_ptr) if out_raw_ptr else None, C.byref(kout))
    _raise_for(st, ctx)
    return kout.value


def knn_graph_batch_device(ptrs, dtype_code: int, ns, dims, k: int, out_idx_ptrs, out_dist_ptrs,
                           options: Optional[KnnGraphOptions] = None, out_raw_ptrs=None) -> list[int]:
    """Many graphs in one pass (evoc_gpu_knn_graph_batch); every pointer is a device pointer.
    Returns k_eff of each request."""
    options = options or KnnGraphOptions(n_neighbors=k)
    ctx = _lib.context(device_of(options))
    o = _to_opts(options, on_device=True)
    m = len(ptrs)
    P = C.c_void_p
    arr = lambda xs: (P * m)(*[P(int(x)) if x else None for x in xs])  # noqa: E731
    n = (C.c_int64 * m)(*[int(v) for v in ns])
    d = (C.c_int64 * m)(*[int(v) for v in dims])
    kout = (C.c_int32 * m)()
    raw = arr(out_raw_ptrs) if out_raw_ptrs is not None else None
    st = _lib.lib().evoc_gpu_knn_graph_batch(ctx.h, C.byref(o), dtype_code, m, arr(ptrs), n, d, int(k),
                                            arr(out_idx_ptrs), arr(out_dist_ptrs), raw, kout)
    _raise_for(st, ctx)
    return list(kout)


def knn_graph_batch(datas, options: KnnGraphOptions, rngs=None):
    """Build the graphs of many embedding sets of one dtype in one pass.  Returns a list of
    (indices, distances) as knn_graph returns them; each result equals knn_graph on that set.
    With `rngs`, each RandomState is advanced by knn_graph's draws."""
    import torch

    datas = [EmbeddingData.wrap(x) for x in datas]
    if options.n_neighbors <= 0:
        raise InvalidNeighbors()
    if not datas:
        return []
    if any(x.nrows() == 0 for x in datas):
        raise EmptyData()
    if rngs is not None:
        for x, r in zip(datas, rngs):
            _advance_rng(r, x, options)
    code = datas[0].dtype_code
    dev = torch.device("cuda", device_of(options))
    xs = [torch.from_numpy(np.ascontiguousarray(x.array)).to(dev) for x in datas]
    ks = [max(1, min(options.n_neighbors, x.nrows() - 1)) for x in datas]
    oi = [torch.empty((x.nrows(), kk), dtype=torch.int32, device=dev) for x, kk in zip(datas, ks)]
    od = [torch.empty((x.nrows(), kk), dtype=torch.float32, device=dev) for x, kk in zip(datas, ks)]
    torch.cuda.current_stream(dev).synchronize()  # the library runs on its own stream
    knn_graph_batch_device([t.data_ptr() for t in xs], code, [x.nrows() for x in datas],
                           [x.array.shape[1] for x in datas], options.n_neighbors, [t.data_ptr() for t in oi],
                           [t.data_ptr() for t in od], options)
    return [(a.cpu().numpy(), b.cpu().numpy()) for a, b in zip(oi, od)]


def autotune(kind: str, n: int, dim: int, k: int, form: str = "auto", cache_path: Optional[str] = None,
             device: int = 0) -> dict:
    """Time the scan's kernel variants for requests of this shape (evoc_gpu_autotune) and keep the
    fastest for this device's context; with cache_path, append it to that tuning cache file.
    kind: "Float32", "Int8" or "UInt8"."""
    code = {"Float32": _lib.DTYPE_F32, "Int8": _lib.DTYPE_I8, "UInt8": _lib.DTYPE_U8}[kind]
    ctx = _lib.context(device)
    buf = C.create_string_buffer(2048)
    st = _lib.lib().evoc_gpu_autotune(ctx.h, code, _lib.FORM_NAMES[form], int(n), int(dim), int(k),
                                     cache_path.encode() if cache_path else None, buf, 2048)
    _raise_for(st, ctx)
    lines = buf.value.decode().strip().splitlines()
    variants = {}
    chosen = None
    for ln in lines:
        if ln.startswith("chosen: "):
            chosen = int(ln.split("variant=")[1].split()[0])
        else:
            v, ms = ln.split()[:2]
            variants[int(v)] = float(ms)
    return {"variants_ms": variants, "chosen": chosen, "report": lines}


def transform_distances_float(distances: np.ndarray) -> np.ndarray:
    """transform_distances_float (src/knn.rs:156-171), host-side helper."""
    d = np.asarray(distances, np.float32)
    out = np.zeros_like(d)
    neg = d < 0
    sim = (-d[neg]).astype(np.float64)
    with np.errstate(divide="ignore"):
        v = np.where(sim >= 1.0, 0.0, np.maximum(-np.log2(sim), 0.0))
    out[neg] = v.astype(np.float32)
    return out
