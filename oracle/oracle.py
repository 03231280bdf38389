"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes wrapper over ``oracle/liborc.so``, the plain-C restatement of the
evoc-rs kNN-graph path (``oracle/evoc_oracle.c`` lists every reference
file:line it follows).  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module, and only as the checker;
the product library (``evoc-rs_b200``) never imports or links it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")
REF_COS_PATH = os.path.join(HERE, "_ref", "libref_fast_cosine.so")

DT_F32, DT_I8, DT_U8 = 0, 1, 2
_DTYPES = {np.dtype(np.float32): DT_F32, np.dtype(np.int8): DT_I8, np.dtype(np.uint8): DT_U8}


class MT(C.Structure):
    """NumPy RandomState MT19937 state (src/numpy_rng.rs:11-17)."""

    _fields_ = [("key", C.c_uint32 * 624), ("pos", C.c_int32), ("has_gauss", C.c_int32), ("gauss", C.c_double)]


class KnnOpts(C.Structure):
    """KnnGraphOptions (src/knn.rs:44-76); <=0 selects the reference default."""

    _fields_ = [
        ("n_neighbors", C.c_int64),
        ("n_trees", C.c_int64),
        ("leaf_size", C.c_int64),
        ("max_candidates", C.c_int64),
        ("max_rptree_depth", C.c_int64),
        ("n_iters", C.c_int64),
        ("delta", C.c_float),
        ("delta_improv", C.c_float),
        ("brute_force_max_n", C.c_int64),
        ("deterministic", C.c_int32),
        ("n_threads", C.c_int32),
    ]


_lib = None


def build(force: bool = False) -> None:
    if force or not os.path.exists(LIB_PATH):
        subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        i64 = C.c_int64
        L.orc_mt_seed.argtypes = [C.POINTER(MT), C.c_uint32]
        L.orc_mt_randint.argtypes = [C.POINTER(MT), i64, i64]
        L.orc_mt_randint.restype = i64
        L.orc_mt_normal.argtypes = [C.POINTER(MT)]
        L.orc_mt_normal.restype = C.c_double
        L.orc_mt_randint3_for_tau.argtypes = [C.POINTER(MT), P]
        L.orc_tau_rand_int.argtypes = [P]
        L.orc_tau_rand_int.restype = C.c_int32
        L.orc_distance.argtypes = [C.c_int, P, i64, i64, C.c_int, i64, i64]
        L.orc_distance.restype = C.c_float
        L.orc_forest.argtypes = [C.c_int, P, i64, i64, i64, i64, i64, C.POINTER(MT), i64, P, i64, C.POINTER(i64)]
        L.orc_forest.restype = i64
        L.orc_knn_graph.argtypes = [C.c_int, P, i64, i64, C.POINTER(KnnOpts), C.POINTER(MT), P, P, P,
                                    C.POINTER(i64), C.POINTER(i64)]
        L.orc_knn_graph.restype = C.c_int
        L.orc_brute_force_knn.argtypes = [C.c_int, P, i64, i64, i64, P, P]
        L.orc_brute_force_knn.restype = C.c_int
        L.orc_exact_knn.argtypes = [C.c_int, P, i64, i64, i64, i64, i64, P, P]
        L.orc_transform.argtypes = [C.c_int, P, i64, P]
        L.orc_smooth_knn_dist.argtypes = [P, i64, i64, C.c_float, P, P]
        L.orc_membership.argtypes = [P, P, i64, i64, P, P, P]
        L.orc_fuzzy_graph.argtypes = [P, P, i64, i64, C.c_float, C.c_int, P, P, P, P, P, i64]
        L.orc_fuzzy_graph.restype = i64
        L.orc_prepare_float.argtypes = [P, i64, i64]
        L.orc_prepare_float.restype = C.c_int
        L.orc_set_strict_cosine.argtypes = [P]
        L.orc_num_threads.restype = C.c_int
        L.orc_set_num_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def dtype_code(a: np.ndarray) -> int:
    return _DTYPES[a.dtype]


def use_reference_cosine(enable: bool = True) -> bool:
    """Route the deterministic f32 cosine through the reference's own compiled
    native/fast_cosine.c (oracle/_ref), when it was built.  Returns whether the
    reference function is now in use."""
    L = lib()
    if enable and os.path.exists(REF_COS_PATH):
        ref = C.CDLL(REF_COS_PATH)
        fn = ref.fast_cosine_numba
        L.orc_set_strict_cosine(C.cast(fn, C.c_void_p))
        return True
    L.orc_set_strict_cosine(None)
    return False


class RandomState:
    """Oracle-side NumPy RandomState (MT19937)."""

    def __init__(self, seed: int):
        self.s = MT()
        lib().orc_mt_seed(C.byref(self.s), C.c_uint32(seed & 0xFFFFFFFF))

    def randint(self, low: int, high: int) -> int:
        return int(lib().orc_mt_randint(C.byref(self.s), low, high))

    def normal(self) -> float:
        return float(lib().orc_mt_normal(C.byref(self.s)))

    def randint3_for_tau(self):
        out = np.zeros(3, np.int64)
        lib().orc_mt_randint3_for_tau(C.byref(self.s), _ptr(out))
        return out

    @property
    def key(self) -> np.ndarray:
        return np.frombuffer(bytes(self.s.key), dtype=np.uint32).copy()

    @property
    def pos(self) -> int:
        return int(self.s.pos)


def knn_graph(data: np.ndarray, n_neighbors: int, rng: RandomState, *, deterministic: bool = True,
              n_threads: int = 1, n_trees: int = 0, n_iters: int = 0, max_candidates: int = 0,
              leaf_size: int = 0, delta: float = 0.001, delta_improv: float = 0.001,
              brute_force_max_n: int = 0, return_raw: bool = False):
    """Restated knn_graph (src/knn.rs:345-454). Returns (indices, distances[, raw, iters])."""
    data = np.ascontiguousarray(data)
    n, d = data.shape
    o = KnnOpts(n_neighbors=n_neighbors, n_trees=n_trees, leaf_size=leaf_size, max_candidates=max_candidates,
                max_rptree_depth=200, n_iters=n_iters, delta=delta, delta_improv=delta_improv,
                brute_force_max_n=brute_force_max_n, deterministic=1 if deterministic else 0,
                n_threads=n_threads)
    kk = max(1, min(n_neighbors, max(n - 1, 0)))
    ind = np.empty((n, kk), np.int32)
    raw = np.empty((n, kk), np.float32)
    dst = np.empty((n, kk), np.float32)
    k_out = C.c_int64(0)
    iters = C.c_int64(0)
    rc = lib().orc_knn_graph(dtype_code(data), _ptr(data), n, d, C.byref(o), C.byref(rng.s), _ptr(ind), _ptr(raw),
                             _ptr(dst), C.byref(k_out), C.byref(iters))
    if rc != 0:
        raise ValueError({1: "empty embedding matrix", 2: "n_neighbors must be positive"}[rc])
    if return_raw:
        return ind, dst, raw, int(iters.value)
    return ind, dst


def forest(data: np.ndarray, n_neighbors: int, n_trees: int, rng: RandomState, leaf_size: int = 0):
    data = np.ascontiguousarray(data)
    n, d = data.shape
    leaf = max(10, n_neighbors) if leaf_size <= 0 else leaf_size
    cap = 4 * n_trees * n * max(leaf, 1) + 1024
    out = np.empty(cap, np.int32)
    w = C.c_int64(0)
    rows = lib().orc_forest(dtype_code(data), _ptr(data), n, d, n_neighbors, n_trees, leaf, C.byref(rng.s), 200,
                            _ptr(out), cap, C.byref(w))
    return out[: rows * w.value].reshape(rows, w.value).copy()


def exact_knn(data: np.ndarray, k: int, row0: int = 0, row1: int | None = None):
    """Exact selection under the CUDA forms' contract (self offered with raw
    -1.0, keep k smallest by (raw, index), rows sorted).  Returns (ind, raw)."""
    data = np.ascontiguousarray(data)
    n, d = data.shape
    row1 = n if row1 is None else row1
    ind = np.empty((row1 - row0, k), np.int32)
    raw = np.empty((row1 - row0, k), np.float32)
    lib().orc_exact_knn(dtype_code(data), _ptr(data), n, d, k, row0, row1, _ptr(ind), _ptr(raw))
    return ind, raw


def brute_force_knn(data: np.ndarray, k: int):
    data = np.ascontiguousarray(data)
    n, d = data.shape
    kk = max(1, min(k, n - 1))
    ind = np.empty((n, kk), np.int32)
    raw = np.empty((n, kk), np.float32)
    lib().orc_brute_force_knn(dtype_code(data), _ptr(data), n, d, k, _ptr(ind), _ptr(raw))
    return ind, raw


def transform(dtype: int, raw: np.ndarray) -> np.ndarray:
    raw = np.ascontiguousarray(raw, np.float32)
    out = np.empty_like(raw)
    lib().orc_transform(dtype, _ptr(raw), raw.size, _ptr(out))
    return out


def distance(data: np.ndarray, a: int, b: int, strict: bool = False) -> float:
    data = np.ascontiguousarray(data)
    n, d = data.shape
    return float(lib().orc_distance(dtype_code(data), _ptr(data), n, d, 1 if strict else 0, a, b))


def prepare_float(x: np.ndarray) -> np.ndarray:
    x = np.array(x, np.float32, copy=True, order="C")
    lib().orc_prepare_float(_ptr(x), x.shape[0], x.shape[1])
    return x


def smooth_knn_dist(dists: np.ndarray, k: float):
    dists = np.ascontiguousarray(dists, np.float32)
    n, kk = dists.shape
    s = np.empty(n, np.float32)
    r = np.empty(n, np.float32)
    lib().orc_smooth_knn_dist(_ptr(dists), n, kk, k, _ptr(s), _ptr(r))
    return s, r


def fuzzy_graph(ind: np.ndarray, dists: np.ndarray, k: float, symmetrize: bool = True):
    """neighbor_graph_matrix: returns (indptr i64, indices i32, data f32, sigma, rho)."""
    ind = np.ascontiguousarray(ind, np.int32)
    dists = np.ascontiguousarray(dists, np.float32)
    n, kk = ind.shape
    cap = 2 * n * kk + 1
    indptr = np.empty(n + 1, np.int64)
    indices = np.empty(cap, np.int32)
    data = np.empty(cap, np.float32)
    s = np.empty(n, np.float32)
    r = np.empty(n, np.float32)
    nnz = lib().orc_fuzzy_graph(_ptr(ind), _ptr(dists), n, kk, k, 1 if symmetrize else 0, _ptr(s), _ptr(r),
                                _ptr(indptr), _ptr(indices), _ptr(data), cap)
    assert nnz >= 0
    return indptr, indices[:nnz].copy(), data[:nnz].copy(), s, r


def set_num_threads(t: int) -> None:
    lib().orc_set_num_threads(t)


def num_threads() -> int:
    return int(lib().orc_num_threads())
