"""Fuzzy simplicial set on the GPU: the host-side mirror of evoc-rs
src/graph_construction.rs.

  smooth_knn_dist          src/graph_construction.rs:16-80   (-> evoc_gpu_smooth_knn_dist)
  neighbor_graph_matrix    src/graph_construction.rs:176-189 (-> evoc_gpu_fuzzy_graph)
The result is returned as a scipy.sparse.csr_matrix (f32 data, sorted
columns), the counterpart of the reference's sprs CsMat<f32>.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .knn import BackendError, EmptyData


def _check(st: int, ctx) -> None:
    if st == _lib.EVOC_OK:
        return
    if st == _lib.EVOC_ERR_EMPTY:
        raise EmptyData()
    raise BackendError(st, ctx.last_error())


def smooth_knn_dist(distances: np.ndarray, k: float, device: int = 0):
    """(sigma, rho), each f32 of length n."""
    d = np.ascontiguousarray(distances, np.float32)
    n, kk = d.shape
    s = np.empty(n, np.float32)
    r = np.empty(n, np.float32)
    ctx = _lib.context(device)
    P = C.c_void_p
    st = _lib.lib().evoc_gpu_smooth_knn_dist(ctx.h, d.ctypes.data_as(P), n, kk, float(k), 0, s.ctypes.data_as(P),
                                             r.ctypes.data_as(P))
    _check(st, ctx)
    return s, r


def neighbor_graph_csr(n_neighbors: float, knn_indices: np.ndarray, knn_dists: np.ndarray, symmetrize: bool = True,
                       device: int = 0):
    """(indptr int64, indices int32, data f32, sigma, rho) of the fuzzy graph."""
    ind = np.ascontiguousarray(knn_indices, np.int32)
    dst = np.ascontiguousarray(knn_dists, np.float32)
    n, k = ind.shape
    cap = 2 * n * k
    indptr = np.empty(n + 1, np.int64)
    indices = np.empty(max(cap, 1), np.int32)
    data = np.empty(max(cap, 1), np.float32)
    sigma = np.empty(n, np.float32)
    rho = np.empty(n, np.float32)
    nnz = C.c_int64(0)
    ctx = _lib.context(device)
    P = C.c_void_p
    st = _lib.lib().evoc_gpu_fuzzy_graph(ctx.h, ind.ctypes.data_as(P), dst.ctypes.data_as(P), n, k,
                                         float(n_neighbors), 1 if symmetrize else 0, 0, sigma.ctypes.data_as(P),
                                         rho.ctypes.data_as(P), indptr.ctypes.data_as(P), indices.ctypes.data_as(P),
                                         data.ctypes.data_as(P), cap, C.byref(nnz))
    _check(st, ctx)
    m = nnz.value
    return indptr, indices[:m].copy(), data[:m].copy(), sigma, rho


def neighbor_graph_matrix(n_neighbors: float, knn_indices: np.ndarray, knn_dists: np.ndarray,
                          symmetrize: bool = True, device: int = 0):
    """scipy.sparse.csr_matrix of the fuzzy union (or of A when symmetrize is False)."""
    import scipy.sparse as sp

    indptr, indices, data, _, _ = neighbor_graph_csr(n_neighbors, knn_indices, knn_dists, symmetrize, device)
    n = len(indptr) - 1
    return sp.csr_matrix((data, indices, indptr), shape=(n, n))
