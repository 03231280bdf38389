"""Minimum spanning tree under mutual-reachability distance on the GPU.

Host-side mirror of build_kdtree + parallel_boruvka (src/kdtree.rs:367-413,
src/boruvka.rs:492-593) as build_cluster_layers calls them
(src/clustering.rs:50-80): evoc_gpu_boruvka_mst in libevoc_gpu.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .knn import BackendError, EmptyData


def parallel_boruvka(data, min_samples: int = 5, device: int = 0, return_core: bool = False):
    """(n - 1, 3) f32 edges (from, to, distance) of the MST of `data` (n x dim f32, dim <= 32) under
    mutual reachability with `min_samples`; with return_core also the n squared core distances."""
    x = np.ascontiguousarray(data, np.float32)
    if x.ndim != 2:
        raise ValueError("data must be a 2-D array")
    n, dim = x.shape
    if n == 0:
        raise EmptyData()
    ctx = _lib.context(device)
    edges = np.zeros((max(n - 1, 0), 3), np.float32)
    core = np.empty(n, np.float32)
    ne = C.c_int64(0)
    P = C.c_void_p
    st = _lib.lib().evoc_gpu_boruvka_mst(ctx.h, x.ctypes.data_as(P), n, dim, int(min_samples), 0,
                                         edges.ctypes.data_as(P), core.ctypes.data_as(P), C.byref(ne))
    if st != _lib.EVOC_OK:
        raise BackendError(st, ctx.last_error())
    edges = edges[: ne.value]
    return (edges, core) if return_core else edges


def parallel_boruvka_device(x_ptr: int, n: int, dim: int, min_samples: int, edges_ptr: int, core_ptr: int = 0,
                            device: int = 0) -> int:
    """Device-pointer form: x (n x dim f32), edges ((n-1) x 3 f32) and core (n f32, optional) on the GPU."""
    ctx = _lib.context(device)
    ne = C.c_int64(0)
    P = C.c_void_p
    st = _lib.lib().evoc_gpu_boruvka_mst(ctx.h, P(x_ptr), n, dim, int(min_samples), 1, P(edges_ptr),
                                         P(core_ptr) if core_ptr else None, C.byref(ne))
    if st != _lib.EVOC_OK:
        raise BackendError(st, ctx.last_error())
    return ne.value
