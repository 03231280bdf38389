"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes wrapper over the KD-tree and Borůvka MST restatement in
``oracle/evoc_oracle_mst.c`` (evoc-rs src/kdtree.rs, src/boruvka.rs,
src/disjoint_set.rs; the file lists the lines it follows).  Only ``tests/``
use it, as the checker.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import oracle as O

_ready = False


def _lib():
    global _ready
    L = O.lib()
    if not _ready:
        P, i64 = C.c_void_p, C.c_int64
        L.orc_kdtree_nodes.argtypes = [i64, i64]
        L.orc_kdtree_nodes.restype = i64
        L.orc_kdtree_build.argtypes = [P, i64, i64, i64, P, P, P, P, P, P, P]
        L.orc_boruvka_mst.argtypes = [P, i64, i64, i64, i64, P, P, P]
        L.orc_boruvka_mst.restype = i64
        _ready = True
    return L


_p = O._ptr


def build_kdtree(data: np.ndarray, leaf_size: int = 40) -> dict:
    """build_kdtree (src/kdtree.rs:367-413): idx_array, idx_start, idx_end, radius, is_leaf, bounds."""
    x = np.ascontiguousarray(data, np.float32)
    n, d = x.shape
    nn = int(_lib().orc_kdtree_nodes(n, leaf_size))
    out = dict(idx_array=np.empty(n, np.int64), idx_start=np.empty(nn, np.int64), idx_end=np.empty(nn, np.int64),
               radius=np.empty(nn, np.float32), is_leaf=np.empty(nn, np.uint8), lo=np.empty((nn, d), np.float32),
               hi=np.empty((nn, d), np.float32))
    _lib().orc_kdtree_build(_p(x), n, d, leaf_size, *(_p(out[k]) for k in
                                                      ("idx_array", "idx_start", "idx_end", "radius", "is_leaf", "lo",
                                                       "hi")))
    return out


def boruvka_mst(data: np.ndarray, min_samples: int = 5, leaf_size: int = 40):
    """parallel_boruvka on build_kdtree(data, 40), reproducible path (src/boruvka.rs:492-593).
    Returns (edges (n-1, 3) f32 of from, to, distance; core distances (squared); idx_array)."""
    x = np.ascontiguousarray(data, np.float32)
    n, d = x.shape
    edges = np.zeros((max(n - 1, 1), 3), np.float32)
    core = np.empty(n, np.float32)
    idx = np.empty(n, np.int64)
    ne = _lib().orc_boruvka_mst(_p(x), n, d, leaf_size, min_samples, _p(edges), _p(core), _p(idx))
    return edges[:ne], core, idx
