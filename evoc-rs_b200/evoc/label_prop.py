"""Label-propagation initialisation and node embedding on the GPU: the host
mirror of evoc-rs src/label_prop.rs and src/embed.rs over the C ABI.

  label_prop_loop          src/label_prop.rs:160-185   (-> evoc_gpu_label_prop_loop)
  label_propagation_init   src/label_prop.rs:464-674   (-> evoc_gpu_label_propagation_init_with_options)
  node_embedding           src/embed.rs:251-369        (-> evoc_gpu_node_embedding)

The graph is a scipy.sparse.csr_matrix (or an (indptr, indices, data, n)
tuple); the random_state is a numpy.random.RandomState, advanced by exactly
the draws the reference makes from its NumpyRandomState.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .knn import BackendError, EmptyData

P = C.c_void_p


def _csr(graph):
    if isinstance(graph, tuple):
        indptr, indices, data, n = graph
    else:
        indptr, indices, data, n = graph.indptr, graph.indices, graph.data, graph.shape[0]
    return (np.ascontiguousarray(indptr, np.int64), np.ascontiguousarray(indices, np.int32),
            np.ascontiguousarray(data, np.float32), int(n))


def _rng_in(rs: np.random.RandomState) -> _lib.NumpyRng:
    name, key, pos, has_gauss, gauss = rs.get_state()
    r = _lib.NumpyRng()
    C.memmove(r.key, np.ascontiguousarray(key, np.uint32).ctypes.data, 624 * 4)
    r.pos, r.has_gauss, r.gauss = int(pos), int(has_gauss), float(gauss)
    return r


def _rng_out(rs: np.random.RandomState, r: _lib.NumpyRng) -> None:
    key = np.frombuffer(bytes(r.key), dtype=np.uint32).copy()
    rs.set_state(("MT19937", key, int(r.pos), int(r.has_gauss), float(r.gauss)))


def _check(st: int, ctx) -> None:
    if st == _lib.EVOC_OK:
        return
    if st == _lib.EVOC_ERR_EMPTY:
        raise EmptyData()
    raise BackendError(st, ctx.last_error())


def _state(random_state):
    if random_state is None:
        return np.random.mtrand._rand
    if isinstance(random_state, (int, np.integer)):
        return np.random.RandomState(int(random_state))
    return random_state


def label_prop_loop(graph, random_state, n_iter: int = 20, approx_n_parts: int = 256, device: int = 0):
    """Partition (int64, n) of the graph's vertices; src/label_prop.rs:160-185 from all -1 labels."""
    indptr, indices, data, n = _csr(graph)
    rs = _state(random_state)
    r = _rng_in(rs)
    out = np.empty(n, np.int64)
    n_parts = C.c_int64(0)
    ctx = _lib.context(device)
    st = _lib.lib().evoc_gpu_label_prop_loop(ctx.h, indptr.ctypes.data_as(P), indices.ctypes.data_as(P),
                                             data.ctypes.data_as(P), n, int(n_iter), int(approx_n_parts),
                                             C.byref(r), 0, out.ctypes.data_as(P), C.byref(n_parts))
    _check(st, ctx)
    _rng_out(rs, r)
    return out


def _lp_options(recursive_init: bool, base_init: str, base_init_threshold: int, upscaling: str) -> _lib.LpOptions:
    if base_init not in _lib.BASE_INITS:
        raise ValueError(f"base_init must be one of {sorted(_lib.BASE_INITS)}")
    if upscaling not in _lib.UPSCALINGS:
        raise ValueError(f"upscaling must be one of {sorted(_lib.UPSCALINGS)}")
    o = _lib.LpOptions()
    o.recursive_init = 1 if recursive_init else 0
    o.base_init = _lib.BASE_INITS[base_init]
    o.base_init_threshold = int(base_init_threshold)
    o.upscaling = _lib.UPSCALINGS[upscaling]
    return o


def label_propagation_init(graph, n_label_prop_iter: int = 20, n_embedding_epochs: int = 50,
                           approx_n_parts: int = 512, n_components: int = 4, scaling: float = 0.5,
                           random_scale: float = 0.1, noise_level: float = 0.5, random_state=None, data=None,
                           device: int = 0, recursive_init: bool = True, base_init: str = "pca",
                           base_init_threshold: int = 64, upscaling: str = "partition_expander") -> np.ndarray:
    """Initial (n, n_components) f32 embedding; src/label_prop.rs:464-494, and with the keyword
    arguments of label_propagation_init_with_options (src/label_prop.rs:497-674): base_init one of
    pca / random / spectral / mds, upscaling one of partition_expander / jitter_expander /
    node_embedding."""
    opt = _lp_options(recursive_init, base_init, base_init_threshold, upscaling)
    indptr, indices, gdata, n = _csr(graph)
    rs = _state(random_state)
    r = _rng_in(rs)
    x = None if data is None else np.ascontiguousarray(data, np.float32)
    dim = 0 if x is None else x.shape[1]
    out = np.empty((n, int(n_components)), np.float32)
    ctx = _lib.context(device)
    st = _lib.lib().evoc_gpu_label_propagation_init_with_options(
        ctx.h, indptr.ctypes.data_as(P), indices.ctypes.data_as(P), gdata.ctypes.data_as(P), n,
        int(n_label_prop_iter), int(n_embedding_epochs), int(approx_n_parts), int(n_components), float(scaling),
        float(random_scale), float(noise_level), C.byref(r), None if x is None else x.ctypes.data_as(P), dim, 0,
        C.byref(opt), out.ctypes.data_as(P))
    _check(st, ctx)
    _rng_out(rs, r)
    return out


def node_embedding(graph, n_components: int, n_epochs: int, initial_embedding=None, initial_alpha: float = 0.1,
                   negative_sample_rate: float = 1.0, noise_level: float = 0.5, random_state=None,
                   reproducible_flag: bool = True, device: int = 0) -> np.ndarray:
    """(n, n_components) f32 embedding; src/embed.rs:251-369 (reproducible epochs)."""
    indptr, indices, gdata, n = _csr(graph)
    rs = _state(random_state)
    r = _rng_in(rs)
    init = None if initial_embedding is None else np.ascontiguousarray(initial_embedding, np.float32)
    if init is not None and init.shape != (n, int(n_components)):
        raise ValueError("initial_embedding must be (n, n_components)")
    out = np.empty((n, int(n_components)), np.float32)
    ctx = _lib.context(device)
    st = _lib.lib().evoc_gpu_node_embedding(
        ctx.h, indptr.ctypes.data_as(P), indices.ctypes.data_as(P), gdata.ctypes.data_as(P), n, int(n_components),
        int(n_epochs), None if init is None else init.ctypes.data_as(P), float(initial_alpha),
        float(negative_sample_rate), float(noise_level), C.byref(r), 1 if reproducible_flag else 0, 0,
        out.ctypes.data_as(P))
    _check(st, ctx)
    _rng_out(rs, r)
    return out


def label_propagation_init_device(indptr_ptr: int, indices_ptr: int, data_ptr: int, n: int, x_ptr: int, dim: int,
                                  out_ptr: int, random_state, n_label_prop_iter: int = 20,
                                  n_embedding_epochs: int = 50, approx_n_parts: int = 512, n_components: int = 4,
                                  scaling: float = 0.5, random_scale: float = 0.1, noise_level: float = 0.5,
                                  device: int = 0):
    """label_propagation_init on device buffers (CSR int64/int32/f32, rows n x dim f32, out n x n_components)."""
    rs = _state(random_state)
    r = _rng_in(rs)
    ctx = _lib.context(device)
    st = _lib.lib().evoc_gpu_label_propagation_init(
        ctx.h, P(indptr_ptr), P(indices_ptr), P(data_ptr), int(n), int(n_label_prop_iter), int(n_embedding_epochs),
        int(approx_n_parts), int(n_components), float(scaling), float(random_scale), float(noise_level),
        C.byref(r), P(x_ptr) if x_ptr else None, int(dim), 1, P(out_ptr))
    _check(st, ctx)
    _rng_out(rs, r)


def node_embedding_device(indptr_ptr: int, indices_ptr: int, data_ptr: int, n: int, n_components: int,
                          n_epochs: int, init_ptr: int, out_ptr: int, random_state, initial_alpha: float = 0.1,
                          negative_sample_rate: float = 1.0, noise_level: float = 0.5, device: int = 0,
                          reproducible: bool = True):
    """node_embedding on device buffers; init_ptr 0 draws the initial embedding."""
    rs = _state(random_state)
    r = _rng_in(rs)
    ctx = _lib.context(device)
    st = _lib.lib().evoc_gpu_node_embedding(
        ctx.h, P(indptr_ptr), P(indices_ptr), P(data_ptr), int(n), int(n_components), int(n_epochs),
        P(init_ptr) if init_ptr else None, float(initial_alpha), float(negative_sample_rate), float(noise_level),
        C.byref(r), 1 if reproducible else 0, 1, P(out_ptr))
    _check(st, ctx)
    _rng_out(rs, r)
