"""ORACLE / TEST INFRASTRUCTURE ONLY.

CPU restatement of evoc-rs's label-propagation initialisation
(src/label_prop.rs:464-674) and its reproducible node embedding
(src/embed.rs:138-369).  The per-element arithmetic runs in
``oracle/evoc_oracle_lp.c`` (through ``oracle/liborc.so``); this module strings
the steps together the way ``label_propagation_init_with_options`` does and
restates the small dense steps (reduction maps, row/column normalisation, PCA
base init) with NumPy, each citing the reference lines it follows.  Only
``tests/`` and the CPU-baseline leg of ``bench.py`` use it, as the checker.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import oracle as O

_ready = False


def _lib():
    global _ready
    L = O.lib()
    if not _ready:
        P, i64, f32, i32 = C.c_void_p, C.c_int64, C.c_float, C.c_int32
        L.orc_lp_iteration.argtypes = [P, P, P, i64, P, P, P]
        L.orc_lp_outliers.argtypes = [P, P, i64, P, P]
        L.orc_lp_remap.argtypes = [P, i64]
        L.orc_lp_loop.argtypes = [P, P, P, i64, P, C.POINTER(O.MT), i32, i64, P]
        L.orc_smmp.argtypes = [i64, i64, P, P, P, P, P, P, i64, P, P, P]
        L.orc_smmp.restype = i64
        L.orc_csr_dense.argtypes = [i64, P, P, P, P, i64, P]
        L.orc_make_epochs_per_sample.argtypes = [P, i64, i32, P]
        L.orc_seg_sum_f32.argtypes = [P, P, i64, i64, P]
        L.orc_node_embedding_serial.argtypes = [i64, P, P, P, i32, i32, P, i32, f32, f32, f32, C.POINTER(O.MT), P, P]
        L.orc_node_embedding_repr.argtypes = [i64, P, P, P, i32, i32, P, i32, f32, f32, f32, C.POINTER(O.MT), i32, P,
                                              P, P]
        _ready = True
    return L


_p = O._ptr


@dataclass
class Csr:
    """CSR matrix: indptr int64 (n+1), indices int32, data f32; rows may be unsorted."""

    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray
    shape: tuple

    @staticmethod
    def make(indptr, indices, data, shape) -> "Csr":
        return Csr(np.ascontiguousarray(indptr, np.int64), np.ascontiguousarray(indices, np.int32),
                   np.ascontiguousarray(data, np.float32), (int(shape[0]), int(shape[1])))

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def rows(self) -> np.ndarray:
        return np.repeat(np.arange(self.shape[0], dtype=np.int64), np.diff(self.indptr))


def mt_from_state(key, pos, has_gauss=0, gauss=0.0) -> O.RandomState:
    """An oracle RandomState at a saved NumPy state (get_state() fields)."""
    r = O.RandomState(0)
    C.memmove(r.s.key, np.ascontiguousarray(key, np.uint32).ctypes.data, 624 * 4)
    r.s.pos = int(pos)
    r.s.has_gauss = int(has_gauss)
    r.s.gauss = float(gauss)
    return r


# ---------------------------------------------------------------- label propagation

def label_prop_iteration(g: Csr, labels: np.ndarray, rng_state=(0, 0, 0)) -> np.ndarray:
    """src/label_prop.rs:39-91."""
    labels = np.ascontiguousarray(labels, np.int64)
    out = np.empty_like(labels)
    rs = np.asarray(rng_state, np.int64)
    _lib().orc_lp_iteration(_p(g.indptr), _p(g.indices), _p(g.data), g.shape[0], _p(labels), _p(rs), _p(out))
    return out


def label_outliers(g: Csr, labels: np.ndarray, rng_state) -> np.ndarray:
    """src/label_prop.rs:94-132 (returns a new array)."""
    labels = np.array(labels, np.int64, copy=True)
    rs = np.asarray(rng_state, np.int64)
    _lib().orc_lp_outliers(_p(g.indptr), _p(g.indices), g.shape[0], _p(labels), _p(rs))
    return labels


def remap_labels(labels: np.ndarray) -> np.ndarray:
    """src/label_prop.rs:135-157 (returns a new array)."""
    labels = np.array(labels, np.int64, copy=True)
    _lib().orc_lp_remap(_p(labels), len(labels))
    return labels


def label_prop_loop(g: Csr, rng: O.RandomState, n_iter: int, approx_n_parts: int, return_seeded: bool = False):
    """src/label_prop.rs:160-185, starting from all -1 labels."""
    n = g.shape[0]
    labels = np.full(n, -1, np.int64)
    seeded = np.empty(n, np.int64)
    _lib().orc_lp_loop(_p(g.indptr), _p(g.indices), _p(g.data), n, _p(labels), C.byref(rng.s), n_iter,
                       approx_n_parts, _p(seeded))
    return (labels, seeded) if return_seeded else labels


# ---------------------------------------------------------------- sparse helpers

def smmp(a: Csr, b: Csr) -> Csr:
    """scipy_csr_matmul, src/csr_matmul.rs:6-59 (SciPy SMMP order)."""
    assert a.shape[1] == b.shape[0]
    blen = np.diff(b.indptr)
    cap = int(blen[a.indices].sum()) + 1 if a.nnz else 1
    cp = np.empty(a.shape[0] + 1, np.int64)
    cj = np.empty(cap, np.int32)
    cd = np.empty(cap, np.float32)
    nnz = _lib().orc_smmp(a.shape[0], b.shape[1], _p(a.indptr), _p(a.indices), _p(a.data), _p(b.indptr),
                          _p(b.indices), _p(b.data), cap, _p(cp), _p(cj), _p(cd))
    assert nnz >= 0
    return Csr.make(cp, cj[:nnz].copy(), cd[:nnz].copy(), (a.shape[0], b.shape[1]))


def csr_matmul_dense(a: Csr, dense: np.ndarray) -> np.ndarray:
    """src/label_prop.rs:233-250: f64 products cast to f32, summed in f32 in CSR order."""
    dense = np.ascontiguousarray(dense, np.float32)
    out = np.empty((a.shape[0], dense.shape[1]), np.float32)
    _lib().orc_csr_dense(a.shape[0], _p(a.indptr), _p(a.indices), _p(a.data), _p(dense), dense.shape[1], _p(out))
    return out


def transpose_sorted(a: Csr) -> Csr:
    """transpose_view().to_csr(): rows of A^T list the source rows in ascending order."""
    rows = a.rows()
    order = np.argsort(a.indices, kind="stable")
    cnt = np.bincount(a.indices, minlength=a.shape[1])
    indptr = np.zeros(a.shape[1] + 1, np.int64)
    np.cumsum(cnt, out=indptr[1:])
    return Csr.make(indptr, rows[order].astype(np.int32), a.data[order], (a.shape[1], a.shape[0]))


def _seq_sum_f32(values: np.ndarray, seg: np.ndarray, nseg: int) -> np.ndarray:
    """Per-segment f32 sum, added one value at a time in storage order."""
    v = np.ascontiguousarray(values, np.float32)
    sg = np.ascontiguousarray(seg, np.int64)
    out = np.empty(nseg, np.float32)
    _lib().orc_seg_sum_f32(_p(v), _p(sg), len(v), nseg, _p(out))
    return out


def normalize_rows_l1(a: Csr) -> Csr:
    """src/label_prop.rs:204-217."""
    s = _seq_sum_f32(np.abs(a.data), a.rows(), a.shape[0])
    s = np.maximum(s, np.float32(1e-12))
    return Csr.make(a.indptr, a.indices, (a.data / s[a.rows()]).astype(np.float32), a.shape)


def normalize_cols_l2(a: Csr) -> Csr:
    """src/label_prop.rs:188-201."""
    sq = _seq_sum_f32((a.data * a.data).astype(np.float32), a.indices, a.shape[1])
    norms = np.maximum(np.sqrt(sq).astype(np.float32), np.float32(1e-12))
    return Csr.make(a.indptr, a.indices, (a.data / norms[a.indices]).astype(np.float32), a.shape)


def partition_reduction_map(part: np.ndarray) -> Csr:
    """src/label_prop.rs:220-230: one 1.0 per labelled row."""
    part = np.asarray(part, np.int64)
    n = len(part)
    n_parts = max(int(part.max()) + 1 if n else 1, 1)
    keep = part >= 0
    indptr = np.zeros(n + 1, np.int64)
    np.cumsum(keep, out=indptr[1:])
    return Csr.make(indptr, part[keep].astype(np.int32), np.ones(int(keep.sum()), np.float32), (n, n_parts))


def hadamard_symmetric(g: Csr) -> Csr:
    """src/label_prop.rs:450-461: G o G^T on G's pattern, rows sorted."""
    rows = g.rows()
    key = rows * g.shape[1] + g.indices
    tkey = g.indices.astype(np.int64) * g.shape[1] + rows
    order = np.argsort(key, kind="stable")
    pos = np.searchsorted(key[order], tkey)
    pos = np.minimum(pos, len(key) - 1)
    found = key[order][pos] == tkey
    other = np.where(found, g.data[order][pos], np.float32(0))
    keep = other != 0
    r, c, v = rows[keep], g.indices[keep], (g.data[keep] * other[keep]).astype(np.float32)
    o = np.lexsort((c, r))
    indptr = np.zeros(g.shape[0] + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=g.shape[0]), out=indptr[1:])
    return Csr.make(indptr, c[o], v[o], g.shape)


# ---------------------------------------------------------------- embeddings

def make_epochs_per_sample(w: np.ndarray, n_epochs: int) -> np.ndarray:
    w = np.ascontiguousarray(w, np.float32)
    out = np.empty_like(w)
    _lib().orc_make_epochs_per_sample(_p(w), len(w), n_epochs, _p(out))
    return out


def node_embedding(g: Csr, n_components: int, n_epochs: int, init, initial_alpha: float,
                   negative_sample_rate: float, noise_level: float, rng: O.RandomState, *,
                   n_run: int = -1, state: bool = False):
    """node_embedding(reproducible_flag=true), src/embed.rs:251-369.  n_run stops after that many
    epochs; state=True also returns (updates, epoch_of_next_negative_sample, epoch_of_next_sample)."""
    n = g.shape[0]
    have = init is not None
    emb = np.array(init, np.float32, copy=True, order="C") if have else np.empty((n, n_components), np.float32)
    upd = np.empty((n, n_components), np.float32)
    eonn = np.empty(g.nnz, np.float32)
    eons = np.empty(g.nnz, np.float32)
    _lib().orc_node_embedding_repr(n, _p(g.indptr), _p(g.indices), _p(g.data), n_components, n_epochs, _p(emb),
                                   1 if have else 0, initial_alpha, negative_sample_rate, noise_level,
                                   C.byref(rng.s), n_run, _p(upd), _p(eonn), _p(eons))
    return (emb, upd, eonn, eons) if state else emb


def node_embedding_serial(g: Csr, n_components: int, n_epochs: int, init, initial_alpha: float,
                          negative_sample_rate: float, noise_level: float, rng: O.RandomState, *,
                          state: bool = False):
    """node_embedding(reproducible_flag=false): in-place SGD in edge order, src/embed.rs:57-135,251-369.
    state=True also returns (epoch_of_next_negative_sample, epoch_of_next_sample)."""
    n = g.shape[0]
    have = init is not None
    emb = np.array(init, np.float32, copy=True, order="C") if have else np.empty((n, n_components), np.float32)
    eonn = np.empty(g.nnz, np.float32)
    eons = np.empty(g.nnz, np.float32)
    _lib().orc_node_embedding_serial(n, _p(g.indptr), _p(g.indices), _p(g.data), n_components, n_epochs, _p(emb),
                                     1 if have else 0, initial_alpha, negative_sample_rate, noise_level,
                                     C.byref(rng.s), _p(eonn), _p(eons))
    return (emb, eonn, eons) if state else emb


def _normalize_small_init(r: np.ndarray) -> np.ndarray:
    """src/label_prop.rs:251-262."""
    mean = np.add.accumulate(r.astype(np.float64).ravel())[-1] / r.size  # f64, element order
    r = (r.astype(np.float64) - mean).astype(np.float32)
    scale = np.float32((r.max() - r.min()) / np.float32(2.0))
    if scale > 0:
        r = (r / scale).astype(np.float32)
    return r


def pca_init(data: np.ndarray, n_components: int) -> np.ndarray:
    """src/label_prop.rs:265-309: f32 column means (rows added in order), f64 thin SVD, signs
    flipped so each right singular vector's largest-|.| entry (the last on ties) is >= 0."""
    data = np.asarray(data, np.float32)
    n, d = data.shape
    mean = np.zeros(d, np.float32)
    for i in range(n):
        mean = (mean + data[i]).astype(np.float32)
    mean = (mean / np.float32(n)).astype(np.float32)
    mat = data.astype(np.float64) - mean.astype(np.float64)
    u, s, vt = np.linalg.svd(mat, full_matrices=False)
    for j in range(vt.shape[0]):
        a = np.abs(vt[j])
        idx = len(a) - 1 - int(np.argmax(a[::-1]))
        if vt[j, idx] < 0:
            vt[j] = -vt[j]
            u[:, j] = -u[:, j]
    k = min(n_components, u.shape[1], len(s))
    out = np.zeros((n, n_components), np.float32)
    out[:, :k] = (u[:, :k] * s[:k]).astype(np.float32)
    return _normalize_small_init(out)


def _ndarray_dot_f32(v: np.ndarray) -> np.float32:
    """ndarray's unrolled f32 dot of a contiguous row with itself (no BLAS feature in the
    reference's build, Cargo.toml:29): eight partial sums over whole blocks of eight, added
    as (0+4), (1+5), (2+6), (3+7) to a zero sum, then the tail in order; separate multiply and add."""
    f = np.float32
    p = [f(0.0)] * 8
    c = 0
    while c + 8 <= len(v):
        for j in range(8):
            p[j] = f(p[j] + f(v[c + j] * v[c + j]))
        c += 8
    s = f(0.0)
    for a, b in ((0, 4), (1, 5), (2, 6), (3, 7)):
        s = f(s + f(p[a] + p[b]))
    for j in range(c, len(v)):
        s = f(s + f(v[j] * v[j]))
    return s


def random_unit_init(n: int, n_components: int, rng: O.RandomState) -> np.ndarray:
    """src/label_prop.rs:311-320: n x c normal(1.0) draws in row order (f32), each row divided by
    the f32 sqrt of its dot with itself when positive."""
    r = np.empty((n, n_components), np.float32)
    for i in range(n):
        for c in range(n_components):
            r[i, c] = np.float32(1.0 * rng.normal())
    for i in range(n):
        norm = np.float32(np.sqrt(_ndarray_dot_f32(r[i])))
        if norm > 0:
            r[i] = (r[i] / norm).astype(np.float32)
    return r


def _pairwise_sq(data: np.ndarray) -> np.ndarray:
    """src/label_prop.rs:322-337: f32, coordinates summed in order, separate multiply and add."""
    x = np.asarray(data, np.float32)
    n, d = x.shape
    sq = np.zeros((n, n), np.float32)
    for c in range(d):
        diff = (x[:, None, c] - x[None, :, c]).astype(np.float32)
        sq = (sq + (diff * diff).astype(np.float32)).astype(np.float32)
    return sq


def _eigh_signed(a: np.ndarray):
    """Symmetric eigen-decomposition in f64 (the CUDA path's; the reference uses faer 0.20.2's f32
    solver, whose eigenvector signs are its own): eigenvalues ascending, each eigenvector's
    largest-|.| entry (the first on ties) made non-negative."""
    w, v = np.linalg.eigh(np.asarray(a, np.float64))
    order = np.argsort(w, kind="stable")
    w, v = w[order], v[:, order]
    for j in range(v.shape[1]):
        i = int(np.argmax(np.abs(v[:, j])))
        if v[i, j] < 0:
            v[:, j] = -v[:, j]
    return w, v


def spectral_init(data: np.ndarray, n_components: int) -> np.ndarray:
    """src/label_prop.rs:364-423: Gaussian affinities with sigma = sqrt of the median positive squared
    distance (floored at 1e-8), the symmetric normalised Laplacian I - D^-1/2 W D^-1/2 in f32,
    eigenvectors 1 .. n_components of the ascending order, then the small-graph normalisation."""
    f = np.float32
    dsq = _pairwise_sq(data)
    n = dsq.shape[0]
    flat = np.sort(dsq[dsq > 0].ravel(), kind="stable")
    sigma = f(max(np.sqrt(f(flat[len(flat) // 2])) if len(flat) else f(1.0), f(1e-8)))
    den = f(f(f(2.0) * sigma) * sigma)
    w = np.zeros((n, n), np.float32)
    for i in range(n):
        for j in range(n):
            if i != j:
                v = f(np.exp(f(-dsq[i, j] / den)))
                if v > f(1e-12):
                    w[i, j] = v
    deg = np.zeros(n, np.float32)
    for i in range(n):
        for j in range(n):
            if w[i, j] != 0:
                deg[i] = f(deg[i] + w[i, j])
    lap = np.eye(n, dtype=np.float32)
    for i in range(n):
        for j in range(n):
            if w[i, j] != 0:
                dn = max(f(np.sqrt(f(deg[i] * deg[j]))), f(1e-12))
                lap[i, j] = f(lap[i, j] - f(w[i, j] / dn))
    _, v = _eigh_signed(lap)
    out = np.zeros((n, n_components), np.float32)
    kc = max(0, min(n_components, n - 1))
    out[:, :kc] = v[:, 1:1 + kc].astype(np.float32)
    return _normalize_small_init(out)


def mds_init(data: np.ndarray, n_components: int) -> np.ndarray:
    """src/label_prop.rs:339-362: B = -0.5 (H D) H in f64 (H = I - 1/n) rounded to f32, the
    eigenvectors of the n_components smallest eigenvalues (ascending order) scaled by
    sqrt(max(lambda, 0)) in f32, then the small-graph normalisation."""
    dsq = _pairwise_sq(data).astype(np.float64)
    n = dsq.shape[0]
    h = np.eye(n) - 1.0 / n
    b = (-0.5 * ((h @ dsq) @ h)).astype(np.float32)
    w, v = _eigh_signed(b)
    out = np.zeros((n, n_components), np.float32)
    kc = min(n_components, n)
    eig = np.sqrt(np.maximum(w[:kc].astype(np.float32), np.float32(0.0))).astype(np.float32)
    out[:, :kc] = (v[:, :kc].astype(np.float32) * eig[None, :]).astype(np.float32)
    return _normalize_small_init(out)


def small_graph_init(data, n: int, n_components: int, base_init: str, rng: O.RandomState) -> np.ndarray:
    """src/label_prop.rs:425-447."""
    if base_init == "random":
        return random_unit_init(n, n_components, rng)
    if data is None:
        raise ValueError("base_init 'pca' requires data")
    if base_init == "pca":
        return pca_init(data, n_components)
    if base_init == "spectral":
        return spectral_init(data, n_components)
    if base_init == "mds":
        return mds_init(data, n_components)
    raise ValueError(base_init)


def _part_layout_plus_noise(part: np.ndarray, layout: np.ndarray, n_components: int, scale: float,
                            rng: O.RandomState) -> np.ndarray:
    """layout[part] (zeros where part < 0) plus normal_scaled(scale) as f32, drawn in row order and
    added in f32 (src/label_prop.rs:628-640, 643-656)."""
    n = len(part)
    out = np.zeros((n, n_components), np.float32)
    ok = part >= 0
    out[ok] = layout[part[ok]]
    for i in range(n):
        for c in range(n_components):
            out[i, c] = np.float32(out[i, c] + np.float32(scale * rng.normal()))
    return out


def label_propagation_init(g: Csr, n_label_prop_iter: int, n_embedding_epochs: int, approx_n_parts: int,
                           n_components: int, scaling: float, random_scale: float, noise_level: float,
                           rng: O.RandomState, data=None, base_init_threshold: int = 64, trace=None,
                           recursive_init: bool = True, base_init: str = "pca",
                           upscaling: str = "partition_expander") -> np.ndarray:
    """label_propagation_init_with_options (src/label_prop.rs:497-674); the defaults are those of
    label_propagation_init (464-494): recursive init, PCA base init, the partition expander."""
    n = g.shape[0]
    if n < base_init_threshold:
        return small_graph_init(data, n, n_components, base_init, rng)
    part = label_prop_loop(g, rng, n_label_prop_iter, approx_n_parts)
    base = partition_reduction_map(part)
    norm = normalize_cols_l2(base)
    norm_t = transpose_sorted(norm)
    reducer = normalize_rows_l1(norm_t)
    reduced_data = csr_matmul_dense(reducer, data) if data is not None else None
    reduced = smmp(smmp(norm_t, g), base)
    reduced = Csr.make(reduced.indptr, reduced.indices, np.clip(reduced.data, 0.0, 1.0), reduced.shape)
    reduced_init = None
    if recursive_init:
        reduced_init = label_propagation_init(reduced, n_label_prop_iter, min(n_embedding_epochs, 255),
                                              approx_n_parts // 4, n_components, scaling, random_scale,
                                              noise_level, rng, reduced_data, base_init_threshold, trace,
                                              recursive_init, base_init, upscaling)
    layout = node_embedding(reduced, n_components, n_embedding_epochs, reduced_init,
                            np.float32(0.001) * np.float32(n_embedding_epochs), 1.0, noise_level, rng)
    if upscaling == "node_embedding":
        result = _part_layout_plus_noise(part, layout, n_components, float(np.float32(random_scale)), rng)
    else:
        sym = hadamard_symmetric(g)
        expander = normalize_rows_l1(smmp(sym, norm))
        part_norm = normalize_rows_l1(norm)
        a = csr_matmul_dense(expander, layout)
        b = csr_matmul_dense(part_norm, layout)
        result = ((a.astype(np.float64) + b.astype(np.float64)) * 0.5).astype(np.float32)
        if upscaling == "jitter_expander":
            quarter = float(np.float32(np.float32(random_scale) / np.float32(4.0)))
            jit = _part_layout_plus_noise(part, layout, n_components, quarter, rng)
            result = ((result.astype(np.float64) + jit.astype(np.float64)) * 0.5).astype(np.float32)
        elif upscaling != "partition_expander":
            raise ValueError(upscaling)
    mean = np.add.accumulate(result.astype(np.float64), axis=0)[-1] / n  # f64, row order
    if trace is not None:
        trace.append(dict(n=n, partition=part, reduced=reduced, reduced_data=reduced_data,
                          reduced_init=reduced_init, layout=layout, pre_scale=result))
    return (np.float64(np.float32(scaling)) * (result.astype(np.float64) - mean)).astype(np.float32)
