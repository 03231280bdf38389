""".npy / .npz ingestion over the C ABI (evoc_npy_open, evoc_npz_open,
evoc_graph_npz_read): arrays are views of a read-only mapping of the file, so
a data set can be handed to the kNN entry points without a host-side copy.
The graph reader takes the reference's CSR and COO layouts
(src/graph_construction.rs:117-154).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .knn import BackendError

_DTYPES = {0: np.float32, 1: np.float64, 2: np.int8, 3: np.uint8, 4: np.int32, 5: np.int64, 6: np.uint32,
           7: np.bool_}


class NpyFile:
    """An opened array; `.array` is a read-only view valid until close()."""

    def __init__(self, path: str, name: str | None = None):
        self._a = _lib.NpyArray()
        L = _lib.lib()
        st = (L.evoc_npy_open(path.encode(), C.byref(self._a)) if name is None else
              L.evoc_npz_open(path.encode(), name.encode(), C.byref(self._a)))
        if st != _lib.EVOC_OK:
            raise BackendError(st, f"cannot read {path}" + (f" member {name}" if name else ""))
        shape = tuple(self._a.shape[i] for i in range(self._a.ndim))
        dt = np.dtype(_DTYPES[self._a.dtype])
        count = int(np.prod(shape)) if shape else 1
        if count == 0:
            flat = np.empty(0, dt)
        else:
            buf = (C.c_char * int(self._a.nbytes)).from_address(self._a.data)
            flat = np.frombuffer(buf, dtype=dt, count=count)
        self.array = flat.reshape(shape, order="F" if self._a.fortran_order else "C")
        self.array.flags.writeable = False

    @property
    def address(self) -> int:
        return int(self._a.data or 0)

    def close(self) -> None:
        if self._a.handle:
            self.array = None
            _lib.lib().evoc_npy_close(C.byref(self._a))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load(path: str, name: str | None = None) -> np.ndarray:
    """The array (a copy, so the file can be closed at once)."""
    with NpyFile(path, name) as f:
        return np.array(f.array, copy=True)


def graph_npz(path: str):
    """(indptr int64, indices int32, data f32, n) of a graph .npz (CSR or COO layout)."""
    L = _lib.lib()
    n, nnz = C.c_int64(0), C.c_int64(0)
    st = L.evoc_graph_npz_read(path.encode(), C.byref(n), C.byref(nnz), None, None, None, 0)
    if st != _lib.EVOC_OK:
        raise BackendError(st, f"cannot read graph {path}")
    indptr = np.empty(n.value + 1, np.int64)
    indices = np.empty(max(nnz.value, 1), np.int32)
    data = np.empty(max(nnz.value, 1), np.float32)
    P = C.c_void_p
    st = L.evoc_graph_npz_read(path.encode(), C.byref(n), C.byref(nnz), indptr.ctypes.data_as(P),
                               indices.ctypes.data_as(P), data.ctypes.data_as(P), len(data))
    if st != _lib.EVOC_OK:
        raise BackendError(st, f"cannot read graph {path}")
    return indptr, indices[:nnz.value].copy(), data[:nnz.value].copy(), n.value
