"""The .npy / .npz readers of the C ABI against NumPy (CPU only; no device needed)."""
import numpy as np
import pytest

import evoc
from evoc import _lib, npy


@pytest.mark.parametrize("dtype,shape", [(np.float32, (3, 5)), (np.float64, (7,)), (np.int8, (2, 3, 4)),
                                         (np.uint8, (0, 4)), (np.int32, ()), (np.int64, (10,)),
                                         (np.uint32, (4, 4)), (np.bool_, (5,))])
@pytest.mark.parametrize("fortran", [False, True])
def test_npy_arrays_read_in_place(tmp_path, dtype, shape, fortran):
    rng = np.random.default_rng(1)
    a = (rng.normal(size=shape) * 50).astype(dtype)
    if fortran:
        a = np.asfortranarray(a)
    p = str(tmp_path / "a.npy")
    np.save(p, a)
    with npy.NpyFile(p) as f:
        assert f.array.dtype == a.dtype and f.array.shape == a.shape
        assert np.array_equal(f.array, a)
        assert not f.array.flags.writeable


def test_npy_version_2_header(tmp_path):
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    p = tmp_path / "v2.npy"
    with open(p, "wb") as fh:
        np.lib.format.write_array(fh, a, version=(2, 0))
    assert np.array_equal(npy.load(str(p)), a)


@pytest.mark.parametrize("compressed", [False, True])
def test_npz_members(tmp_path, compressed):
    rng = np.random.default_rng(2)
    arrs = {"x": rng.normal(size=(300, 17)).astype(np.float32), "idx": np.arange(1000, dtype=np.int64),
            "flags": rng.integers(0, 2, 64).astype(np.uint8)}
    p = str(tmp_path / "m.npz")
    (np.savez_compressed if compressed else np.savez)(p, **arrs)
    for name, a in arrs.items():
        assert np.array_equal(npy.load(p, name), a)
        assert np.array_equal(npy.load(p, name + ".npy"), a)


def test_graph_npz_csr_and_coo_layouts(tmp_path):
    import scipy.sparse as sp

    rng = np.random.default_rng(3)
    n = 500
    r = rng.integers(0, n, 4000)
    c = rng.integers(0, n, 4000)
    w = rng.uniform(0.1, 1.0, 4000).astype(np.float32)
    coo = tmp_path / "g_coo.npz"  # with repeated (row, column) pairs
    np.savez(coo, rows=r.astype(np.int32), cols=c.astype(np.int32), data=w, shape=np.array([n, n], np.int64))
    m = sp.coo_matrix((w, (r, c)), shape=(n, n)).tocsr()
    m.sum_duplicates()
    m.sort_indices()
    ip, ix, dt, nn = npy.graph_npz(str(coo))
    assert nn == n and np.array_equal(ip, m.indptr) and np.array_equal(ix, m.indices)
    assert np.allclose(dt, m.data, rtol=1e-6)
    csr = tmp_path / "g_csr.npz"
    np.savez(csr, indptr=m.indptr.astype(np.int64), indices=m.indices.astype(np.int32), data=m.data.astype(np.float32),
             shape=np.array([n, n], np.int64))
    ip2, ix2, dt2, _ = npy.graph_npz(str(csr))
    assert np.array_equal(ip2, m.indptr) and np.array_equal(ix2, m.indices)
    assert np.array_equal(dt2, m.data.astype(np.float32))


def test_graph_npz_from_golden_csr(tmp_path):
    """The golden fuzzy graph written in the reference's graph_csr.npz layout reads back unchanged."""
    import os

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "lp_medium_800.npz"))
    p = tmp_path / "graph_csr.npz"
    np.savez(p, indptr=z["graph_csr_indptr"], indices=z["graph_csr_indices"], data=z["graph_csr_data"],
             shape=z["graph_csr_shape"])
    ip, ix, dt, n = npy.graph_npz(str(p))
    assert n == 800 and np.array_equal(ip, z["graph_csr_indptr"]) and np.array_equal(ix, z["graph_csr_indices"])
    assert np.array_equal(dt.view(np.uint32), z["graph_csr_data"].view(np.uint32))


def test_errors(tmp_path):
    with pytest.raises(evoc.BackendError):
        npy.load(str(tmp_path / "missing.npy"))
    bad = tmp_path / "bad.npy"
    bad.write_bytes(b"not an npy file at all")
    with pytest.raises(evoc.BackendError):
        npy.load(str(bad))
    be = tmp_path / "be.npy"
    np.save(be, np.arange(4, dtype=">f4"))
    with pytest.raises(evoc.BackendError):
        npy.load(str(be))
    cx = tmp_path / "cx.npy"
    np.save(cx, np.zeros(3, np.complex64))
    with pytest.raises(evoc.BackendError):
        npy.load(str(cx))
    z = tmp_path / "z.npz"
    np.savez(z, a=np.zeros(3))
    with pytest.raises(evoc.BackendError):
        npy.load(str(z), "nope")
    import ctypes as C

    g = tmp_path / "g.npz"
    np.savez(g, indptr=np.array([0, 1, 2], np.int64), indices=np.array([1, 0], np.int32),
             data=np.ones(2, np.float32), shape=np.array([2, 2], np.int64))
    n, nnz = C.c_int64(0), C.c_int64(0)
    ip = np.empty(3, np.int64)
    ix = np.empty(1, np.int32)
    dt = np.empty(1, np.float32)
    P = C.c_void_p
    st = _lib.lib().evoc_graph_npz_read(str(g).encode(), C.byref(n), C.byref(nnz), ip.ctypes.data_as(P),
                                        ix.ctypes.data_as(P), dt.ctypes.data_as(P), 1)
    assert st == _lib.EVOC_ERR_ARG and nnz.value == 2  # cap below nnz


def _npy_with_header(path, header: str, payload: bytes):
    h = header.encode("latin1")
    pad = 64 - (10 + len(h) + 1) % 64
    h = h + b" " * pad + b"\n"
    with open(path, "wb") as fh:
        fh.write(b"\x93NUMPY\x01\x00" + len(h).to_bytes(2, "little") + h + payload)


@pytest.mark.parametrize("shape", ["(4611686018427387904, 4)", "(9223372036854775807, 2)",
                                   "(4294967296, 4294967296, 2)", "(2305843009213693952,)"])
def test_overflowing_shape_is_rejected(tmp_path, shape):
    """A shape whose element count or byte size wraps 64 bits must not pass the size check."""
    p = str(tmp_path / "wrap.npy")
    _npy_with_header(p, "{'descr': '<f4', 'fortran_order': False, 'shape': %s, }" % shape, b"\0" * 64)
    with pytest.raises(evoc.BackendError):
        npy.load(p)


def test_zip_extra_field_past_its_region_is_rejected(tmp_path):
    """A ZIP64 extra field whose size runs past the central-directory entry is refused."""
    import io
    import struct
    import zipfile

    p = tmp_path / "x.npz"
    body = io.BytesIO()
    np.save(body, np.arange(6, dtype=np.float32))
    zi = zipfile.ZipInfo("a.npy")
    zi.extra = struct.pack("<HH", 0xCAFE, 4) + b"abcd"  # one private extra field of 4 bytes
    with zipfile.ZipFile(p, "w") as zf:
        zf.writestr(zi, body.getvalue())
    assert np.array_equal(npy.load(str(p), "a"), np.arange(6, dtype=np.float32))  # well-formed: readable
    raw = bytearray(p.read_bytes())
    at = raw.rfind(b"PK\x01\x02")
    nlen, xlen = struct.unpack_from("<HH", raw, at + 28)
    assert xlen >= 4
    struct.pack_into("<H", raw, at + 46 + nlen + 2, 0xFFF0)  # first extra field claims 65,520 bytes
    p.write_bytes(bytes(raw))
    with pytest.raises(evoc.BackendError):
        npy.load(str(p), "a")


@pytest.mark.gpu
def test_mapped_rows_feed_knn_graph(tmp_path):
    """Rows read in place from an .npy file go to the kNN entry point as they are."""
    rng = np.random.default_rng(4)
    x = rng.normal(size=(2000, 48)).astype(np.float32)
    p = str(tmp_path / "x.npy")
    np.save(p, x)
    opts = evoc.KnnGraphOptions(n_neighbors=10, form="fp32")
    want = evoc.knn_graph(x, opts)
    with npy.NpyFile(p) as f:
        got = evoc.knn_graph(f.array, opts)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1].view(np.uint32), want[1].view(np.uint32))
