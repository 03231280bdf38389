"""The C-ABI library loads and exports every entry point include/evoc_gpu.h
declares.  No compute calls: these run without a GPU."""
import ctypes as C
import os
import subprocess

import pytest

from evoc import _lib


@pytest.fixture(scope="module")
def libpath():
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    return _lib.LIB_PATH


def test_header_declares_entry_points():
    syms = _lib.header_symbols()
    for s in ("evoc_gpu_knn_graph", "evoc_gpu_ctx_create", "evoc_gpu_ctx_destroy", "evoc_gpu_last_error"):
        assert s in syms


def test_library_exports_every_header_symbol(libpath):
    L = C.CDLL(libpath)
    missing = [s for s in _lib.header_symbols() if not hasattr(L, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True).stdout
    for s in _lib.header_symbols():
        assert f" T {s}" in out, s


def test_version_and_default_opts(libpath):
    L = _lib.lib()
    assert L.evoc_gpu_version() >= 100
    o = _lib.default_opts()
    assert o.struct_size == C.sizeof(_lib.Opts)
    assert o.form == _lib.FORM_AUTO and o.oversample == 0  # automatic: ceil(2.5 k) candidates
    assert abs(o.delta - 0.001) < 1e-9 and abs(o.delta_improv - 0.001) < 1e-9
    assert o.scan_type == 0 and o.certify == 1  # FP16 operands, every row certified
    assert o.strict_precision == 0 and o.brute_force_max_n == 0  # KnnGraphOptions' default (src/knn.rs:72)


def test_null_context_is_rejected(libpath):
    L = _lib.lib()
    assert L.evoc_gpu_knn_graph(None, None, 0, None, 0, 0, 0, None, None, None, None) == _lib.EVOC_ERR_ARG
    assert L.evoc_gpu_last_error(None) == b"null context"


def test_build_targets_sm100a_only():
    mk = open(os.path.join(_lib.PKG_ROOT, "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_struct_layouts_match_the_header(tmp_path):
    """sizeof/offsetof of every ABI struct as gcc sees the header, against the ctypes mirror."""
    fields = {
        "evoc_gpu_opts": _lib.Opts,
        "evoc_gpu_server_opts": _lib.ServerOpts,
        "evoc_gpu_server_counters": _lib.ServerCounters,
        "evoc_gpu_job_info": _lib.JobInfo,
        "evoc_numpy_rng": _lib.NumpyRng,
        "evoc_npy_array": _lib.NpyArray,
    }
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{_lib.HEADER_PATH}"', "int main(void) {"]
    for name, cls in fields.items():
        src.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for f, _ in cls._fields_:
            src.append(f'  printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    src += ["  return 0;", "}"]
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Werror", str(c), "-o", str(exe)])
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        s, f, v = line.split()
        got[(s, f)] = int(v)
    for name, cls in fields.items():
        assert got[(name, "size")] == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert got[(name, f)] == getattr(cls, f).offset, (name, f)


def test_server_rejects_bad_arguments_without_a_device(libpath):
    L = _lib.lib()
    o = _lib.ServerOpts()
    L.evoc_gpu_server_default_opts(C.byref(o))
    assert o.struct_size == C.sizeof(_lib.ServerOpts)
    assert o.budget_bytes == 150 * 10**9 and o.max_inflight == 4
    h = C.c_void_p()
    o.struct_size = 1
    assert L.evoc_gpu_server_create(C.byref(o), C.byref(h)) == _lib.EVOC_ERR_ARG
    o.struct_size = C.sizeof(_lib.ServerOpts)
    o.max_inflight = 0
    assert L.evoc_gpu_server_create(C.byref(o), C.byref(h)) == _lib.EVOC_ERR_ARG
    assert not h.value
    jid = C.c_int64(7)
    assert L.evoc_gpu_server_submit(None, None, 0, None, 0, 0, 0, None, 0, C.byref(jid)) == _lib.EVOC_ERR_ARG
    assert L.evoc_gpu_server_poll(None, 1) == _lib.EVOC_ERR_ARG
    assert L.evoc_gpu_server_now_ns() > 0
