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
    assert o.form == _lib.FORM_AUTO and o.oversample == 2
    assert abs(o.delta - 0.001) < 1e-9 and abs(o.delta_improv - 0.001) < 1e-9


def test_null_context_is_rejected(libpath):
    L = _lib.lib()
    assert L.evoc_gpu_knn_graph(None, None, 0, None, 0, 0, 0, None, None, None, None) == _lib.EVOC_ERR_ARG
    assert L.evoc_gpu_last_error(None) == b"null context"


def test_build_targets_sm100a_only():
    mk = open(os.path.join(_lib.PKG_ROOT, "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk
