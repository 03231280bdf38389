"""Backend selection and the strict_precision rule (src/rlx_backend/mod.rs), on the CPU.

The GPU build has one backend, Cuda.  resolve() defaults to Strict as the
reference does and reports it as not built here; strict_precision calls that
the GPU cannot make bit-identical to Strict are refused before any RNG draw.
"""
import numpy as np
import pytest

import evoc
from evoc import backend as B


def test_resolve_defaults_to_strict_which_is_not_built(monkeypatch):
    monkeypatch.delenv("EVOC_BACKEND", raising=False)
    with pytest.raises(B.NotEnabled) as e:
        B.ComputeBackend.resolve(None)
    assert e.value.backend is B.ComputeBackend.Strict and "Cuda" in str(e.value)
    assert B.ComputeBackend.resolve(B.ComputeBackend.Cuda) is B.ComputeBackend.Cuda
    monkeypatch.setenv("EVOC_BACKEND", "cuda")
    assert B.ComputeBackend.resolve(None) is B.ComputeBackend.Cuda
    assert B.ComputeBackend.backends_for_run() == [B.ComputeBackend.Cuda]
    monkeypatch.setenv("EVOC_BACKEND", "rocm")
    with pytest.raises(B.NotEnabled) as e:
        B.ComputeBackend.resolve(None)
    assert e.value.feature == "rlx-rocm"
    monkeypatch.setenv("EVOC_BACKEND", "tpu")
    assert B.ComputeBackend.from_env() is None
    with pytest.raises(B.UnknownEnv):
        B.ComputeBackend.backends_for_run()
    monkeypatch.delenv("EVOC_BACKEND")
    assert B.ComputeBackend.backends_for_run() == [B.ComputeBackend.Cuda]


def test_env_aliases():
    table = {"strict": "Strict", "cpu": "Cpu", "cuda": "Cuda", "mlx": "Mlx", "metal": "Mlx", "rocm": "Rocm",
             "wgpu": "Wgpu", "gpu": "Wgpu"}
    import os

    old = os.environ.get("EVOC_BACKEND")
    try:
        for v, name in table.items():
            os.environ["EVOC_BACKEND"] = v
            assert B.ComputeBackend.from_env() is getattr(B.ComputeBackend, name)
    finally:
        if old is None:
            os.environ.pop("EVOC_BACKEND", None)
        else:
            os.environ["EVOC_BACKEND"] = old


@pytest.mark.parametrize("dtype,bfmax", [(np.float32, 10**9), (np.int8, 0), (np.uint8, 99)])
def test_strict_precision_refused_before_any_rng_draw(dtype, bfmax):
    """f32 (always NN-descent in the reference) and integer data above brute_force_max_n cannot be
    bit-identical to Strict: the call raises and the caller's RandomState is untouched."""
    x = (np.random.default_rng(0).standard_normal((100, 16)) * 40).astype(dtype)
    opts = evoc.KnnGraphOptions(n_neighbors=5, brute_force_max_n=bfmax)
    rng = np.random.RandomState(7)
    before = rng.get_state()[1].copy(), rng.get_state()[2]
    be = B.make_backend(B.ComputeBackend.Cuda)
    with pytest.raises(B.StrictPrecisionUnavailable):
        be.knn_graph(x, opts, rng, strict_precision=True)
    with pytest.raises(evoc.BackendError):
        evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=5, brute_force_max_n=bfmax, strict_precision=True),
                       rng)
    assert np.array_equal(rng.get_state()[1], before[0]) and rng.get_state()[2] == before[1]


def test_strict_bits_available_only_for_the_integer_brute_force_branch():
    xi = np.zeros((50, 8), np.int8)
    xu = np.zeros((50, 8), np.uint8)
    xf = np.zeros((50, 8), np.float32)
    o = evoc.KnnGraphOptions(n_neighbors=5, brute_force_max_n=50)
    assert B.strict_bits_available(xi, o) and B.strict_bits_available(xu, o)
    assert not B.strict_bits_available(xf, o)
    assert not B.strict_bits_available(xi, evoc.KnnGraphOptions(n_neighbors=5, brute_force_max_n=49))
