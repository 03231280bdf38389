"""Backend selection, mirroring src/rlx_backend/mod.rs.

ComputeBackend (src/rlx_backend/mod.rs:21-34) keeps the reference's variants
and its EVOC_BACKEND parsing (47-58).  Only ``Cuda`` is built here: it is the
drop-in for RlxBackend::knn_graph (135-144) and runs libevoc_gpu.so.  The
other variants belong to the CPU crate and raise NotEnabled, as the reference
does for a backend whose Cargo feature is off (96-105, 191-202).  resolve()
defaults to ``Strict`` as the reference does, so a caller that names no
backend is told that this build has none but ``Cuda`` instead of silently
getting the GPU.

strict_precision (src/rlx_backend/mod.rs:133-144): "requires bitwise-identical
results to Strict, or the implementation must delegate to the strict
reference path".  There is no CPU path here to delegate to, so the rule is
explicit: with strict_precision the call succeeds only where the GPU
reproduces the Strict bits -- i8/u8 data with n <= brute_force_max_n, the
reference's brute-force branch (src/knn.rs:189-281,418-421), replayed in the
reference's heap order -- and otherwise raises StrictPrecisionUnavailable
before any RNG draw, leaving the caller's RandomState untouched.
"""
from __future__ import annotations

import dataclasses
import enum
import os

from . import knn as _knn


class BackendError(_knn.KnnError):
    pass


class UnknownEnv(BackendError):
    def __init__(self):
        super().__init__("unknown EVOC_BACKEND (use strict|cpu|cuda|mlx|metal|rocm|wgpu|gpu)")


class NotEnabled(BackendError):
    def __init__(self, backend, feature):
        if backend is ComputeBackend.Strict:
            msg = ("compute backend `strict` is the evoc-rs CPU crate, which this GPU build does not contain; "
                   "select ComputeBackend.Cuda (or EVOC_BACKEND=cuda)")
        else:
            msg = f"compute backend `{backend}` not enabled at compile time (enable Cargo feature `{feature}`)"
        super().__init__(msg)
        self.backend = backend
        self.feature = feature


class StrictPrecisionUnavailable(BackendError):
    def __init__(self):
        super().__init__("strict_precision: the Strict backend's results come from its RP-forest NN-descent "
                         "(src/knn.rs:423-445), which no GPU form reproduces bit for bit; only i8/u8 data with "
                         "n <= brute_force_max_n (the reference's brute-force branch) is bit-identical here. "
                         "Pass strict_precision=False to take the exact GPU search")


class ComputeBackend(enum.Enum):
    Strict = "strict"
    Cpu = "cpu"
    Cuda = "cuda"
    Mlx = "mlx"
    Rocm = "rocm"
    Wgpu = "wgpu"

    def __str__(self):
        return self.value

    @classmethod
    def from_env(cls):
        v = os.environ.get("EVOC_BACKEND")
        if v is None:
            return None
        table = {"strict": cls.Strict, "cpu": cls.Cpu, "cuda": cls.Cuda, "mlx": cls.Mlx, "metal": cls.Mlx,
                 "rocm": cls.Rocm, "wgpu": cls.Wgpu, "gpu": cls.Wgpu}
        return table.get(v)

    @classmethod
    def available(cls):
        return [cls.Cuda]

    def is_enabled(self) -> bool:
        return self is ComputeBackend.Cuda

    @classmethod
    def backends_for_run(cls):
        """src/rlx_backend/mod.rs:81-93: the EVOC_BACKEND backend (resolved), else every available one."""
        if "EVOC_BACKEND" in os.environ:
            explicit = cls.from_env()
            if explicit is None:
                raise UnknownEnv()
            return [cls.resolve(explicit)]
        return cls.available()

    @classmethod
    def resolve(cls, explicit=None):
        """An explicit backend or EVOC_BACKEND, defaulting to Strict (src/rlx_backend/mod.rs:93-105)."""
        kind = explicit or cls.from_env() or cls.Strict
        if not kind.is_enabled():
            raise NotEnabled(kind, _feature_name(kind))
        return kind


def _feature_name(kind: ComputeBackend) -> str:
    return {ComputeBackend.Cpu: "rlx-cpu", ComputeBackend.Cuda: "rlx-cuda", ComputeBackend.Mlx: "rlx-mlx",
            ComputeBackend.Rocm: "rlx-rocm", ComputeBackend.Wgpu: "rlx-wgpu",
            ComputeBackend.Strict: "strict"}[kind]


def strict_bits_available(data, opts: _knn.KnnGraphOptions) -> bool:
    """Whether the GPU gives the Strict backend's bits for this call: the integer brute-force branch."""
    data = _knn.EmbeddingData.wrap(data)
    return data.kind != "Float32" and data.nrows() <= opts.brute_force_max_n


class CudaBackend:
    """RlxBackend implementation backed by libevoc_gpu.so."""

    def kind(self) -> ComputeBackend:
        return ComputeBackend.Cuda

    def knn_graph(self, data, opts: _knn.KnnGraphOptions, rng, strict_precision: bool = False):
        if strict_precision and not strict_bits_available(data, opts):
            raise StrictPrecisionUnavailable()
        return _knn.knn_graph(data, dataclasses.replace(opts, strict_precision=bool(strict_precision)), rng)


def make_backend(kind: ComputeBackend):
    kind = ComputeBackend.resolve(kind)
    return CudaBackend()
