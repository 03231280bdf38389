"""Backend selection, mirroring src/rlx_backend/mod.rs.

ComputeBackend (src/rlx_backend/mod.rs:21-34) keeps the reference's variants
and its EVOC_BACKEND parsing (47-58).  Only ``Cuda`` is implemented here: it is
the drop-in for RlxBackend::knn_graph (135-144) and runs libevoc_gpu.so.  The
other variants belong to the CPU crate and raise NotEnabled, as the reference
does for a backend whose Cargo feature is off (96-105, 191-202).
"""
from __future__ import annotations

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
        super().__init__(f"compute backend `{backend}` not enabled at compile time (enable Cargo feature `{feature}`)")
        self.backend = backend
        self.feature = feature


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
    def resolve(cls, explicit=None):
        kind = explicit or cls.from_env() or cls.Cuda
        if not kind.is_enabled():
            raise NotEnabled(kind, _feature_name(kind))
        return kind


def _feature_name(kind: ComputeBackend) -> str:
    return {ComputeBackend.Cpu: "rlx-cpu", ComputeBackend.Cuda: "rlx-cuda", ComputeBackend.Mlx: "rlx-mlx",
            ComputeBackend.Rocm: "rlx-rocm", ComputeBackend.Wgpu: "rlx-wgpu",
            ComputeBackend.Strict: "strict"}[kind]


class CudaBackend:
    """RlxBackend implementation backed by libevoc_gpu.so."""

    def kind(self) -> ComputeBackend:
        return ComputeBackend.Cuda

    def knn_graph(self, data, opts: _knn.KnnGraphOptions, rng, strict_precision: bool = False):
        # strict_precision asks for the Strict backend's exact bits; the GPU
        # forms are exact searches whose results the test suite pins instead.
        return _knn.knn_graph(data, opts, rng)


def make_backend(kind: ComputeBackend):
    kind = ComputeBackend.resolve(kind)
    return CudaBackend()
