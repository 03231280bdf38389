"""Loader for libevoc_gpu.so (the C ABI declared in include/evoc_gpu.h).

There is no CPU fallback: if the library is missing or no CUDA device is
present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libevoc_gpu.so")
HEADER_PATH = os.path.join(os.path.dirname(PKG_ROOT), "include", "evoc_gpu.h")

EVOC_OK = 0
EVOC_ERR_EMPTY = 1
EVOC_ERR_K = 2
EVOC_ERR_ARG = 3
EVOC_ERR_OOM = 4
EVOC_ERR_TIMEOUT = 5
EVOC_ERR_CUDA = 6
EVOC_ERR_UNSUPPORTED = 7
EVOC_ERR_CANCELLED = 8
EVOC_ERR_PENDING = 9

DTYPE_F32, DTYPE_I8, DTYPE_U8 = 0, 1, 2
FORM_AUTO, FORM_FP32, FORM_BF16_RERANK, FORM_EXACT_INT, FORM_NNDESCENT, FORM_POPCOUNT = 0, 1, 2, 3, 4, 5
FORM_NAMES = {"auto": FORM_AUTO, "fp32": FORM_FP32, "bf16_rerank": FORM_BF16_RERANK,
              "half_rerank": FORM_BF16_RERANK, "exact_int": FORM_EXACT_INT, "nndescent": FORM_NNDESCENT,
              "popcount": FORM_POPCOUNT}
SCAN_TYPES = {"fp16": 0, "bf16": 1}


class Opts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("form", C.c_int32),
        ("oversample", C.c_int32),
        ("buffers_on_device", C.c_int32),
        ("deterministic", C.c_int32),
        ("n_iters", C.c_int32),
        ("max_candidates", C.c_int32),
        ("delta", C.c_float),
        ("delta_improv", C.c_float),
        ("row_begin", C.c_int64),
        ("row_end", C.c_int64),
        ("strict_precision", C.c_int32),
        ("scan_type", C.c_int32),
        ("brute_force_max_n", C.c_int64),
        ("certify", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


_lib = None
_lock = threading.Lock()


def build() -> None:
    """Compile libevoc_gpu.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.check_call(["make", "-s", "-C", PKG_ROOT, "-j8"])


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"libevoc_gpu.so not built at {LIB_PATH}; run build()")
            L = C.CDLL(LIB_PATH)
            P = C.c_void_p
            i32, i64 = C.c_int32, C.c_int64
            L.evoc_gpu_version.restype = C.c_int
            L.evoc_gpu_default_opts.argtypes = [C.POINTER(Opts)]
            L.evoc_gpu_ctx_create.argtypes = [C.c_int, C.POINTER(P)]
            L.evoc_gpu_ctx_destroy.argtypes = [P]
            L.evoc_gpu_last_error.argtypes = [P]
            L.evoc_gpu_last_error.restype = C.c_char_p
            L.evoc_gpu_knn_graph.argtypes = [P, C.POINTER(Opts), i32, P, i64, i64, i32, P, P, P, C.POINTER(i32)]
            L.evoc_gpu_knn_graph_raw.argtypes = [P, C.POINTER(Opts), i32, P, i64, i64, i32, P, P, P, P,
                                                 C.POINTER(i32)]
            L.evoc_gpu_ctx_stream.argtypes = [P]
            L.evoc_gpu_ctx_stream.restype = P
            L.evoc_gpu_profile_enable.argtypes = [P, C.c_int]
            L.evoc_gpu_profile_count.argtypes = [P]
            L.evoc_gpu_profile_stage.argtypes = [P, C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_float)]
            L.evoc_gpu_last_launch_count.argtypes = [P]
            L.evoc_gpu_last_certify.argtypes = [P, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)]
            L.evoc_gpu_set_wait_limit.argtypes = [P, C.c_uint64, C.c_uint64]
            L.evoc_gpu_last_nndescent.argtypes = [P, C.POINTER(i32), C.POINTER(i64), C.POINTER(i64)]
            L.evoc_gpu_set_symmetric_scan.argtypes = [P, C.c_int64]
            L.evoc_gpu_last_symmetric.argtypes = [P, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64),
                                                  C.POINTER(i64)]
            _bind_optional(L)
            _lib = L
    return _lib


def _bind_optional(L) -> None:
    """Signatures of entry points added by later parts of the library."""
    P = C.c_void_p
    i32, i64 = C.c_int32, C.c_int64
    if hasattr(L, "evoc_gpu_fuzzy_graph"):
        L.evoc_gpu_fuzzy_graph.argtypes = [P, P, P, i64, i32, C.c_float, i32, i32, P, P, P, P, P, i64,
                                           C.POINTER(i64)]
    if hasattr(L, "evoc_gpu_smooth_knn_dist"):
        L.evoc_gpu_smooth_knn_dist.argtypes = [P, P, i64, i32, C.c_float, i32, P, P]
    if hasattr(L, "evoc_gpu_autotune"):
        L.evoc_gpu_autotune.argtypes = [P, i32, i32, i64, i64, i32, C.c_char_p, C.c_char_p, i32]
        L.evoc_gpu_tune_load.argtypes = [P, C.c_char_p]
    if hasattr(L, "evoc_gpu_knn_graph_batch"):
        L.evoc_gpu_knn_graph_batch.argtypes = [P, C.POINTER(Opts), i32, i32, P, P, P, i32, P, P, P, P]
    if hasattr(L, "evoc_gpu_label_propagation_init"):
        f32 = C.c_float
        L.evoc_gpu_label_prop_loop.argtypes = [P, P, P, P, i64, i32, i64, C.POINTER(NumpyRng), i32, P,
                                               C.POINTER(i64)]
        L.evoc_gpu_label_propagation_init.argtypes = [P, P, P, P, i64, i32, i32, i64, i32, f32, f32, f32,
                                                      C.POINTER(NumpyRng), P, i64, i32, P]
        L.evoc_gpu_node_embedding.argtypes = [P, P, P, P, i64, i32, i32, P, f32, f32, f32, C.POINTER(NumpyRng),
                                              i32, i32, P]
    if hasattr(L, "evoc_gpu_label_propagation_init_with_options"):
        f32 = C.c_float
        L.evoc_gpu_label_propagation_init_with_options.argtypes = [
            P, P, P, P, i64, i32, i32, i64, i32, f32, f32, f32, C.POINTER(NumpyRng), P, i64, i32,
            C.POINTER(LpOptions), P]
        L.evoc_lp_options_default.argtypes = [C.POINTER(LpOptions)]
        L.evoc_lp_options_default.restype = None
    if hasattr(L, "evoc_gpu_peak_ffma"):
        L.evoc_gpu_peak_ffma.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    if hasattr(L, "evoc_gpu_boruvka_mst"):
        L.evoc_gpu_boruvka_mst.argtypes = [P, P, i64, i32, i32, i32, P, P, C.POINTER(i64)]
    if hasattr(L, "evoc_npy_open"):
        L.evoc_npy_open.argtypes = [C.c_char_p, C.POINTER(NpyArray)]
        L.evoc_npz_open.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(NpyArray)]
        L.evoc_npy_close.argtypes = [C.POINTER(NpyArray)]
        L.evoc_npy_close.restype = None
        L.evoc_graph_npz_read.argtypes = [C.c_char_p, C.POINTER(i64), C.POINTER(i64), P, P, P, i64]
    if hasattr(L, "evoc_gpu_server_create"):
        L.evoc_gpu_server_default_opts.argtypes = [C.POINTER(ServerOpts)]
        L.evoc_gpu_server_create.argtypes = [C.POINTER(ServerOpts), C.POINTER(P)]
        L.evoc_gpu_server_destroy.argtypes = [P]
        L.evoc_gpu_server_now_ns.restype = i64
        L.evoc_gpu_server_submit.argtypes = [P, C.POINTER(Opts), i32, P, i64, i64, i32, P, i32, C.POINTER(i64)]
        L.evoc_gpu_server_request_bytes.argtypes = [P, C.POINTER(Opts), i32, i64, i64, i32, C.POINTER(i64),
                                                    C.POINTER(i64)]
        L.evoc_gpu_server_poll.argtypes = [P, i64]
        L.evoc_gpu_server_wait.argtypes = [P, i64, i64]
        L.evoc_gpu_server_wait_any.argtypes = [P, i64, C.POINTER(i64)]
        L.evoc_gpu_server_result.argtypes = [P, i64, P, P, C.POINTER(i32), i32]
        L.evoc_gpu_server_result_device.argtypes = [P, i64, C.POINTER(P), C.POINTER(P), C.POINTER(i32)]
        L.evoc_gpu_server_release.argtypes = [P, i64]
        L.evoc_gpu_server_cancel.argtypes = [P, i64]
        L.evoc_gpu_server_job_info.argtypes = [P, i64, C.POINTER(JobInfo)]
        L.evoc_gpu_server_stats.argtypes = [P, C.POINTER(ServerCounters)]
        L.evoc_gpu_server_stage_count.argtypes = [P]
        L.evoc_gpu_server_stage.argtypes = [P, C.c_int, C.c_char_p, i32, C.POINTER(C.c_double), C.POINTER(i64)]
        L.evoc_gpu_server_lane_busy_ms.argtypes = [P]
        L.evoc_gpu_server_lane_busy_ms.restype = C.c_double


class NumpyRng(C.Structure):
    """evoc_numpy_rng: the fields of numpy.random.RandomState.get_state()."""

    _fields_ = [("key", C.c_uint32 * 624), ("pos", C.c_int32), ("has_gauss", C.c_int32), ("gauss", C.c_double)]


class LpOptions(C.Structure):
    """evoc_lp_options: label_propagation_init_with_options's keyword arguments."""

    _fields_ = [("recursive_init", C.c_int32), ("base_init", C.c_int32), ("base_init_threshold", C.c_int64),
                ("upscaling", C.c_int32), ("reserved", C.c_int32 * 3)]


BASE_INITS = {"pca": 0, "random": 1, "spectral": 2, "mds": 3}
UPSCALINGS = {"partition_expander": 0, "jitter_expander": 1, "node_embedding": 2}


class NpyArray(C.Structure):
    """evoc_npy_array."""

    _fields_ = [("data", C.c_void_p), ("nbytes", C.c_int64), ("shape", C.c_int64 * 8), ("ndim", C.c_int32),
                ("dtype", C.c_int32), ("fortran_order", C.c_int32), ("reserved", C.c_int32), ("handle", C.c_void_p)]


class ServerOpts(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("device", C.c_int32),
        ("budget_bytes", C.c_int64),
        ("max_inflight", C.c_int32),
        ("profile", C.c_int32),
        ("batch_max", C.c_int32),
        ("small_lanes", C.c_int32),
        ("admission", C.c_int32),
        ("reserved", C.c_int32 * 1),
    ]


class ServerCounters(C.Structure):
    _fields_ = [(name, C.c_int64) for name in (
        "submitted", "completed", "failed", "cancelled", "rejected", "pending", "running", "bytes_in_use",
        "peak_bytes", "budget_bytes", "workspace_bytes", "workspace_misses", "lanes", "batches", "batched")]


class JobInfo(C.Structure):
    _fields_ = [
        ("submit_ns", C.c_int64),
        ("admit_ns", C.c_int64),
        ("done_ns", C.c_int64),
        ("n", C.c_int64),
        ("dim", C.c_int64),
        ("dtype", C.c_int32),
        ("k_eff", C.c_int32),
        ("lane", C.c_int32),
        ("status", C.c_int32),
        ("error", C.c_char * 160),
    ]


SUBMIT_BORROW = 1


def header_symbols() -> list[str]:
    """Function names declared in include/evoc_gpu.h."""
    import re

    src = open(HEADER_PATH).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(evoc_gpu_[a-z0-9_]+)\s*\(", src)))


def default_opts() -> Opts:
    o = Opts()
    lib().evoc_gpu_default_opts(C.byref(o))
    return o


class Context:
    """One evoc_gpu_ctx (a CUDA stream plus scratch on one device)."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        rc = lib().evoc_gpu_ctx_create(device, C.byref(self.h))
        if rc != EVOC_OK:
            raise RuntimeError(f"evoc_gpu_ctx_create(device={device}) failed with status {rc}")
        self.device = device

    def last_error(self) -> str:
        return lib().evoc_gpu_last_error(self.h).decode()

    @property
    def stream_ptr(self) -> int:
        """The context's cudaStream_t (for torch.cuda.ExternalStream)."""
        return int(lib().evoc_gpu_ctx_stream(self.h) or 0)

    def profile(self, enable: bool = True) -> None:
        lib().evoc_gpu_profile_enable(self.h, 1 if enable else 0)

    def stages(self) -> list[tuple[str, float]]:
        """(name, milliseconds) of each stage of the last call, device-timed."""
        out = []
        buf = C.create_string_buffer(64)
        ms = C.c_float(0.0)
        for i in range(lib().evoc_gpu_profile_count(self.h)):
            if lib().evoc_gpu_profile_stage(self.h, i, buf, 64, C.byref(ms)) == EVOC_OK:
                out.append((buf.value.decode(), float(ms.value)))
        return out

    def launches(self) -> int:
        return int(lib().evoc_gpu_last_launch_count(self.h))

    def peak_ffma(self) -> float:
        """FP32 FMA TFLOP/s of this device, measured by a hand-written kernel."""
        t, ms = C.c_double(0.0), C.c_double(0.0)
        if lib().evoc_gpu_peak_ffma(self.h, C.byref(t), C.byref(ms)) != EVOC_OK:
            raise RuntimeError(self.last_error())
        return t.value

    def set_wait_limit(self, ns: int, producer_delay_ns: int = 0) -> None:
        """Limit of each pipeline wait in the tensor-core scan (0: the 4 s default); producer_delay_ns
        delays the scan's producer (tests of the timeout path)."""
        if lib().evoc_gpu_set_wait_limit(self.h, int(ns), int(producer_delay_ns)) != EVOC_OK:
            raise ValueError(self.last_error())

    def nndescent_stats(self) -> dict:
        """Iterations, distance evaluations and gathered row bytes of the last NN-descent call."""
        it, ev, rb = C.c_int32(0), C.c_int64(0), C.c_int64(0)
        lib().evoc_gpu_last_nndescent(self.h, C.byref(it), C.byref(ev), C.byref(rb))
        return {"iterations": it.value, "distance_evals": ev.value, "row_bytes": rb.value}

    def certify_counts(self) -> dict:
        """Rows the last 16-bit-form call certified (checked), rescanned with 256 candidates
        (second_pass), and rescanned exactly in FP32 (exact_rescan)."""
        a, b, c = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        lib().evoc_gpu_last_certify(self.h, C.byref(a), C.byref(b), C.byref(c))
        return {"checked": a.value, "second_pass": b.value, "exact_rescan": c.value}

    def set_symmetric_scan(self, min_rows: int) -> None:
        """16-bit-form self-joins of at least min_rows rows take the symmetric scan (0 or
        negative: never, the default)."""
        if lib().evoc_gpu_set_symmetric_scan(self.h, int(min_rows)) != EVOC_OK:
            raise ValueError(self.last_error())

    def symmetric_stats(self) -> dict:
        """The last call's symmetric scan: sample rows of its pre-scan (0: not taken), mailbox
        capacity per row, the most mailbox keys a row was offered, rows that overflowed."""
        a, b, c, d = C.c_int64(0), C.c_int64(0), C.c_int64(0), C.c_int64(0)
        lib().evoc_gpu_last_symmetric(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(d))
        return {"sample_rows": a.value, "mailbox_cap": b.value, "max_offers": c.value, "overflowed": d.value}

    def close(self) -> None:
        if self.h:
            lib().evoc_gpu_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    with _lock:
        ctx = _contexts.get(device)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _contexts[device] = ctx
    return ctx
