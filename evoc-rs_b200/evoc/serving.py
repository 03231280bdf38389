"""Continuous-batching kNN-graph server: the host-side mirror of the evoc_gpu_server C ABI.

Requests of any n, dim and dtype are submitted as they arrive; the library's
lanes (one CUDA stream and scratch each) admit the oldest request that fits
the HBM budget, so several requests run on the device at once and a request
arriving while others run starts as soon as a lane and memory are free.
Each request's graph stays in HBM until `result` copies it out (or `release`
drops it).

The per-request call mirrors knn_graph (src/knn.rs:345-359): same options,
same k clamp, same errors (EmptyData, InvalidNeighbors), and the same RNG draw
contract -- submit advances the caller's RandomState exactly as knn_graph does.
evoc-rs itself has no server; its fit_predict builds one data set's graph at a
time (src/clustering.rs:650-716).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .knn import BackendError, EmbeddingData, EmptyData, InvalidNeighbors, KnnGraphOptions, _advance_rng, _to_opts


class JobCancelled(BackendError):
    def __init__(self, job: int):
        super().__init__(_lib.EVOC_ERR_CANCELLED, f"job {job} was cancelled")


class Server:
    """One evoc_gpu_server on one device."""

    def __init__(self, budget_bytes: int = 150 * 10**9, max_inflight: int = 4, device: int = 0,
                 profile: bool = False, batch_max: int = 64, small_lanes: int = 0, admission: str = "oldest"):
        L = _lib.lib()
        o = _lib.ServerOpts()
        L.evoc_gpu_server_default_opts(C.byref(o))
        o.device = int(device)
        o.budget_bytes = int(budget_bytes)
        o.max_inflight = int(max_inflight)
        o.profile = 1 if profile else 0
        o.batch_max = int(batch_max)
        o.small_lanes = int(small_lanes)  # lanes for requests under 65,536 rows only
        if admission not in ("oldest", "smallest"):
            raise ValueError("admission must be 'oldest' or 'smallest'")
        o.admission = 0 if admission == "oldest" else 1  # oldest request first, or smallest scan first
        self.h = C.c_void_p()
        rc = L.evoc_gpu_server_create(C.byref(o), C.byref(self.h))
        if rc != _lib.EVOC_OK:
            raise BackendError(rc, f"evoc_gpu_server_create(device={device}, lanes={max_inflight}) failed")
        self.device = device
        self._keep: dict[int, object] = {}  # host arrays the server reads in place

    # -- submission ---------------------------------------------------------------------------
    def submit(self, data, options: KnnGraphOptions, rng=None, *, borrow: bool = False) -> int:
        """Queue one request (host rows).  With borrow=True the server reads the array in place
        (no copy at submit); the array is kept alive here until the job is fetched or released."""
        data = EmbeddingData.wrap(data)
        if options.n_neighbors <= 0:
            raise InvalidNeighbors()
        if data.nrows() == 0:
            raise EmptyData()
        tau = _advance_rng(rng, data, options) if rng is not None else None
        arr = np.ascontiguousarray(data.array)
        n, dim = arr.shape
        o = _to_opts(options)
        jid = C.c_int64(0)
        P = C.c_void_p
        rc = _lib.lib().evoc_gpu_server_submit(self.h, C.byref(o), data.dtype_code, arr.ctypes.data_as(P), n, dim,
                                               int(options.n_neighbors),
                                               tau.ctypes.data_as(P) if tau is not None else None,
                                               _lib.SUBMIT_BORROW if borrow else 0, C.byref(jid))
        self._raise(rc, "submit")
        if borrow:
            self._keep[jid.value] = arr
        return jid.value

    def submit_device(self, ptr: int, dtype_code: int, n: int, dim: int, options: KnnGraphOptions,
                      tau: Optional[np.ndarray] = None, keep_alive=None) -> int:
        """Queue one request whose rows are already on the server's device (e.g. a torch tensor's
        data_ptr()); `keep_alive` is held until the job is fetched or released."""
        if options.n_neighbors <= 0:
            raise InvalidNeighbors()
        if n == 0:
            raise EmptyData()
        o = _to_opts(options, on_device=True)
        jid = C.c_int64(0)
        P = C.c_void_p
        t = None if tau is None else np.ascontiguousarray(tau, np.int64)
        rc = _lib.lib().evoc_gpu_server_submit(self.h, C.byref(o), dtype_code, P(ptr), n, dim,
                                               int(options.n_neighbors), t.ctypes.data_as(P) if t is not None else None,
                                               0, C.byref(jid))
        self._raise(rc, "submit")
        if keep_alive is not None:
            self._keep[jid.value] = keep_alive
        return jid.value

    def request_bytes(self, dtype_code: int, n: int, dim: int, options: KnnGraphOptions,
                      on_device: bool = False) -> tuple[int, int]:
        """(resident, workspace) bytes a request is admitted against on a lane holding no buffers."""
        o = _to_opts(options, on_device=on_device)
        res, ws = C.c_int64(0), C.c_int64(0)
        rc = _lib.lib().evoc_gpu_server_request_bytes(self.h, C.byref(o), dtype_code, n, dim,
                                                      int(options.n_neighbors), C.byref(res), C.byref(ws))
        self._raise(rc, "request_bytes")
        return res.value, ws.value

    # -- completion ---------------------------------------------------------------------------
    def poll(self, job: int) -> int:
        return int(_lib.lib().evoc_gpu_server_poll(self.h, job))

    def done(self, job: int) -> bool:
        return self.poll(job) != _lib.EVOC_ERR_PENDING

    def wait(self, job: int, timeout: Optional[float] = None) -> int:
        ms = -1 if timeout is None else int(timeout * 1000)
        return int(_lib.lib().evoc_gpu_server_wait(self.h, job, ms))

    def wait_any(self, timeout: Optional[float] = None) -> Optional[tuple[int, int]]:
        """(job, status) of the next finished job not yet reported, or None on timeout."""
        ms = -1 if timeout is None else int(timeout * 1000)
        jid = C.c_int64(0)
        rc = _lib.lib().evoc_gpu_server_wait_any(self.h, ms, C.byref(jid))
        if rc == _lib.EVOC_ERR_TIMEOUT and jid.value == 0:
            return None
        return jid.value, int(rc)

    def result(self, job: int, *, keep_resident: bool = False, out=None):
        """(indices int32 (n,k), distances f32 (n,k)) of a job, as knn_graph returns them."""
        self.wait(job)
        info = self.info(job)  # read before the result call releases the job
        n, k = info["n"], info["k_eff"]
        if out is not None:
            ind, dst = out
        else:
            ind = np.empty((n, k), np.int32)
            dst = np.empty((n, k), np.float32)
        kout = C.c_int32(0)
        P = C.c_void_p
        rc = _lib.lib().evoc_gpu_server_result(self.h, job, ind.ctypes.data_as(P), dst.ctypes.data_as(P),
                                               C.byref(kout), 1 if keep_resident else 0)
        if not keep_resident:
            self._keep.pop(job, None)
        if rc == _lib.EVOC_ERR_CANCELLED:
            raise JobCancelled(job)
        if rc != _lib.EVOC_OK:
            raise BackendError(rc, info["error"] or f"job {job} failed")
        return ind, dst

    def result_device(self, job: int) -> tuple[int, int, int]:
        """(indices ptr, distances ptr, k) of a finished job's graph in HBM."""
        pi, pd = C.c_void_p(), C.c_void_p()
        kout = C.c_int32(0)
        rc = _lib.lib().evoc_gpu_server_result_device(self.h, job, C.byref(pi), C.byref(pd), C.byref(kout))
        self._raise(rc, f"result_device({job})")
        return int(pi.value or 0), int(pd.value or 0), kout.value

    def release(self, job: int) -> None:
        _lib.lib().evoc_gpu_server_release(self.h, job)
        self._keep.pop(job, None)

    def cancel(self, job: int) -> None:
        self._raise(_lib.lib().evoc_gpu_server_cancel(self.h, job), f"cancel({job})")

    # -- introspection ------------------------------------------------------------------------
    def info(self, job: int) -> dict:
        ji = _lib.JobInfo()
        rc = _lib.lib().evoc_gpu_server_job_info(self.h, job, C.byref(ji))
        self._raise(rc, f"job_info({job})")
        return {"submit_ns": ji.submit_ns, "admit_ns": ji.admit_ns, "done_ns": ji.done_ns, "n": ji.n,
                "dim": ji.dim, "dtype": ji.dtype, "k_eff": ji.k_eff, "lane": ji.lane, "status": ji.status,
                "error": ji.error.decode(errors="replace")}

    def stats(self) -> dict:
        c = _lib.ServerCounters()
        self._raise(_lib.lib().evoc_gpu_server_stats(self.h, C.byref(c)), "stats")
        return {name: int(getattr(c, name)) for name, _ in _lib.ServerCounters._fields_}

    def stage_totals(self) -> dict:
        """{stage: (summed device ms, requests)} over all finished requests (profile=True)."""
        L = _lib.lib()
        out = {}
        buf = C.create_string_buffer(64)
        ms, cnt = C.c_double(0.0), C.c_int64(0)
        for i in range(L.evoc_gpu_server_stage_count(self.h)):
            if L.evoc_gpu_server_stage(self.h, i, buf, 64, C.byref(ms), C.byref(cnt)) == _lib.EVOC_OK:
                out[buf.value.decode()] = (float(ms.value), int(cnt.value))
        return out

    def lane_busy_ms(self) -> float:
        """Host time the lanes spent on requests, summed over lanes."""
        return float(_lib.lib().evoc_gpu_server_lane_busy_ms(self.h))

    @staticmethod
    def now_ns() -> int:
        """The clock of the job times (CLOCK_MONOTONIC), in ns."""
        return int(_lib.lib().evoc_gpu_server_now_ns())

    def close(self) -> None:
        if self.h:
            _lib.lib().evoc_gpu_server_destroy(self.h)
            self.h = C.c_void_p()
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _raise(rc: int, what: str) -> None:
        if rc == _lib.EVOC_OK:
            return
        if rc == _lib.EVOC_ERR_EMPTY:
            raise EmptyData()
        if rc == _lib.EVOC_ERR_K:
            raise InvalidNeighbors()
        if rc == _lib.EVOC_ERR_OOM:
            raise BackendError(rc, f"{what}: request does not fit the HBM budget")
        raise BackendError(rc, f"{what} failed")
