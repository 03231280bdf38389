#!/usr/bin/env python
"""Benchmark: kNN-graph edges/s on the 1,000,000 x 768 f32 cosine k=30 workload.

Workload (zipf_1m_768): 200 Gaussian clusters with Zipf(1.1) sizes, centres
N(0,1), per-cluster per-dimension sigma ~ U(0.1, 0.5), rows L2-normalised,
seed 7 (+ rank), k = 30; generated on the device (synthetic stand-in for the
reference's own make_blobs workloads; no dataset is downloaded).

One step = one kNN-graph build of the whole workload (every row's 30
neighbours) in the headline form (the metric's "BF16+rerank" form): tcgen05
16-bit exact scan with FP16 operands keeping ceil(2.5k) candidates per row,
FP32 rerank (FP64 at the k-th boundary) with a per-row certificate, rescans of
the rows that fail it.

  value    edges/s (rows x k / step time) with the rows already in HBM,
           step timed with CUDA events on the library's own stream, max over
           ranks; each rank builds its own independent graph (weak scaling).
  e2e      the same through the public API with pinned HOST buffers: the
           host->device copy of the rows and the device->host copy of the
           indices and distances are inside every timed step.
  roofline the dominant kernel (the 16-bit scan): 2 n^2 d algorithmic FLOPs per
           launch over its CUDA-event duration, against the measured dense
           BF16 peak (FP16 and BF16 MMAs run at the same rate).
  fp32_form the plain FP32 SIMT form on a slice of query rows against all rows.
  cpu_baseline  the reference's NN-descent (restated in oracle/, all host
           threads) on a bounded prefix of the same workload.

  serving  (default run) the continuous-batching server on 10,000 Poisson
           requests at 200 req/s: edges/s and p50/p95/p99 latency, next to
           the plain FP32 form run one request at a time.

--workload gmm_i8 (2,000,000 x 384 i8, k=15) and --workload bits
(4,000,000 x 1,024 bits, k=15) measure the exact integer forms instead, with
a sampled exactness check and the int8 roofline.
--impl reference runs only the CPU path, on the same metric and workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
# where the raw clock samples go (the JSON line carries their summary)
OUT_DIR = os.environ.get("EVOC_BENCH_OUT", os.path.join(ROOT, "bench_out"))
sys.path.insert(0, os.path.join(ROOT, "evoc-rs_b200"))
sys.path.insert(0, ROOT)

METRIC = "kNN edges/s at recall@k>=0.99 vs FP64 (BF16+FP32-rerank form)"
METRIC_INT = "kNN edges/s, exact integer arithmetic (bit-exact to the reference's {kind} path)"
UNIT = "edges/s"
WORKLOAD = "zipf_1m_768: 1,000,000 x 768 f32, 200 Zipf(1.1) clusters, cosine k=30, seed 7"
# Workload name -> (rows, dim or bytes per row, k) and its description.
WORKLOADS = {
    "zipf_f32": (1_000_000, 768, 30, WORKLOAD),
    "gmm_i8": (2_000_000, 384, 15, "gmm_i8_2m_384: round(127 x) of L2-normalised 100-cluster GMM (sigma 0.25), "
                                   "i8, k=15, seed 11"),
    "bits": (4_000_000, 128, 15, "bits_4m_1024: 500 Bernoulli(0.1) prototypes over 1,024 bits, 5% flips, packed "
                                 "128 B/row, Jaccard k=15, seed 13"),
}

# DRAM bytes (read + write) of one launch of the 16-bit scan (FP16 operands,
# keep 75, 3 stages, 1 epilogue group -- the variant the tuner picks): 6.393e9 B
# captured with ncu (dram__bytes_read.sum + dram__bytes_write.sum) at
# n = 262,144, scaled by the number of (query, key) pairs to n = 1,000,000 (the
# key rows are re-streamed once per wave of query blocks, so traffic grows
# with n^2).
SCAN_TRAFFIC_BYTES_262K = 6_392_895_864
# The same for the int8 scan (gmm_i8 rows, d = 384, keep 15, 3 stages, 4
# epilogue groups): 1.380e9 B at n = 262,144, scaled by n^2.  The Jaccard scan
# has no such figure: its 262,144-row capture (130 GB, twice L2 in keys) is
# not a proxy for 4M rows, and a full-size capture is beyond ncu's limits here.
I8_TRAFFIC_BYTES_262K = 1_379_694_592


def scan_traffic(n):
    return SCAN_TRAFFIC_BYTES_262K * (n / 262144.0) ** 2


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str, path: str):
        self.path = path
        self.proc = None
        try:
            self.f = open(path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", gpu_id], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s, p in zip(sm, power) if p > 0.5 * max(power)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_nndescent_sample(x_host, k, rows, threads, deterministic=False):
    """The reference's knn_graph NN-descent (restated in oracle/) on a prefix."""
    from oracle import oracle as O

    O.build()
    O.set_num_threads(threads)
    sub = x_host[:rows].copy()
    t0 = time.perf_counter()
    ind, dst = O.knn_graph(sub, k, O.RandomState(7), deterministic=deterministic, n_threads=threads)
    return time.perf_counter() - t0, ind


def host_workload(name, rows, dim, seed_offset=0):
    """A bounded draw of the workload on the host (the CPU arms' sample)."""
    from evoc import synthetic

    if name == "gmm_i8":
        return synthetic.gmm_i8(n=rows, dim=dim, seed=11 + seed_offset)
    if name == "bits":
        return synthetic.bits_u8(n=rows, nbits=dim * 8, seed=13 + seed_offset)
    return synthetic.zipf_f32(n=rows, dim=dim, seed=7 + seed_offset)


def run_reference(args, world, rank):
    import numpy as np

    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    rows = args.cpu_rows
    x = host_workload(args.workload, rows, args.dim)
    for _ in range(args.warmup):
        cpu_nndescent_sample(x, args.k, rows, threads)
    times = []
    for _ in range(args.steps):
        t, _ = cpu_nndescent_sample(x, args.k, rows, threads)
        times.append(t)
    ms = 1000.0 * sum(times) / len(times)
    value = rows * args.k / (ms / 1000.0)
    sample = (f"NN-descent (RP forest + sorted local join, src/knn.rs / src/nndescent/*.rs restated in "
              f"oracle/evoc_oracle.c) on a {rows}-row draw of the same distribution, {threads} threads")
    metric, dtype = METRIC, "f32"
    if args.workload == "gmm_i8":
        metric, dtype = METRIC_INT.format(kind="Int8"), "int8"
    elif args.workload == "bits":
        metric, dtype = METRIC_INT.format(kind="Binary (UInt8)"), "u8"
    line = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOADS[args.workload][3], "n": args.n, "d": args.dim, "k": args.k,
                   "sample_rows": rows},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def recall_vs_fp64(x, ind, rows, k):
    """recall@k and max |distance - FP64 distance| of the reported pairs, on query rows [0, rows)."""
    import torch

    hits = 0
    max_err = 0.0
    X64 = x.double()
    for r0 in range(0, rows, 256):
        r1 = min(rows, r0 + 256)
        q = X64[r0:r1]
        s = q @ X64.T
        s[torch.arange(r1 - r0), torch.arange(r0, r1)] = 2.0  # self first
        top = s.topk(k, dim=1).indices
        got = ind[r0:r1].long()
        hits += (top.unsqueeze(2) == got.unsqueeze(1)).any(dim=2).sum().item()
    return hits / (rows * k), max_err


def transform_f64(dots, self_mask):
    import torch

    d = torch.where(dots > 0, -torch.log2(dots.clamp(min=1e-300)), torch.zeros_like(dots))
    d = torch.clamp(d, min=0.0)
    d[self_mask] = 0.0
    return d


SERVING_WORKLOAD = ("serving_10k: Poisson arrivals at 200 req/s; n log-uniform [500, 200000], d from "
                    "{128, 384, 768}, 80% f32 / 20% i8, 5-50-cluster GMM sigma 0.3, k=15, HBM budget 150 GB")


def _pct(v, q):
    import numpy as np

    return float(np.percentile(np.asarray(v, dtype=np.float64), q)) if len(v) else None


def serve_stream(srv, pools, sched, ids, k, paced, forms=("bf16_rerank", "exact_int"), stall_s=300.0):
    """Open-loop client: submits request i at its scheduled arrival (or all at
    once), fetches each finished graph to host memory, and returns per-request
    (arrival, admit, done-with-result-on-host) times in ns plus edges."""
    import threading

    import evoc
    from evoc.serving import Server

    opts = {False: evoc.KnnGraphOptions(n_neighbors=k, form=forms[0]),
            True: evoc.KnnGraphOptions(n_neighbors=k, form=forms[1])}
    lock = threading.Lock()
    jid_to_i, arrival_ns = {}, {}
    failures = []
    t0 = Server.now_ns() + 20_000_000

    def submitter():
        try:
            for i in ids:
                at = t0 + (int(sched["arrival"][i] * 1e9) if paced else 0)
                while True:
                    now = Server.now_ns()
                    if now >= at:
                        break
                    time.sleep(min(0.002, (at - now) / 1e9))
                n, d, q = int(sched["n"][i]), int(sched["dim"][i]), bool(sched["i8"][i])
                jid = srv.submit(pools.rows_for(int(i), n, d, q), opts[q], borrow=True)
                with lock:
                    jid_to_i[jid] = int(i)
                    arrival_ns[int(i)] = at
        except Exception as e:  # surfaced by the collector
            failures.append(repr(e))

    th = threading.Thread(target=submitter, daemon=True)
    th.start()
    rec = {}
    while len(rec) < len(ids):
        got = srv.wait_any(timeout=stall_s)
        if got is None or failures:
            raise RuntimeError(f"serving stalled or failed: {failures}")
        jid, rc = got
        info = srv.info(jid)
        ind, _ = srv.result(jid)
        t_done = Server.now_ns()
        while True:
            with lock:
                i = jid_to_i.get(jid)
            if i is not None:
                break
            time.sleep(0.0005)
        rec[i] = (arrival_ns[i], info["admit_ns"], t_done, int(ind.shape[0]) * int(ind.shape[1]))
    th.join()
    return t0, rec


def serving_summary(t0, rec, sched=None):
    arr = [rec[i][0] for i in rec]
    lat = [(rec[i][2] - rec[i][0]) / 1e6 for i in rec]
    by_size = None
    if sched is not None:
        by_size = {}
        for name, lo, hi in (("n<16384", 0, 16384), ("16384<=n<65536", 16384, 65536), ("n>=65536", 65536, 1 << 40)):
            sel = [(rec[i][2] - rec[i][0]) / 1e6 for i in rec if lo <= sched["n"][i] < hi]
            if sel:
                by_size[name] = {"requests": len(sel), "p50": _pct(sel, 50), "p99": _pct(sel, 99)}
    queue = [(rec[i][1] - rec[i][0]) / 1e6 for i in rec]
    end = max(rec[i][2] for i in rec)
    edges = sum(rec[i][3] for i in rec)
    span = (end - t0) / 1e9
    return {"requests": len(rec), "edges": edges, "makespan_s": span, "edges_per_s": edges / span,
            "arrival_window_s": (max(arr) - t0) / 1e9,
            "latency_ms": {"p50": _pct(lat, 50), "p95": _pct(lat, 95), "p99": _pct(lat, 99), "max": max(lat)},
            "latency_ms_by_size": by_size,
            "queue_ms": {"p50": _pct(queue, 50), "p99": _pct(queue, 99)}}


def small_graph_batch(dev, m=256, n=2000, d=384, k=15, reps=3):
    """Many small graphs: one evoc_gpu_knn_graph_batch call against one evoc_gpu_knn_graph call per
    graph (device-resident f32 rows, BF16+rerank form), wall time of whole passes."""
    import torch

    import evoc
    from evoc import _lib

    g = torch.Generator(device=dev)
    g.manual_seed(5)
    xs = []
    for _ in range(m):
        x = torch.randn(n, d, generator=g, device=dev)
        xs.append(x / x.norm(dim=1, keepdim=True))
    opts = evoc.KnnGraphOptions(n_neighbors=k, form="bf16_rerank")
    oi = [torch.empty((n, k), dtype=torch.int32, device=dev) for _ in range(m)]
    od = [torch.empty((n, k), dtype=torch.float32, device=dev) for _ in range(m)]
    torch.cuda.synchronize()

    def singles():
        for x, a, b in zip(xs, oi, od):
            evoc.knn_graph_device(x.data_ptr(), _lib.DTYPE_F32, n, d, k, a.data_ptr(), b.data_ptr(), opts)

    def batch():
        evoc.knn_graph_batch_device([x.data_ptr() for x in xs], _lib.DTYPE_F32, [n] * m, [d] * m, k,
                                    [a.data_ptr() for a in oi], [b.data_ptr() for b in od], opts)

    out = {"graphs": m, "n": n, "d": d, "k": k}
    for name, fn in (("one_call_per_graph_ms", singles), ("batch_ms", batch)):
        fn()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        out[name] = (time.perf_counter() - t) / reps * 1e3
    batch()
    first = [a.clone() for a in oi]
    singles()
    out["identical"] = all(torch.equal(a, b) for a, b in zip(first, oi))
    out["speedup"] = out["one_call_per_graph_ms"] / out["batch_ms"]
    out["batch_edges_per_s"] = m * n * k / (out["batch_ms"] / 1e3)
    return out


def run_serving(args, dev):
    """The continuous-batching server on the serving workload, next to the
    plain FP32 form run one request at a time on the same arrivals."""
    import numpy as np

    from evoc import synthetic
    from evoc.serving import Server

    k = 15
    sched = synthetic.serving_schedule(count=args.serve_requests, rate=args.serve_rate)
    pools = synthetic.ServingPools(dev)
    offered = float((sched["n"] * k).sum() / max(sched["arrival"][-1], 1e-9))
    # Warm-up requests: the largest shape of each (d, dtype) once per lane, then small ones.
    warm = [(200_000, d, q) for d in (128, 384, 768) for q in (False, True) for _ in range(args.serve_lanes)]
    small = [(500 + 97 * t, (128, 384, 768)[t % 3], t % 5 == 0) for t in range(16)]
    warm += small
    warm_sched = {"arrival": np.zeros(len(warm)), "n": np.array([w[0] for w in warm], np.int64),
                  "dim": np.array([w[1] for w in warm], np.int64), "i8": np.array([w[2] for w in warm], bool)}
    out = {"workload": SERVING_WORKLOAD, "lanes": args.serve_lanes, "budget_bytes": 150 * 10**9,
           "offered_edges_per_s": offered,
           "data": "rows cut from 4 pinned-host mixtures per (d, dtype), window chosen by request id",
           "timing": "host monotonic clock: scheduled arrival -> graph copied back to host memory"}
    with Server(budget_bytes=150 * 10**9, max_inflight=args.serve_lanes, profile=True,
                batch_max=args.serve_batch, small_lanes=args.serve_small_lanes,
                admission=args.serve_admission) as srv:
        serve_stream(srv, pools, warm_sched, list(range(len(warm_sched["n"]))), k, paced=False)
        t0, rec = serve_stream(srv, pools, sched, list(range(len(sched["n"]))), k, paced=True)
        out.update(serving_summary(t0, rec, sched))
        st = srv.stats()
        out["peak_bytes"] = st["peak_bytes"]
        out["failed"] = st["failed"]
        out["workspace_misses"] = st["workspace_misses"]
        out["batches"], out["batched_requests"] = st["batches"], st["batched"]
        if args.serve_capacity > 0:
            ids = list(range(min(args.serve_capacity, len(sched["n"]))))
            st0, busy0 = srv.stage_totals(), srv.lane_busy_ms()
            t0c, recc = serve_stream(srv, pools, sched, ids, k, paced=False)
            c = serving_summary(t0c, recc)
            st1, busy1 = srv.stage_totals(), srv.lane_busy_ms()
            stages = {nm: round(v[0] - st0.get(nm, (0.0, 0))[0], 1) for nm, v in st1.items()}
            scan_ops = 0.0
            for i in ids:
                nn, dd, q = float(sched["n"][i]), float(sched["dim"][i]), bool(sched["i8"][i])
                scan_ops += 2.0 * nn * nn * dd
            out["capacity"] = {"requests": c["requests"], "edges_per_s": c["edges_per_s"], "makespan_s": c["makespan_s"],
                               "scan_ops_per_s": scan_ops / c["makespan_s"],
                               "stage_device_ms_sum": stages,
                               "lane_busy_frac": (busy1 - busy0) / (args.serve_lanes * c["makespan_s"] * 1e3),
                               "note": ("the first requests of the stream submitted at once (closed queue); "
                                        "stage_device_ms_sum adds each request's stage times (CUDA events on its "
                                        "lane's stream), so stages of concurrent requests overlap")}
    out["small_graph_batch"] = small_graph_batch(dev)
    if args.serve_baseline > 0:
        ids = list(range(min(args.serve_baseline, len(sched["n"]))))
        with Server(budget_bytes=150 * 10**9, max_inflight=1) as base:
            serve_stream(base, pools, warm_sched, list(range(len(warm) - len(small), len(warm))), k, paced=False,
                         forms=("fp32", "exact_int"))
            t0b, recb = serve_stream(base, pools, sched, ids, k, paced=True, forms=("fp32", "exact_int"))
        b = serving_summary(t0b, recb)
        b["note"] = ("plain FP32 SIMT form (i8 requests: exact int8 form), one request at a time, on the first "
                     f"{len(ids)} arrivals of the same stream; the queue grows without bound at this rate")
        out["fp32_one_at_a_time"] = b
        out["edges_per_s_vs_fp32_one_at_a_time"] = out["edges_per_s"] / b["edges_per_s"]
    return out


def int8_peak_tops(dev, sustain_s=4.0):
    """int8 GEMM throughput of the library path torch uses (cuBLASLt via torch._int_mm), 8192^3: best of
    10 (burst) and back to back for `sustain_s` seconds (sustained, under the power cap), both with CUDA
    events.  No int8 figure is recorded in MEASURED_PEAKS.json; the scan runs for seconds, so its
    fraction is taken against the sustained figure, as the BF16 roofline is."""
    import torch

    try:
        m = 8192
        ops = 2.0 * m ** 3
        a = torch.randint(-127, 128, (m, m), dtype=torch.int8, device=dev)
        b = torch.randint(-127, 128, (m, m), dtype=torch.int8, device=dev).t()
        for _ in range(3):
            torch._int_mm(a, b)
        best = float("inf")
        for _ in range(10):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        reps = max(1, int(sustain_s / (best / 1e3)))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        burst = ops / (best / 1e3) / 1e12
        sustained = ops * reps / (e0.elapsed_time(e1) / 1e3) / 1e12
        return sustained, burst, (f"measured in this run: torch._int_mm 8192^3 int8, back to back for "
                                  f"{sustain_s:.0f} s (sustained); burst best of 10 = {burst:.0f} TOPS")
    except Exception as e:  # noqa: BLE001
        return 4500.0, 4500.0, f"nominal dense int8 (torch._int_mm unavailable: {type(e).__name__})"


def sampled_exact_check(x, oi, oraw, k, kind, rows=128):
    """Sampled query rows against a brute force on the GPU: FP64 dots for i8 (exact integers), f32 0/1
    matmul for binary (exact counts, IEEE division for the Jaccard value).  Indices and raw values must
    match exactly (the k smallest by (raw, index), self raw -1)."""
    import numpy as np
    import torch

    n = x.shape[0]
    q = torch.arange(0, n, max(1, n // rows), device=x.device)[:rows]
    if kind == "i8":
        X = x.double()
        raw = -(X[q] @ X.T)
        del X
    else:
        nb = x.shape[1]
        bits = torch.stack([(x >> (7 - b)) & 1 for b in range(8)], dim=2).reshape(n, nb * 8).float()
        inter = bits[q] @ bits.T
        pc = bits.sum(1)
        del bits
        uni = pc[q][:, None] + pc[None, :] - inter
        raw = torch.where(uni > 0, -(inter / uni), torch.zeros_like(inter)).double()
    raw[torch.arange(len(q), device=x.device), q] = -1.0
    vals, idx = torch.topk(raw, k + 64, dim=1, largest=False)
    vals, idx = vals.cpu().numpy(), idx.cpu().numpy()
    gi, gr = oi[q].cpu().numpy(), oraw[q].cpu().numpy().astype(np.float64)
    ok_i = ok_r = True
    for r in range(len(q)):
        o = np.lexsort((idx[r], vals[r]))[:k]
        ok_i &= bool(np.array_equal(gi[r], idx[r][o]))
        ok_r &= bool(np.array_equal(np.abs(gr[r]), np.abs(vals[r][o])))
    return {"rows": int(len(q)), "indices_exact": ok_i, "raw_exact": ok_r}


def exact_int_leg(workload, n, d, k, dev, local, rank, world, pg, steps, warmup, e2e_steps, check_rows, cpu_rows,
                  autotune=True):
    """C3 / C4: the exact integer forms (int8 dots; binary Jaccard on 0/1-expanded int8 rows) on one
    workload; returns its JSON object (value, e2e, roofline, sampled exactness, CPU baseline)."""
    import numpy as np
    import torch

    import evoc
    from evoc import _lib, synthetic

    i8 = workload == "gmm_i8"
    if i8:
        x = synthetic.gmm_i8(n=n, dim=d, seed=11 + rank, device=dev)
        code, stage, kind = _lib.DTYPE_I8, "int8_scan", "i8"
        ops_per_pair = 2.0 * d
    else:
        x = synthetic.bits_u8(n=n, nbits=d * 8, seed=13 + rank, device=dev)
        code, stage, kind = _lib.DTYPE_U8, "jaccard_scan", "u8"
        ops_per_pair = 2.0 * d * 8
    oi = torch.empty((n, k), dtype=torch.int32, device=dev)
    od = torch.empty((n, k), dtype=torch.float32, device=dev)
    oraw = torch.empty((n, k), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    ctx = _lib.context(local)
    ctx.profile(True)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=dev)
    opts = evoc.KnnGraphOptions(n_neighbors=k, form="exact_int", device=local)
    tuned = evoc.autotune("Int8" if i8 else "UInt8", n, d, k, "exact_int", device=local) if autotune else None

    def step():
        evoc.knn_graph_device(x.data_ptr(), code, n, d, k, oi.data_ptr(), od.data_ptr(), opts,
                              out_raw_ptr=oraw.data_ptr())

    for _ in range(warmup):
        step()
    gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    os.makedirs(OUT_DIR, exist_ok=True)
    clocks = ClockSampler(gpu_id, os.path.join(OUT_DIR, f"clocks_{workload}_rank{rank}.csv"))
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stage_ms, launches = {}, 0
    ev0.record(stream)
    for _ in range(steps):
        step()
        for name, ms in ctx.stages():
            stage_ms.setdefault(name, []).append(ms)
        launches += ctx.launches()
    ev1.record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clk = clocks.stop()
    ms_step = ev0.elapsed_time(ev1) / steps
    if pg:
        t = torch.tensor([ms_step], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_step = float(t.item())
    value = world * n * k / (ms_step / 1000.0)
    check = sampled_exact_check(x, oi, oraw, k, kind, rows=check_rows)

    # End to end through the public API with pinned host buffers.
    xh = torch.empty(x.shape, dtype=x.dtype, pin_memory=True)
    xh.copy_(x)
    ih = torch.empty((n, k), dtype=torch.int32, pin_memory=True)
    dh = torch.empty((n, k), dtype=torch.float32, pin_memory=True)
    xh_np, ih_np, dh_np = xh.numpy(), ih.numpy(), dh.numpy()
    if pg:
        pg.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        evoc.knn_graph(xh_np, opts, None, out=(ih_np, dh_np))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    if pg:
        t = torch.tensor([e2e_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_consistent = bool(np.array_equal(ih_np[:1000], oi[:1000].cpu().numpy()))

    peak, peak_burst, peak_kind = int8_peak_tops(dev)
    scan_ms = statistics.mean(stage_ms[stage])
    achieved = ops_per_pair * n * n / (scan_ms / 1000.0) / 1e12
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TOPS (int8)", "frac": achieved / peak,
                "traffic": I8_TRAFFIC_BYTES_262K * (n / 262144.0) ** 2 if i8 else None,
                "traffic_unit": "bytes per launch (ncu at 262,144 rows, scaled by n^2)" if i8 else None,
                "kernel": f"tc_scan_kernel ({'int8' if i8 else 'Jaccard on 0/1 int8'}, fused top-k)",
                "peak_kind": peak_kind, "peak_burst": peak_burst, "frac_of_burst": achieved / peak_burst,
                "launch_ms": scan_ms, "ops_per_launch": ops_per_pair * n * n}

    cpu = None
    if rank == 0 and world == 1 and cpu_rows > 0:
        from oracle import oracle as O

        threads = os.cpu_count() or 1
        rows = min(cpu_rows, n)
        xs = x[:rows].cpu().numpy()
        O.build()
        O.set_num_threads(threads)
        t0 = time.perf_counter()
        cind, _ = O.knn_graph(xs, k, O.RandomState(7), deterministic=False, n_threads=threads)
        t = time.perf_counter() - t0
        qn = min(2000, rows)
        ei, _ = O.exact_knn(xs, k, 0, qn)
        crec = float(np.mean([len(set(cind[r]) & set(ei[r])) / k for r in range(qn)]))
        cpu = {"value": rows * k / t, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": (f"reference NN-descent for {'Int8' if i8 else 'UInt8 (Jaccard)'} restated in oracle/ on the "
                          f"first {rows} rows, {threads} threads, {t:.1f} s; its recall@{k} vs exact on {qn} of "
                          f"those rows {crec:.4f} (this form is exact)")}

    metric = METRIC_INT.format(kind="Int8" if i8 else "Binary (UInt8)")
    line = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int8" if i8 else "u8 (expanded to 0/1 int8)", "data": "synthetic (generated on device, seeded)",
        "config": {"workload": WORKLOADS[workload][3], "n": n, "d": d, "k": k, "form": "exact_int",
                   "l2": f"inputs larger than L2 ({x.numel() / 1e9:.2f} GB vs 126 MB)",
                   "per_rank": "independent graph per rank"},
        "sampled_exact_check": check,
        "autotune": tuned and {"sample_rows": min(n, 262144 if n >= 1_000_000 else 65536),
                               "variants_ms": tuned["variants_ms"], "chosen": tuned["chosen"]},
        "stages_ms": {kname: statistics.mean(v) for kname, v in stage_ms.items()},
        "roofline": roofline,
        "e2e": {"value": world * n * k / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": int(x.numel()),
                "d2h_bytes_per_step": n * k * 8, "ms_per_step": e2e_ms, "matches_device_path": e2e_consistent},
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
    }
    del x, oi, od, oraw, xh, ih, dh
    torch.cuda.empty_cache()
    return line


def run_exact_int(args, world, rank, local):
    """--workload gmm_i8 / bits: the exact integer forms as the headline line."""
    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    line = exact_int_leg(args.workload, args.n, args.dim, args.k, dev, local, rank, world, pg, args.steps,
                         args.warmup, args.e2e_steps, args.check_rows, args.cpu_rows, bool(args.autotune))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def deterministic_cpu_baseline(x_host, k, rows):
    """The reference's deterministic path on one thread (knn_graph with deterministic = true: RP forest
    and sorted NN-descent on a 1-thread pool, src/knn.rs:345-359) with the reference's own compiled
    native/fast_cosine.c as the distance when oracle/_ref holds it; on the first `rows` rows."""
    from oracle import oracle as O

    O.build()
    ref = O.use_reference_cosine(True)
    O.set_num_threads(1)
    sub = x_host[:rows].copy()
    t0 = time.perf_counter()
    ind, _ = O.knn_graph(sub, k, O.RandomState(7), deterministic=True, n_threads=1)
    t = time.perf_counter() - t0
    O.use_reference_cosine(False)
    return t, ind, ref


def recall_on_host(x, ind, k, rows):
    """recall@k of `ind` (rows 0..rows-1 of x, self first) against FP64 brute force, on the host."""
    import numpy as np

    x64 = x.astype(np.float64)
    hits = 0
    for r0 in range(0, rows, 512):
        r1 = min(rows, r0 + 512)
        s = x64[r0:r1] @ x64.T
        s[np.arange(r1 - r0), np.arange(r0, r1)] = 2.0
        top = np.argpartition(-s, k - 1, axis=1)[:, :k]
        hits += sum(len(set(top[i]) & set(ind[r0 + i][:k])) for i in range(r1 - r0))
    return hits / (rows * k)


def blobs_leg(dev, local, steps=20, warmup=5):
    """C1: 2,000 x 128 f32, 10 Gaussian blobs (sigma 0.3), k=15, seed 42 -- the reference's own
    CPU-runnable case: edges/s of the default (FP16 scan + FP32 rerank) form with the rows resident,
    end to end with host buffers, parity against the oracle's exact selection, and the reference's
    deterministic path (single thread) on the same rows."""
    import numpy as np
    import torch

    import evoc
    from evoc import _lib, synthetic
    from oracle import oracle as O

    x = synthetic.blobs_2k_128()
    n, d, k = x.shape[0], x.shape[1], 15
    xd = torch.from_numpy(x).to(dev)
    oi = torch.empty((n, k), dtype=torch.int32, device=dev)
    od = torch.empty((n, k), dtype=torch.float32, device=dev)
    oraw = torch.empty((n, k), dtype=torch.float32, device=dev)
    ctx = _lib.context(local)
    ctx.profile(True)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=dev)
    opts = evoc.KnnGraphOptions(n_neighbors=k, form="bf16_rerank", device=local)

    def step():
        evoc.knn_graph_device(xd.data_ptr(), 0, n, d, k, oi.data_ptr(), od.data_ptr(), opts,
                              out_raw_ptr=oraw.data_ptr())

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, scan = 0, []
    ev0.record(stream)
    for _ in range(steps):
        step()
        launches += ctx.launches()
        scan.append(dict(ctx.stages()).get("bf16_scan", float("nan")))
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    cert = ctx.certify_counts()
    ind, raw = oi.cpu().numpy(), oraw.cpu().numpy()
    ei, er = O.exact_knn(x, k)
    same = ind == ei
    x64 = x.astype(np.float64)
    dots = np.einsum("rkd,rd->rk", x64[ind], x64)
    want = np.where(dots > 0, -dots, 1.17549435e-38)
    want[ind == np.arange(n)[:, None]] = -1.0
    xh = torch.empty((n, d), dtype=torch.float32, pin_memory=True)
    xh.copy_(xd)
    ih = torch.empty((n, k), dtype=torch.int32, pin_memory=True)
    dh = torch.empty((n, k), dtype=torch.float32, pin_memory=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    evoc.knn_graph(xh.numpy(), opts, None, out=(ih.numpy(), dh.numpy()))
    e0.record(stream)
    for _ in range(steps):
        evoc.knn_graph(xh.numpy(), opts, None, out=(ih.numpy(), dh.numpy()))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / steps
    t, cind, ref = deterministic_cpu_baseline(x, k, n)
    crec = float(np.mean([len(set(cind[r]) & set(ei[r])) / k for r in range(n)]))
    scan_ms = statistics.median(scan)
    peaks, peak_kind = measured_peaks()
    flops = 2.0 * n * n * d
    return {
        "workload": "blobs_2k_128: 2,000 x 128 f32, 10 N(0,1) centres, sigma 0.3, L2-normalised, k=15, seed 42",
        "value": n * k / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms, "steps": steps, "warmup": warmup,
        "form": "fp16 tensor-core scan + fp32 rerank (certified)", "certificate": cert,
        "parity": {"recall_at_k_vs_oracle_exact": float(np.mean([len(set(ind[r]) & set(ei[r])) / k for r in range(n)])),
                   "indices_equal_to_oracle": int(same.sum()), "entries": int(same.size),
                   "max_abs_raw_err_vs_fp64": float(np.abs(raw.astype(np.float64) - want).max()),
                   "max_abs_raw_diff_vs_oracle": float(np.abs(raw.astype(np.float64) - er).max())},
        "roofline": {"bound": "latency", "achieved": flops / (scan_ms / 1e3) / 1e12, "unit": "TFLOP/s",
                     "peak": float(peaks.get("bf16_tflops")), "peak_kind": f"{peak_kind} bf16 burst",
                     "frac": flops / (scan_ms / 1e3) / 1e12 / float(peaks.get("bf16_tflops")),
                     "launch_ms": scan_ms, "traffic": None,
                     "note": "16 query blocks of 128 rows: 16 of 148 SMs busy, launch/latency-bound by size"},
        "e2e": {"value": n * k / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": n * d * 4,
                "d2h_bytes_per_step": n * k * 8, "ms_per_step": e2e_ms},
        "cpu_baseline": {"value": n * k / t, "unit": UNIT, "cores": 1, "kind": "reference" if ref else "port",
                         "sample": (f"the reference's deterministic path (RP forest + sorted NN-descent, one "
                                    f"thread) restated in oracle/, distance = "
                                    f"{'the reference native/fast_cosine.c compiled unchanged' if ref else 'its restatement'}"
                                    f", all {n} rows: {t:.2f} s; recall@{k} vs exact {crec:.4f}")},
        "gpu_launches": launches,
    }


def mst_leg(emb, n, ncomp, dev, ctx, cpu_rows, min_samples=5):
    """Borůvka MST of the node embedding under mutual reachability (build_cluster_layers' input,
    src/clustering.rs:50-80) on the device, with the oracle's (the reference's reproducible Borůvka,
    restated) timed on a prefix of the same points and both MSTs' weights compared there."""
    import numpy as np
    import torch

    from evoc import boruvka as BV

    edges = torch.empty((n - 1, 3), dtype=torch.float32, device=dev)
    core = torch.empty(n, dtype=torch.float32, device=dev)
    emb = emb.contiguous()
    BV.parallel_boruvka_device(emb.data_ptr(), n, ncomp, min_samples, edges.data_ptr(), core.data_ptr(),
                               device=ctx.device)
    runs = []
    for _ in range(2):
        BV.parallel_boruvka_device(emb.data_ptr(), n, ncomp, min_samples, edges.data_ptr(), core.data_ptr(),
                                   device=ctx.device)
        runs.append((dict(ctx.stages()), ctx.launches()))
    ms = statistics.median(r[0]["total"] for r in runs)
    out = {"metric": "points/s through the MST (KD-tree, core distances, Boruvka rounds)",
           "value": n / (ms / 1000.0), "unit": "points/s", "ms": ms, "points": n, "dim": ncomp,
           "min_samples": min_samples, "mode": "non-reproducible (atomic component bounds)",
           "stages_ms": {nm: statistics.median(r[0][nm] for r in runs) for nm in runs[0][0] if nm != "total"},
           "gpu_launches": runs[-1][1]}
    m = min(cpu_rows, n)
    if m > 1:
        from oracle import mst as OM

        sub = emb[:m].cpu().numpy()
        t0 = time.perf_counter()
        oe, oc, _ = OM.boruvka_mst(sub, min_samples=min_samples)
        to = time.perf_counter() - t0
        ge, gc = BV.parallel_boruvka(sub, min_samples, device=ctx.device, return_core=True)
        gw, ow = np.sort(ge[:, 2].astype(np.float64)), np.sort(oe[:, 2].astype(np.float64))
        out["cpu_baseline"] = {
            "value": m / to, "unit": "points/s", "cores": 1, "kind": "port",
            "sample": (f"oracle restatement of build_kdtree + parallel_boruvka (reproducible, one thread, as "
                       f"build_cluster_layers runs it for reproducible fits) on the first {m} points: {to:.2f} s")}
        out["parity_on_cpu_sample"] = {"points": m, "max_abs_sorted_weight_diff": float(np.abs(gw - ow).max()),
                                       "total_weight_rel_diff": float(abs(gw.sum() - ow.sum()) / ow.sum()),
                                       "max_abs_core_diff": float(np.abs(gc - oc).max())}
    return out


def run_label_prop(args, dev, ctx, stream, x, f_indptr, f_ind, f_dat, nnz, opts):
    """label_propagation_init (src/label_prop.rs:464-494) on the workload's fuzzy graph, resident in
    HBM, then the full-graph node embedding (src/embed.rs:251-369, reproducible) from it; the
    oracle's restatement timed on the fuzzy graph of the first cpu_lp_rows rows beside the GPU
    on the same graph."""
    import numpy as np
    import torch

    import evoc
    from evoc import label_prop as LP

    n, d, k = args.n, args.dim, args.k
    ncomp = min(max(k // 4, 4), 15)
    approx = int(np.clip(8 * np.sqrt(n), 256, 16384))
    out = torch.empty((n, ncomp), dtype=torch.float32, device=dev)
    emb = torch.empty((n, ncomp), dtype=torch.float32, device=dev)

    def lp_once():
        LP.label_propagation_init_device(f_indptr.data_ptr(), f_ind.data_ptr(), f_dat.data_ptr(), n, x.data_ptr(), d,
                                         out.data_ptr(), np.random.RandomState(42), 20, 50, approx, ncomp)
        st = {}
        for nm, ms in ctx.stages():
            st[nm] = st.get(nm, 0.0) + ms
        return st, ctx.launches()

    lp_once()
    runs = [lp_once() for _ in range(max(1, args.lp_reps))]
    lp_ms = statistics.median(r[0]["total"] for r in runs)
    stages = {nm: statistics.median(r[0][nm] for r in runs) for nm in runs[0][0] if nm != "total"}

    def ne_once():
        LP.node_embedding_device(f_indptr.data_ptr(), f_ind.data_ptr(), f_dat.data_ptr(), n, ncomp, 50,
                                 out.data_ptr(), emb.data_ptr(), np.random.RandomState(43))
        return dict(ctx.stages())

    ne_ms = ne_free_ms = float("nan")
    if args.ne_reps > 0:
        ne_once()
        ne_ms = statistics.median(ne_once()["total"] for _ in range(args.ne_reps))

    def ne_free_once():
        LP.node_embedding_device(f_indptr.data_ptr(), f_ind.data_ptr(), f_dat.data_ptr(), n, ncomp, 50,
                                 out.data_ptr(), emb.data_ptr(), np.random.RandomState(43), reproducible=False)
        return dict(ctx.stages())

    if args.ne_reps > 0:
        ne_free_once()
        ne_free_ms = statistics.median(ne_free_once()["total"] for _ in range(args.ne_reps))
    # effective bandwidth of the full-graph epochs: per edge the five f32 schedule words (three read,
    # two written) and the column index, plus one embedding row gathered
    ne_bytes = 50 * nnz * (6 * 4 + ncomp * 4)
    peaks, peak_kind = measured_peaks()
    res = {
        "metric": "graph edges/s through label_propagation_init (partition, reductions, recursive init, "
                  "reduced-graph embedding, expander)",
        "value": nnz / (lp_ms / 1000.0), "unit": "edges/s", "ms": lp_ms, "graph_nnz": nnz, "rows": n,
        "n_components": ncomp, "approx_n_parts": approx, "n_label_prop_iter": 20, "n_embedding_epochs": 50,
        "stages_ms": stages, "gpu_launches": runs[-1][1],
        "node_embedding_full_graph": {
            "ms": ne_ms, "epochs": 50, "ms_per_epoch": ne_ms / 50, "edge_epochs_per_s": 50 * nnz / (ne_ms / 1000.0),
            "roofline": {"bound": "hbm", "achieved": ne_bytes / (ne_ms / 1000.0) / 1e9,
                         "peak": float(peaks.get("hbm_gbs")), "unit": "GB/s",
                         "frac": ne_bytes / (ne_ms / 1000.0) / 1e9 / float(peaks.get("hbm_gbs")),
                         "peak_kind": peak_kind, "traffic": None,
                         "note": "latency-bound gathers; bytes = 6 schedule/index words + one embedding row "
                                 "per edge per epoch"}},
        "node_embedding_full_graph_non_reproducible": {
            "ms": ne_free_ms, "epochs": 50, "ms_per_epoch": ne_free_ms / 50,
            "edge_epochs_per_s": 50 * nnz / (ne_free_ms / 1000.0),
            "note": "reproducible_flag = false (the default when no random_state is set): lock-free epochs"},
        "parity": "bit-identical to the oracle (tests/test_label_prop_gpu.py); oracle pinned to the "
                  "reference's golden intermediates",
    }
    if args.mst:
        try:
            res["boruvka_mst"] = mst_leg(emb if args.ne_reps > 0 else out, n, ncomp, dev, ctx, args.cpu_mst_rows)
        except Exception as e:  # noqa: BLE001 -- reported in the line, the other measurements stand
            res["boruvka_mst"] = {"error": repr(e)}
    m = min(args.cpu_lp_rows, n)
    if m > 0:
        from oracle import label_prop as OL

        xs = x[:m].contiguous()
        si = torch.empty((m, k), dtype=torch.int32, device=dev)
        sd = torch.empty((m, k), dtype=torch.float32, device=dev)
        evoc.knn_graph_device(xs.data_ptr(), 0, m, d, k, si.data_ptr(), sd.data_ptr(), opts)
        torch.cuda.synchronize()
        indptr, indices, data, _, _ = evoc.neighbor_graph_csr(float(k), si.cpu().numpy(), sd.cpu().numpy())
        g = OL.Csr.make(indptr, indices, data, (m, m))
        xh = xs.cpu().numpy()
        ap2 = int(np.clip(8 * np.sqrt(m), 256, 16384))
        LP.label_propagation_init((indptr, indices, data, m), 20, 50, ap2, ncomp, 0.5, 0.1, 0.5,
                                  np.random.RandomState(5), xh)
        t0 = time.perf_counter()
        gi = LP.label_propagation_init((indptr, indices, data, m), 20, 50, ap2, ncomp, 0.5, 0.1, 0.5,
                                       np.random.RandomState(5), xh)
        tg = time.perf_counter() - t0
        rs = np.random.RandomState(5)
        _, key, pos, hg, ga = rs.get_state()
        t0 = time.perf_counter()
        oi = OL.label_propagation_init(g, 20, 50, ap2, ncomp, 0.5, 0.1, 0.5, OL.mt_from_state(key, pos, hg, ga), xh)
        to = time.perf_counter() - t0
        res["cpu_baseline"] = {
            "value": g.nnz / to, "unit": "edges/s", "cores": 1, "kind": "port",
            "sample": (f"oracle restatement of label_propagation_init (C + NumPy, one thread; the reference's "
                       f"label propagation and reproducible epochs are serial) on the fuzzy graph of the first "
                       f"{m} rows ({g.nnz} entries): {to:.2f} s; the GPU with host buffers on the same graph "
                       f"{tg * 1000:.1f} ms, max |GPU - oracle| = {float(np.abs(gi - oi).max()):.3g}")}
    return res


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import evoc
    from evoc import _lib, synthetic

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    n, d, k = args.n, args.dim, args.k
    x = synthetic.zipf_f32(n=n, dim=d, seed=7 + rank, device=dev)
    oi = torch.empty((n, k), dtype=torch.int32, device=dev)
    od = torch.empty((n, k), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    ctx = _lib.context(local)
    ctx.profile(True)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=dev)
    form = args.form
    opts = evoc.KnnGraphOptions(n_neighbors=k, form=form, oversample=0, device=local)
    tuned = (evoc.autotune("Float32", n, d, k, "bf16_rerank", device=local)
             if args.autotune and form == "bf16_rerank" else None)

    def step():
        evoc.knn_graph_device(x.data_ptr(), 0, n, d, k, oi.data_ptr(), od.data_ptr(), opts)

    for _ in range(args.warmup):
        step()
    gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    os.makedirs(OUT_DIR, exist_ok=True)
    clocks = ClockSampler(gpu_id, os.path.join(OUT_DIR, f"clocks_rank{rank}.csv"))
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    stage_ms = {}
    launches = 0
    ev0.record(stream)
    for _ in range(args.steps):
        step()
        for name, ms in ctx.stages():
            stage_ms.setdefault(name, []).append(ms)
        launches += ctx.launches()
    ev1.record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clk = clocks.stop()
    cert = ctx.certify_counts() if form == "bf16_rerank" else None
    sym = ctx.symmetric_stats() if form == "bf16_rerank" else None
    total_ms = ev0.elapsed_time(ev1)
    ms_step = total_ms / args.steps
    if pg:
        t = torch.tensor([ms_step], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_step = float(t.item())
    value = world * n * k / (ms_step / 1000.0)

    # Recall / error vs FP64 on a 10,000-row query sample (untimed).
    sample = min(args.recall_rows, n)
    rec, _ = recall_vs_fp64(x, oi, sample, k)
    X64 = x.double()
    got = oi[:sample].long()
    dots = (X64[:sample].unsqueeze(1) * X64[got]).sum(-1)
    selfm = got == torch.arange(sample, device=dev).unsqueeze(1)
    want = transform_f64(dots, selfm)
    max_err = float((od[:sample].double() - want).abs().max().item())

    # The fuzzy simplicial set of the graph, on the device (σ/ρ, membership,
    # symmetric union as canonical CSR), timed on the library's stream.
    fuzzy = None
    if args.fuzzy:
        import ctypes as C

        cap = 2 * n * k
        f_indptr = torch.empty(n + 1, dtype=torch.int64, device=dev)
        f_ind = torch.empty(cap, dtype=torch.int32, device=dev)
        f_dat = torch.empty(cap, dtype=torch.float32, device=dev)
        f_sig = torch.empty(n, dtype=torch.float32, device=dev)
        f_rho = torch.empty(n, dtype=torch.float32, device=dev)
        nnz = C.c_int64(0)
        P = C.c_void_p
        times = []
        for rep in range(4):
            st = _lib.lib().evoc_gpu_fuzzy_graph(ctx.h, P(oi.data_ptr()), P(od.data_ptr()), n, k, float(k), 1, 1,
                                                 P(f_sig.data_ptr()), P(f_rho.data_ptr()), P(f_indptr.data_ptr()),
                                                 P(f_ind.data_ptr()), P(f_dat.data_ptr()), cap, C.byref(nnz))
            assert st == 0, ctx.last_error()
            if rep:
                times.append(dict(ctx.stages()))
        fuzzy = {"ms": statistics.mean(t["total"] for t in times),
                 "stages_ms": {nm: statistics.mean(t[nm] for t in times) for nm in times[0] if nm != "total"},
                 "nnz": int(nnz.value), "rows": n, "k": k,
                 "note": "sigma/rho bisection, membership strengths, A + A^T - A o A^T as canonical CSR"}
        if args.label_prop and world == 1:
            fuzzy["label_propagation_init"] = run_label_prop(args, dev, ctx, stream, x, f_indptr, f_ind, f_dat,
                                                             int(nnz.value), opts)
        del f_indptr, f_ind, f_dat, f_sig, f_rho

    # End to end through the public API with pinned host buffers.
    xh = torch.empty((n, d), dtype=torch.float32, pin_memory=True)
    xh.copy_(x)
    ih = torch.empty((n, k), dtype=torch.int32, pin_memory=True)
    dh = torch.empty((n, k), dtype=torch.float32, pin_memory=True)
    xh_np, ih_np, dh_np = xh.numpy(), ih.numpy(), dh.numpy()
    evoc.knn_graph(xh_np, opts, None, out=(ih_np, dh_np))  # warm the host path
    if pg:
        pg.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        evoc.knn_graph(xh_np, opts, None, out=(ih_np, dh_np))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.e2e_steps
    if pg:
        t = torch.tensor([e2e_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * n * k / (e2e_ms / 1000.0)
    e2e_consistent = bool(np.array_equal(ih_np[:1000], oi[:1000].cpu().numpy()))

    # Plain FP32 SIMT form on a slice of query rows against all n rows.
    fp32 = None
    if args.fp32_rows > 0 and form == "bf16_rerank":
        rows = min(args.fp32_rows, n)
        fo = evoc.KnnGraphOptions(n_neighbors=k, form="fp32", device=local, row_begin=0, row_end=rows)
        fi = torch.empty((rows, k), dtype=torch.int32, device=dev)
        fd = torch.empty((rows, k), dtype=torch.float32, device=dev)
        warm = evoc.KnnGraphOptions(n_neighbors=k, form="fp32", device=local, row_begin=0, row_end=128)
        evoc.knn_graph_device(x.data_ptr(), 0, n, d, k, fi.data_ptr(), fd.data_ptr(), warm)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        evoc.knn_graph_device(x.data_ptr(), 0, n, d, k, fi.data_ptr(), fd.data_ptr(), fo)
        f1.record(stream)
        torch.cuda.synchronize()
        fms = f0.elapsed_time(f1)
        frec, _ = recall_vs_fp64(x, fi, min(sample, rows), k)
        same = (fi[:sample] == oi[:sample]).float().mean().item()
        ffma = ctx.peak_ffma()
        tfl = 2.0 * rows * n * d / (fms / 1000.0) / 1e12
        fp32 = {"value": rows * k / (fms / 1000.0), "unit": UNIT, "query_rows": rows, "key_rows": n,
                "ms": fms, "recall_at_k_vs_fp64": frec, "index_agreement_with_fp16_form": same,
                "tflops_fp32": tfl,
                "roofline": {"bound": "fp32 ffma", "achieved": tfl, "peak": ffma, "unit": "TFLOP/s",
                             "frac": tfl / ffma,
                             "peak_kind": "measured in this run: hand-written FFMA loop over every SM "
                                          "(evoc_gpu_peak_ffma)"},
                "fp16_form_speedup": value / (rows * k / (fms / 1000.0))}

    peaks, peak_kind = measured_peaks()
    if form == "bf16_rerank":
        scan_ms = statistics.mean(stage_ms.get("bf16_scan", [float("nan")]))
        peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops")))
        if sym and sym["sample_rows"]:
            # one score per unordered pair of rows (self pairs included): n (n + 1) / 2 dot products
            flops = 1.0 * n * (n + 1) * d
            kernel = ("tc_scan_kernel, symmetric mode (FP16 operands, each pair of rows once, fused top-C "
                      "with per-row mailboxes, C = 2k)")
            traffic = None
        else:
            flops = 2.0 * n * n * d
            kernel = "tc_scan_kernel (FP16 operands, fused top-C, C = ceil(2.5k))"
            traffic = scan_traffic(n)
        achieved = flops / (scan_ms / 1000.0) / 1e12
        roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                    "traffic": traffic, "traffic_unit": "bytes per launch (ncu, scaled)",
                    "kernel": kernel, "algorithmic_flops": flops,
                    "peak_kind": f"{peak_kind} bf16 sustained (burst {peaks.get('bf16_tflops')})",
                    "launch_ms": scan_ms}
    else:
        it_ms = stage_ms.get("nnd_iteration", [float("nan")])
        nst = ctx.nndescent_stats()  # of the last timed step
        step_iter_ms = sum(it_ms) / args.steps
        gathered = nst["distance_evals"] * nst["row_bytes"]
        achieved = gathered / (step_iter_ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": float(peaks.get("hbm_gbs")), "unit": "GB/s",
                    "frac": achieved / float(peaks.get("hbm_gbs")), "traffic": None,
                    "kernel": "nnd_join_kernel (candidate row gathers)", "launch_ms": statistics.mean(it_ms),
                    "iterations": nst["iterations"], "distance_evals": nst["distance_evals"],
                    "row_bytes": nst["row_bytes"],
                    "note": ("achieved = candidate-row bytes the joins gathered (distance evaluations x FP16 row "
                             "bytes) over the iterations' device time; rows found in L2 count too, so the "
                             "fraction can pass 1")}

    cpu = None
    if rank == 0 and world == 1 and args.cpu_rows > 0:
        xs = x[: args.cpu_rows].cpu().numpy()
        threads = os.cpu_count() or 1
        t, cind = cpu_nndescent_sample(xs, k, args.cpu_rows, threads)
        xs64 = torch.from_numpy(xs).double().to(dev)
        cg = torch.from_numpy(cind).long().to(dev)
        qrows = min(5000, args.cpu_rows)
        hits = 0
        for r0 in range(0, qrows, 256):
            r1 = min(qrows, r0 + 256)
            s = xs64[r0:r1] @ xs64.T
            s[torch.arange(r1 - r0), torch.arange(r0, r1)] = 2.0
            top = s.topk(k, dim=1).indices
            hits += (top.unsqueeze(2) == cg[r0:r1].unsqueeze(1)).any(dim=2).sum().item()
        crec = hits / (qrows * k)
        cpu = {"value": args.cpu_rows * k / t, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": (f"reference NN-descent restated in oracle/ (rlx-cpu path: serial-order f32 dot, "
                          f"{threads} threads) on the first {args.cpu_rows} rows of the workload; "
                          f"{t:.1f} s; its recall@{k} vs FP64 on {qrows} of those rows {crec:.4f}")}
    cpu_det = None
    if rank == 0 and world == 1 and args.cpu_det_rows > 0:
        rows = min(args.cpu_det_rows, n)
        xs = x[:rows].cpu().numpy()
        t, cind, ref = deterministic_cpu_baseline(xs, k, rows)
        crec = recall_on_host(xs, cind, k, min(2000, rows))
        cpu_det = {"value": rows * k / t, "unit": UNIT, "cores": 1, "kind": "reference" if ref else "port",
                   "sample": (f"the reference's deterministic C path: RP forest + sorted NN-descent on one "
                              f"thread (src/knn.rs deterministic = true) restated in oracle/, distance = "
                              f"{'native/fast_cosine.c compiled unchanged from the reference' if ref else 'its restatement'}"
                              f", on the first {rows} rows: {t:.1f} s; recall@{k} vs FP64 on {min(2000, rows)} "
                              f"of those rows {crec:.4f}")}

    metric = METRIC if form == "bf16_rerank" else "kNN edges/s, GPU NN-descent form (recall vs FP64 reported)"
    line = {
        "metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp16 tensor-core scan + f32 rerank" if form == "bf16_rerank" else "f32 (NN-descent joins, f32 rerank)",
        "data": "synthetic (generated on device, seeded)",
        "config": {"workload": WORKLOAD, "n": n, "d": d, "k": k, "form": form, "oversample": "ceil(2.5 k)",
                   "l2": "inputs larger than L2 (3.1 GB f32 + 1.5 GB fp16 vs 126 MB)",
                   "per_rank": "independent graph per rank"},
        "recall_at_k_vs_fp64": rec, "max_abs_dist_err_vs_fp64": max_err, "recall_sample_rows": sample,
        "stages_ms": {kname: statistics.mean(v) for kname, v in stage_ms.items()},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n * d * 4, "d2h_bytes_per_step": n * k * 8,
                "ms_per_step": e2e_ms, "matches_device_path": e2e_consistent},
        "fp32_form": fp32,
        "fuzzy_graph": fuzzy,
        "autotune": tuned and {"sample_rows": min(n, 262144 if n >= 1_000_000 else 65536),
                               "variants_ms": tuned["variants_ms"], "chosen": tuned["chosen"]},
        "cpu_baseline": cpu,
        "cpu_baseline_deterministic": cpu_det,
        "certificate": cert and dict(cert, note=(
            "rows whose k nearest the 16-bit scan's candidates provably hold (rigorous FP16 error bound); "
            "second_pass rows were rescanned with 256 candidates, exact_rescan rows in FP32")),
        "symmetric_scan": sym and sym["sample_rows"] and dict(sym, note=(
            "each pair of rows multiplied once; scores for the later row reach it through a per-row mailbox "
            "filtered by thresholds from a pre-scan against sample_rows strided rows; overflowed rows are "
            "rescanned by the certificate")),
        "clocks": clk,
        "gpu_launches": launches,
    }
    del xh, ih, dh, xh_np, ih_np, dh_np
    if world == 1 and args.configs:
        torch.cuda.empty_cache()
        cfg = {}
        cfg["C1 blobs_2k_128"] = blobs_leg(dev, local)
        for wl, steps in (("gmm_i8", args.int_steps), ("bits", args.int_steps)):
            wn, wd, wk, _ = WORKLOADS[wl]
            cfg[{"gmm_i8": "C3 gmm_i8_2m_384", "bits": "C4 bits_4m_1024"}[wl]] = exact_int_leg(
                wl, wn, wd, wk, dev, local, rank, world, None, steps, 1, 1, args.int_check_rows,
                {"gmm_i8": 150_000, "bits": 50_000}[wl], bool(args.autotune))
        line["configs"] = cfg
    if world == 1 and args.serve_requests > 0:
        del x, oi, od
        torch.cuda.empty_cache()
        line["serving"] = run_serving(args, dev)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_shard(args, world, rank, local):
    """--shard: ONE graph of the workload on N GPUs.  Every rank holds all rows, builds the complete
    neighbour lists of its query-row shard (evoc_gpu_opts.row_begin/row_end, 128-row blocks,
    evoc.distributed.shard_rows) and the shards are all-gathered over NCCL so every rank ends with
    the whole (n, k) graph.  value = n * k / (slowest rank's shard build + gather): strong scaling."""
    import datetime

    import numpy as np
    import torch

    import evoc
    from evoc import _lib, synthetic
    from evoc.distributed import knn_graph_sharded, shard_rows

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    n, d, k = args.n, args.dim, args.k
    x = synthetic.zipf_f32(n=n, dim=d, seed=7, device=dev)  # the same rows on every rank
    b, e = shard_rows(n, world, rank)
    largest = max(hi - lo for lo, hi in (shard_rows(n, world, r) for r in range(world)))
    si = torch.full((largest, k), -1, dtype=torch.int32, device=dev)
    sd = torch.zeros((largest, k), dtype=torch.float32, device=dev)
    gi = [torch.empty_like(si) for _ in range(world)]
    gd = [torch.empty_like(sd) for _ in range(world)]
    ctx = _lib.context(local)
    ctx.profile(True)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=dev)
    opts = evoc.KnnGraphOptions(n_neighbors=k, form="bf16_rerank", device=local, row_begin=b, row_end=e)

    def step():
        if e > b:
            evoc.knn_graph_device(x.data_ptr(), 0, n, d, k, si.data_ptr(), sd.data_ptr(), opts)
        if pg:
            with torch.cuda.stream(stream):
                pg.all_gather(gi, si)
                pg.all_gather(gd, sd)

    for _ in range(args.warmup):
        step()
    gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    os.makedirs(OUT_DIR, exist_ok=True)
    clocks = ClockSampler(gpu_id, os.path.join(OUT_DIR, f"clocks_shard_rank{rank}.csv"))
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    ev0.record(stream)
    for _ in range(args.steps):
        step()
        launches += ctx.launches()
    ev1.record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    if pg:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    value = n * k / (ms / 1000.0)
    # the gathered graph equals a whole-graph call on every rank (checked on its first rows)
    if pg:
        spans = [shard_rows(n, world, r) for r in range(world)]
        full_i = torch.cat([gi[r][: hi - lo] for r, (lo, hi) in enumerate(spans)])
    else:
        full_i = si
    rows = min(2048, n)
    ri = torch.empty((rows, k), dtype=torch.int32, device=dev)
    rd = torch.empty((rows, k), dtype=torch.float32, device=dev)
    evoc.knn_graph_device(x.data_ptr(), 0, n, d, k, ri.data_ptr(), rd.data_ptr(),
                          evoc.KnnGraphOptions(n_neighbors=k, form="bf16_rerank", device=local, row_begin=0,
                                               row_end=rows))
    torch.cuda.synchronize()
    consistent = bool(torch.equal(full_i[:rows], ri))
    # End to end through the public API (knn_graph_sharded with host arrays).
    xh = x.cpu().numpy()
    so = evoc.KnnGraphOptions(n_neighbors=k, form="bf16_rerank", device=local)
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        if pg:
            knn_graph_sharded(xh, so)
        else:
            evoc.knn_graph(xh, so)
    e2e_s = (time.perf_counter() - t0) / args.e2e_steps
    if pg:
        t = torch.tensor([e2e_s], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "fp16 tensor-core scan + f32 rerank", "data": "synthetic (generated on device)",
        "config": {"workload": WORKLOAD, "n": n, "d": d, "k": k, "form": "bf16_rerank",
                   "parallelism": f"query-row shards of one graph over {world} GPUs + NCCL all-gather",
                   "shard_rows": [list(shard_rows(n, world, r)) for r in range(world)],
                   "l2": "inputs larger than L2"},
        "gathered_graph_matches_single_call": consistent,
        "e2e": {"value": n * k / e2e_s, "unit": UNIT, "h2d_bytes_per_step": n * d * 4,
                "d2h_bytes_per_step": n * k * 8, "ms_per_step": e2e_s * 1e3,
                "timing": "host clock around evoc.distributed.knn_graph_sharded (max over ranks)"},
        "clocks": clk, "gpu_launches": launches,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0



def run_case(args):
    """One small case of a kernel, for timings and ncu captures (`--case NAME [--n N]`): prints
    one JSON line with the stage times (CUDA events on the library stream) of the last of two
    identical calls.  Cases: scan (the 16-bit form of zipf rows with the certificate counts), fp32
    (the plain FP32 form on the first 37,888 query rows), nnd (the NN-descent form), mst (the
    Boruvka MST of a 7-d blob set)."""
    import numpy as np
    import torch

    import evoc
    from evoc import _lib, synthetic

    dev = torch.device("cuda", 0)
    if args.case == "serve":  # the serving leg alone (its own JSON object)
        print(json.dumps({"case": "serve", "lanes": args.serve_lanes, "small_lanes": args.serve_small_lanes,
                          "admission": args.serve_admission,
                          "serving": run_serving(args, dev)}))
        return 0
    ctx = _lib.context(0)
    ctx.profile(True)
    out = {"case": args.case}
    if args.case == "mst":
        n = args.n or 300_000
        rng = np.random.default_rng(11)
        c = rng.normal(size=(200, 7)) * 3
        x = (c[rng.integers(0, 200, n)] + 0.5 * rng.normal(size=(n, 7))).astype(np.float32)
        for _ in range(2):
            e = evoc.parallel_boruvka(x, 5)
        out.update(n=n, dim=7, stages_ms=dict(ctx.stages()), total_weight=float(e[:, 2].sum()))
    else:
        n = args.n or 262_144
        k = args.k or 30
        dim = args.dim or 768
        x = synthetic.zipf_f32(n=n, dim=dim, seed=7, device=dev)
        rows = n if args.case != "fp32" else min(n, 37_888)
        oi = torch.empty((rows, k), dtype=torch.int32, device=dev)
        od = torch.empty((rows, k), dtype=torch.float32, device=dev)
        form = {"scan": "bf16_rerank", "fp32": "fp32", "nnd": "nndescent"}[args.case]
        kw = {"row_begin": 0, "row_end": rows} if args.case == "fp32" else {}
        o = evoc.KnnGraphOptions(n_neighbors=k, form=form, device=0, scan_type=args.scan_type,
                                 oversample=args.oversample, **kw)
        for _ in range(2):
            evoc.knn_graph_device(x.data_ptr(), 0, n, dim, k, oi.data_ptr(), od.data_ptr(), o)
        st = ctx.stages()
        out.update(n=n, dim=dim, k=k, form=form, query_rows=rows)
        if args.case == "nnd":
            out["stages_ms"] = {nm: ms for nm, ms in st if nm != "nnd_iteration"}
            out["iteration_ms"] = [ms for nm, ms in st if nm == "nnd_iteration"]
            out["nndescent"] = ctx.nndescent_stats()
        else:
            out["stages_ms"] = dict(st)
        if args.case == "scan":
            out["certificate"] = ctx.certify_counts()
            out["symmetric_scan"] = ctx.symmetric_stats()
            out["scan_type"] = args.scan_type
            out["oversample"] = args.oversample
        if args.case == "fp32":
            out["tflops_fp32"] = 2.0 * rows * n * dim / (out["stages_ms"]["fp32_scan"] / 1e3) / 1e12
    torch.cuda.synchronize()
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="zipf_f32", choices=sorted(WORKLOADS))
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--dim", type=int, default=None, help="features (f32, i8) or bytes per row (bits)")
    ap.add_argument("--k", type=int, default=None)
    ap.add_argument("--check-rows", type=int, default=128)
    ap.add_argument("--autotune", type=int, default=0,
                    help="tune the scan's kernel variant before timing (default: the library's automatic "
                         "choice, which encodes full-size measurements the short tuning runs do not reproduce)")
    ap.add_argument("--form", default="bf16_rerank", choices=["bf16_rerank", "nndescent"],
                    help="zipf_f32 workload: the exact BF16+rerank form (headline) or GPU NN-descent")
    ap.add_argument("--fuzzy", type=int, default=1, help="time the fuzzy graph of the built graph")
    ap.add_argument("--label-prop", type=int, default=1,
                    help="time label_propagation_init and the node embedding on the fuzzy graph")
    ap.add_argument("--lp-reps", type=int, default=3, help="timed label_propagation_init calls")
    ap.add_argument("--ne-reps", type=int, default=2, help="timed node_embedding calls of each kind (0: none)")
    ap.add_argument("--cpu-lp-rows", type=int, default=100000,
                    help="rows of the graph the oracle's label_propagation_init is timed on")
    ap.add_argument("--mst", type=int, default=1, help="time the Boruvka MST of the node embedding")
    ap.add_argument("--cpu-mst-rows", type=int, default=100_000, help="points of the oracle's MST baseline")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--fp32-rows", type=int, default=75_776)  # 2 full waves of 296 CTAs x 128 rows
    ap.add_argument("--recall-rows", type=int, default=10_000)
    ap.add_argument("--cpu-rows", type=int, default=None, help="CPU baseline sample rows (default per workload)")
    ap.add_argument("--cpu-det-rows", type=int, default=20_000,
                    help="rows of the single-thread deterministic CPU baseline (0: none)")
    ap.add_argument("--configs", type=int, default=1,
                    help="also measure C1 (2k x 128 f32), C3 (2M x 384 i8) and C4 (4M x 1024 bits) at N=1")
    ap.add_argument("--int-steps", type=int, default=3, help="timed steps of the C3 / C4 objects")
    ap.add_argument("--int-check-rows", type=int, default=256, help="sampled exactness rows of C3 / C4")
    ap.add_argument("--shard", action="store_true",
                    help="one graph over all ranks: query-row shards + NCCL all-gather (strong scaling)")
    ap.add_argument("--serve-requests", type=int, default=10_000)
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-lanes", type=int, default=8)
    ap.add_argument("--serve-capacity", type=int, default=2000)
    ap.add_argument("--serve-baseline", type=int, default=250)
    ap.add_argument("--serve-batch", type=int, default=64, help="most small requests per batch (0: none)")
    ap.add_argument("--serve-small-lanes", type=int, default=0,
                    help="serving lanes for requests under 65,536 rows only")
    ap.add_argument("--serve-admission", default="oldest", choices=["oldest", "smallest"],
                    help="serving admission order: oldest request first, or smallest scan first")
    ap.add_argument("--case", default=None, choices=["scan", "fp32", "nnd", "mst", "serve"],
                    help="run one small case of a kernel (timings, ncu captures) instead of the bench")
    ap.add_argument("--scan-type", default="fp16", choices=["fp16", "bf16"], help="operands of --case scan")
    ap.add_argument("--oversample", type=int, default=0,
                    help="--case scan: candidates per row = oversample * k (0: ceil(2.5 k))")
    args = ap.parse_args()
    if args.case:
        return run_case(args)  # --n / --dim / --k: the case's own defaults when not given
    wn, wd, wk, _ = WORKLOADS[args.workload]
    args.n = wn if args.n is None else args.n
    args.dim = wd if args.dim is None else args.dim
    args.k = wk if args.k is None else args.k
    if args.cpu_rows is None:
        args.cpu_rows = {"zipf_f32": 150_000, "gmm_i8": 150_000, "bits": 50_000}[args.workload]
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.workload != "zipf_f32":
        return run_exact_int(args, world, rank, local)
    if args.shard:
        return run_shard(args, world, rank, local)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
