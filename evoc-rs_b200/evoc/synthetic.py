"""Seeded synthetic embedding sets with the shapes and value distributions of
the benchmark workloads.  No public dataset is involved: each generator
documents the distribution it draws.

  blobs_2k_128     2,000 x 128 f32: 10 centres ~ N(0,1), 200 points each,
                   noise sigma 0.3, rows L2-normalised, seed 42
  zipf_1m_768      1,000,000 x 768 f32: 200 clusters, Zipf(1.1) sizes
                   (largest-remainder rounding), centres ~ N(0,1), per-cluster
                   per-dimension sigma ~ U(0.1, 0.5), rows L2-normalised, seed 7
  gmm_i8_2m_384    2,000,000 x 384 i8: round(127 x) of L2-normalised
                   100-cluster equal-weight mixture (sigma 0.25), clipped to
                   [-127, 127], seed 11
  bits_4m_1024     4,000,000 x 128 u8 (1,024 bits): 500 Bernoulli(0.1)
                   prototypes, each row copies a uniform prototype and flips
                   each bit with p = 0.05, packed big-endian, seed 13
  serving_10k      10,000 requests, Poisson arrivals at 200 req/s; per
                   request n log-uniform in [500, 200,000], d uniform from
                   {128, 384, 768}, f32 (80%) or i8 (20%, round(127 x));
                   each request's rows are a window of one of a few
                   5-50-cluster Gaussian mixtures (sigma 0.3, L2-normalised),
                   chosen and placed by the request id (seed 17)
Rows are emitted in a seeded random order (not grouped by cluster).
Large sets are generated on a CUDA device with torch when one is given.
"""
from __future__ import annotations

import numpy as np


def _zipf_sizes(n: int, clusters: int, s: float) -> np.ndarray:
    w = np.arange(1, clusters + 1, dtype=np.float64) ** (-s)
    exact = n * w / w.sum()
    base = np.floor(exact).astype(np.int64)
    rem = n - int(base.sum())
    order = np.argsort(-(exact - base), kind="stable")
    base[order[:rem]] += 1
    return base


def blobs(n_per: int = 200, centres: int = 10, dim: int = 128, noise: float = 0.3, seed: int = 42) -> np.ndarray:
    rng = np.random.RandomState(seed)
    c = rng.standard_normal((centres, dim))
    lab = np.repeat(np.arange(centres), n_per)
    x = c[lab] + noise * rng.standard_normal((centres * n_per, dim))
    x = x[rng.permutation(len(x))]
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    return x.astype(np.float32)


def blobs_2k_128() -> np.ndarray:
    return blobs()


def zipf_f32(n: int = 1_000_000, dim: int = 768, clusters: int = 200, s: float = 1.1, seed: int = 7,
             device=None) -> np.ndarray:
    """Zipf-sized anisotropic Gaussian clusters (f32, L2-normalised)."""
    sizes = _zipf_sizes(n, clusters, s)
    if device is None:
        rng = np.random.default_rng(seed)
        centres = rng.standard_normal((clusters, dim)).astype(np.float32)
        sig = rng.uniform(0.1, 0.5, (clusters, dim)).astype(np.float32)
        lab = np.repeat(np.arange(clusters), sizes)
        lab = lab[rng.permutation(n)]
        x = np.empty((n, dim), np.float32)
        step = 65536
        for s0 in range(0, n, step):
            l = lab[s0:s0 + step]
            z = rng.standard_normal((len(l), dim), dtype=np.float32)
            v = centres[l] + sig[l] * z
            v /= np.linalg.norm(v, axis=1, keepdims=True)
            x[s0:s0 + step] = v
        return x
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    centres = torch.randn(clusters, dim, generator=g, device=device)
    sig = torch.rand(clusters, dim, generator=g, device=device) * 0.4 + 0.1
    lab = torch.repeat_interleave(torch.arange(clusters, device=device), torch.as_tensor(sizes, device=device))
    lab = lab[torch.randperm(n, generator=g, device=device)]
    x = torch.empty(n, dim, device=device)
    step = 131072
    for s0 in range(0, n, step):
        l = lab[s0:s0 + step]
        v = centres[l] + sig[l] * torch.randn(len(l), dim, generator=g, device=device)
        x[s0:s0 + step] = v / v.norm(dim=1, keepdim=True)
    return x


def gmm_i8(n: int = 2_000_000, dim: int = 384, clusters: int = 100, sigma: float = 0.25, seed: int = 11,
           device=None):
    if device is None:
        rng = np.random.default_rng(seed)
        centres = rng.standard_normal((clusters, dim)).astype(np.float32)
        lab = rng.integers(0, clusters, n)
        out = np.empty((n, dim), np.int8)
        step = 65536
        for s0 in range(0, n, step):
            l = lab[s0:s0 + step]
            v = centres[l] + sigma * rng.standard_normal((len(l), dim), dtype=np.float32)
            v /= np.linalg.norm(v, axis=1, keepdims=True)
            out[s0:s0 + step] = np.clip(np.round(127.0 * v), -127, 127).astype(np.int8)
        return out
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    centres = torch.randn(clusters, dim, generator=g, device=device)
    lab = torch.randint(0, clusters, (n,), generator=g, device=device)
    out = torch.empty(n, dim, dtype=torch.int8, device=device)
    step = 131072
    for s0 in range(0, n, step):
        l = lab[s0:s0 + step]
        v = centres[l] + sigma * torch.randn(len(l), dim, generator=g, device=device)
        v = v / v.norm(dim=1, keepdim=True)
        out[s0:s0 + step] = torch.clamp(torch.round(127.0 * v), -127, 127).to(torch.int8)
    return out


def bits_u8(n: int = 4_000_000, nbits: int = 1024, protos: int = 500, p_on: float = 0.1, p_flip: float = 0.05,
            seed: int = 13, device=None):
    nbytes = nbits // 8
    if device is None:
        rng = np.random.default_rng(seed)
        P = rng.random((protos, nbits)) < p_on
        lab = rng.integers(0, protos, n)
        out = np.empty((n, nbytes), np.uint8)
        step = 65536
        for s0 in range(0, n, step):
            l = lab[s0:s0 + step]
            rows = P[l] ^ (rng.random((len(l), nbits)) < p_flip)
            out[s0:s0 + step] = np.packbits(rows, axis=1)
        return out
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    P = torch.rand(protos, nbits, generator=g, device=device) < p_on
    lab = torch.randint(0, protos, (n,), generator=g, device=device)
    weights = (2 ** torch.arange(7, -1, -1, device=device)).to(torch.int32)
    out = torch.empty(n, nbytes, dtype=torch.uint8, device=device)
    step = 131072
    for s0 in range(0, n, step):
        l = lab[s0:s0 + step]
        rows = P[l] ^ (torch.rand(len(l), nbits, generator=g, device=device) < p_flip)
        packed = (rows.view(len(l), nbytes, 8).to(torch.int32) * weights).sum(-1)
        out[s0:s0 + step] = packed.to(torch.uint8)
    return out


def serving_schedule(count: int = 10_000, rate: float = 200.0, n_lo: int = 500, n_hi: int = 200_000,
                     dims=(128, 384, 768), p_i8: float = 0.2, seed: int = 17) -> dict:
    """Arrival times (s, first at 0), n, d and dtype of each request of the serving workload."""
    rng = np.random.RandomState(seed)
    gaps = rng.exponential(1.0 / rate, count)
    arrival = np.cumsum(gaps) - gaps[0]
    n = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), count)).astype(np.int64)
    dim = np.asarray(dims, np.int64)[rng.randint(0, len(dims), count)]
    i8 = rng.random_sample(count) < p_i8
    return {"arrival": arrival, "n": n, "dim": dim, "i8": i8}


class ServingPools:
    """Row pools the serving requests are cut from: for each d, `mixtures`
    Gaussian mixtures of 5..50 equal-weight clusters (centres N(0,1), sigma
    0.3, rows L2-normalised) of `rows` rows, as f32 and as i8 (round(127 x),
    clipped), in pinned host memory.  Request i reads mixture i % mixtures at a
    seeded offset, so requests differ in data as well as in shape."""

    def __init__(self, device, rows: int = 200_000, dims=(128, 384, 768), mixtures: int = 4, seed: int = 17):
        import torch

        self.rows, self.mixtures = rows, mixtures
        self.pool = {}
        g = torch.Generator(device=device)
        g.manual_seed(seed)
        clusters = np.linspace(5, 50, mixtures).round().astype(int)
        for d in dims:
            for m in range(mixtures):
                c = int(clusters[m])
                centres = torch.randn(c, d, generator=g, device=device)
                lab = torch.randint(0, c, (rows,), generator=g, device=device)
                v = centres[lab] + 0.3 * torch.randn(rows, d, generator=g, device=device)
                v = v / v.norm(dim=1, keepdim=True)
                f = torch.empty((rows, d), dtype=torch.float32, pin_memory=True)
                f.copy_(v)
                q = torch.empty((rows, d), dtype=torch.int8, pin_memory=True)
                q.copy_(torch.clamp(torch.round(127.0 * v), -127, 127).to(torch.int8))
                self.pool[(int(d), m, False)] = f.numpy()
                self.pool[(int(d), m, True)] = q.numpy()
                del v, centres, lab

    def rows_for(self, request_id: int, n: int, dim: int, i8: bool) -> np.ndarray:
        m = request_id % self.mixtures
        off = np.random.RandomState(request_id).randint(0, self.rows - n + 1)
        return self.pool[(int(dim), m, bool(i8))][off:off + n]
