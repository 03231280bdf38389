"""One kNN graph on several GPUs: query rows sharded across ranks.

Every rank holds all n rows and computes the complete neighbour lists of its
contiguous slice of query rows with the library's row-slice option
(`row_begin` / `row_end` of evoc_gpu_opts); the slices are then gathered so
every rank ends with the whole (n, k) graph.  The only exchange is that final
gather -- the search itself has no collective.  This is the multi-GPU layout
of the exact forms (the reference's CPU path has no counterpart; its rayon
threads share one address space).

One process per GPU, `torch.distributed` for the gather (NCCL on GPUs; gloo
runs the same code on CPU, which the tests use).
"""
from __future__ import annotations

import os
from dataclasses import replace
from typing import Callable, Optional

import numpy as np

from .knn import EmbeddingData, EmptyData, InvalidNeighbors, KnnGraphOptions, _advance_rng

BLOCK = 128  # query rows per scan block: shards start on block boundaries


def shard_rows(n: int, world: int, rank: int) -> tuple[int, int]:
    """[begin, end) of this rank's query rows: contiguous, balanced in 128-row blocks; empty when
    there are fewer blocks than ranks."""
    blocks = (n + BLOCK - 1) // BLOCK
    lo = blocks * rank // world
    hi = blocks * (rank + 1) // world
    return min(n, lo * BLOCK), min(n, hi * BLOCK)


def rank_device(options: KnnGraphOptions) -> int:
    """The GPU a rank computes on: options.device when set, else the device torch made current
    (torchrun ranks call torch.cuda.set_device(LOCAL_RANK)), else LOCAL_RANK."""
    if options.device is not None:
        return int(options.device)
    import torch

    if torch.cuda.is_available() and torch.cuda.is_initialized():
        return int(torch.cuda.current_device())
    return int(os.environ.get("LOCAL_RANK", "0"))


def _local_gpu(data: EmbeddingData, options: KnnGraphOptions, begin: int, end: int):
    from .knn import knn_graph

    return knn_graph(data, replace(options, row_begin=begin, row_end=end))


def knn_graph_sharded(data, options: KnnGraphOptions, rng=None, *, group=None,
                      compute: Optional[Callable] = None):
    """The whole (indices, distances) graph on every rank, each rank computing its query-row shard.
    `compute(data, options, begin, end)` builds one shard (default: the GPU library) on the rank's
    device (options.device, resolved by rank_device); it must return int32 (end-begin, k) indices
    and f32 distances.  The caller's RandomState is advanced by knn_graph's draws, as on one GPU."""
    import torch
    import torch.distributed as dist

    data = EmbeddingData.wrap(data)
    if options.n_neighbors <= 0:
        raise InvalidNeighbors()
    n = data.nrows()
    if n == 0:
        raise EmptyData()
    if rng is not None:
        _advance_rng(rng, data, options)
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    k = max(1, min(options.n_neighbors, n - 1))
    begin, end = shard_rows(n, world, rank)
    options = replace(options, device=rank_device(options))
    if end > begin:
        ind, dst = (compute or _local_gpu)(data, options, begin, end)
    else:
        ind, dst = np.empty((0, k), np.int32), np.empty((0, k), np.float32)
    # Gather the slices: pad to the largest shard (shards differ by at most one block).
    largest = max(e - b for b, e in (shard_rows(n, world, r) for r in range(world)))
    backend = dist.get_backend(group)
    dev = torch.device("cuda", options.device) if backend == "nccl" else torch.device("cpu")
    pi = torch.full((largest, k), -1, dtype=torch.int32, device=dev)
    pd = torch.zeros((largest, k), dtype=torch.float32, device=dev)
    pi[: end - begin] = torch.from_numpy(np.ascontiguousarray(ind))
    pd[: end - begin] = torch.from_numpy(np.ascontiguousarray(dst))
    gi = [torch.empty_like(pi) for _ in range(world)]
    gd = [torch.empty_like(pd) for _ in range(world)]
    dist.all_gather(gi, pi, group=group)
    dist.all_gather(gd, pd, group=group)
    out_i = np.empty((n, k), np.int32)
    out_d = np.empty((n, k), np.float32)
    for r in range(world):
        b, e = shard_rows(n, world, r)
        out_i[b:e] = gi[r][: e - b].cpu().numpy()
        out_d[b:e] = gd[r][: e - b].cpu().numpy()
    return out_i, out_d
