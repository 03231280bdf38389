"""Multi-GPU layout of one graph (query rows sharded across ranks), on CPU.

Two gloo ranks run the sharding and gather logic of evoc.distributed with the
oracle's exact selection standing in for the per-GPU shard (the GPU shard is
evoc_gpu_knn_graph with row_begin/row_end, tested on the GPU elsewhere); the
gathered graph must equal the oracle's whole graph.  A rank that fails before
the gather must make the other rank's collective end with an error within the
process group's timeout.
"""
import datetime
import os
import socket

import numpy as np
import pytest

from evoc.distributed import shard_rows


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n,world", [(1, 2), (128, 2), (1000, 2), (1000, 3), (4097, 4), (300, 8)])
def test_shards_cover_rows_once_and_balance(n, world):
    spans = [shard_rows(n, world, r) for r in range(world)]
    covered = np.zeros(n, int)
    for b, e in spans:
        assert 0 <= b <= e <= n and (b % 128 == 0 or b == n)
        covered[b:e] += 1
    assert np.all(covered == 1)
    sizes = [e - b for b, e in spans]
    assert max(sizes) - min(sizes) <= 128


def _data(n, d, seed):
    r = np.random.default_rng(seed)
    x = r.normal(size=(6, d))[r.integers(0, 6, n)] + 0.3 * r.normal(size=(n, d))
    return (x / np.linalg.norm(x, axis=1, keepdims=True)).astype(np.float32)


def _oracle_shard(data, options, begin, end):
    from oracle import oracle as O

    # the shard is built on the rank's own GPU: LOCAL_RANK here (no CUDA in these processes)
    assert options.device == int(os.environ["LOCAL_RANK"]), (options.device, os.environ["LOCAL_RANK"])
    x = data.array
    k = max(1, min(options.n_neighbors, len(x) - 1))
    ind, raw = O.exact_knn(x, k, begin, end)
    return ind, O.transform(O.DT_F32, raw)


def _rank_main(rank, world, port, n, d, k, out_dir, fail_rank):
    import torch.distributed as dist

    import evoc
    from evoc.distributed import knn_graph_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["LOCAL_RANK"] = str(rank)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=6))
    try:
        if rank == fail_rank:
            raise RuntimeError("rank failed before the gather")
        x = _data(n, d, 5)
        rng = np.random.RandomState(3)
        ind, dst = knn_graph_sharded(x, evoc.KnnGraphOptions(n_neighbors=k), rng, compute=_oracle_shard)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), ind=ind, dst=dst, rng=rng.get_state()[1])
    except RuntimeError as e:
        if rank == fail_rank:
            raise
        with open(os.path.join(out_dir, f"rank{rank}.err"), "w") as f:
            f.write(repr(e))
    finally:
        if rank != fail_rank:
            try:
                dist.destroy_process_group()
            except Exception:
                pass


@pytest.mark.parametrize("n,world", [(700, 2), (300, 3)])
def test_sharded_graph_equals_whole_graph(tmp_path, n, world):
    import torch.multiprocessing as mp

    from oracle import oracle as O

    O.build()
    d, k = 24, 10
    mp.spawn(_rank_main, args=(world, _free_port(), n, d, k, str(tmp_path), -1), nprocs=world, join=True)
    x = _data(n, d, 5)
    ei, er = O.exact_knn(x, k)
    ed = O.transform(O.DT_F32, er)
    rng = np.random.RandomState(3)
    import evoc
    from evoc.knn import _advance_rng

    _advance_rng(rng, evoc.EmbeddingData.wrap(x), evoc.KnnGraphOptions(n_neighbors=k))
    for r in range(world):
        z = np.load(tmp_path / f"rank{r}.npz")
        assert np.array_equal(z["ind"], ei)
        assert np.array_equal(z["dst"].view(np.uint32), ed.view(np.uint32))
        assert np.array_equal(z["rng"], rng.get_state()[1])  # the RNG contract holds on every rank


def test_failed_rank_is_detected_by_the_other(tmp_path):
    import multiprocessing as mp
    import time

    from oracle import oracle as O

    O.build()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, 400, 16, 5, str(tmp_path), 1)) for r in range(2)]
    t0 = time.time()
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=60)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank still waits after the other failed"
    assert procs[1].exitcode != 0
    # rank 0's gather ended with an error (peer gone or timeout), well within the bound
    assert (tmp_path / "rank0.err").exists() and not (tmp_path / "rank0.npz").exists()
    assert time.time() - t0 < 60


def _gpu_rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    import evoc
    from evoc.distributed import knn_graph_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        x = _data(3000, 96, 8)
        for form in ("bf16_rerank", "fp32"):
            # one GPU here, so both ranks name device 0 explicitly
            ind, dst = knn_graph_sharded(x, evoc.KnnGraphOptions(n_neighbors=15, form=form, device=0))
            np.savez(os.path.join(out_dir, f"gpu_{form}_rank{rank}.npz"), ind=ind, dst=dst)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_gpu_graph_equals_single_gpu_graph(tmp_path):
    """Two ranks, each computing its query-row shard with the GPU library (both on device 0: their
    kernels are independent and the gather is gloo on the host), assemble the single-call graph."""
    import torch.multiprocessing as mp

    import evoc

    mp.spawn(_gpu_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    x = _data(3000, 96, 8)
    for form in ("bf16_rerank", "fp32"):
        wi, wd = evoc.knn_graph(x, evoc.KnnGraphOptions(n_neighbors=15, form=form))
        for r in range(2):
            z = np.load(tmp_path / f"gpu_{form}_rank{r}.npz")
            assert np.array_equal(z["ind"], wi) and np.array_equal(z["dst"].view(np.uint32), wd.view(np.uint32))
