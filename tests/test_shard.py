"""Sharding a job over ranks: byte-balanced contiguous partition, in-order
reassembly, and a gloo world-size-2 run (CPU) in which each rank compresses
its range with the oracle and rank 0 gathers the streams."""
import os
import queue
import socket
import gzip

import numpy as np
import pytest
import torch.multiprocessing as mp

from gpzip_b200 import shard
from gpzip_b200 import workloads as W


def test_partition_is_contiguous_and_complete():
    rng = np.random.default_rng(0)
    for world in (1, 2, 3, 4, 8):
        for k in (0, 1, 3, 17, 100):
            sizes = [int(x) for x in rng.integers(0, 1 << 20, size=k)]
            parts = shard.partition(sizes, world)
            assert len(parts) == world
            assert parts[0][0] == 0 and parts[-1][1] == k
            for (a, b), (c, d) in zip(parts, parts[1:]):
                assert a <= b == c <= d


def test_partition_balances_bytes():
    rng = np.random.default_rng(1)
    sizes = [int(x) for x in rng.integers(1, 1 << 16, size=2000)]
    total = sum(sizes)
    for world in (2, 4, 8):
        for lo, hi in shard.partition(sizes, world):
            share = sum(sizes[lo:hi])
            assert abs(share - total / world) <= max(sizes)


def test_partition_rejects_bad_world():
    with pytest.raises(ValueError):
        shard.partition([1, 2], 0)


def test_assemble_detects_missing_and_duplicates():
    assert shard.assemble([(0, [b"a"]), (1, [b"b", b"c"])], 3) == [b"a", b"b", b"c"]
    with pytest.raises(ValueError):
        shard.assemble([(0, [b"a"])], 2)
    with pytest.raises(ValueError):
        shard.assemble([(0, [b"a", b"b"]), (1, [b"x"])], 2)


def _items():
    kinds = ["text", "logs", "binary"]
    sizes = [70_000, 5, 300_000, 0, 131_072, 200_001, 12_345]
    return [W.GENERATORS[kinds[i % 3]](n, seed=40 + i).tobytes() if n else b"" for i, n in enumerate(sizes)]


def _oracle_compress(items):
    from oracle import oracle as O
    return [O.gzip_chunk(x, 131072) for x in items]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        out = shard.compress_distributed(_items(), _oracle_compress)
        if rank == 0:
            q.put([bytes(x) for x in out])
        else:
            assert out is None
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_gloo_matches_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = None
    try:
        for _ in range(240):
            try:
                got = q.get(timeout=1)
                break
            except queue.Empty:
                if any(p.exitcode not in (None, 0) for p in procs):
                    break
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.exitcode is None:
                p.kill()
    assert got is not None, [p.exitcode for p in procs]
    assert all(p.exitcode == 0 for p in procs)
    items = _items()
    want = _oracle_compress(items)
    assert got == want
    for it, g in zip(items, got):
        assert gzip.decompress(g) == it  # every member, concatenated
