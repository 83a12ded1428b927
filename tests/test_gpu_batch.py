"""Batched, plain, device-resident and serving paths against each other and the oracle (GPU).

All comparisons are byte-exact: the path is integer work end to end.
"""
import ctypes
import threading
import zlib

import numpy as np
import pytest

from gpzip_b200 import native
from gpzip_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def uneven_items(count=24, seed=5):
    rng = np.random.default_rng(seed)
    items = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1), np.log(3 << 20))))
        kind = ["text", "logs", "binary"][i % 3]
        items.append(W.GENERATORS[kind](n, seed=100 + i).tobytes())
    items[3] = b""
    items[7] = b"x"
    return items


def test_batch_plain_oracle_uneven(ctx):
    items = uneven_items()
    got = ctx.compress_batch(items)
    plain = ctx.compress_batch_plain(items)
    for it, g, p in zip(items, got, plain):
        assert g == p
        assert g == O.gzip_chunk(it, 131072, threads=8)


def test_page_locked_inputs_upload_directly(ctx):
    # inputs in page-locked memory skip the staging copy; the bytes are the
    # same as from pageable inputs, including ragged and empty items and
    # items that start at odd offsets inside the pinned buffer
    import torch
    items = uneven_items(count=12, seed=8)
    total = sum(len(x) for x in items) + 3 * len(items)
    pinned = torch.empty(total, dtype=torch.uint8, pin_memory=True).numpy()
    views, off = [], 1
    for it in items:
        pinned[off:off + len(it)] = np.frombuffer(it, dtype=np.uint8) if it else []
        views.append(pinned[off:off + len(it)])
        off += len(it) + 3
    got = ctx.compress_batch(views)
    want = ctx.compress_batch(items)
    assert got == want
    for it, g in zip(items, got):
        assert g == O.gzip_chunk(it, 131072, threads=8)


def test_graph_reuse_across_batch_sizes(ctx):
    # same size bucket, different member/tile counts: the captured graph reads
    # the batch dimensions from device memory
    a = [W.text(300_000, seed=1).tobytes(), W.logs(200_000, seed=2).tobytes()]
    b = [W.binary(150_001, seed=3).tobytes()]
    c = [W.text(40_000, seed=4).tobytes()] * 5
    for items in (a, b, c, a):
        for it, g in zip(items, ctx.compress_batch(items)):
            assert g == O.gzip_chunk(it, 131072)


def test_every_launch_shape_gives_the_same_bytes(ctx):
    # logs, and binary data whose tiles hold more distinct hashes than one
    # join pass takes
    data = W.logs(700_000, seed=9).tobytes() + W.binary(300_000, seed=19).tobytes()
    want = O.gzip_chunk(data, 131072)
    keep = ctx.get_shape()
    for lt in (1024, 768, 512):
        for wt in (1024, 512, 256):
            for et in (512, 256):
                ctx.set_shape(native.Shape(lt, 0, wt, 0, et, 0))
                assert ctx.compress_chunk(data) == want, (lt, wt, et)
    ctx.set_shape(keep)


def test_device_api_matches_host_api(ctx):
    import torch
    items = [W.text(500_000, seed=11).tobytes(), W.binary(123_457, seed=12).tobytes(), b"", b"ab"]
    offs, lens, pos = [], [], 0
    for it in items:
        offs.append(pos)
        lens.append(len(it))
        pos += (max(len(it), 1) + 15) // 16 * 16
    packed = np.zeros(pos + 64, dtype=np.uint8)
    for it, o in zip(items, offs):
        packed[o:o + len(it)] = np.frombuffer(it, dtype=np.uint8)
    d_in = torch.from_numpy(packed).cuda()
    cap = sum(ctx.bound(len(it)) for it in items) + 1024
    d_out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    oo = ctx.compress_device(d_in.data_ptr(), offs, lens, d_out.data_ptr(), cap)
    host = d_out[:oo[-1]].cpu().numpy().copy()
    ctx.frame_host(host)
    want = ctx.compress_batch(items)
    for i, w in enumerate(want):
        assert host[oo[i]:oo[i + 1]].tobytes() == w


def test_short_output_buffer_is_reported(ctx):
    L = native.load()
    data = np.frombuffer(W.text(10_000, seed=3).tobytes(), dtype=np.uint8)
    out = np.zeros(16, dtype=np.uint8)
    n = ctypes.c_size_t()
    rc = L.gpz_compress_chunk(ctx._h, data.ctypes.data, data.size, 5, out.ctypes.data, out.size, ctypes.byref(n))
    assert rc == 6 and n.value > 16  # GPZ_E_SPACE, with the needed size
    assert ctx.compress_chunk(data) == O.gzip_chunk(data.tobytes(), 131072)  # context still usable


def test_concurrent_chunk_calls_are_batched():
    # ParallelChunkedWriter's workers call the ChunkFn concurrently: the
    # calls are combined into shared passes, and every caller gets exactly
    # the bytes of a lone call, also with one short output buffer in the mix
    items = [W.GENERATORS[["text", "logs", "binary"][i % 3]](int(n), seed=500 + i).tobytes()
             for i, n in enumerate(np.random.default_rng(6).integers(1, 3 << 20, size=48))]
    items[5] = b""
    with native.Context() as c:
        want = [bytes(x) for x in c.compress_batch(items)]
        c.host_times(reset=True)
        got = [None] * len(items)
        errs = []
        start = threading.Barrier(16)
        L = c.L

        def worker(k):
            start.wait()
            for i in range(k, len(items), 16):
                if i == 7:
                    a = np.frombuffer(items[i], dtype=np.uint8)
                    small = np.zeros(8, dtype=np.uint8)
                    n = ctypes.c_size_t()
                    rc = L.gpz_compress_chunk(c._h, a.ctypes.data, a.size, 5, small.ctypes.data, 8, ctypes.byref(n))
                    if rc != 6 or n.value != len(want[i]):
                        errs.append((i, rc, n.value))
                try:
                    got[i] = c.compress_chunk(items[i])
                except Exception as e:  # noqa: BLE001
                    errs.append((i, e))

        th = [threading.Thread(target=worker, args=(k,)) for k in range(16)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        passes = c.host_times()["passes"]
    assert not errs, errs
    assert got == want
    assert passes < len(items) + 1  # at least two calls shared a pass


def test_whole_chunk_member_mode():
    data = W.logs(3 << 20, seed=21).tobytes()
    with native.Context(member_bytes=2 << 20) as c2:
        got = c2.compress_chunk(data)
    assert got == O.gzip_chunk(data, 2 << 20)
    assert zlib.decompress(got[:len(got)], 31) is not None


def test_serving_alone_equals_mix(ctx):
    rng = np.random.default_rng(4)
    reqs = []
    for i in range(40):
        n = int(np.exp(rng.uniform(np.log(4096), np.log(6 << 20))))
        reqs.append(W.GENERATORS[["text", "logs", "binary"][i % 3]](n, seed=300 + i).tobytes())
    tickets = [None] * len(reqs)

    def submitter(lo, hi):
        for i in range(lo, hi):
            tickets[i] = ctx.submit(reqs[i])

    ths = [threading.Thread(target=submitter, args=(k * 10, (k + 1) * 10)) for k in range(4)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    mixed = [ctx.poll(t, ctx.bound(len(r)), wait_ms=60_000) for t, r in zip(tickets, reqs)]
    for r, m in zip(reqs, mixed):
        assert m is not None
        assert m == ctx.compress_chunk(r)  # alone, same bytes
    st = ctx.serve_stats()
    assert st["completed"] >= len(reqs) and st["batches"] >= 1


def test_serving_pending_space_and_admission():
    with native.Context(pool_bytes=64 << 20) as c:
        data = W.text(3 << 20, seed=8).tobytes()
        t = c.submit(data)
        r = c.poll(t, 16, wait_ms=60_000)  # too small at first: the result is kept, then fetched whole
        assert r == O.gzip_chunk(data, 131072)
    # a fresh context with a tiny cap rejects what it cannot queue
    with native.Context(pool_bytes=1 << 20) as c:
        with pytest.raises(native.GpzError) as e:
            c.submit(b"z" * (2 << 20))
        assert e.value.status == native.GPZ_E_ADMISSION
        st = c.serve_stats()
        assert st["rejected"] == 1


def test_fixed_block_mode():
    # GPZ_FLAG_FIXED_BLOCKS: every member is the fixed-Huffman block the
    # reference falls back to (deflate.rs:752-799), byte for byte
    import gzip
    items = [W.text(300_000, seed=81).tobytes(), W.binary(131_072, seed=82).tobytes(), b"", b"q",
             W.logs(70_001, seed=83).tobytes()]
    with native.Context(flags=native.GPZ_FLAG_FIXED_BLOCKS) as c:
        for it in items:
            got = c.compress_chunk(it)
            assert got == O.gzip_chunk_fixed(it, 131072)
            assert gzip.decompress(got) == it
        for it, g in zip(items, c.compress_batch(items)):
            assert g == O.gzip_chunk_fixed(it, 131072)


def test_device_writer_matches_the_oracle(ctx):
    # the streaming writer over the device path: 2 MiB chunks, 16 in flight,
    # members in order; bytes equal the oracle's per-chunk gzip streams
    import io
    data = W.logs((9 << 20) + 4321, seed=30).tobytes()
    out = io.BytesIO()
    with native.Writer(out, ctx=ctx, chunk_size=2 << 20, max_in_flight=3) as w:
        for i in range(0, len(data), 700_000):
            w.write(data[i:i + 700_000])
    want = b"".join(O.gzip_chunk(data[i:i + (2 << 20)], 131072, threads=8) for i in range(0, len(data), 2 << 20))
    assert out.getvalue() == want
    assert bytes(ctx.inflate(out.getvalue())) == data


def test_bounded_wait_times_out_and_the_context_recovers():
    """Every host wait for the device is bounded by the context's wait limit.
    With a limit of 0 a call whose device work is still running gives up with
    GPZ_E_TIMEOUT; the next call waits for that work before it reuses the
    buffers, and its bytes are the same as ever."""
    data = W.logs(96 << 20, seed=12)
    items = [np.ascontiguousarray(data[i:i + (2 << 20)]) for i in range(0, data.size, 2 << 20)]
    with native.Context() as c:
        want = c.compress_batch(items)
        c.set_wait_ms(0)
        with pytest.raises(native.GpzError) as e:
            c.compress_batch(items)
        assert e.value.status == native.GPZ_E_TIMEOUT
        c.set_wait_ms(60_000)
        assert c.compress_batch(items) == want
        assert c.compress_chunk(items[0]) == want[0]


def test_hybrid_writer_on_the_device(ctx):
    """The `--backend auto` composition on the device: the hybrid chunk
    function in a writer with CPU workers + GPU permits in flight.  Every
    chunk the GPU took equals the oracle's bytes, every CPU chunk is zlib's
    level-5 member, the stream is in input order and gzip -t accepts it."""
    import gzip
    import io
    import subprocess
    import tempfile
    data = W.logs(40 << 20, seed=31).tobytes()
    chunk = 2 << 20
    with native.Hybrid(ctx=ctx, gpu_permits=8, warmup_chunks=4) as h:
        out = io.BytesIO()
        with native.Writer(out, hybrid=h, chunk_size=chunk, max_in_flight=8 + 8) as w:
            for i in range(0, len(data), 1 << 20):
                w.write(data[i:i + (1 << 20)])
        cpu, gpu = h.stats()
    got = out.getvalue()
    assert cpu >= 4 and gpu >= 1 and cpu + gpu == len(data) // chunk
    pos, on_gpu = 0, 0
    for i in range(0, len(data), chunk):
        c = data[i:i + chunk]
        a = O.gzip_chunk(c, 131072, threads=8)
        if got.startswith(a, pos):
            pos += len(a)
            on_gpu += 1
        else:
            b = native.cpu_gzip_chunk(c, 5)
            assert got.startswith(b, pos)
            pos += len(b)
    assert pos == len(got) and on_gpu == gpu
    assert gzip.decompress(got) == data
    with tempfile.NamedTemporaryFile(suffix=".gz") as f:
        f.write(got)
        f.flush()
        subprocess.run(["gzip", "-t", f.name], check=True)
