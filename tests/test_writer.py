"""The streaming chunked writer (gpz_writer_*, the reference's
ParallelChunkedWriter, crates/gpzip-codec-cpu/src/parallel.rs:28-229) on the
CPU, with the oracle as its chunk function: chunking, member order, the
flush rule, sticky errors, and a tar stream packed through it as pack_tar
does (crates/gpzip-core/src/archive/pack.rs:144-176).  The device-backed
writer is checked in tests/test_gpu_batch.py."""
import gzip
import io
import tarfile

import numpy as np
import pytest

from gpzip_b200 import native
from gpzip_b200 import workloads as W
from oracle import oracle as O

CHUNK = 256 * 1024


def oracle_fn(b: bytes) -> bytes:
    return O.gzip_chunk(b, 131072)


def expected(data: bytes, chunk: int) -> bytes:
    return b"".join(oracle_fn(data[i:i + chunk]) for i in range(0, len(data), chunk))


@pytest.mark.parametrize("max_in_flight", [1, 3, 16])
def test_members_in_input_order(max_in_flight):
    data = W.logs(5 * CHUNK + 12_345, seed=2).tobytes()
    out = io.BytesIO()
    with native.Writer(out, chunk_fn=oracle_fn, chunk_size=CHUNK, max_in_flight=max_in_flight) as w:
        rng = np.random.default_rng(max_in_flight)
        pos = 0
        while pos < len(data):  # uneven writes, some across chunk boundaries
            n = int(rng.integers(1, 3 * CHUNK // 2))
            w.write(data[pos:pos + n])
            pos += n
    assert out.getvalue() == expected(data, CHUNK)
    assert gzip.decompress(out.getvalue()) == data


def test_sink_view_gives_the_same_stream():
    # the sink may take each run of members as a view of the library's
    # buffer (valid during the call) instead of a bytes copy
    data = W.text(4 * CHUNK + 999, seed=9).tobytes()
    out, kinds = io.BytesIO(), set()

    class Sink:
        def write(self, b):
            kinds.add(type(b).__name__)
            return out.write(b)

    with native.Writer(Sink(), chunk_fn=oracle_fn, chunk_size=CHUNK, max_in_flight=4, sink_view=True) as w:
        w.write(data)
    assert kinds == {"memoryview"}
    assert out.getvalue() == expected(data, CHUNK)


def test_flush_does_not_cut_chunks_and_empty_input_writes_nothing():
    data = W.text(3 * CHUNK - 7, seed=3).tobytes()
    out = io.BytesIO()
    with native.Writer(out, chunk_fn=oracle_fn, chunk_size=CHUNK, max_in_flight=2) as w:
        for i in range(0, len(data), 1000):
            w.write(data[i:i + 1000])
            w.flush()
    assert out.getvalue() == expected(data, CHUNK)
    empty = io.BytesIO()
    with native.Writer(empty, chunk_fn=oracle_fn, chunk_size=CHUNK):
        pass
    assert empty.getvalue() == b""


def test_errors_are_sticky():
    calls = []

    def failing(b):
        calls.append(len(b))
        if len(calls) == 2:
            raise RuntimeError("chunk 2 failed")
        return oracle_fn(b)

    out = io.BytesIO()
    w = native.Writer(out, chunk_fn=failing, chunk_size=CHUNK, max_in_flight=1)
    data = W.binary(6 * CHUNK, seed=4).tobytes()
    with pytest.raises(native.GpzError) as e:
        for i in range(0, len(data), CHUNK):
            w.write(data[i:i + CHUNK])
        w.close()
    assert e.value.status == native.GPZ_E_SINK
    with pytest.raises(native.GpzError):
        w.close()  # still reports it
    assert out.getvalue() == oracle_fn(data[:CHUNK])  # nothing after the failed chunk

    class BadSink:
        def write(self, b):
            raise OSError("disk full")

    w2 = native.Writer(BadSink(), chunk_fn=oracle_fn, chunk_size=CHUNK)
    w2.write(b"x" * 100)
    with pytest.raises(native.GpzError) as e2:
        w2.close()
    assert e2.value.status == native.GPZ_E_SINK


def test_bad_arguments():
    with pytest.raises(ValueError):
        native.Writer(io.BytesIO())
    with pytest.raises(native.GpzError):
        native.Writer(io.BytesIO(), chunk_fn=oracle_fn, chunk_size=0)
    with pytest.raises(native.GpzError):
        native.Writer(io.BytesIO(), chunk_fn=oracle_fn, max_in_flight=0)


def test_tar_stream_packs_and_unpacks(tmp_path):
    files = {f"dir/f{i}.log": W.logs(int(n), seed=10 + i).tobytes() if n else b""
             for i, n in enumerate([0, 1, 50_000, 300_000, 700_001])}
    out = io.BytesIO()
    with native.Writer(out, chunk_fn=oracle_fn, chunk_size=CHUNK, max_in_flight=4) as w:
        with tarfile.open(fileobj=w, mode="w|", format=tarfile.GNU_FORMAT) as tb:
            for name, body in files.items():
                ti = tarfile.TarInfo(name)
                ti.size = len(body)
                ti.mtime = 0
                tb.addfile(ti, io.BytesIO(body))
    raw = gzip.decompress(out.getvalue())
    assert out.getvalue() == expected(raw, CHUNK)
    with tarfile.open(fileobj=io.BytesIO(raw), mode="r:") as tr:
        got = {m.name: tr.extractfile(m).read() for m in tr.getmembers()}
    assert got == files


def test_chunk_calls_run_concurrently():
    """Up to max_in_flight chunk calls run at once (the reference spawns one
    rayon task per chunk, parallel.rs:91-129), and the members still reach
    the sink in input order."""
    import threading
    import time
    lock = threading.Lock()
    live = [0, 0]  # now, peak

    def slow(b):
        with lock:
            live[0] += 1
            live[1] = max(live[1], live[0])
        time.sleep(0.05)  # releases the GIL: calls overlap if the writer lets them
        with lock:
            live[0] -= 1
        return oracle_fn(b)

    data = W.text(8 * CHUNK + 99, seed=7).tobytes()
    out = io.BytesIO()
    with native.Writer(out, chunk_fn=slow, chunk_size=CHUNK, max_in_flight=4) as w:
        w.write(data)
    assert out.getvalue() == expected(data, CHUNK)
    assert 1 < live[1] <= 4


def test_failed_chunk_ends_the_stream_in_input_order():
    """With calls in flight together, the chunks before the failed one are
    written and nothing from it on, whatever order the calls finish in."""
    import time
    data = W.logs(8 * CHUNK, seed=8).tobytes()
    bad = data[3 * CHUNK:4 * CHUNK]

    def fn(b):
        if b == bad:
            raise RuntimeError("chunk 3 failed")
        if b == data[:CHUNK]:
            time.sleep(0.2)  # the first chunk finishes last
        return oracle_fn(b)

    out = io.BytesIO()
    w = native.Writer(out, chunk_fn=fn, chunk_size=CHUNK, max_in_flight=8)
    with pytest.raises(native.GpzError) as e:
        try:
            w.write(data)  # may already report the failure
        finally:
            w.close()  # waits for the chunks in flight, then reports it
    assert e.value.status == native.GPZ_E_SINK
    assert out.getvalue() == expected(data[:3 * CHUNK], CHUNK)
