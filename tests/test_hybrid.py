"""The hybrid CPU + GPU chunk function (gpz_hybrid_*, the reference's
HybridGzipCompressor, crates/gpzip-cli/src/hybrid.rs:103-147) on the CPU,
with stand-in functions for the device: warm-up chunks on the CPU, permit
accounting (never more GPU calls at once than permits), GPU errors returned
without a CPU retry, and the writer composed as the reference composes it.
The device-backed hybrid is checked in tests/test_gpu_batch.py."""
import gzip
import io
import threading
import time
import zlib

import pytest

from gpzip_b200 import native
from gpzip_b200 import workloads as W
from oracle import oracle as O

CHUNK = 256 * 1024


def zlib_member(b: bytes, level: int = 5) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, 31)
    return c.compress(b) + c.flush()


def test_cpu_chunk_is_a_zlib_gzip_member():
    for data in (b"", b"x", W.text(300_000, seed=1).tobytes(), W.binary(70_000, seed=2).tobytes()):
        for level in (1, 5, 9):
            g = native.cpu_gzip_chunk(data, level)
            assert g == zlib_member(data, level)
            assert gzip.decompress(g) == data


class FakeGpu:
    """Stands in for the device: the oracle's bytes, slowly, counting how
    many calls overlap."""

    def __init__(self, fail_on=None, delay=0.02):
        self.lock = threading.Lock()
        self.live = 0
        self.peak = 0
        self.calls = 0
        self.fail_on = fail_on
        self.delay = delay

    def __call__(self, b):
        with self.lock:
            self.live += 1
            self.calls += 1
            self.peak = max(self.peak, self.live)
        try:
            time.sleep(self.delay)
            if self.fail_on is not None and b == self.fail_on:
                raise RuntimeError("device failed")
            return O.gzip_chunk(b, 131072)
        finally:
            with self.lock:
                self.live -= 1


@pytest.mark.parametrize("permits", [1, 3])
def test_permits_bound_gpu_calls_and_output_is_in_order(permits):
    data = W.logs(24 * CHUNK + 777, seed=3).tobytes()
    chunks = [data[i:i + CHUNK] for i in range(0, len(data), CHUNK)]
    gpu = FakeGpu()
    cpu_workers = 4
    with native.Hybrid(gpu_permits=permits, warmup_chunks=4, gpu_fn=gpu) as h:
        out = io.BytesIO()
        with native.Writer(out, hybrid=h, chunk_size=CHUNK, max_in_flight=cpu_workers + permits) as w:
            w.write(data)
        cpu, gpu_n = h.stats()
    assert cpu + gpu_n == len(chunks)
    assert gpu.calls == gpu_n and gpu_n > 0 and cpu >= 4
    assert gpu.peak <= permits
    # every member is either the device's bytes or the CPU's, in input order
    got = out.getvalue()
    pos = 0
    for c in chunks:
        a, b = O.gzip_chunk(c, 131072), zlib_member(c)
        if got.startswith(a, pos):
            pos += len(a)
        else:
            assert got.startswith(b, pos)
            pos += len(b)
    assert pos == len(got)
    assert gzip.decompress(got) == data


def test_warmup_chunks_stay_on_the_cpu():
    gpu = FakeGpu(delay=0)
    with native.Hybrid(gpu_permits=8, warmup_chunks=4, gpu_fn=gpu) as h:
        for k in range(6):
            g = h.chunk(bytes([k]) * 1000)
            assert gzip.decompress(g) == bytes([k]) * 1000
        assert h.stats() == (4, 2)
    with native.Hybrid(gpu_permits=0, warmup_chunks=0, gpu_fn=gpu) as h:
        h.chunk(b"abc")
        assert h.stats() == (1, 0)


def test_gpu_error_is_returned_without_cpu_retry():
    bad = b"z" * 5000
    gpu = FakeGpu(fail_on=bad, delay=0)
    with native.Hybrid(gpu_permits=1, warmup_chunks=0, gpu_fn=gpu) as h:
        with pytest.raises(native.GpzError):
            h.chunk(bad)
        assert h.stats() == (0, 1)
        assert gzip.decompress(h.chunk(b"ok" * 100)) == b"ok" * 100  # the permit came back


def test_no_device_means_every_chunk_on_the_cpu():
    """Without a usable CUDA device the context cannot be made, and the
    hybrid leaves every chunk to the CPU (hybrid.rs:128-137)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with native.Hybrid(gpu_permits=4, warmup_chunks=0) as h:
        data = W.text(3 * CHUNK, seed=4).tobytes()
        out = io.BytesIO()
        with native.Writer(out, hybrid=h, chunk_size=CHUNK, max_in_flight=6) as w:
            w.write(data)
        assert h.stats() == (3, 0)
        assert out.getvalue() == b"".join(zlib_member(data[i:i + CHUNK]) for i in range(0, len(data), CHUNK))
