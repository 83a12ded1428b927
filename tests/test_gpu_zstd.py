"""The device zstd codec (GPZ_CODEC_ZSTD) against the oracle's restatement,
byte for byte, and against libzstd's decoder (GPU)."""
import io

import numpy as np
import pytest

from gpzip_b200 import native
from gpzip_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def zctx():
    with native.Context(codec=native.GPZ_CODEC_ZSTD) as c:
        yield c


def items():
    rng = np.random.default_rng(11)
    out = [b"", b"x", b"abcabcabcabcabc" * 10, rng.integers(0, 256, 5000, dtype=np.uint8).tobytes(),
           bytes(200_000), W.text(131_073, seed=5).tobytes(), rng.integers(0, 3, 4097, dtype=np.uint8).tobytes()]
    for kind, seed in (("text", 0), ("logs", 1), ("binary", 2)):
        out.append(W.GENERATORS[kind](2 << 20, seed=seed).tobytes())
    for i in range(12):
        n = int(np.exp(rng.uniform(np.log(1), np.log(3 << 20))))
        out.append(W.GENERATORS[["text", "logs", "binary"][i % 3]](n, seed=400 + i).tobytes())
    return out


def test_batch_equals_oracle_and_decodes(zctx):
    its = items()
    got = zctx.compress_batch(its)
    for it, g in zip(its, got):
        assert g == O.zstd_chunk(it, 131072)
        assert O.zstd_decompress(g, len(it)) == it


def test_chunk_calls_and_plain_path(zctx):
    its = items()[:10]
    for it in its:
        assert zctx.compress_chunk(it) == O.zstd_chunk(it, 131072)
    assert zctx.compress_batch_plain(its) == zctx.compress_batch(its)


def test_two_mib_members():
    data = W.logs(3 << 20, seed=21).tobytes()
    with native.Context(codec=native.GPZ_CODEC_ZSTD, member_bytes=2 << 20) as c:
        got = c.compress_chunk(data)
    assert got == O.zstd_chunk(data, 2 << 20)
    assert O.zstd_decompress(got, len(data)) == data


def test_writer_writes_a_zstd_stream(zctx):
    """The streaming writer over the zstd context: one frame per 2 MiB chunk,
    in order, one zstd stream (as the reference's ZstdCompressor writes)."""
    data = W.logs((9 << 20) + 4321, seed=30).tobytes()
    out = io.BytesIO()
    with native.Writer(out, ctx=zctx, chunk_size=2 << 20, max_in_flight=3) as w:
        for i in range(0, len(data), 700_000):
            w.write(data[i:i + 700_000])
    want = b"".join(O.zstd_chunk(data[i:i + (2 << 20)], 131072) for i in range(0, len(data), 2 << 20))
    assert out.getvalue() == want
    assert O.zstd_decompress(out.getvalue(), len(data)) == data


def test_full_logs_workload_decodes(zctx):
    data = W.config_logs_tar()
    chunks = [np.ascontiguousarray(data[o:o + n]) for o, n in W.chunk_spans(data.size, 2 << 20)]
    got = zctx.compress_batch(chunks)
    stream = b"".join(bytes(g) for g in got)
    assert O.zstd_decompress(stream, data.size) == data.tobytes()
    for k in (0, 16, len(chunks) - 1):
        assert bytes(got[k]) == O.zstd_chunk(chunks[k], 131072)
