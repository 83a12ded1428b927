"""The named workloads at their full sizes (GPU), through the batched host
API with 2 MiB chunks: the 8 MiB text stream byte for byte against the
oracle; the 64 MiB logs tar and the 272 MiB mixed binary stream through
size-independent properties (every member inflates back to its chunk, the
streams are exactly the concatenation of valid gzip members, sampled chunks
equal the oracle's)."""
import zlib

import numpy as np
import pytest

from gpzip_b200 import native
from gpzip_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu
CHUNK = 2 << 20


def chunks_of(data):
    return [np.ascontiguousarray(data[o:o + n]) for o, n in W.chunk_spans(data.size, CHUNK)]


def members(stream: bytes):
    """Splits a concatenation of gzip members; every member must be valid."""
    out, pos = [], 0
    view = memoryview(stream)
    while pos < len(stream):
        d = zlib.decompressobj(31)
        body = d.decompress(view[pos:])
        assert d.eof, "truncated member"
        used = len(stream) - pos - len(d.unused_data)
        out.append(body)
        pos += used
    return out


def test_text_8mib_exact(ctx):
    data = W.config_text()
    items = chunks_of(data)
    got = ctx.compress_batch(items)
    for it, g in zip(items, got):
        assert g == O.gzip_chunk(it.tobytes(), 131072, threads=8)


@pytest.mark.parametrize("name", ["logs", "binary"])
def test_full_config_properties(ctx, name):
    data = W.config_logs_tar() if name == "logs" else W.config_binary()
    items = chunks_of(data)
    got = ctx.compress_batch(items)
    rng = np.random.default_rng(5)
    sample = set(int(x) for x in rng.choice(len(items), size=3, replace=False)) | {len(items) - 1}
    for k, (it, g) in enumerate(zip(items, got)):
        ms = members(bytes(g))
        assert len(ms) == max(1, -(-it.size // 131072))
        assert b"".join(ms) == it.tobytes()
        if k in sample:
            assert g == O.gzip_chunk(it.tobytes(), 131072, threads=8)
