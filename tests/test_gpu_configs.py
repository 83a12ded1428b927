"""The named workloads at their full sizes (GPU), through the batched host
API with 2 MiB chunks, compared chunk by chunk with the oracle's output.

The oracle's per-chunk SHA-256 digests are committed in
tests/golden/config_digests.json (made by tests/golden/make_config_digests.py,
which checks that every oracle chunk inflates back to its input).  Every
chunk of every set is compared, not a sample:

* text     8 MiB, 4 chunks, 128 KiB members;
* logs     the 64 MiB log ustar stream, 33 chunks;
* binary   272 MiB mixed binary, 136 chunks;
* uneven   the 1,000-file mix, 1,245 chunks (each file cut on its own);
* member2m text, logs and binary inputs of 3 x 2 MiB + 12,345 bytes with
           2 MiB members (whole-chunk mode).

Each stream must also be a concatenation of valid gzip members that inflate
back to the chunk (zlib), a property that holds whatever the digests say.
"""
import hashlib
import json
import os
import zlib

import numpy as np
import pytest

from gpzip_b200 import native
from gpzip_b200 import workloads as W

CHUNK = 2 << 20
HERE = os.path.dirname(os.path.abspath(__file__))
DIGESTS = json.load(open(os.path.join(HERE, "golden", "config_digests.json")))["sets"]


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


def check_set(got, items, want, member):
    assert len(got) == len(items) == want["chunks"]
    bad = []
    for k, (it, g) in enumerate(zip(items, got)):
        g = bytes(g)
        if hashlib.sha256(g).hexdigest() != want["chunk_sha256"][k]:
            bad.append((k, len(g), want["gzip_len"][k]))
        ms = members(g)
        assert len(ms) == max(1, -(-it.size // member))
        assert b"".join(ms) == it.tobytes()
    assert not bad, f"{len(bad)} of {len(items)} chunks differ from the oracle (chunk, got len, want len): {bad[:8]}"


def uneven_chunks():
    items = []
    for _, _, data in W.uneven_files(1000, seed=3):
        items.extend(chunks_of(data))
    return items


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["text", "logs", "binary"])
def test_named_config_every_chunk(ctx, name):
    data = {"text": W.config_text, "logs": W.config_logs_tar, "binary": W.config_binary}[name]()
    want = DIGESTS[name]
    assert W.digest(data) == want["input_sha256"], "workload generator drifted"
    items = chunks_of(data)
    check_set(ctx.compress_batch(items), items, want, 131072)


@pytest.mark.gpu
def test_uneven_mix_every_chunk(ctx):
    items = uneven_chunks()
    want = DIGESTS["uneven"]
    assert hashlib.sha256(b"".join(W.digest(x).encode() for x in items)).hexdigest() == want["input_sha256"]
    check_set(ctx.compress_batch(items), items, want, 131072)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["text", "logs", "binary"])
def test_member2m_every_chunk(name):
    n = 3 * CHUNK + 12_345
    data = {"text": lambda: W.text(n, seed=7), "logs": lambda: W.logs(n, seed=8),
            "binary": lambda: W.binary(n, seed=9)}[name]()
    want = DIGESTS["member2m"][name]
    assert W.digest(data) == want["input_sha256"]
    items = chunks_of(data)
    with native.Context(member_bytes=2 << 20) as c2:
        check_set(c2.compress_batch(items), items, want, 2 << 20)


def test_digest_fixture_pinned_on_cpu():
    """The committed digests are the oracle's: the first text chunk and the
    2 MiB-member binary tail are recomputed here (CPU, under a second)."""
    from oracle import oracle as O
    data = W.config_text()
    assert W.digest(data) == DIGESTS["text"]["input_sha256"]
    first = data[:CHUNK]
    assert hashlib.sha256(O.gzip_chunk(first, 131072, threads=4)).hexdigest() == DIGESTS["text"]["chunk_sha256"][0]
    n = 3 * CHUNK + 12_345
    tail = W.binary(n, seed=9)[3 * CHUNK:]
    assert (hashlib.sha256(O.gzip_chunk(tail, 2 << 20)).hexdigest()
            == DIGESTS["member2m"]["binary"]["chunk_sha256"][-1])
    for name in ("text", "logs", "binary", "uneven"):
        s = DIGESTS[name]
        assert len(s["chunk_sha256"]) == len(s["gzip_len"]) == s["chunks"]
    assert DIGESTS["logs"]["chunks"] == 33 and DIGESTS["binary"]["chunks"] == 136
    assert DIGESTS["uneven"]["chunks"] == 1245
