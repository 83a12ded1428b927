"""Device path vs the CPU oracle: packed tokens, walked tokens and gzip bytes.

Bit-exact is the bar for every comparison here (integer and byte work).
Inputs: the reference's own test inputs (lz77_hash.rs:725-767,
deflate.rs:1030-1127), edge sizes around the 4 KiB segment and the 128 KiB
member boundaries, and 2 MiB chunks of the three synthetic generators.
"""
import zlib

import numpy as np
import pytest

from gpzip_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MEMBER = 128 * 1024


def ref_inputs():
    yield "empty", b""
    yield "one", b"a"
    yield "no_match_32", bytes(range(32))
    yield "abc_repeat_lz", b"abcabcabcabcabcabcabcabc" * 8
    yield "abc_repeat_deflate", b"abcabcabcabcabcabcabc" * 8
    yield "self_overlap_q", b"q" * 64
    yield "self_overlap_x", b"x" * 64
    yield "pseudo_random_2048", bytes((i * 2654435761) & 0xFF for i in range(2048))
    yield "pseudo_random_1500", bytes((i * 2654435761) & 0xFF for i in range(1500))
    yield "lines_512", b"".join(f"line {i}: the quick brown fox\n".encode() for i in range(512))
    yield "lines_256", b"".join(f"line {i}: the quick brown fox\n".encode() for i in range(256))


def edge_inputs():
    rng = np.random.default_rng(11)
    for n in (2, 3, 4, 5, 17, 4095, 4096, 4097, 4098, 8191, 8193, 36863, 36865, 131071, 131072, 131073,
              131074, 262149):
        kind = n % 3
        if kind == 0:
            a = rng.integers(0, 256, size=n, dtype=np.uint8)
        elif kind == 1:
            a = rng.integers(0, 3, size=n, dtype=np.uint8)
        else:
            a = W.text(n, seed=n)
        yield f"edge_{n}", a.tobytes()
    yield "zeros_200k", bytes(200_000)
    yield "ones_run_70k", b"\x01" * 70_000


def expected(data: bytes, member=MEMBER):
    pps, toks = [], []
    for off in range(0, max(len(data), 1), member):
        piece = data[off:off + member]
        pp = O.match_find(piece)
        pps.append(pp)
        toks.append(O.greedy_walk(pp, piece))
    pp = np.concatenate(pps) if pps else np.zeros(0, np.uint32)
    tok = np.concatenate(toks) if toks else np.zeros(0, np.uint32)
    return pp, tok, O.gzip_chunk(data, member)


def check(ctx, name, data, member=MEMBER):
    pp, tok, gz = ctx.debug_chunk(data)
    epp, etok, egz = expected(data, member)
    assert pp.size == len(data)
    if len(data):
        bad = np.nonzero(pp != epp)[0]
        assert bad.size == 0, f"{name}: pp differs at {bad[:8]} got {pp[bad[:4]]} want {epp[bad[:4]]}"
    assert tok.size == etok.size and np.array_equal(tok, etok), f"{name}: walked tokens differ"
    assert gz == egz, f"{name}: gzip bytes differ ({len(gz)} vs {len(egz)})"
    out, rest = b"", gz
    while rest:
        d = zlib.decompressobj(31)
        out += d.decompress(rest)
        rest = d.unused_data
    assert out == bytes(data), f"{name}: round trip failed"


@pytest.mark.parametrize("name,data", list(ref_inputs()), ids=[n for n, _ in ref_inputs()])
def test_reference_inputs(ctx, name, data):
    check(ctx, name, data)


@pytest.mark.parametrize("name,data", list(edge_inputs()), ids=[n for n, _ in edge_inputs()])
def test_edge_sizes(ctx, name, data):
    check(ctx, name, data)


@pytest.mark.parametrize("gen", ["text", "logs", "binary"])
def test_two_mib_chunk(ctx, gen):
    data = W.GENERATORS[gen](2 << 20, seed=7).tobytes()
    check(ctx, gen, data)


def test_batch_matches_single(ctx):
    items = [W.text(5000, seed=1).tobytes(), b"", W.binary(300_000, seed=3).tobytes(), b"z" * 10,
             W.logs(1 << 20, seed=4).tobytes()]
    outs = ctx.compress_batch(items)
    for it, o in zip(items, outs):
        assert o == O.gzip_chunk(it, MEMBER)
    plain = ctx.compress_batch_plain(items)
    assert plain == outs
