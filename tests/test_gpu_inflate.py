"""GPU decompression of gpzip-written gzip streams (gpz_inflate) through the C
ABI: the output equals the input that was compressed, for the device
compressor's own streams, the oracle's, fixed-block members and zlib-built
members of every block type, overlapping and chained matches; damaged
streams fail with GPZ_E_DATA."""
import struct
import zlib

import numpy as np
import pytest

from gpzip_b200 import native
from gpzip_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def member(deflate: bytes, data: bytes) -> bytes:
    return O.GZIP_HEADER + deflate + struct.pack("<II", zlib.crc32(data), len(data) & 0xFFFFFFFF)


def raw_deflate(data: bytes, level: int, strategy: int = zlib.Z_DEFAULT_STRATEGY) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, -15, 8, strategy)
    return c.compress(data) + c.flush()


def test_round_trip_of_the_device_compressor(ctx):
    for kind, n, seed in (("logs", (8 << 20) + 1536, 1), ("text", 3 << 20, 2), ("binary", (4 << 20) + 5, 3)):
        data = W.GENERATORS[kind](n, seed=seed).tobytes()
        gz = bytes(ctx.compress_chunk(data))
        assert bytes(ctx.inflate(gz)) == data
        assert ctx.inflate_device_ms() > 0


def test_many_items_and_empty_members(ctx):
    items = [W.GENERATORS[["text", "logs", "binary"][i % 3]](int(n), seed=60 + i).tobytes()
             for i, n in enumerate(np.random.default_rng(3).integers(0, 400_000, size=40))]
    items[4] = b""
    items[9] = b"z"
    gz = b"".join(bytes(x) for x in ctx.compress_batch(items))
    assert bytes(ctx.inflate(gz)) == b"".join(items)
    assert bytes(ctx.inflate(b"")) == b""


def test_fixed_blocks_and_zlib_members(ctx):
    data = [W.logs(131_072, seed=5).tobytes(), W.text(90_000, seed=6).tobytes(), b"\0" * 70_000,
            np.random.default_rng(7).integers(0, 256, 60_000, dtype=np.uint8).tobytes(), W.text(700_000, seed=8).tobytes()]
    parts, want = [O.gzip_member_fixed(data[0])], [data[0]]
    for d in data:
        for level, strat in ((0, 0), (1, 0), (6, zlib.Z_FIXED), (9, zlib.Z_RLE), (6, zlib.Z_HUFFMAN_ONLY)):
            parts.append(member(raw_deflate(d, level, strat), d))
            want.append(d)
    assert bytes(ctx.inflate(b"".join(parts))) == b"".join(want)


def test_overlapping_and_chained_matches(ctx):
    # runs whose matches overlap their own output (distance 1 or 3) and
    # chains of matches that copy from earlier matches: the expansion
    # kernel resolves them in order
    rng = np.random.default_rng(13)
    block = rng.integers(0, 256, 3000, dtype=np.uint8).tobytes()
    data = [b"\0" * 300_000, b"abc" * 100_001, (b"x" * 5 + b"yz") * 40_000, block * 60,
            b"".join(block[: int(k)] for k in rng.integers(1, 3000, size=80))]
    parts, want = [], []
    for d in data:
        parts.append(bytes(ctx.compress_chunk(d)))
        want.append(d)
        for level in (1, 9):
            parts.append(member(raw_deflate(d, level), d))
            want.append(d)
    assert bytes(ctx.inflate(b"".join(parts))) == b"".join(want)


def test_page_locked_buffers(ctx):
    import torch
    data = W.logs(3 << 20, seed=11).tobytes()
    gz = bytes(ctx.compress_chunk(data))
    src = torch.empty(len(gz), dtype=torch.uint8, pin_memory=True).numpy()
    src[:] = np.frombuffer(gz, dtype=np.uint8)
    dst = torch.empty(len(data), dtype=torch.uint8, pin_memory=True).numpy()
    assert bytes(ctx.inflate(src, out=dst)) == data


def test_members_that_do_not_settle_page_locked(ctx):
    # binary and text members: runs of codes of one length keep speculative
    # decodes misaligned, so many members go through the tail kernels
    # (candidate sub-spans and the walk); the output goes straight from the
    # expansion kernel into the page-locked buffer
    import torch
    data = W.binary((8 << 20) + 777, seed=14).tobytes() + W.text(3 << 20, seed=15).tobytes()
    gz = b"".join(bytes(ctx.compress_chunk(data[o:o + (2 << 20)])) for o in range(0, len(data), 2 << 20))
    src = torch.empty(len(gz), dtype=torch.uint8, pin_memory=True).numpy()
    src[:] = np.frombuffer(gz, dtype=np.uint8)
    dst = torch.empty(len(data), dtype=torch.uint8, pin_memory=True).numpy()
    for _ in range(2):  # the scratch of the first call is reused by the second
        dst[:] = 0
        assert bytes(ctx.inflate(src, out=dst)) == data
    # a flipped bit inside a binary member's data: that member fails (the
    # serial decoder gives the status), and the context stays usable
    bad = bytearray(gz)
    bad[len(gz) // 3] ^= 0x10
    with pytest.raises(native.GpzError) as e:
        ctx.inflate(bytes(bad))
    assert e.value.status == native.GPZ_E_DATA
    assert bytes(ctx.inflate(gz)) == data


def test_damaged_streams_fail_and_leave_the_context_usable(ctx):
    data = W.text(600_000, seed=12).tobytes()
    gz = bytearray(ctx.compress_chunk(data))
    cases = []
    bad_crc = bytearray(gz)
    bad_crc[-8] ^= 1  # the last member's CRC
    cases.append(bad_crc)
    bad_size = bytearray(gz)
    bad_size[-4] ^= 1  # the last member's ISIZE
    cases.append(bad_size)
    flipped = bytearray(gz)
    flipped[200] ^= 0x10  # inside the first member's DEFLATE data
    cases.append(flipped)
    cases.append(gz[:-3])  # truncated
    for c in cases:
        with pytest.raises(native.GpzError) as e:
            ctx.inflate(bytes(c))
        assert e.value.status == native.GPZ_E_DATA
    assert bytes(ctx.inflate(bytes(gz))) == data
    with pytest.raises(native.GpzError):
        ctx.inflate(zlib.compress(data))  # not gzip at all
