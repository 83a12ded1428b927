"""The member decoder of the GPU inflate path (gpzip_b200/csrc/gpz_inflate_core.h)
built for the host with one lane, under AddressSanitizer and UBSan, against
zlib: every block type and zlib strategy, gpzip's own members, and mutated
streams, which must either fail with a status or decode exactly as zlib
does.  The device build runs the same code with 32 lanes."""
import os
import random
import shutil
import struct
import subprocess
import zlib

import numpy as np
import pytest

from gpzip_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def decoder(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path_factory.mktemp("infl") / "inflate_host")
    flags = ["-O1", "-g", "-std=c++17", "-Wall", "-Wextra", "-Werror"]
    san = ["-fsanitize=address,undefined", "-fno-sanitize-recover=all"]
    src = [os.path.join(ROOT, "tests", "c", "inflate_host.cpp"), "-I", os.path.join(ROOT, "gpzip_b200", "csrc")]
    r = subprocess.run([cxx, *flags, *san, *src, "-o", exe], capture_output=True, text=True)
    if r.returncode != 0:  # no sanitizer runtime: plain build
        r = subprocess.run([cxx, *flags, *src, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


PARALLEL = {}  # the last run's "parallel: <taken> of <records>" from inflate_host


def run(decoder, tmp_path, cases):
    """cases: list of (deflate bytes, isize) -> list of (status, output)."""
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as f:
        for data, isize in cases:
            f.write(struct.pack("<II", len(data), isize))
            f.write(data)
    r = subprocess.run([decoder, str(fin), str(fout)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    PARALLEL.clear()
    for line in r.stderr.splitlines():
        if line.startswith("parallel: "):
            taken, _, records = line[len("parallel: "):].partition(" of ")
            PARALLEL.update(taken=int(taken), records=int(records))
    res = []
    with open(fout, "rb") as f:
        for _ in cases:
            st, n = struct.unpack("<II", f.read(8))
            res.append((st, f.read(n)))
    return res


def raw_deflate(data: bytes, level: int, strategy: int = zlib.Z_DEFAULT_STRATEGY) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, -15, 8, strategy)
    return c.compress(data) + c.flush()


def inputs():
    rng = np.random.default_rng(11)
    return {
        "empty": b"",
        "one": b"x",
        "text": W.text(100_000, seed=1).tobytes(),
        "logs": W.logs(131_072, seed=2).tobytes(),
        "binary": W.binary(131_072, seed=3).tobytes(),
        "runs": b"\0" * 70_000 + b"ab" * 20_000 + bytes(rng.integers(0, 3, 5000, dtype=np.uint8)),
        "random": rng.integers(0, 256, 50_000, dtype=np.uint8).tobytes(),
        "large": W.text(700_000, seed=4).tobytes(),  # several blocks per stream
    }


def test_every_zlib_level_and_strategy(decoder, tmp_path):
    cases, want = [], []
    strategies = [zlib.Z_DEFAULT_STRATEGY, zlib.Z_FILTERED, zlib.Z_HUFFMAN_ONLY, zlib.Z_RLE, zlib.Z_FIXED]
    for name, data in inputs().items():
        for level in (0, 1, 6, 9):
            for strat in strategies:
                cases.append((raw_deflate(data, level, strat), len(data)))
                want.append(data)
    got = run(decoder, tmp_path, cases)
    for (st, out), w, (c, _) in zip(got, want, cases):
        assert st == 0 and out == w, (st, len(c), len(w))


def test_gpzip_members(decoder, tmp_path):
    from oracle import oracle as O
    cases, want = [], []
    for kind in ("text", "logs", "binary"):
        data = W.GENERATORS[kind](131_072 * 3 + 999, seed=7).tobytes()
        gz = O.gzip_chunk(data, 131072)
        # split at the fixed 10-byte header; every member is header + deflate + trailer
        pos = 0
        while pos < len(gz):
            nxt = gz.find(O.GZIP_HEADER, pos + 10)
            end = nxt if nxt >= 0 else len(gz)
            member = gz[pos:end]
            crc, isize = struct.unpack("<II", member[-8:])
            cases.append((member[10:-8], isize))
            want.append(zlib.decompress(member, 31))
            pos = end
    got = run(decoder, tmp_path, cases)
    for (st, out), w in zip(got, want):
        assert st == 0 and out == w
    # every gpzip member is one dynamic block: the parallel decode (128
    # lanes, checked against the serial tokens by the harness) takes them all
    assert PARALLEL == {"taken": len(cases), "records": len(cases)}


def test_parallel_decode_of_zlib_members(decoder, tmp_path):
    # single-block zlib members (one final dynamic block below ~16 KiB of
    # output at level 6 on text) go the parallel way; the multi-block ones
    # are left to the serial decoder; the harness exits 6 if the parallel
    # tokens differ from the serial ones or a rejected member is taken
    cases = []
    for n in (1, 100, 3000, 20_000, 60_000, 200_000):
        for kind in ("text", "logs", "binary"):
            data = W.GENERATORS[kind](n, seed=n % 97).tobytes()
            for level in (1, 6, 9):
                cases.append((raw_deflate(data, level), len(data)))
    run(decoder, tmp_path, cases)
    assert 0 < PARALLEL["taken"] < PARALLEL["records"]


def test_fixed_block_members(decoder, tmp_path):
    from oracle import oracle as O
    data = W.logs(131_072, seed=5).tobytes()
    member = O.gzip_member_fixed(data)
    got = run(decoder, tmp_path, [(member[10:-8], len(data))])
    assert got[0] == (0, data)


def test_wrong_sizes_fail(decoder, tmp_path):
    data = W.text(20_000, seed=8).tobytes()
    d = raw_deflate(data, 6)
    got = run(decoder, tmp_path, [(d, len(data) - 1), (d, len(data) + 1), (d + b"\0", len(data)), (d[:-1], len(data))])
    assert got[0][0] == 7   # output longer than ISIZE
    assert got[1][0] == 9   # output shorter than ISIZE
    assert got[2][0] == 10  # data ends before the trailer
    assert got[3][0] != 0   # truncated


def test_mutated_streams_fail_or_match_zlib(decoder, tmp_path):
    rnd = random.Random(12)
    base = []
    for name, data in inputs().items():
        if name in ("empty", "large"):
            continue
        for level, strat in ((1, zlib.Z_DEFAULT_STRATEGY), (9, zlib.Z_DEFAULT_STRATEGY), (6, zlib.Z_FIXED), (0, 0)):
            base.append((raw_deflate(data, level, strat), len(data)))
    cases = []
    for _ in range(600):
        d, isize = rnd.choice(base)
        b = bytearray(d)
        op = rnd.randrange(4)
        if op == 0 and b:
            i = rnd.randrange(len(b))
            b[i] ^= 1 << rnd.randrange(8)
        elif op == 1 and b:
            i = rnd.randrange(min(len(b), 64))  # the block header
            b[i] = rnd.randrange(256)
        elif op == 2:
            b = b[:rnd.randrange(len(b) + 1)]
        else:
            i = rnd.randrange(len(b) + 1)
            b[i:i] = bytes(rnd.randrange(256) for _ in range(rnd.randrange(1, 9)))
        cases.append((bytes(b), isize if rnd.random() < 0.9 else rnd.randrange(0, 2 * isize + 10)))
    got = run(decoder, tmp_path, cases)
    ok = 0
    for (st, out), (c, isize) in zip(got, cases):
        if st != 0:
            continue
        ok += 1
        z = zlib.decompressobj(-15)
        ref = z.decompress(c) + z.flush()
        assert z.eof and not z.unused_data and ref == out
    assert ok < len(cases)


def test_member_split_and_sizes_on_the_host():
    # gpz_inflate_size cuts the stream at gpzip's fixed header and sums the
    # ISIZE trailers; it needs no device
    from gpzip_b200 import native
    from oracle import oracle as O
    data = W.logs(131_072 * 5 + 77, seed=9).tobytes()
    gz = O.gzip_chunk(data, 131072)
    assert native.inflate_size(gz) == (6, len(data))
    assert native.inflate_size(b"") == (0, 0)
    two = gz + O.gzip_chunk(b"abc", 131072)
    assert native.inflate_size(two) == (7, len(data) + 3)
    for bad in (b"\x1f\x8b\x08\x08" + gz[4:], gz[:17], b"x" + gz):
        with pytest.raises(native.GpzError) as e:
            native.inflate_size(bad)
        assert e.value.status == native.GPZ_E_DATA
    # an ISIZE beyond what the member's data can expand to is refused
    forged = bytearray(O.gzip_chunk(b"hello", 131072))
    forged[-4:] = struct.pack("<I", 1 << 30)
    with pytest.raises(native.GpzError):
        native.inflate_size(bytes(forged))


def split_like_the_reference(buf: bytes):
    """(members, output bytes) as parallel_decompress.rs:36-58 cuts a stream:
    every header occurrence, scanning on 10 bytes past each one, then the
    ISIZE trailers summed; None where gpz_inflate_size must refuse."""
    from oracle import oracle as O
    if not buf:
        return (0, 0)
    if len(buf) < 18 or buf[:10] != O.GZIP_HEADER:
        return None
    starts, p = [0], 10
    while p + 10 <= len(buf):
        q = buf.find(O.GZIP_HEADER, p)
        if q < 0:
            break
        starts.append(q)
        p = q + 10
    total = 0
    for i, b in enumerate(starts):
        e = starts[i + 1] if i + 1 < len(starts) else len(buf)
        if e - b < 18:
            return None
        isize = struct.unpack("<I", buf[e - 4:e])[0]
        if isize > 1032 * (e - b - 18 + 1):
            return None
        total += isize
    return (len(starts), total)


def test_member_split_of_a_long_stream_in_pieces():
    # streams of several MiB are searched in pieces on several threads;
    # members of every size, headers right at piece edges (a member every
    # few hundred bytes in one stretch), and members too short to be valid
    from gpzip_b200 import native
    from oracle import oracle as O
    rng = np.random.default_rng(31)

    def member(n):
        body = rng.integers(0, 255, n, dtype=np.uint8).tobytes().replace(b"\x1f\x8b", b"\x1f\x8c")
        return O.GZIP_HEADER + body + struct.pack("<II", 0, min(n, 1000))

    sizes = [int(x) for x in rng.integers(0, 200_000, 60)] + [int(x) for x in rng.integers(0, 600, 4000)]
    rng.shuffle(sizes)
    stream = b"".join(member(n) for n in sizes)
    assert len(stream) > 6 << 20
    assert native.inflate_size(stream) == split_like_the_reference(stream)
    # a member shorter than its header and trailer: both refuse
    bad = stream[:3_000_000] + O.GZIP_HEADER + b"xy" + stream[3_000_000:]
    assert split_like_the_reference(bad) is None
    with pytest.raises(native.GpzError):
        native.inflate_size(bad)


@pytest.fixture(scope="module")
def lanes_decoder(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path_factory.mktemp("infl32") / "inflate_lanes")
    src = [os.path.join(ROOT, "tests", "c", "inflate_lanes.cpp"), "-I", os.path.join(ROOT, "gpzip_b200", "csrc")]
    r = subprocess.run([cxx, "-O2", "-std=c++20", "-pthread", "-Wall", "-Wextra", "-Werror", *src, "-o", exe],
                       capture_output=True, text=True)
    if r.returncode != 0 and "barrier" in r.stderr:
        pytest.skip("no std::barrier")
    assert r.returncode == 0, r.stderr
    return exe


def test_32_lane_build_matches_zlib(lanes_decoder, tmp_path):
    # the device build's lane-cooperative paths (NL = 32) on 32 host threads:
    # strided staging and table fills, copies with distances below 32 (the
    # modulo path the one-lane build never takes), flushes; every lane must
    # return the same status
    from oracle import oracle as O
    rng = np.random.default_rng(21)
    runs = b"ab" * 3000 + b"\0" * 5000 + bytes(rng.integers(0, 4, 3000, dtype=np.uint8)) + b"xyz" * 2000
    cases, want = [], []
    for data in (runs, W.text(40_000, seed=22).tobytes(), W.binary(50_000, seed=23).tobytes(), b"", b"q"):
        for level, strat in ((0, 0), (1, zlib.Z_DEFAULT_STRATEGY), (9, zlib.Z_RLE), (6, zlib.Z_FIXED)):
            cases.append((raw_deflate(data, level, strat), len(data)))
            want.append(data)
    data = W.logs(131_072, seed=24).tobytes()
    member = O.gzip_chunk(data, 131072)
    cases.append((member[10:-8], len(data)))
    want.append(data)
    d = raw_deflate(runs, 6)
    cases += [(d[:len(d) // 2], len(runs)), (d, len(runs) - 5)]
    want += [None, None]
    got = run(lanes_decoder, tmp_path, cases)
    for (st, out), w in zip(got, want):
        if w is None:
            assert st != 0
        else:
            assert st == 0 and out == w
