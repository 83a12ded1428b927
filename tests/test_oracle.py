"""CPU checks of the oracle itself (no GPU).

Pins the C oracle (oracle/gpz_oracle.c) against:
  * the independent pure-Python restatement (oracle/pyref.py);
  * the reference's own property tests: Huffman lengths (huffman.rs:158-232),
    round trips (deflate.rs:1018-1127, lz77_hash.rs:713-767), the fixed member
    header GPZIP_HEADER (parallel_decompress.rs:29);
  * the CRC-32 check value crc32("123456789") = 0xCBF43926 (crc32fast, the
    dependency behind deflate.rs:974) and zlib's crc32;
  * zlib 1.3 inflate and GNU gzip -t on every member;
  * the committed golden fixtures (tests/golden/golden.json).
"""
import hashlib
import json
import os
import shutil
import subprocess
import zlib

import numpy as np
import pytest

from oracle import oracle as O
from oracle import pyref as P

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.json")


def inflate_all(gz: bytes) -> bytes:
    out, rest = b"", gz
    while rest:
        d = zlib.decompressobj(31)
        out += d.decompress(rest)
        rest = d.unused_data
    return out


REF_INPUTS = {
    "empty": b"",
    "single_byte": b"a",
    "no_matches": bytes(range(32)),
    "obvious_repeat": b"abcabcabcabcabcabcabc" * 8,
    "obvious_repeat_24": b"abcabcabcabcabcabcabcabc" * 8,
    "self_overlap": b"x" * 64,
    "self_overlap_q": b"q" * 64,
    "pseudo_random": bytes((i * 2654435761) & 0xFF for i in range(1500)),
    "pseudo_random_2048": bytes((i * 2654435761) & 0xFF for i in range(2048)),
    "larger_text": b"".join(f"line {i}: the quick brown fox\n".encode() for i in range(256)),
}


@pytest.mark.parametrize("name", sorted(REF_INPUTS))
def test_c_oracle_matches_python_restatement(name):
    data = REF_INPUTS[name]
    pp = O.match_find(data)
    assert list(pp) == P.match_find(data)
    tok = O.greedy_walk(pp, data)
    assert list(tok) == P.greedy_walk(list(pp), data)
    assert P.reconstruct(list(tok)) == data
    assert O.encode_block_fast(tok) == P.encode_block_fast(list(tok))
    assert O.gzip_member(data) == P.gzip_member(data)


@pytest.mark.parametrize("seed", range(6))
def test_c_oracle_matches_python_random(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 12000))
    alphabet = int(rng.choice([2, 4, 16, 256]))
    data = rng.integers(0, alphabet, size=n, dtype=np.uint8).tobytes()
    assert list(O.match_find(data)) == P.match_find(data)
    assert O.gzip_chunk(data, 4096) == P.gzip_chunk(data, 4096)


@pytest.mark.parametrize("name", sorted(REF_INPUTS))
def test_round_trip_brute_force_tokens(name):
    """deflate.rs:1074-1084: brute-force tokens -> walk -> encode -> gzip -> inflate."""
    data = REF_INPUTS[name]
    pp = O.brute_lz77(data, 4096)
    assert list(pp) == P.brute_lz77(data, 4096)
    tok = O.greedy_walk(pp, data)
    gz = P.gzip_wrap(O.encode_block_fast(tok), data)
    assert inflate_all(gz) == data


def test_member_header_is_gpzip_header():
    """parallel_decompress.rs:29 scans for exactly this header."""
    gpzip_header = bytes([0x1F, 0x8B, 0x08, 0x00, 0, 0, 0, 0, 0x00, 0xFF])
    for data in REF_INPUTS.values():
        assert O.gzip_member(data)[:10] == gpzip_header


def test_crc32_check_value():
    assert O.crc32(b"123456789") == 0xCBF43926
    rng = np.random.default_rng(3)
    for n in (0, 1, 7, 4096, 100_000):
        b = rng.integers(0, 256, size=n, dtype=np.uint8).tobytes()
        assert O.crc32(b) == zlib.crc32(b) & 0xFFFFFFFF


# huffman.rs:158-232
def test_huffman_empty():
    assert all(x == 0 for x in O.build_code_lengths([0] * 10, 15))


def test_huffman_single_symbol():
    f = [0] * 10
    f[3] = 100
    lens = O.build_code_lengths(f, 15)
    assert lens[3] == 1 and sum(lens) == 1


def test_huffman_balanced():
    assert all(x == 3 for x in O.build_code_lengths([1] * 8, 15))


def test_huffman_skewed():
    lens = O.build_code_lengths([100, 50, 25, 10, 5, 2, 1, 1], 15)
    assert lens[0] <= lens[7]


def test_huffman_length_limit_and_kraft():
    lens = O.build_code_lengths(list(range(1, 21)), 6)
    assert all(x <= 6 for x in lens)
    assert sum(2.0 ** -int(x) for x in lens if x) <= 1.0 + 1e-9


def test_huffman_fibonacci_needs_halving():
    fib = [1, 1]
    while len(fib) < 30:
        fib.append(fib[-1] + fib[-2])
    lens = O.build_code_lengths(fib, 15)
    assert max(lens) <= 15
    assert list(lens) == P.build_code_lengths(fib, 15)
    assert sum(2.0 ** -int(x) for x in lens if x) <= 1.0 + 1e-9


def test_canonical_prefix_property():
    lens = [3, 3, 3, 3, 3, 2, 4, 4]
    codes = P.canonical_codes(lens)
    for i in range(len(lens)):
        for j in range(len(lens)):
            if i != j and lens[j] < lens[i]:
                assert codes[i] >> (lens[i] - lens[j]) != codes[j]


def test_multi_member_chunk_and_gzip_t(tmp_path):
    rng = np.random.default_rng(9)
    data = (b"the quick brown fox " * 20000) + rng.integers(0, 256, size=70000, dtype=np.uint8).tobytes()
    gz = O.gzip_chunk(data, 131072, threads=4)
    assert gz == O.gzip_chunk(data, 131072, threads=1)
    assert inflate_all(gz) == data
    # 16 members for a 2 MiB chunk, as gzip_chunk_fn splits it (gpu.rs:193-208)
    assert gz.count(bytes([0x1F, 0x8B, 0x08, 0x00, 0, 0, 0, 0, 0, 0xFF])) >= -(-len(data) // 131072)
    if shutil.which("gzip"):
        p = tmp_path / "x.gz"
        p.write_bytes(gz)
        assert subprocess.run(["gzip", "-t", str(p)]).returncode == 0


def test_golden_fixtures():
    g = json.load(open(GOLDEN))
    assert g["member_bytes"] == O.MEMBER_BYTES
    for group in ("reference", "extra"):
        for name, e in g[group].items():
            if "input_hex" not in e:
                continue
            data = bytes.fromhex(e["input_hex"])
            assert list(O.match_find(data)) == e["pp"], name
            assert list(O.tokens(data)) == e["walked"], name
            assert O.gzip_chunk(data).hex() == e["gzip_hex"], name


def test_golden_fixtures_synthetic():
    from gpzip_b200 import workloads as W
    g = json.load(open(GOLDEN))["extra"]
    for gen, seed in (("text", 0), ("logs", 1), ("binary", 2)):
        e = g[f"{gen}_2MiB_seed{seed}"]
        data = W.GENERATORS[gen](2 << 20, seed=seed).tobytes()
        assert hashlib.sha256(data).hexdigest() == e["input_sha256"], gen
        gz = O.gzip_chunk(data, threads=8)
        assert hashlib.sha256(gz).hexdigest() == e["gzip_sha256"], gen


def test_cpu_baseline_gzip_chunks():
    rng = np.random.default_rng(2)
    data = (b"abc def ghi " * 300000) + rng.integers(0, 256, size=5000, dtype=np.uint8).tobytes()
    gz = O.cpu_gzip_chunks(data, 2 << 20, 5, threads=4)
    assert inflate_all(gz) == data


def test_fixed_block_matches_python_restatement():
    # write_fixed_block_fast (deflate.rs:763-799): the C oracle's fixed block
    # equals the pure-Python restatement's and inflates back
    import gzip
    from gpzip_b200 import workloads as W
    for i, kind in enumerate(("text", "logs", "binary")):
        data = W.GENERATORS[kind](12_000, seed=70 + i).tobytes()
        toks = O.tokens(data)
        assert O.encode_block_fixed(toks) == P._encode_fixed([int(t) for t in toks])
        assert gzip.decompress(O.gzip_chunk_fixed(data)) == data
    assert gzip.decompress(O.gzip_chunk_fixed(b"")) == b""
