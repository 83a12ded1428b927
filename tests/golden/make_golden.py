"""Generates tests/golden/golden.json: known answers for the gzip path.

The reference ships no golden vectors for packed tokens or DEFLATE bytes, so
these are this project's own known answers, produced by the C oracle and, for
every input small enough, by the independent pure-Python restatement too; the
script refuses to write anything if the two disagree or if zlib cannot inflate
a member back to its input.

Inputs: the reference's own test inputs (crates/gpzip-codec-gpu/src/gpu/
lz77_hash.rs:725-767 and deflate.rs:1030-1127), a few edge sizes, and 2 MiB of
each synthetic generator.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import zlib

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gpzip_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import pyref as P  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
PY_LIMIT = 20_000  # inputs up to this size are also run through pyref


def reference_inputs():
    return {
        "empty": b"",
        "single_byte": b"a",
        "no_matches_32": bytes(range(32)),
        "obvious_repeat_lz77_hash": b"abcabcabcabcabcabcabcabc" * 8,
        "obvious_repeat_deflate": b"abcabcabcabcabcabcabc" * 8,
        "self_overlap_q64": b"q" * 64,
        "self_overlap_x64": b"x" * 64,
        "pseudo_random_2048": bytes((i * 2654435761) & 0xFF for i in range(2048)),
        "pseudo_random_1500": bytes((i * 2654435761) & 0xFF for i in range(1500)),
        "larger_text_512": b"".join(f"line {i}: the quick brown fox\n".encode() for i in range(512)),
        "larger_text_256": b"".join(f"line {i}: the quick brown fox\n".encode() for i in range(256)),
    }


def extra_inputs():
    rng = np.random.Generator(np.random.PCG64(1234))
    d = {
        "edge_4097_ternary": rng.integers(0, 3, size=4097, dtype=np.uint8).tobytes(),
        "edge_40000_text": W.text(40_000, seed=5).tobytes(),
        "edge_131073_binary": W.binary(131_073, seed=6).tobytes(),
        "zeros_70000": bytes(70_000),
    }
    for gen, seed in (("text", 0), ("logs", 1), ("binary", 2)):
        d[f"{gen}_2MiB_seed{seed}"] = W.GENERATORS[gen](2 << 20, seed=seed).tobytes()
    return d


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()


def inflate_all(gz: bytes) -> bytes:
    out, rest = b"", gz
    while rest:
        d = zlib.decompressobj(31)
        out += d.decompress(rest)
        rest = d.unused_data
    return out


def entry(name: str, data: bytes) -> dict:
    members = [data[o:o + O.MEMBER_BYTES] for o in range(0, max(len(data), 1), O.MEMBER_BYTES)]
    pps = [O.match_find(m) for m in members]
    toks = [O.greedy_walk(pp, m) for pp, m in zip(pps, members)]
    gz = O.gzip_chunk(data)
    if inflate_all(gz) != data:
        raise SystemExit(f"{name}: zlib does not inflate the oracle output")
    if len(data) <= PY_LIMIT:
        ppp = P.match_find(data)
        pt = P.greedy_walk(ppp, data)
        if list(np.concatenate(pps)) != ppp or list(np.concatenate(toks)) != pt:
            raise SystemExit(f"{name}: C oracle and Python restatement disagree on tokens")
        if P.gzip_chunk(data) != gz:
            raise SystemExit(f"{name}: C oracle and Python restatement disagree on bytes")
    pp = np.concatenate(pps).astype("<u4")
    tok = np.concatenate(toks).astype("<u4")
    e = {
        "n": len(data),
        "input_sha256": sha(data),
        "pp_sha256": sha(pp.tobytes()),
        "tokens": int(tok.size),
        "tokens_sha256": sha(tok.tobytes()),
        "gzip_len": len(gz),
        "gzip_sha256": sha(gz),
        "pyref_checked": len(data) <= PY_LIMIT,
    }
    if len(data) <= 2048:
        e["input_hex"] = data.hex()
        e["pp"] = [int(x) for x in pp]
        e["walked"] = [int(x) for x in tok]
        e["gzip_hex"] = gz.hex()
    return e


def main():
    res = {"member_bytes": O.MEMBER_BYTES, "reference": {}, "extra": {}}
    for k, v in reference_inputs().items():
        res["reference"][k] = entry(k, v)
    for k, v in extra_inputs().items():
        res["extra"][k] = entry(k, v)
    with open(OUT, "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
    print(OUT)


if __name__ == "__main__":
    main()
