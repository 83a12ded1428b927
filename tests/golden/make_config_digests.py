"""Generates tests/golden/config_digests.json: the oracle's gzip output for
every 2 MiB chunk of every named workload, as SHA-256 digests.

The reference ships no token or byte vectors for this path, so these are
this project's own known answers from the C oracle (the restatement of
lz77_hash_lookup.wgsl:45-119, lz77.rs:260-284 and deflate.rs:752-980 in
oracle/gpz_oracle.c).  They let the GPU tests and the benchmark compare
every chunk of the full-size workloads, not a sample, in a fraction of a
second; computing them takes the oracle a few minutes.

Sets (chunks of 2 MiB, the remainder last, as ParallelChunkedWriter cuts):

* ``text``    8 MiB text, seed 0 (4 chunks), 128 KiB members;
* ``logs``    the 64 MiB log ustar stream, seed 1 (33 chunks);
* ``binary``  272 MiB mixed binary, seed 2 (136 chunks);
* ``uneven``  the 1,000-file mix, seed 3, each file cut on its own
              (1,245 chunks);
* ``member2m`` one input per generator of 3 x 2 MiB + 12,345 bytes (a tail
              that is no multiple of 4096), with 2 MiB members.

Every digest is checked before it is written: each chunk's stream must
inflate back to the chunk through zlib.

Run from the repository root:  python tests/golden/make_config_digests.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time
import zlib

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gpzip_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "config_digests.json")
CHUNK = 2 << 20
MEMBER = 128 << 10
MEMBER_2M = 2 << 20
THREADS = os.cpu_count() or 1


def sha(b) -> str:
    return hashlib.sha256(memoryview(np.ascontiguousarray(b))).hexdigest()


def inflate_all(gz: bytes) -> bytes:
    out, rest = [], gz
    while rest:
        d = zlib.decompressobj(31)
        out.append(d.decompress(rest))
        if not d.eof:
            raise SystemExit("truncated member in oracle output")
        rest = d.unused_data
    return b"".join(out)


def chunk_set(items, member: int) -> dict:
    digests, lens = [], []
    for it in items:
        gz = O.gzip_chunk(it, member, threads=THREADS)
        if inflate_all(gz) != it.tobytes():
            raise SystemExit("oracle output does not inflate back to its chunk")
        digests.append(hashlib.sha256(gz).hexdigest())
        lens.append(len(gz))
    return {"member_bytes": member, "chunks": len(items), "chunk_sha256": digests, "gzip_len": lens,
            "input_bytes": int(sum(int(x.size) for x in items)), "gzip_bytes": int(sum(lens))}


def chunks_of(data: np.ndarray):
    return [np.ascontiguousarray(data[o:o + n]) for o, n in W.chunk_spans(data.size, CHUNK)]


def uneven_chunks():
    items = []
    for _, _, data in W.uneven_files(1000, seed=3):
        items.extend(chunks_of(data))
    return items


def member2m_inputs():
    n = 3 * CHUNK + 12_345
    return {"text": W.text(n, seed=7), "logs": W.logs(n, seed=8), "binary": W.binary(n, seed=9)}


def main():
    res = {"chunk_bytes": CHUNK, "sets": {}}
    named = {"text": W.config_text, "logs": W.config_logs_tar, "binary": W.config_binary}
    for name, gen in named.items():
        t0 = time.time()
        data = gen()
        e = chunk_set(chunks_of(data), MEMBER)
        e["input_sha256"] = sha(data)
        res["sets"][name] = e
        print(f"{name}: {e['chunks']} chunks, {time.time() - t0:.1f} s", flush=True)
    t0 = time.time()
    items = uneven_chunks()
    e = chunk_set(items, MEMBER)
    e["input_sha256"] = hashlib.sha256(b"".join(sha(x).encode() for x in items)).hexdigest()
    e["input_digest_kind"] = "sha256 over the concatenated hex sha256 of every chunk"
    res["sets"]["uneven"] = e
    print(f"uneven: {e['chunks']} chunks, {time.time() - t0:.1f} s", flush=True)
    m2 = {}
    for name, data in member2m_inputs().items():
        e = chunk_set(chunks_of(data), MEMBER_2M)
        e["input_sha256"] = sha(data)
        m2[name] = e
    res["sets"]["member2m"] = m2
    with open(OUT, "w") as f:
        json.dump(res, f, indent=0, sort_keys=True)
    print(OUT)


if __name__ == "__main__":
    main()
