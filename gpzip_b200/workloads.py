"""Seeded synthetic workloads for the gzip compression path.

The reference measures on harvested corpora that are not available here, so
these generators stand in for them with the shapes, sizes and value
distributions the benchmark configurations name:

* ``text``   -- English-like text: 5,000-word seeded vocabulary, word lengths
  geometric with mean 5, letters a-z, Zipf(1.1) word frequencies, spaces,
  a newline every 60-100 characters, punctuation with p = 0.05.
* ``logs``   -- ``YYYY-MM-DDTHH:MM:SS.ffffff host-NN svc[PID]: <template>``
  lines: 200 templates with 0-4 integer/hex/IPv4 fields, templates Zipf(1.3),
  exponential timestamp gaps with mean 2 ms, PIDs from a pool of 50.  The
  64 MiB log config is wrapped as a one-file ustar stream (512-byte header,
  the data, 1,024 bytes of end-of-archive zeros).
* ``binary`` -- 64 KiB regions: 35% uniform random bytes, 25% runs of zero or
  one byte value (lengths 16-4096), 25% copies of earlier 8-512-byte spans at
  distances 1-32768, 15% bytes i.i.d. from a seeded Zipf(1.0) 256-entry table.
* ``uneven`` -- 1,000 files with log-uniform sizes 1 KiB-8 MiB, each from one
  of the three generators (equal thirds).
* ``serving`` -- Poisson arrivals with log-uniform request sizes 4 KiB-16 MiB.

Everything is numpy PCG64 with fixed seeds, so every run sees the same bytes;
``digest`` gives a SHA-256 for the record.
"""
from __future__ import annotations

import hashlib

import numpy as np

MiB = 1 << 20
KiB = 1 << 10
CHUNK_BYTES = 2 * MiB

_LETTERS = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz", dtype=np.uint8)
_PUNCT = np.frombuffer(b".,;:!?", dtype=np.uint8)


def digest(data) -> str:
    return hashlib.sha256(memoryview(np.ascontiguousarray(data))).hexdigest()


def _zipf_p(n: int, s: float) -> np.ndarray:
    p = 1.0 / np.arange(1, n + 1, dtype=np.float64) ** s
    return p / p.sum()


def _scatter_pieces(pieces_off: np.ndarray, pieces_len: np.ndarray, src: np.ndarray) -> np.ndarray:
    """Concatenate src[off:off+len] for each piece, vectorised."""
    total = int(pieces_len.sum())
    starts = np.cumsum(pieces_len) - pieces_len
    idx = np.repeat(pieces_off - starts, pieces_len) + np.arange(total, dtype=np.int64)
    return src[idx]


def text(nbytes: int, seed: int = 0) -> np.ndarray:
    """English-like text of exactly nbytes bytes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    vocab_len = rng.geometric(0.2, size=5000).astype(np.int64)
    vocab_bytes = _LETTERS[rng.integers(0, 26, size=int(vocab_len.sum()))]
    vocab_off = np.cumsum(vocab_len) - vocab_len
    p = _zipf_p(5000, 1.1)
    out_parts = []
    have = 0
    col = 0  # characters already on the current line when a batch starts
    target = int(rng.integers(60, 101))
    while have < nbytes:
        nw = max(1024, (nbytes - have) // 5 + 1024)
        w = rng.choice(5000, size=nw, p=p)
        wl = vocab_len[w]
        punct = rng.random(nw) < 0.05
        pch = _PUNCT[rng.integers(0, 6, size=nw)]
        # piece = word [+ punctuation] + separator
        piece_len = wl + punct + 1
        ends = np.cumsum(piece_len)
        total = int(ends[-1])
        buf = np.empty(total, dtype=np.uint8)
        word_start = ends - piece_len
        widx = np.repeat(word_start - (np.cumsum(wl) - wl), wl) + np.arange(int(wl.sum()),
                                                                           dtype=np.int64)
        buf[widx] = _scatter_pieces(vocab_off[w], wl, vocab_bytes)
        buf[(word_start + wl)[punct]] = pch[punct]
        sep_pos = ends - 1
        buf[sep_pos] = ord(" ")
        # a newline every U[60,100] characters, at the first separator at or
        # past the target column
        line_start = -col
        while True:
            k = int(np.searchsorted(sep_pos, line_start + target, side="left"))
            if k >= sep_pos.size:
                break
            buf[sep_pos[k]] = ord("\n")
            line_start = int(sep_pos[k]) + 1
            target = int(rng.integers(60, 101))
        col = total - line_start
        out_parts.append(buf)
        have += total
    return np.concatenate(out_parts)[:nbytes]


_SERVICES = ["auth", "api", "db", "cache", "queue", "sched", "web", "mail", "dns", "proxy",
             "store", "search"]
_LOG_WORDS = ("request completed failed started connection closed opened user session token "
              "retry timeout upstream downstream latency bytes sent received error warning ok "
              "client server handshake cache miss hit flush commit rollback query rows worker "
              "job queued dequeued heartbeat lease renewed expired shard replica primary").split()


def _log_templates(rng: np.random.Generator):
    temps = []
    for _ in range(200):
        svc = _SERVICES[int(rng.integers(0, len(_SERVICES)))]
        nwords = int(rng.integers(3, 11))
        words = [_LOG_WORDS[int(i)] for i in rng.integers(0, len(_LOG_WORDS), size=nwords)]
        nfields = int(rng.integers(0, 5))
        kinds = [int(k) for k in rng.integers(0, 3, size=nfields)]  # 0 int, 1 hex, 2 ipv4
        slots = sorted(int(s) for s in rng.integers(0, nwords + 1, size=nfields))
        parts, fi = [], 0
        for wi in range(nwords + 1):
            while fi < nfields and slots[fi] == wi:
                parts.append(("f", kinds[fi]))
                fi += 1
            if wi < nwords:
                parts.append(("w", words[wi]))
        temps.append((svc, parts))
    return temps


def logs(nbytes: int, seed: int = 1) -> np.ndarray:
    """Log lines of exactly nbytes bytes (the last line is cut)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    temps = _log_templates(rng)
    p = _zipf_p(200, 1.3)
    pids = rng.integers(100, 65536, size=50)
    t_us = 1_700_000_000 * 1_000_000  # fixed epoch start
    out = []
    have = 0
    import datetime as _dt
    epoch = _dt.datetime(1970, 1, 1)
    while have < nbytes:
        m = 20000
        tid = rng.choice(200, size=m, p=p)
        gaps = rng.exponential(2000.0, size=m).astype(np.int64) + 1
        hosts = rng.integers(0, 32, size=m)
        pidx = rng.integers(0, 50, size=m)
        fvals = rng.integers(0, 1 << 32, size=(m, 4), dtype=np.uint64)
        lines = []
        for i in range(m):
            t_us += int(gaps[i])
            sec, us = divmod(t_us, 1_000_000)
            ts = (epoch + _dt.timedelta(seconds=sec)).strftime("%Y-%m-%dT%H:%M:%S")
            svc, parts = temps[int(tid[i])]
            msg, fi = [], 0
            for kind, val in parts:
                if kind == "w":
                    msg.append(val)
                else:
                    v = int(fvals[i, fi])
                    fi += 1
                    if val == 0:
                        msg.append(str(v % 100000))
                    elif val == 1:
                        msg.append(f"0x{v:08x}")
                    else:
                        msg.append(f"{v >> 24 & 255}.{v >> 16 & 255}.{v >> 8 & 255}.{v & 255}")
            lines.append(f"{ts}.{us:06d} host-{int(hosts[i]):02d} {svc}[{int(pids[pidx[i]])}]: "
                         f"{' '.join(msg)}\n")
        blob = "".join(lines).encode()
        out.append(np.frombuffer(blob, dtype=np.uint8))
        have += len(blob)
    return np.concatenate(out)[:nbytes]


def ustar(name: str, payload: np.ndarray) -> np.ndarray:
    """One-file ustar stream: 512-byte header, payload padded to 512, 1,024 zero bytes."""
    hdr = bytearray(512)
    nb = name.encode()[:99]
    hdr[0:len(nb)] = nb
    hdr[100:108] = b"0000644\0"
    hdr[108:116] = b"0000000\0"
    hdr[116:124] = b"0000000\0"
    hdr[124:136] = f"{payload.size:011o}\0".encode()
    hdr[136:148] = b"00000000000\0"
    hdr[156:157] = b"0"
    hdr[257:263] = b"ustar\0"
    hdr[263:265] = b"00"
    hdr[148:156] = b"        "
    chk = sum(hdr)
    hdr[148:156] = f"{chk:06o}\0 ".encode()
    pad = (-payload.size) % 512
    return np.concatenate([np.frombuffer(bytes(hdr), dtype=np.uint8), payload,
                           np.zeros(pad + 1024, dtype=np.uint8)])


def binary(nbytes: int, seed: int = 2) -> np.ndarray:
    """Mixed-entropy binary in 64 KiB regions."""
    rng = np.random.Generator(np.random.PCG64(seed))
    region = 64 * KiB
    nreg = -(-nbytes // region)
    out = np.empty(nreg * region, dtype=np.uint8)
    kinds = rng.choice(4, size=nreg, p=[0.35, 0.25, 0.25, 0.15])
    zipf_table = rng.permutation(256).astype(np.uint8)
    zp = _zipf_p(256, 1.0)
    for r in range(nreg):
        base = r * region
        k = int(kinds[r])
        if k == 0:
            out[base:base + region] = rng.integers(0, 256, size=region, dtype=np.uint8)
        elif k == 1:
            pos = 0
            while pos < region:
                ln = int(rng.integers(16, 4097))
                val = 0 if rng.random() < 0.5 else int(rng.integers(0, 256))
                end = min(region, pos + ln)
                out[base + pos:base + end] = val
                pos = end
        elif k == 2:
            pos = 0
            if base == 0:  # nothing earlier to copy: seed with random bytes
                out[0:4096] = rng.integers(0, 256, size=4096, dtype=np.uint8)
                pos = 4096
            while pos < region:
                ln = int(rng.integers(8, 513))
                dist = int(rng.integers(1, 32769))
                at = base + pos
                dist = min(dist, at)
                end = min(region, pos + ln)
                ln = end - pos
                src = at - dist
                if dist >= ln:
                    out[at:at + ln] = out[src:src + ln]
                else:
                    pat = out[src:at]
                    reps = -(-ln // dist)
                    out[at:at + ln] = np.tile(pat, reps)[:ln]
                pos = end
        else:
            out[base:base + region] = zipf_table[rng.choice(256, size=region, p=zp)]
    return out[:nbytes]


GENERATORS = {"text": text, "logs": logs, "binary": binary}


def config_text() -> np.ndarray:
    """8 MiB text, seed 0 (4 chunks of 2 MiB)."""
    return text(8 * MiB, seed=0)


def config_logs_tar() -> np.ndarray:
    """64 MiB of log lines, seed 1, as a one-file ustar stream (32 full chunks + tail)."""
    return ustar("logs.txt", logs(64 * MiB, seed=1))


def config_binary() -> np.ndarray:
    """272 MiB mixed-entropy binary, seed 2 (136 chunks)."""
    return binary(272 * MiB, seed=2)


def uneven_files(count: int = 1000, seed: int = 3, scale: float = 1.0):
    """(name, kind, bytes) for the uneven-size file mix.

    Sizes are log-uniform in [1 KiB, 8 MiB]; kinds cycle text/logs/binary in a
    seeded shuffle with equal thirds.  ``scale`` < 1 shrinks every file (for
    quick tests) while keeping the size distribution's shape.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = np.exp(rng.uniform(np.log(KiB), np.log(8 * MiB), size=count)).astype(np.int64)
    sizes = np.maximum(1, (sizes * scale).astype(np.int64))
    kinds = np.array(["text", "logs", "binary"] * (count // 3 + 1))[:count]
    rng.shuffle(kinds)
    seeds = rng.integers(0, 2**31, size=count)
    # generate each kind once as a long stream and cut files from it at
    # seeded offsets: identical statistics, far less generator overhead
    need = {k: int(sizes[kinds == k].max(initial=0)) for k in GENERATORS}
    pools = {}
    for k, gen in GENERATORS.items():
        pool_size = max(need[k] * 4, 32 * MiB) if need[k] else 0
        pools[k] = gen(pool_size, seed=seed * 100 + list(GENERATORS).index(k)) if pool_size else None
    files = []
    for i in range(count):
        k = str(kinds[i])
        pool = pools[k]
        off = int(np.random.Generator(np.random.PCG64(int(seeds[i]))).integers(
            0, pool.size - sizes[i] + 1))
        files.append((f"file{i:04d}.{k}", k, pool[off:off + int(sizes[i])]))
    return files


def chunk_spans(nbytes: int, chunk: int = CHUNK_BYTES):
    """(offset, length) chunks of at most `chunk` bytes, the remainder last."""
    return [(o, min(chunk, nbytes - o)) for o in range(0, nbytes, chunk)]


def serving_arrivals(rate: float, seconds: float, seed: int = 4, min_size: int = 4 * KiB,
                     max_size: int = 16 * MiB):
    """Poisson arrival times (s), log-uniform sizes and content kinds."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = int(rate * seconds * 1.2) + 16
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    t = t[t < seconds]
    m = t.size
    sizes = np.exp(rng.uniform(np.log(min_size), np.log(max_size), size=m)).astype(np.int64)
    kinds = rng.integers(0, 3, size=m)
    offs = rng.random(m)
    return t, sizes, kinds, offs
