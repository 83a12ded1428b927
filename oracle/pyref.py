"""Pure-Python restatement of the reference GPU gzip path (TEST INFRASTRUCTURE).

A second, independent restatement of skmtkytr/gpzip's GPU codec arithmetic,
written separately from the C oracle (oracle/gpz_oracle.c) so the two can be
checked against each other on small inputs.  Loops are plain Python: use it for
inputs of a few tens of KiB at most.

Citations are paths inside crates/gpzip-codec-gpu/src/ of the reference.
"""
from __future__ import annotations

import heapq
import zlib

HASH_BITS = 16  # gpu/lz77_hash.rs:43
MIN_MATCH = 3  # gpu/lz77_hash.rs:46
MAX_MATCH = 258  # gpu/lz77_hash.rs:47
WINDOW = 32 * 1024  # gpu/lz77_hash.rs:48
SEG_LOG2 = 12  # gpu/lz77_hash.rs:68
MEMBER_BYTES = 128 * 1024  # gpu.rs:160
META_ORDER = [16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15]  # gpu/deflate.rs:17-19
GZIP_HEADER = bytes([0x1F, 0x8B, 0x08, 0x00, 0, 0, 0, 0, 0x00, 0xFF])  # gpu/deflate.rs:965-972

# RFC 1951 3.2.5 rows (base, extra, symbol): gpu/deflate.rs:99-129, 147-178
LEN_ROWS = [(3, 0, 257), (4, 0, 258), (5, 0, 259), (6, 0, 260), (7, 0, 261), (8, 0, 262),
            (9, 0, 263), (10, 0, 264), (11, 1, 265), (13, 1, 266), (15, 1, 267), (17, 1, 268),
            (19, 2, 269), (23, 2, 270), (27, 2, 271), (31, 2, 272), (35, 3, 273), (43, 3, 274),
            (51, 3, 275), (59, 3, 276), (67, 4, 277), (83, 4, 278), (99, 4, 279), (115, 4, 280),
            (131, 5, 281), (163, 5, 282), (195, 5, 283), (227, 5, 284), (258, 0, 285)]
DIST_ROWS = [(1, 0, 0), (2, 0, 1), (3, 0, 2), (4, 0, 3), (5, 1, 4), (7, 1, 5), (9, 2, 6),
             (13, 2, 7), (17, 3, 8), (25, 3, 9), (33, 4, 10), (49, 4, 11), (65, 5, 12),
             (97, 5, 13), (129, 6, 14), (193, 6, 15), (257, 7, 16), (385, 7, 17), (513, 8, 18),
             (769, 8, 19), (1025, 9, 20), (1537, 9, 21), (2049, 10, 22), (3073, 10, 23),
             (4097, 11, 24), (6145, 11, 25), (8193, 12, 26), (12289, 12, 27), (16385, 13, 28),
             (24577, 13, 29)]


def hash3(b: bytes, p: int) -> int:
    """gpu/lz77_hash_build.wgsl:36-43."""
    x = (b[p] << 16) | (b[p + 1] << 8) | b[p + 2]
    return ((x * 0x9E3779B1) & 0xFFFFFFFF) >> (32 - HASH_BITS)


def match_find(b: bytes) -> list[int]:
    """Per-position packed tokens (length<<16 | dist-or-byte).

    Build: gpu/lz77_hash_build.wgsl:45-54; lookup: gpu/lz77_hash_lookup.wgsl:45-119.
    The [hash][segment] tables are dicts whose missing keys read as the
    sentinels (0xFFFFFFFF for oldest, 0 for newest), which is what the reset at
    gpu/lz77_hash.rs:584-587 leaves in the dense tables.
    """
    n = len(b)
    oldest: dict[tuple[int, int], int] = {}
    newest: dict[tuple[int, int], int] = {}
    for p in range(n):
        if p + 2 >= n:
            break
        key = (hash3(b, p), p >> SEG_LOG2)
        oldest[key] = min(oldest.get(key, 0xFFFFFFFF), p + 1)
        newest[key] = max(newest.get(key, 0), p + 1)

    def try_candidate(raw: int, p: int, cur_best: int):
        if raw == 0 or raw == 0xFFFFFFFF:
            return None
        cand = raw - 1
        if cand >= p:
            return None
        dist = p - cand
        if dist > WINDOW:
            return None
        if b[cand:cand + 3] != b[p:p + 3]:
            return None
        length = 3
        while length < MAX_MATCH and p + length < n and b[cand + length] == b[p + length]:
            length += 1
        return (length, dist) if length > cur_best else None

    out = []
    for p in range(n):
        if p + 2 >= n:
            out.append(b[p])
            continue
        h = hash3(b, p)
        best_len, best_dist = 0, 0
        for seg in range(p >> SEG_LOG2, -1, -1):
            r = try_candidate(newest.get((h, seg), 0), p, best_len)
            if r:
                best_len, best_dist = r
            if best_len >= MAX_MATCH:
                break
            if best_len < 16:
                r = try_candidate(oldest.get((h, seg), 0xFFFFFFFF), p, best_len)
                if r:
                    best_len, best_dist = r
                if best_len >= MAX_MATCH:
                    break
        out.append(b[p] if best_len == 0 else (best_len << 16) | best_dist)
    return out


def brute_lz77(b: bytes, window: int) -> list[int]:
    """gpu/deflate.rs:992-1016 (cpu_lz77 used by the reference encoder tests)."""
    n = len(b)
    out = []
    for pos in range(n):
        best_len = best_dist = 0
        for prev in range(max(0, pos - window), pos):
            length = 0
            while pos + length < n and length < 258 and b[prev + length] == b[pos + length]:
                length += 1
            if length > best_len:
                best_len, best_dist = length, pos - prev
        out.append((best_len << 16) | best_dist if best_len >= 3 else b[pos])
    return out


def greedy_walk(pp: list[int], b: bytes) -> list[int]:
    """gpu/lz77.rs:260-284 (lazy one-step walk)."""
    pp = [int(t) for t in pp]
    out, p, n = [], 0, len(pp)
    while p < n:
        t = pp[p]
        ln = t >> 16
        if ln == 0:
            out.append(t)
            p += 1
            continue
        if p + 1 < n:
            nl = pp[p + 1] >> 16
            if nl != 0 and nl > ln:
                out.append(b[p])
                p += 1
                continue
        out.append(t)
        p += ln
    return out


def reconstruct(tokens: list[int]) -> bytes:
    """gpu/lz77.rs:288-304."""
    tokens = [int(t) for t in tokens]
    out = bytearray()
    for t in tokens:
        ln, lo = t >> 16, t & 0xFFFF
        if ln == 0:
            out.append(lo)
        else:
            start = len(out) - lo
            for i in range(ln):
                out.append(out[start + i])
    return bytes(out)


def _standard_huffman(freq: list[int]) -> list[int]:
    """gpu/huffman.rs:63-117: heap on (freq, id), internal ids from n."""
    n = len(freq)
    heap = [(f, i) for i, f in enumerate(freq) if f > 0]
    heapq.heapify(heap)
    children: dict[int, tuple[int, int]] = {}
    next_id = n
    while len(heap) > 1:
        f1, i1 = heapq.heappop(heap)
        f2, i2 = heapq.heappop(heap)
        children[next_id] = (i1, i2)
        heapq.heappush(heap, (f1 + f2, next_id))
        next_id += 1
    lens = [0] * n
    stack = [(heap[0][1], 0)]
    while stack:
        node, depth = stack.pop()
        if node < n:
            lens[node] = max(depth, 1)
        else:
            l, r = children[node]
            stack.append((l, depth + 1))
            stack.append((r, depth + 1))
    return lens


def build_code_lengths(freq: list[int], max_bits: int):
    """gpu/huffman.rs:26-60 (try_build_code_lengths); None where it returns None."""
    used = [i for i, f in enumerate(freq) if f > 0]
    if not used:
        return [0] * len(freq)
    if len(used) == 1:
        lens = [0] * len(freq)
        lens[used[0]] = 1
        return lens
    if (len(used) - 1).bit_length() > max_bits:  # ceil(log2(used))
        return None
    work = list(freq)
    while True:
        lens = _standard_huffman(work)
        if max(lens) <= max_bits:
            return lens
        work = [f // 2 if f > 1 else f for f in work]


def canonical_codes(lens: list[int]) -> list[int]:
    """gpu/huffman.rs:122-152."""
    mx = max(lens) if lens else 0
    if mx == 0:
        return [0] * len(lens)
    bl = [0] * (mx + 1)
    for l in lens:
        if l:
            bl[l] += 1
    nxt = [0] * (mx + 1)
    code = 0
    for bits in range(1, mx + 1):
        code = (code + bl[bits - 1]) << 1
        nxt[bits] = code
    codes = [0] * len(lens)
    for s, l in enumerate(lens):
        if l:
            codes[s] = nxt[l]
            nxt[l] += 1
    return codes


def _rev(code: int, bits: int) -> int:
    return int(format(code, f"0{bits}b")[::-1], 2) if bits else 0


def _row(rows, v):
    best = rows[0]
    for r in rows:
        if r[0] <= v:
            best = r
        else:
            break
    return best


def _rle(lens: list[int]):
    """gpu/deflate.rs:254-326: (code, extra_bits, extra_value) entries."""
    out, i, n = [], 0, len(lens)
    while i < n:
        cur, run = lens[i], 1
        while i + run < n and lens[i + run] == cur:
            run += 1
        if cur == 0:
            while run >= 11:
                m = min(run, 138)
                out.append((18, 7, m - 11)); run -= m; i += m
            while run >= 3:
                m = min(run, 10)
                out.append((17, 3, m - 3)); run -= m; i += m
            while run > 0:
                out.append((0, 0, 0)); run -= 1; i += 1
        else:
            out.append((cur, 0, 0)); i += 1; run -= 1
            while run >= 3:
                m = min(run, 6)
                out.append((16, 2, m - 3)); run -= m; i += m
            while run > 0:
                out.append((cur, 0, 0)); run -= 1; i += 1
    return out


class _Bits:
    """LSB-first packer (gpu/deflate.rs:697-745)."""

    def __init__(self):
        self.acc = 0
        self.n = 0

    def put(self, value: int, count: int):
        self.acc |= value << self.n
        self.n += count

    def finish(self) -> bytes:
        return self.acc.to_bytes((self.n + 7) // 8, "little") if self.n else b""


def encode_block_fast(tokens: list[int]) -> bytes:
    """gpu/deflate.rs:752-761 -> try_write_dynamic_block_fast (830-959)."""
    tokens = [int(t) for t in tokens]
    lit = [0] * 286
    dist = [0] * 30
    for t in tokens:
        ln, lo = t >> 16, t & 0xFFFF
        if ln == 0:
            lit[lo] += 1
        else:
            lit[_row(LEN_ROWS, ln)[2]] += 1
            dist[_row(DIST_ROWS, lo)[2]] += 1
    lit[256] += 1
    ll = build_code_lengths(lit, 15)
    dl = build_code_lengths(dist, 15)
    if ll is None or dl is None:
        return _encode_fixed(tokens)
    used_d = [i for i, l in enumerate(dl) if l > 0]
    if not used_d:
        dl[0] = dl[1] = 1
    elif len(used_d) == 1:
        only = used_d[0]
        dl[only] = 1
        dl[1 - min(only, 1)] = 1
    if sum(1 for l in ll if l > 0) < 2:
        ll[0] = 1
        ll[256] = 1
    lc, dc = canonical_codes(ll), canonical_codes(dl)
    nlit = 286
    while nlit > 257 and ll[nlit - 1] == 0:
        nlit -= 1
    ndist = 30
    while ndist > 1 and dl[ndist - 1] == 0:
        ndist -= 1
    rle = _rle(ll[:nlit] + dl[:ndist])
    mf = [0] * 19
    for c, _, _ in rle:
        mf[c] += 1
    ml = build_code_lengths(mf, 7)
    if ml is None:
        return _encode_fixed(tokens)
    mc = canonical_codes(ml)
    hclen = 19
    while hclen > 4 and ml[META_ORDER[hclen - 1]] == 0:
        hclen -= 1
    w = _Bits()
    w.put(0b101, 3)
    w.put(nlit - 257, 5)
    w.put(ndist - 1, 5)
    w.put(hclen - 4, 4)
    for i in range(hclen):
        w.put(ml[META_ORDER[i]], 3)
    for c, eb, ev in rle:
        w.put(_rev(mc[c], ml[c]), ml[c])
        if eb:
            w.put(ev, eb)
    for t in tokens:
        ln, lo = t >> 16, t & 0xFFFF
        if ln == 0:
            w.put(_rev(lc[lo], ll[lo]), ll[lo])
        else:
            base, extra, sym = _row(LEN_ROWS, ln)
            w.put(_rev(lc[sym], ll[sym]), ll[sym])
            if extra:
                w.put(ln - base, extra)
            dbase, dextra, dsym = _row(DIST_ROWS, lo)
            w.put(_rev(dc[dsym], dl[dsym]), dl[dsym])
            if dextra:
                w.put(lo - dbase, dextra)
    w.put(_rev(lc[256], ll[256]), ll[256])
    return w.finish()


def _encode_fixed(tokens: list[int]) -> bytes:
    """gpu/deflate.rs:763-799 (unreachable in practice)."""
    def code(sym):
        if sym <= 143:
            return 0x30 + sym, 8
        if sym <= 255:
            return 0x190 + sym - 144, 9
        if sym <= 279:
            return sym - 256, 7
        return 0xC0 + sym - 280, 8

    w = _Bits()
    w.put(0b011, 3)
    for t in tokens:
        ln, lo = t >> 16, t & 0xFFFF
        if ln == 0:
            c, b = code(lo)
            w.put(_rev(c, b), b)
        else:
            base, extra, sym = _row(LEN_ROWS, ln)
            c, b = code(sym)
            w.put(_rev(c, b), b)
            if extra:
                w.put(ln - base, extra)
            dbase, dextra, dsym = _row(DIST_ROWS, lo)
            w.put(_rev(dsym, 5), 5)
            if dextra:
                w.put(lo - dbase, dextra)
    w.put(0, 7)
    return w.finish()


def gzip_wrap(deflate: bytes, original: bytes) -> bytes:
    """gpu/deflate.rs:962-980."""
    crc = zlib.crc32(original) & 0xFFFFFFFF
    return GZIP_HEADER + deflate + crc.to_bytes(4, "little") + (len(original) & 0xFFFFFFFF).to_bytes(4, "little")


def gzip_member(b: bytes) -> bytes:
    """gpu.rs:271-287 (encode_one) for one member."""
    toks = greedy_walk(match_find(b), b) if b else []
    return gzip_wrap(encode_block_fast(toks), b)


def gzip_chunk(b: bytes, member_bytes: int = MEMBER_BYTES) -> bytes:
    """gpu.rs:193-208 (gzip_chunk_fn)."""
    if len(b) <= member_bytes:
        return gzip_member(b)
    return b"".join(gzip_member(b[i:i + member_bytes]) for i in range(0, len(b), member_bytes))
