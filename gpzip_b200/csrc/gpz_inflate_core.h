// gpz_inflate_core.h -- RFC 1951 decoder for one gzip member, written once
// for two builds:
//   * CUDA (NL = 32): one warp decodes one member.  Every lane runs the same
//     decode on the same data (lane-uniform control flow), and the lanes
//     share the wide work: staging input, filling lookup tables, copying
//     matches and flushing output.
//   * host C++ (NL = 1): the same code on one thread, which the CPU tests
//     check against zlib.
// The decoder writes bytes, or (the token form) the member's tokens, which
// the device expands into bytes in a kernel of its own.  The second half of
// this file holds the parallel decode of a member that is one dynamic block
// (decode_span and its helpers; inflate_member_par runs its steps on the
// host for the tests), which the device uses for gpzip's members.
//
// It replaces, for gpzip-written archives, the per-member GzDecoder of
// crates/gpzip-codec-cpu/src/parallel_decompress.rs:63-113 (flate2).  The
// decoder follows RFC 1951 directly: block types 0 (stored), 1 (fixed) and
// 2 (dynamic), canonical Huffman codes (RFC 1951 3.2.2), the code-length
// alphabet and its repeat codes 16/17/18 (3.2.7), and the length / distance
// tables of 3.2.5.  It checks what zlib's inflate checks and reports, never
// writes outside the member's output range, and never reads outside its
// input range: every failure is a status code.
#pragma once

#include <stdint.h>

#if defined(GPZI_HOST_LANES)
#include <barrier>
#endif

#if defined(__CUDACC__)
#define GPZI_FN __host__ __device__ __forceinline__
#else
#define GPZI_FN inline
#endif

namespace gpzi {

constexpr uint32_t kRing = 32768;   // window ring of the last 32 KiB of output
constexpr uint32_t kStage = 4096;   // input bytes staged at a time
constexpr uint32_t kFlush = 4096;   // output flushed to its destination in steps of this
constexpr int kFastBits = 9;        // first-level table index width

// status codes of one member
enum : uint32_t {
    kOk = 0,
    kErrBlockType = 1,   // block type 3
    kErrStoredLen = 2,   // LEN != ~NLEN
    kErrCodeLens = 3,    // bad code-length code or repeat
    kErrCodeSet = 4,     // over-subscribed or incomplete code
    kErrSymbol = 5,      // a code that no symbol has, or litlen 286/287, dist 30/31
    kErrDistance = 6,    // distance beyond the start of the member
    kErrOutput = 7,      // output longer than ISIZE
    kErrInput = 8,       // ran past the end of the member's deflate bytes
    kErrLength = 9,      // output shorter than ISIZE
    kErrTrailing = 10,   // deflate data ends before the trailer
    kErrCrc = 11,        // CRC-32 differs from the trailer (set by the CRC pass)
    kErrEmptyLen = 12,   // a table without any code is used
};

// Decoded entries carry what the decoder needs next, so it never maps a
// symbol again: bits 0-3 code length (fast table; 0 = not in the fast
// table), bits 4-5 kind, then per table kind
//   litlen:  kind 0 literal (byte in bits 8-15), 1 length (base in bits
//            8-16, extra bits in 17-19), 2 end of block, 3 invalid (286, 287)
//   dist:    kind 0 (base in bits 8-22, extra bits in 24-27), 3 invalid (30, 31)
//   meta:    kind 0, the code-length symbol in bits 8-15
enum : uint32_t { kTabMeta = 0, kTabLit = 1, kTabDist = 2 };
struct Table {
    uint32_t fast[1 << kFastBits];  // entries of codes of <= kFastBits bits, 0 otherwise
    uint16_t count[16];             // codes of each length
    uint16_t sym[320];              // symbols ordered by (length, value)
};

// The ring comes last: the token form (TOK) never touches it, and its
// kernel allocates only the bytes before it (kSharedTokBytes).
struct Shared {
    alignas(4) uint8_t stage[kStage + 16];
    Table lit, dist;
    uint8_t lens[320];
    uint32_t bcast;  // a value lane 0 computed, for every lane
    uint8_t ring[kRing];
};
constexpr size_t kSharedTokBytes = sizeof(Shared) - kRing;

#if defined(GPZI_HOST_LANES)
// Host test build with NL host threads standing in for the lanes of a warp
// (tests/c/inflate_lanes.cpp): lane_sync is a barrier across them.
inline std::barrier<>* g_lanes = nullptr;
#endif

GPZI_FN void lane_sync() {
#if defined(__CUDA_ARCH__)
    __syncwarp();
#elif defined(GPZI_HOST_LANES)
    g_lanes->arrive_and_wait();
#endif
}

// Lane-uniform bit reader over the member's deflate bytes src[0, len).
// Input is staged kStage + 16 bytes at a time by all lanes (zeros past
// len).  Bits of buf at and above cnt are always the stream's next bits (or
// zero), so a refill may OR the next eight bytes in at cnt (libdeflate's
// branch-free refill).  Reading past the end yields zeros; the loops stop
// once pos is more than 8 bytes past len, and the exact check at the end
// catches a smaller overrun.
template <int NL>
struct Bits {
    const uint8_t* src;
    uint32_t len;
    uint32_t pos;   // next input byte not yet counted in cnt
    uint64_t buf;
    uint32_t cnt;   // valid bits in buf
    uint32_t lane;
    uint32_t base;  // input offset of s.stage[0], a multiple of 4

    GPZI_FN void restage(Shared& s, uint32_t p) {
        lane_sync();  // every lane is done with the old stage
        base = p & ~3u;
        for (uint32_t k = lane; k < kStage + 16; k += NL)
            s.stage[k] = base + k < len ? src[base + k] : (uint8_t)0;
        lane_sync();
    }
    // afterwards at least 56 bits are valid
    GPZI_FN void refill(Shared& s) {
        if (pos - base > kStage) restage(s, pos);
        const uint32_t off = pos - base, i = off >> 2, sh = (off & 3u) * 8u;
        const uint32_t* w = reinterpret_cast<const uint32_t*>(s.stage);
        uint64_t v = ((uint64_t)w[i + 1] << 32 | w[i]) >> sh;
        if (sh) v |= (uint64_t)w[i + 2] << (64u - sh);
        buf |= v << cnt;
        const uint32_t nb = (63u - cnt) >> 3;
        pos += nb;
        cnt += nb * 8u;
    }
    GPZI_FN uint32_t peek(uint32_t n) const { return (uint32_t)(buf & ((1ull << n) - 1ull)); }
    GPZI_FN void drop(uint32_t n) {
        buf >>= n;
        cnt -= n;
    }
    GPZI_FN uint32_t take(Shared& s, uint32_t n) {  // n <= 32
        if (cnt < n) refill(s);
        const uint32_t v = peek(n);
        drop(n);
        return v;
    }
    // bits consumed so far, padding included
    GPZI_FN uint64_t consumed() const { return 8ull * pos - cnt; }
    GPZI_FN bool overrun() const { return consumed() > 8ull * len; }
    GPZI_FN bool far_past_end() const { return pos > len + 8u; }
};

struct LenDist {
    uint32_t base;
    uint32_t extra;
};
// RFC 1951 3.2.5 by arithmetic (no tables): length symbol 257 + i
GPZI_FN LenDist len_row(uint32_t i) {
    if (i >= 28u) return LenDist{258u, 0u};
    if (i < 8u) return LenDist{i + 3u, 0u};
    const uint32_t e = (i >> 2) - 1u;
    return LenDist{((4u + (i & 3u)) << e) + 3u, e};
}
// distance code i (0..29)
GPZI_FN LenDist dist_row(uint32_t i) {
    if (i < 4u) return LenDist{i + 1u, 0u};
    const uint32_t e = (i >> 1) - 1u;
    return LenDist{((2u + (i & 1u)) << e) + 1u, e};
}
// position i of the code-length code lengths: 16, 17, 18, 0, 8, 7, 9, 6, ...
GPZI_FN uint32_t meta_order(uint32_t i) {
    if (i < 3u) return 16u + i;
    if (i == 3u) return 0u;
    const uint32_t k = i - 4u;
    return (k & 1u) ? 7u - (k >> 1) : 8u + (k >> 1);
}

GPZI_FN uint32_t pack_entry(uint32_t kind, uint32_t sym, uint32_t l) {
    if (kind == kTabLit) {
        if (sym < 256u) return l | (sym << 8);
        if (sym == 256u) return l | (2u << 4);
        if (sym > 285u) return l | (3u << 4);
        const LenDist r = len_row(sym - 257u);
        return l | (1u << 4) | (r.base << 8) | (r.extra << 17);
    }
    if (kind == kTabDist) {
        if (sym > 29u) return l | (3u << 4);
        const LenDist r = dist_row(sym);
        return l | (r.base << 8) | (r.extra << 24);
    }
    return l | (sym << 8);
}

// Builds t from code lengths lens[0, n): counts, the symbols in canonical
// order (lane 0), then the first-level table (all lanes).  As zlib's
// inflate_table: an over-subscribed code is an error, and so is an
// incomplete one, except for a single code of length 1 in the litlen and
// distance codes (meta = false); a code with no symbols at all is accepted
// (empty = true) and fails only when used.
template <int NL>
GPZI_FN uint32_t build_table(Shared& s, Table& t, uint32_t kind, const uint8_t* lens, uint32_t n, uint32_t lane,
                             bool& empty) {
    const bool meta = kind == kTabMeta;
    if (lane == 0) {
        uint32_t st = kOk;
        uint16_t offs[16];
        for (int i = 0; i < 16; i++) t.count[i] = 0;
        for (uint32_t i = 0; i < n; i++) t.count[lens[i]]++;
        int left = 1, maxlen = 0;  // codes of the current length still unassigned
        for (int l = 1; l < 16; l++) {
            if (t.count[l]) maxlen = l;
            if (left < 0) continue;
            left = 2 * left - t.count[l];
            if (left < 0) st = kErrCodeSet;
        }
        if (st == kOk && left > 0 && maxlen > 0 && (meta || maxlen > 1)) st = kErrCodeSet;
        offs[1] = 0;
        for (int l = 1; l < 15; l++) offs[l + 1] = (uint16_t)(offs[l] + t.count[l]);
        if (st == kOk)
            for (uint32_t i = 0; i < n; i++)
                if (lens[i]) t.sym[offs[lens[i]]++] = (uint16_t)i;
        t.count[0] = 0;
        s.bcast = st;
    }
    lane_sync();
    const uint32_t st = s.bcast;
    uint32_t total = 0;
    for (int l = 1; l < 16; l++) total += t.count[l];
    empty = total == 0;
    if (st != kOk) {
        lane_sync();
        return st;
    }
    // first-level entries: index = the next kFastBits stream bits (first
    // stream bit in bit 0); canonical walk over at most kFastBits lengths
    for (uint32_t idx = lane; idx < (1u << kFastBits); idx += NL) {
        uint32_t code = 0, first = 0, index = 0, e = 0;
        for (uint32_t l = 1; l <= (uint32_t)kFastBits; l++) {
            code |= (idx >> (l - 1)) & 1u;
            const uint32_t c = t.count[l];
            if (code - first < c) {
                e = pack_entry(kind, t.sym[index + code - first], l);
                break;
            }
            index += c;
            first += c;
            first <<= 1;
            code <<= 1;
        }
        t.fast[idx] = e;
    }
    lane_sync();
    return kOk;
}

// One code's entry (see Table); refills so that at least 15 bits are
// available.  Codes longer than kFastBits are walked length by length
// (RFC 1951 3.2.2).
template <int NL>
GPZI_FN uint32_t decode_entry(Shared& s, Bits<NL>& b, const Table& t, uint32_t kind, uint32_t& err) {
    if (b.cnt < 15) b.refill(s);
    const uint32_t e = t.fast[b.peek(kFastBits)];
    if (e) {
        b.drop(e & 15u);
        return e;
    }
    uint32_t code = 0, first = 0, index = 0;
    for (uint32_t l = 1; l < 16; l++) {
        code |= (uint32_t)(b.buf >> (l - 1)) & 1u;
        const uint32_t c = t.count[l];
        if (code - first < c) {
            b.drop(l);
            return pack_entry(kind, t.sym[index + code - first], 0u);
        }
        index += c;
        first += c;
        first <<= 1;
        code <<= 1;
    }
    err = kErrSymbol;
    return 0;
}


// Output state: bytes [0, o) of the member are produced, [0, flushed) of
// them already copied to dst; the ring holds the last kRing bytes.  In the
// token form (TOK) nothing is copied: every literal and match goes to
// tok[nt++] instead (a literal as its byte, a match as length << 16 |
// distance), and expand_tokens or the device's expansion kernel makes the
// bytes later.
template <int NL, bool TOK>
struct Out {
    uint8_t* dst;
    uint32_t cap;  // ISIZE
    uint32_t o;
    uint32_t flushed;
    uint32_t lane;
    uint32_t* tok;
    uint32_t nt;

    GPZI_FN void flush(Shared& s, uint32_t upto) {
        if constexpr (!TOK) {
            lane_sync();
            for (uint32_t k = flushed + lane; k < upto; k += NL) dst[k] = s.ring[k & (kRing - 1)];
            flushed = upto;
        }
    }
    GPZI_FN void maybe_flush(Shared& s) {
        if constexpr (!TOK)
            if (o - flushed >= kFlush) flush(s, flushed + kFlush);
    }
};

// The bytes of a token stream (serial; the host check of the token form).
GPZI_FN void expand_tokens(const uint32_t* tok, uint32_t nt, uint8_t* dst) {
    uint32_t o = 0;
    for (uint32_t i = 0; i < nt; i++) {
        const uint32_t v = tok[i], l = v >> 16;
        if (!l) {
            dst[o++] = (uint8_t)v;
            continue;
        }
        const uint32_t d = v & 0xFFFFu;
        for (uint32_t q = 0; q < l; q++) dst[o + q] = dst[o - d + q];
        o += l;
    }
}

// The code tables of one block into s.lit and s.dist: the fixed codes for
// type 1 (RFC 1951 3.2.6), the codes of the header read from b for type 2
// (3.2.7).  Returns a status; lit_empty / dist_empty tell whether a table
// has no code at all (an error only once it is used).
template <int NL>
GPZI_FN uint32_t read_block_tables(Shared& s, Bits<NL>& b, uint32_t lane, uint32_t type, bool& lit_empty,
                                   bool& dist_empty) {
    uint32_t err = kOk;
    if (type == 1) {
        lane_sync();
        if (lane == 0) {
            for (int i = 0; i < 144; i++) s.lens[i] = 8;
            for (int i = 144; i < 256; i++) s.lens[i] = 9;
            for (int i = 256; i < 280; i++) s.lens[i] = 7;
            for (int i = 280; i < 288; i++) s.lens[i] = 8;
            for (int i = 288; i < 320; i++) s.lens[i] = 5;
        }
        lane_sync();
        build_table<NL>(s, s.lit, kTabLit, s.lens, 288, lane, lit_empty);
        build_table<NL>(s, s.dist, kTabDist, s.lens + 288, 32, lane, dist_empty);
    } else {
        const uint32_t hlit = b.take(s, 5) + 257, hdist = b.take(s, 5) + 1, hclen = b.take(s, 4) + 4;
        lane_sync();
        if (lane == 0)
            for (int i = 0; i < 19; i++) s.lens[i] = 0;
        for (uint32_t i = 0; i < hclen; i++) {
            const uint32_t v = b.take(s, 3);
            if (lane == 0) s.lens[meta_order(i)] = (uint8_t)v;
        }
        lane_sync();
        if (hlit > 286 || hdist > 30) {
            return kErrCodeLens;
        }
        bool cl_empty = false;
        if (build_table<NL>(s, s.lit, kTabMeta, s.lens, 19, lane, cl_empty) != kOk || cl_empty) {
            return kErrCodeLens;
        }
        // the litlen and distance code lengths as one sequence (3.2.7)
        uint32_t i = 0, prev = 0;
        const uint32_t nl = hlit + hdist;
        while (i < nl) {
            const uint32_t sym = (decode_entry<NL>(s, b, s.lit, kTabMeta, err) >> 8) & 255u;
            if (err) return err;
            uint32_t rep = 1, val = sym;
            if (sym == 16) {
                if (i == 0) {
                    return kErrCodeLens;
                }
                val = prev;
                rep = 3 + b.take(s, 2);
            } else if (sym == 17) {
                val = 0;
                rep = 3 + b.take(s, 3);
            } else if (sym == 18) {
                val = 0;
                rep = 11 + b.take(s, 7);
            }
            if (i + rep > nl) {
                return kErrCodeLens;
            }
            lane_sync();
            if (lane == 0)
                for (uint32_t r = 0; r < rep; r++) s.lens[i + r] = (uint8_t)val;
            lane_sync();
            prev = val;
            i += rep;
        }
        if (err) return err;
        if (b.far_past_end()) {
            return kErrInput;
        }
        if (s.lens[256] == 0) {  // no end-of-block code
            return kErrCodeLens;
        }
        // distance lengths moved to s.lens[288, 318) (from the top down:
        // the ranges may overlap and the target lies above), litlen
        // lengths stay in s.lens[0, hlit)
        if (lane == 0) {
            for (uint32_t q = 30; q-- > 0;) s.lens[288 + q] = q < hdist ? s.lens[hlit + q] : (uint8_t)0;
            s.lens[318] = s.lens[319] = 0;
        }
        lane_sync();
        if (build_table<NL>(s, s.lit, kTabLit, s.lens, hlit, lane, lit_empty) != kOk ||
            build_table<NL>(s, s.dist, kTabDist, s.lens + 288, 30, lane, dist_empty) != kOk) {
            return kErrCodeSet;
        }
    }
    return kOk;
}

// Decodes one member's deflate data src[0, len) into dst[0, isize), or, in
// the token form (TOK), into its tokens tok[0, *ntok) (at most isize of
// them; dst is not written).  Returns a status code; on kOk exactly isize
// bytes were produced and the data ended exactly at len.  Both forms make
// the same checks and return the same status.
template <int NL, bool TOK = false>
GPZI_FN uint32_t inflate_member(Shared& s, uint32_t lane, const uint8_t* src, uint32_t len, uint8_t* dst,
                                uint32_t isize, uint32_t* tok = nullptr, uint32_t* ntok = nullptr) {
    Bits<NL> b{src, len, 0u, 0ull, 0u, lane, 0u};
    Out<NL, TOK> out{dst, isize, 0u, 0u, lane, tok, 0u};
    b.restage(s, 0);
    uint32_t err = kOk;
    bool last = false;
    // every block consumes at least 3 bits and every symbol at least 1, and
    // past the end of the input the reader yields zero bits and the
    // overrun checks stop the loops
    while (!last && err == kOk) {
        if (b.far_past_end()) {
            err = kErrInput;
            break;
        }
        last = b.take(s, 1) != 0;
        const uint32_t type = b.take(s, 2);
        if (type == 0) {
            // stored: to a byte boundary, LEN, NLEN, then LEN raw bytes
            b.drop(b.cnt & 7u);
            const uint32_t ln = b.take(s, 16), nl = b.take(s, 16);
            if ((ln ^ 0xFFFFu) != nl) {
                err = kErrStoredLen;
                break;
            }
            if (out.o + ln > out.cap) {
                err = kErrOutput;
                break;
            }
            // whole bytes still in the bit buffer come first
            uint32_t k = 0;
            for (; k < ln && b.cnt >= 8; k++) {
                if (lane == 0) {
                    if constexpr (TOK) out.tok[out.nt + k] = (uint32_t)b.peek(8);
                    else s.ring[(out.o + k) & (kRing - 1)] = (uint8_t)b.peek(8);
                }
                b.drop(8);
            }
            out.o += k;
            out.nt += k;
            // then straight from the input, at most kFlush / 2 bytes a round
            // so that the unflushed part always fits the ring; the bit
            // buffer is empty and its look-ahead stale from here
            if (k < ln) b.buf = 0;
            while (k < ln) {
                const uint32_t step = ln - k < kFlush / 2 ? ln - k : kFlush / 2;
                lane_sync();
                for (uint32_t q = lane; q < step; q += NL) {
                    const uint32_t p = b.pos + q;
                    const uint8_t v = p < len ? src[p] : (uint8_t)0;
                    if constexpr (TOK) out.tok[out.nt + q] = v;
                    else s.ring[(out.o + q) & (kRing - 1)] = v;
                }
                b.pos += step;
                k += step;
                out.o += step;
                out.nt += step;
                out.maybe_flush(s);
            }
            if (b.overrun()) err = kErrInput;
            out.maybe_flush(s);
            continue;
        }
        if (type == 3) {
            err = kErrBlockType;
            break;
        }
        bool lit_empty = false, dist_empty = false;
        err = read_block_tables<NL>(s, b, lane, type, lit_empty, dist_empty);
        if (err) break;
        // symbols up to the end of the block
        for (;;) {
            if (b.far_past_end()) {
                err = kErrInput;
                break;
            }
            const uint32_t e = decode_entry<NL>(s, b, s.lit, kTabLit, err);
            if (err) break;
            const uint32_t kind = (e >> 4) & 3u;
            if (kind == 0u) {
                if (out.o >= out.cap) {
                    err = kErrOutput;
                    break;
                }
                if constexpr (TOK) {
                    if (lane == 0) out.tok[out.nt] = (e >> 8) & 0xFFu;
                    out.nt++;
                } else {
                    s.ring[out.o & (kRing - 1)] = (uint8_t)(e >> 8);  // every lane, the same byte
                }
                out.o++;
                out.maybe_flush(s);
                continue;
            }
            if (kind == 2u) break;
            if (kind == 3u) {
                err = kErrSymbol;
                break;
            }
            const uint32_t lx = (e >> 17) & 7u;
            const uint32_t mlen = ((e >> 8) & 511u) + (lx ? b.take(s, lx) : 0u);
            if (dist_empty) {
                err = kErrEmptyLen;
                break;
            }
            const uint32_t de = decode_entry<NL>(s, b, s.dist, kTabDist, err);
            if (err) break;
            if (((de >> 4) & 3u) == 3u) {
                err = kErrSymbol;
                break;
            }
            const uint32_t dx = (de >> 24) & 15u;
            const uint32_t d = ((de >> 8) & 0x7FFFu) + (dx ? b.take(s, dx) : 0u);
            if (d > out.o) {
                err = kErrDistance;
                break;
            }
            if (out.o + mlen > out.cap) {
                err = kErrOutput;
                break;
            }
            if constexpr (TOK) {
                if (lane == 0) out.tok[out.nt] = (mlen << 16) | d;
                out.nt++;
            } else if (d >= NL && d <= kRing - NL) {
                // byte o + k = byte o + k - d, which precedes this step of
                // NL bytes, and no write of a step hits a slot that the same
                // step reads
                for (uint32_t k0 = 0; k0 < mlen; k0 += NL) {
                    const uint32_t k = k0 + lane;
                    lane_sync();
                    if (k < mlen) s.ring[(out.o + k) & (kRing - 1)] = s.ring[(out.o + k - d) & (kRing - 1)];
                }
            } else {
                // byte o + k = byte o - d + (k mod d), which precedes o; each
                // step reads before any lane writes
                for (uint32_t k0 = 0; k0 < mlen; k0 += NL) {
                    const uint32_t k = k0 + lane;
                    lane_sync();
                    uint8_t v = 0;
                    if (k < mlen) v = s.ring[(out.o - d + (d >= mlen ? k : k % d)) & (kRing - 1)];
                    lane_sync();
                    if (k < mlen) s.ring[(out.o + k) & (kRing - 1)] = v;
                }
            }
            out.o += mlen;
            out.maybe_flush(s);
        }
    }
    if (err == kOk) {
        if (b.overrun()) err = kErrInput;
        else if (out.o != out.cap) err = kErrLength;
        else if ((b.consumed() + 7u) / 8u != len) err = kErrTrailing;
    }
    if (err == kOk) out.flush(s, out.o);
    if (ntok) *ntok = out.nt;
    lane_sync();
    return err;
}


// ---- Parallel decode of a member that is one dynamic block ----
//
// gpzip writes every member as one dynamic-Huffman block, and a member's
// serial decode (one symbol after another, each needing the last one's
// length) is the whole cost of k_inflate_tok.  The block's symbol bits,
// from the end of its header to the end of the data, are therefore cut into
// R spans of equal bit length, one per lane, and every lane decodes its span
// on its own.  A lane that starts in the middle of a code decodes garbage at
// first, but Huffman codes resynchronise within a few symbols, so its exit
// -- the first symbol start at or after the next span's first bit -- is
// almost always the true one.  Rounds repeat with each lane starting at its
// left neighbour's exit from the round before, until no start changes.
// Then every start is a true symbol boundary (lane 0's is, and a lane's
// exit from a true start is true), and the last round's token and byte
// counts are exact.  A final pass writes the tokens at offsets from a scan
// of those counts and checks every distance against the output position.
// Whatever the serial decoder would reject, and a member that does not
// settle within kParRounds, is left to the serial decoder, so failing
// members get exactly its status codes.

constexpr uint64_t kSpanEnd = ~0ull;      // the end-of-block code came first
constexpr uint64_t kSpanBad = ~0ull - 1;  // an invalid code, distance or length
constexpr uint32_t kParRounds = 2;        // rounds before the unsettled rest becomes a tail
constexpr uint64_t kParMinSpanBits = 256; // shortest span worth a lane of its own
// The rest of a block that has not settled (the tail) is cut into sub-spans
// of kSubBits, and each sub-span is decoded from each of the kCands bit
// offsets after its first bit.  Walking the sub-spans in order then picks,
// for each, the candidate that starts where the one before it ended.  A
// symbol takes at most kMaxSymBits = 15 + 5 + 15 + 13 bits, so the true
// start lies less than that after the first bit; on gpzip's members it lay
// within 24 bits at 99.8 % of the boundaries, and the walk decodes a
// sub-span itself where it lies further.
constexpr uint64_t kSubBits = 2048;
constexpr uint32_t kCands = 32;
constexpr uint32_t kMaxSymBits = 48;


// Per-lane bit reader straight from the member's bytes (zeros past len).
struct LaneBits {
    const uint8_t* src;
    uint32_t len;
    uint32_t pos;  // next byte not yet in buf
    uint32_t cnt;  // valid bits in buf
    uint64_t buf;

    // afterwards at least 56 bits are valid.  Away from the end, eight
    // bytes come from three aligned words loaded at once; in the last 12
    // bytes they are read one by one.
    GPZI_FN void refill() {
        if (pos + 12u <= len) {
            const uintptr_t at = (uintptr_t)(src + pos);
            const uint32_t* w = reinterpret_cast<const uint32_t*>(at & ~(uintptr_t)3);
            const uint32_t sh = (uint32_t)(at & 3u) * 8u;
            uint64_t v = ((uint64_t)w[1] << 32 | w[0]) >> sh;
            if (sh) v |= (uint64_t)w[2] << (64u - sh);
            buf |= v << cnt;
            const uint32_t nb = (63u - cnt) >> 3;
            pos += nb;
            cnt += nb * 8u;
            return;
        }
        while (cnt <= 56u) {
            buf |= (uint64_t)(pos < len ? src[pos] : 0u) << cnt;
            pos++;
            cnt += 8u;
        }
    }
    GPZI_FN void seek(uint64_t bit) {
        pos = (uint32_t)(bit >> 3);
        buf = 0;
        cnt = 0;
        refill();
        drop((uint32_t)(bit & 7u));
    }
    GPZI_FN uint32_t peek(uint32_t n) const { return (uint32_t)(buf & ((1ull << n) - 1ull)); }
    GPZI_FN void drop(uint32_t n) {
        buf >>= n;
        cnt -= n;
    }
    GPZI_FN uint32_t take(uint32_t n) {  // n <= 32
        if (cnt < n) refill();
        const uint32_t v = peek(n);
        drop(n);
        return v;
    }
    GPZI_FN uint64_t bitpos() const { return 8ull * pos - cnt; }
};

// One code's entry from t (see Table), as decode_entry; bad if no symbol
// has the code.
GPZI_FN uint32_t lane_entry(const Table& t, LaneBits& b, uint32_t kind, bool& bad) {
    if (b.cnt < 15) b.refill();
    const uint32_t e = t.fast[b.peek(kFastBits)];
    if (e) {
        b.drop(e & 15u);
        return e;
    }
    uint32_t code = 0, first = 0, index = 0;
    for (uint32_t l = 1; l < 16; l++) {
        code |= (uint32_t)(b.buf >> (l - 1)) & 1u;
        const uint32_t c = t.count[l];
        if (code - first < c) {
            b.drop(l);
            return pack_entry(kind, t.sym[index + code - first], 0u);
        }
        index += c;
        first += c;
        first <<= 1;
        code <<= 1;
    }
    bad = true;
    return 0;
}

// What a lane found in its span: its exit (the first symbol start at or
// after the span's stop bit, or kSpanEnd / kSpanBad), the bit after the
// end-of-block code (with kSpanEnd), and the tokens and bytes of the
// symbols that start in the span.
struct Span {
    uint64_t exit;
    uint64_t end;
    uint32_t ntok;
    uint32_t nbytes;
};

// A candidate's result packed into 64 bits: the exit as an offset from the
// next sub-span's first bit (< kMaxSymBits; kCandEnd: the end-of-block code
// came first, kCandBad: anything else), the end-of-block code's end bit as an
// offset from the sub-span's first bit, and its tokens and bytes.
constexpr uint32_t kCandEnd = 254u, kCandBad = 255u;
GPZI_FN uint64_t pack_cand(const Span& r, uint64_t first, uint64_t next_first) {
    uint64_t code = kCandBad, endoff = 0;
    if (r.exit == kSpanEnd) {
        code = kCandEnd;
        endoff = r.end - first;
    } else if (r.exit != kSpanBad && r.exit >= next_first && r.exit - next_first < kMaxSymBits) {
        code = r.exit - next_first;
    }
    if (endoff >= (1u << 13) || r.ntok >= (1u << 13) || r.nbytes >= (1u << 21)) code = kCandBad;
    return code | endoff << 8 | (uint64_t)r.ntok << 21 | (uint64_t)r.nbytes << 34;
}

// Decodes the symbols of the block (tables lit, dist) that start at bit
// `start` and below `stop`.  A start of kSpanEnd or kSpanBad is passed
// on as the exit.  Spans never count more than isize bytes.  With tok (the
// final pass) the tokens are written to tok[0, ntok) (a literal as its
// byte, a match as length << 16 | distance), and every match is checked to
// reach no further back than the member's start and no further than ISIZE:
// obase is the number of bytes before the span.
GPZI_FN Span decode_span(const Table& lit, const Table& dist, const uint8_t* src, uint32_t len, uint64_t start,
                         uint64_t stop, uint32_t* tok, uint32_t obase, uint32_t isize) {
    Span r{kSpanBad, 0ull, 0u, 0u};
    if (start == kSpanEnd || start == kSpanBad) {
        r.exit = start;
        return r;
    }
    LaneBits b{src, len, 0u, 0u, 0ull};
    b.seek(start);
    const uint64_t data_bits = 8ull * len;
    uint64_t p = start;
    // every symbol takes at least one bit, so the loop ends within
    // data_bits + 1 rounds
    while (p < stop) {
        if (p >= data_bits) return r;  // the data ended without an end-of-block code
        bool bad = false;
        const uint32_t e = lane_entry(lit, b, kTabLit, bad);
        if (bad) return r;
        const uint32_t kind = (e >> 4) & 3u;
        if (kind == 0u) {
            if (r.nbytes >= isize || (tok && (uint64_t)obase + r.nbytes >= isize)) return r;
            if (tok) tok[r.ntok] = (e >> 8) & 0xFFu;
            r.ntok++;
            r.nbytes++;
        } else if (kind == 2u) {
            r.exit = kSpanEnd;
            r.end = b.bitpos();
            return r;
        } else if (kind == 3u) {
            return r;
        } else {
            const uint32_t lx = (e >> 17) & 7u;
            const uint32_t mlen = ((e >> 8) & 511u) + (lx ? b.take(lx) : 0u);
            const uint32_t de = lane_entry(dist, b, kTabDist, bad);
            if (bad || ((de >> 4) & 3u) == 3u) return r;
            const uint32_t dx = (de >> 24) & 15u;
            const uint32_t d = ((de >> 8) & 0x7FFFu) + (dx ? b.take(dx) : 0u);
            if (r.nbytes > isize || isize - r.nbytes < mlen) return r;
            if (tok) {
                const uint64_t o = (uint64_t)obase + r.nbytes;  // output bytes before this match
                if (d > o || o > isize || isize - o < mlen) return r;
                tok[r.ntok] = (mlen << 16) | d;
            }
            r.ntok++;
            r.nbytes += mlen;
        }
        p = b.bitpos();
    }
    r.exit = p;
    return r;
}

// The block's first symbol bit when the member is one final dynamic block
// whose header and tables are valid (tables built in s.lit, s.dist), else
// 0: the serial decoder takes the member.
template <int NL>
GPZI_FN uint64_t par_header(Shared& s, uint32_t lane, const uint8_t* src, uint32_t len) {
    Bits<NL> b{src, len, 0u, 0ull, 0u, lane, 0u};
    b.restage(s, 0);
    const bool last = b.take(s, 1) != 0;
    const uint32_t type = b.take(s, 2);
    if (!last || type != 2u) return 0;
    bool lit_empty = false, dist_empty = false;
    if (read_block_tables<NL>(s, b, lane, type, lit_empty, dist_empty) != kOk || lit_empty || b.overrun()) return 0;
    return b.consumed();
}

// Lanes used for a block whose symbols take `bits` bits: spans of at least
// kParMinSpanBits, at most max_lanes of them.
GPZI_FN uint32_t par_lanes(uint64_t bits, uint32_t max_lanes) {
    const uint64_t r = bits / kParMinSpanBits;
    return r < 1u ? 1u : r > max_lanes ? max_lanes : (uint32_t)r;
}

#if !defined(__CUDACC__)
#include <vector>

// The parallel decode with its lanes run one after another (the host check
// of the device's path in gpz_inflate.cu, which runs the same steps with
// one thread per lane): true when it takes the member, with the tokens in
// tok[0, *ntok); false when the member is left to the serial decoder.
inline bool inflate_member_par(Shared& s, const uint8_t* src, uint32_t len, uint32_t isize, uint32_t max_lanes,
                               uint32_t* tok, uint32_t* ntok) {
    constexpr uint32_t kMax = 128;
    if (max_lanes < 1u || max_lanes > kMax) return false;
    const uint64_t h = par_header<1>(s, 0, src, len);
    if (!h || h >= 8ull * len) return false;
    const uint64_t bits = 8ull * len - h;
    const uint32_t R = par_lanes(bits, max_lanes);
    const uint64_t span = (bits + R - 1) / R;
    uint64_t start[kMax], stop[kMax], next[kMax];
    Span res[kMax];
    for (uint32_t k = 0; k < R; k++) {
        start[k] = h + k * span;
        stop[k] = k + 1 < R ? h + (k + 1) * span : kSpanBad - 1;
    }
    for (uint32_t round = 0; round < kParRounds; round++) {
        for (uint32_t k = 0; k < R; k++) res[k] = decode_span(s.lit, s.dist, src, len, start[k], stop[k], nullptr, 0u, isize);
        bool settled = true;
        for (uint32_t k = 0; k < R; k++) {
            next[k] = k ? res[k - 1].exit : start[k];
            settled = settled && next[k] == start[k];
        }
        if (settled || round + 1 == kParRounds) break;
        for (uint32_t k = 0; k < R; k++) start[k] = next[k];
    }
    // lanes before the first one whose start moved decoded from true starts;
    // one lane decodes the rest from that lane's next (true) start
    uint32_t f = R;
    for (uint32_t k = 0; k < R && f == R; k++)
        if (next[k] != start[k]) f = k;
    uint64_t end = 0, bytes = 0, toks = 0;
    bool ended = false, fits = true;
    for (uint32_t k = 0; k < f && fits; k++) {
        const Span g = decode_span(s.lit, s.dist, src, len, start[k], stop[k], tok + toks, (uint32_t)bytes, isize);
        fits = g.exit == res[k].exit && g.ntok == res[k].ntok && g.nbytes == res[k].nbytes && bytes <= isize;
        if (start[k] != kSpanEnd && g.exit == kSpanEnd) {
            end = g.end;
            ended = true;
        }
        toks += g.ntok;
        bytes += g.nbytes;
    }
    if (fits && f < R && !ended && bytes <= isize && next[f] != kSpanEnd) {
        // the tail from next[f] (a true start): every sub-span from each of
        // its kCands first bits, then the walk that picks one per sub-span
        const uint64_t t0 = next[f];
        const uint64_t tail = t0 < 8ull * len ? 8ull * len - t0 : 0ull;
        const uint32_t Q = (uint32_t)((tail + kSubBits - 1) / kSubBits);
        std::vector<uint64_t> cand((size_t)Q * kCands);
        for (uint32_t q = 0; q < Q; q++) {
            const uint64_t first = t0 + q * kSubBits, nf = first + kSubBits;
            for (uint32_t j = 0; j < kCands; j++)
                cand[(size_t)q * kCands + j] = pack_cand(
                    decode_span(s.lit, s.dist, src, len, first + j, q + 1 < Q ? nf : kSpanBad - 1, nullptr, 0u, isize),
                    first, nf);
        }
        uint64_t e = t0;
        fits = t0 != kSpanBad;
        for (uint32_t q = 0; q < Q && fits && !ended; q++) {
            const uint64_t first = t0 + q * kSubBits, nf = first + kSubBits, stop = q + 1 < Q ? nf : kSpanBad - 1;
            const uint64_t c = e - first < kCands ? cand[(size_t)q * kCands + (e - first)]
                                                  : pack_cand(decode_span(s.lit, s.dist, src, len, e, stop, nullptr,
                                                                          0u, isize),
                                                              first, nf);
            const uint32_t code = (uint32_t)(c & 255u);
            if (code == kCandBad || bytes > isize) {
                fits = false;
                break;
            }
            const Span g = decode_span(s.lit, s.dist, src, len, e, stop, tok + toks, (uint32_t)bytes, isize);
            fits = pack_cand(g, first, nf) == c;
            toks += g.ntok;
            bytes += g.nbytes;
            if (code == kCandEnd) {
                end = first + ((c >> 8) & 8191u);
                ended = true;
            } else {
                e = nf + code;
            }
        }
    }
    if (!fits || !ended || end > 8ull * len || (end + 7) / 8 != len || bytes != isize) return false;
    *ntok = (uint32_t)toks;
    return true;
}
#endif

}  // namespace gpzi
