// gpz_zstd.cu -- zstd frames (RFC 8878) from the gzip path's tokens: the
// chunk-parallel zstd codec of the reference (ZstdCompressor::chunk_fn,
// crates/gpzip-codec-cpu/src/compress.rs:76-126: one frame per chunk) on the
// device.  The match finder and the lazy walk are the gzip path's
// (k_segtab .. k_walk_mark); these kernels replace its Huffman stages.
//
// Frame of one input: a 6-byte header (magic, no content size, no
// checksum, a 64 KiB window: every match is at most 32768 bytes back), then
// one block per 4 KiB tile of each member.  A tile's block holds the walked
// tokens that start in the tile (tile_ntok of them, stored by k_walk_mark
// at the tile's place in `tok`), so it decodes the input from the tile's
// walk entry to the next tile's entry, and every block is independent:
//   literals   raw, with a 1-, 2- or 3-byte header;
//   sequences  the count, then modes 0 (the predefined literal-length,
//              offset and match-length distributions) and one FSE
//              bitstream; a sequence is the literals since the last match
//              plus a match; every offset is sent as distance + 3;
// and a block whose content is not smaller than the bytes it decodes to is
// stored raw.  The last block of the frame carries the last-block flag; an
// empty input is one empty raw block.
//
//   k_zblock  one CTA per tile, in shared memory: literal and match
//             counts and the literals scattered by ballots; each sequence's
//             codes; the three FSE state chains (literal lengths, match
//             lengths, offsets) run last sequence to first, one lane each,
//             recording the states; then every thread packs a run of
//             sequences' bits at offsets from a block scan.  The block
//             content goes to the tile's slice of `pp` (free after the
//             walk).  The last CTA places every member and tile.
//   k_zcopy   per tile: the block header and content (or the raw input) to
//             the batch output; per input, the frame header.
#include <cuda_runtime.h>

#include <cstdint>

#include "gpz_internal.h"

namespace {

// FSE encoding table of one of the three predefined distributions.
struct ZTab {
    uint16_t state[64];  // encoder states of each symbol, by symbol, as size + cell
    int32_t find[53];    // first index of the symbol's states minus its count
    uint32_t nbits[53];  // (max bits << 16) - (count << max bits)
    int32_t log;
};
// Every table the block encoder reads.  Each CTA keeps a copy in shared
// memory: the threads of a warp index it with different symbols.
struct ZConst {
    ZTab t[3];  // literal lengths, match lengths, offsets
    uint32_t ll_base[36];
    uint32_t ml_base[53];
    uint8_t ll_code[64];
    uint8_t ml_code[128];
    uint8_t ll_bits[36];
    uint8_t ml_bits[53];
    uint8_t pad[3];
};
static_assert(sizeof(ZConst) % 4 == 0, "ZConst is copied in words");
__constant__ ZConst c_z;

constexpr int kZThreads = 128;  // one CTA per tile
constexpr int kZWarps = kZThreads / 32;
constexpr int kCopyThreads = 128;
constexpr uint32_t kCompressed = 1u << 31;
constexpr uint32_t kZMaxSeq = (GPZ_SEG + 2u) / 3u;  // a tile's matches start at least 3 bytes apart
constexpr uint32_t kZBuf = GPZ_SEG + 320u;          // content bytes; a tile decodes to at most 4096 + 257

// literal-length and match-length codes (RFC 8878 3.1.1.3.2.1.1)
__device__ __forceinline__ uint32_t ll_code(const ZConst& z, uint32_t ll) {
    return ll < 64u ? z.ll_code[ll] : 31u - __clz(ll) + 19u;
}
__device__ __forceinline__ uint32_t ml_code(const ZConst& z, uint32_t ml) {
    const uint32_t m = ml - 3u;
    return m < 128u ? z.ml_code[m] : 31u - __clz(m) + 36u;
}

// Shared memory of k_zblock: one tile at a time.
struct ZBlockSmem {
    ZConst z;
    uint32_t out[kZBuf / 4];   // the block content, little-endian
    uint16_t mpos[kZMaxSeq];   // token index of each match, in order
    uint8_t sym[3][kZMaxSeq];  // literal-length, match-length and offset code of each sequence
    uint8_t st[3][kZMaxSeq];   // each stream's state before the sequence is encoded, minus the table size
    uint32_t cnt[kZWarps][2];  // literals and matches of each warp's share of the tokens
    uint32_t part[kZWarps];    // bit counts of each warp's sequences
    uint32_t fin[3];           // the streams' states after the first sequence
    uint32_t tile;
};

// ORs the n low bits of f into `out` at bit g (LSB first); n <= 64.
__device__ __forceinline__ void or_bits(uint32_t* out, uint32_t g, unsigned long long f, uint32_t n) {
    if (!n) return;
    const uint32_t w = g >> 5, s = g & 31u;
    const unsigned long long lo = f << s;
    atomicOr(&out[w], (uint32_t)lo);
    if (s + n > 32u) atomicOr(&out[w + 1], (uint32_t)(lo >> 32));
    if (s + n > 64u) atomicOr(&out[w + 2], (uint32_t)(f >> (64u - s)));
}

// Bits of stream j's state for sequence k: the value and its width.
__device__ __forceinline__ uint32_t state_bits(const ZBlockSmem& sm, int j, uint32_t k, uint32_t& nb) {
    const ZTab& tb = sm.z.t[j];
    const uint32_t state = sm.st[j][k] + (1u << tb.log);
    nb = (state + tb.nbits[sm.sym[j][k]]) >> 16;
    return state & ((1u << nb) - 1u);
}

// Bits that sequence k adds to the stream (the last sequence, which is
// encoded first, only sets the states and adds no state bits).
__device__ __forceinline__ uint32_t seq_nbits(const ZBlockSmem& sm, uint32_t k, bool first) {
    uint32_t n = sm.z.ll_bits[sm.sym[0][k]] + sm.z.ml_bits[sm.sym[1][k]] + sm.sym[2][k];
    if (!first) {
        uint32_t nb;
        for (int j = 0; j < 3; j++) {
            state_bits(sm, j, k, nb);
            n += nb;
        }
    }
    return n;
}

// The fields of sequence k in stream order: the offset, match-length and
// literal-length state bits, then the literal-length, match-length and
// offset extra bits.
__device__ __forceinline__ unsigned long long seq_fields(const ZBlockSmem& sm, const uint32_t* tok, uint32_t k,
                                                         bool first, uint32_t& n) {
    const ZConst& z = sm.z;
    const uint32_t i = sm.mpos[k];
    const uint32_t ll = i - (k ? sm.mpos[k - 1] + 1u : 0u);
    const uint32_t v = tok[i];
    const uint32_t ml = v >> 16, off = (v & 0xFFFFu) + 3u;
    const uint32_t llc = sm.sym[0][k], mlc = sm.sym[1][k], ofc = sm.sym[2][k];
    unsigned long long f = 0;
    n = 0;
    if (!first) {
        for (int j = 2; j >= 0; j--) {
            uint32_t nb;
            const uint32_t x = state_bits(sm, j, k, nb);
            f |= (unsigned long long)x << n;
            n += nb;
        }
    }
    f |= (unsigned long long)(ll - z.ll_base[llc]) << n;
    n += z.ll_bits[llc];
    f |= (unsigned long long)(ml - z.ml_base[mlc]) << n;
    n += z.ml_bits[mlc];
    f |= (unsigned long long)(off - (1u << ofc)) << n;
    n += ofc;
    return f;
}

// True in the last CTA of the grid to finish (its global writes, and every
// other CTA's, are visible to it).
__device__ bool z_last_cta(uint32_t* counter) {
    __shared__ bool s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == gridDim.x - 1u;
    __syncthreads();
    if (s_last) __threadfence();
    return s_last;
}

// Member and tile placement: a member's output is the frame header (its
// input's first member), then each tile's 3-byte block header and content
// (an empty input: one empty block); an exclusive scan over the members
// gives their offsets.
__device__ void z_place(const BatchParams& bp) {
    __shared__ unsigned long long s_wsum[kZThreads / 32];
    __shared__ unsigned long long s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t nmembers = bp.dims[1];
    if (tid == 0) s_carry = bp.out_base;
    __syncthreads();
    for (uint32_t base = 0; base < nmembers; base += kZThreads) {
        const uint32_t m = base + tid;
        unsigned long long v = 0;
        if (m < nmembers) {
            const MemberDesc md = bp.members[m];
            uint32_t total = (md.frame & GPZ_MEMBER_FIRST) ? GPZ_ZSTD_FRAME_HDR : 0u;
            if (md.ntiles == 0) total += 3u;
            for (uint32_t i = 0; i < md.ntiles; i++) {
                const uint32_t z = __ldcg(&bp.tile_zinfo[md.tile_base + i]);
                bp.tile_bitoff[md.tile_base + i] = total;
                total += 3u + (z & ~kCompressed);
            }
            MemberOut mo{};
            mo.deflate_bytes = total;
            mo.len = md.len;
            mo.frame_bytes = 0;
            bp.member_out[m] = mo;
            v = total;
        }
        unsigned long long x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_wsum[warp] = x;
        __syncthreads();
        unsigned long long before = 0;
        for (int q = 0; q < warp; q++) before += s_wsum[q];
        if (m < nmembers) bp.member_out[m].gz_off = s_carry + before + x - v;
        __syncthreads();
        if (tid == 0)
            for (int q = 0; q < kZThreads / 32; q++) s_carry += s_wsum[q];
        __syncthreads();
    }
}

// ------------------------------------------------------------------ k_zblock

__global__ void __launch_bounds__(kZThreads) k_zblock(BatchParams bp) {
    __shared__ ZBlockSmem sm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&c_z);
        uint32_t* d = reinterpret_cast<uint32_t*>(&sm.z);
        for (uint32_t i = tid; i < sizeof(ZConst) / 4; i += kZThreads) d[i] = src[i];
    }
    const ZConst& z = sm.z;
    uint8_t* ob = reinterpret_cast<uint8_t*>(sm.out);
    const uint32_t ntiles = bp.dims[0];
    for (;;) {
        if (tid == 0) sm.tile = atomicAdd(&bp.counters[GPZ_CNT_HUFF], 1u);
        for (uint32_t i = tid; i < kZBuf / 4; i += kZThreads) sm.out[i] = 0u;
        __syncthreads();
        const uint32_t t = sm.tile;
        if (t >= ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        const uint32_t start = td.seg << GPZ_SEG_LOG2;
        // the bytes this block decodes to: from this tile's walk entry to
        // the next tile's (or the member's end)
        const uint32_t b0 = start + bp.tile_entry[t];
        const uint32_t b1 = td.seg + 1u < md.ntiles ? start + GPZ_SEG + bp.tile_entry[t + 1] : md.len;
        const uint32_t rawlen = b1 > b0 ? b1 - b0 : 0u;
        const uint32_t ntok = min(bp.tile_ntok[t], GPZ_SEG);
        const uint32_t* tok = bp.tok + md.in_off + start;
        // each warp takes a quarter of the tokens and counts its literals
        // and matches
        const uint32_t span = (ntok + kZThreads - 1u) / kZThreads * 32u;
        const uint32_t w0 = min(ntok, (uint32_t)warp * span), w1 = min(ntok, w0 + span);
        uint32_t nl = 0, nm = 0;
        for (uint32_t c = w0; c < w1; c += 32u) {
            const uint32_t i = c + lane;
            const uint32_t v = i < w1 ? tok[i] : 0u;
            nl += __popc(__ballot_sync(0xFFFFFFFFu, i < w1 && (v >> 16) == 0u));
            nm += __popc(__ballot_sync(0xFFFFFFFFu, i < w1 && (v >> 16) != 0u));
        }
        if (lane == 0) {
            sm.cnt[warp][0] = nl;
            sm.cnt[warp][1] = nm;
        }
        __syncthreads();
        uint32_t nlit = 0, nseq = 0, lbase = 0, mbase = 0;
        for (int w = 0; w < kZWarps; w++) {
            if (w == warp) {
                lbase = nlit;
                mbase = nseq;
            }
            nlit += sm.cnt[w][0];
            nseq += sm.cnt[w][1];
        }
        const uint32_t lh = nlit < 32u ? 1u : nlit < 4096u ? 2u : 3u;
        const uint32_t sh = nseq < 128u ? 1u : nseq < 0x7F00u ? 2u : 3u;
        const uint32_t q = lh + nlit;                      // the sequences section
        const uint32_t body = q + sh + (nseq ? 1u : 0u);  // the FSE bitstream
        // the content is used only when it is smaller than the bytes it
        // decodes to
        bool comp = body < rawlen;
        if (rawlen > kZBuf || nseq > kZMaxSeq) {
            // a tile decodes to at most 4096 + 257 bytes and its matches
            // start at least 3 bytes apart, so this is never reached
            if (tid == 0) atomicOr(bp.err, GPZ_ERRBIT_BITS);
            comp = false;
        }
        uint32_t csize = body;
        if (comp) {
            // literals in token order, and the token index of each match
            for (uint32_t c = w0; c < w1; c += 32u) {
                const uint32_t i = c + lane;
                const uint32_t v = i < w1 ? tok[i] : 0u;
                const bool lit = i < w1 && (v >> 16) == 0u, mat = i < w1 && (v >> 16) != 0u;
                const uint32_t bl = __ballot_sync(0xFFFFFFFFu, lit), bm = __ballot_sync(0xFFFFFFFFu, mat);
                if (lit) ob[lh + lbase + __popc(bl & lt)] = (uint8_t)v;
                if (mat) sm.mpos[mbase + __popc(bm & lt)] = (uint16_t)i;
                lbase += __popc(bl);
                mbase += __popc(bm);
            }
            if (tid == 0) {
                if (lh == 1u) {
                    ob[0] = (uint8_t)(nlit << 3);
                } else if (lh == 2u) {
                    ob[0] = (uint8_t)(((nlit & 15u) << 4) | 4u);
                    ob[1] = (uint8_t)(nlit >> 4);
                } else {
                    ob[0] = (uint8_t)(((nlit & 15u) << 4) | 12u);
                    ob[1] = (uint8_t)(nlit >> 4);
                    ob[2] = (uint8_t)(nlit >> 12);
                }
                if (sh == 1u) {
                    ob[q] = (uint8_t)nseq;
                } else if (sh == 2u) {
                    ob[q] = (uint8_t)((nseq >> 8) + 0x80u);
                    ob[q + 1] = (uint8_t)nseq;
                } else {
                    ob[q] = 0xFF;
                    ob[q + 1] = (uint8_t)(nseq - 0x7F00u);
                    ob[q + 2] = (uint8_t)((nseq - 0x7F00u) >> 8);
                }
                if (nseq) ob[q + sh] = 0;  // predefined modes
            }
            __syncthreads();
        }
        if (comp && nseq) {
            // each sequence's codes
            for (uint32_t k = tid; k < nseq; k += kZThreads) {
                const uint32_t i = sm.mpos[k];
                const uint32_t v = tok[i];
                sm.sym[0][k] = (uint8_t)ll_code(z, i - (k ? sm.mpos[k - 1] + 1u : 0u));
                sm.sym[1][k] = (uint8_t)ml_code(z, v >> 16);
                sm.sym[2][k] = (uint8_t)(31u - __clz((v & 0xFFFFu) + 3u));
            }
            __syncthreads();
            // the three FSE state chains, last sequence to first: one lane
            // each (literal lengths, match lengths, offsets)
            if (warp == 0 && lane < 3) {
                const ZTab& tb = z.t[lane];
                const uint32_t size = 1u << tb.log;
                const uint8_t* sy = sm.sym[lane];
                uint8_t* so = sm.st[lane];
                uint32_t s = sy[nseq - 1u];
                const uint32_t nb0 = (tb.nbits[s] + (1u << 15)) >> 16;
                uint32_t state = tb.state[(int32_t)(((nb0 << 16) - tb.nbits[s]) >> nb0) + tb.find[s]];
#pragma unroll 4
                for (int k = (int)nseq - 2; k >= 0; k--) {
                    s = sy[k];
                    const uint32_t nb = (state + tb.nbits[s]) >> 16;
                    so[k] = (uint8_t)(state - size);
                    state = tb.state[(int32_t)(state >> nb) + tb.find[s]];
                }
                sm.fin[lane] = state;
            }
            __syncthreads();
            // bit offsets: every thread takes a run of sequences in stream
            // order (slot p holds sequence nseq - 1 - p), then a block scan
            const uint32_t per = (nseq + kZThreads - 1u) / kZThreads;
            const uint32_t p0 = min(nseq, (uint32_t)tid * per), p1 = min(nseq, p0 + per);
            uint32_t mine = 0;
            for (uint32_t p = p0; p < p1; p++) mine += seq_nbits(sm, nseq - 1u - p, p == 0u);
            uint32_t x = mine;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) sm.part[warp] = x;
            __syncthreads();
            uint32_t before = x - mine, total = 0;
            for (int w = 0; w < kZWarps; w++) {
                if (w < warp) before += sm.part[w];
                total += sm.part[w];
            }
            // the stream ends with the three final states and a 1 bit
            csize = body + ((total + 18u + 7u) >> 3);
            comp = csize < rawlen;
            if (comp) {
                uint32_t g = body * 8u + before;
                for (uint32_t p = p0; p < p1; p++) {
                    uint32_t n;
                    const unsigned long long f = seq_fields(sm, tok, nseq - 1u - p, p == 0u, n);
                    or_bits(sm.out, g, f, n);
                    g += n;
                }
                if (tid == 0) {
                    const unsigned long long f = (unsigned long long)(sm.fin[1] & 63u) |
                                                 ((unsigned long long)(sm.fin[2] & 31u) << 6) |
                                                 ((unsigned long long)(sm.fin[0] & 63u) << 11) | (1ull << 17);
                    or_bits(sm.out, body * 8u + total, f, 18u);
                }
            }
            __syncthreads();
        }
        if (comp) {
            uint32_t* dst = bp.pp + md.in_off + start;  // the tile's slice of pp, free after the walk
            for (uint32_t i = tid; i < (csize + 3u) / 4u; i += kZThreads) dst[i] = sm.out[i];
        }
        if (tid == 0) bp.tile_zinfo[t] = comp ? (csize | kCompressed) : rawlen;
        __syncthreads();
    }
    if (z_last_cta(&bp.counters[GPZ_CNT_HUFF_DONE])) z_place(bp);
}

// ------------------------------------------------------------------ k_zcopy

__global__ void __launch_bounds__(kCopyThreads) k_zcopy(BatchParams bp) {
    uint8_t* out = reinterpret_cast<uint8_t*>(bp.out_words);  // member offsets are absolute
    const uint32_t ntiles = bp.dims[0], nmembers = bp.dims[1];
    const int tid = threadIdx.x;
    // frame headers, and the empty block of an empty input
    for (uint32_t m = blockIdx.x * kCopyThreads + tid; m < nmembers; m += gridDim.x * kCopyThreads) {
        const MemberDesc md = bp.members[m];
        const unsigned long long o = bp.member_out[m].gz_off;
        if (md.frame & GPZ_MEMBER_FIRST) {
            const uint8_t hdr[GPZ_ZSTD_FRAME_HDR] = {0x28, 0xB5, 0x2F, 0xFD, 0x00, 0x30};
            for (uint32_t k = 0; k < GPZ_ZSTD_FRAME_HDR; k++) out[o + k] = hdr[k];
        }
        if (md.ntiles == 0) {
            const unsigned long long e = o + ((md.frame & GPZ_MEMBER_FIRST) ? GPZ_ZSTD_FRAME_HDR : 0u);
            out[e] = (md.frame & GPZ_MEMBER_LAST) ? 1u : 0u;
            out[e + 1] = 0;
            out[e + 2] = 0;
        }
    }
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        const uint32_t z = bp.tile_zinfo[t];
        const bool comp = (z & kCompressed) != 0u;
        const uint32_t size = z & ~kCompressed;
        const unsigned long long o = bp.member_out[td.member].gz_off + bp.tile_bitoff[t];
        const bool last = (md.frame & GPZ_MEMBER_LAST) && td.seg + 1u == md.ntiles;
        if (tid == 0) {
            const uint32_t h = (last ? 1u : 0u) | ((comp ? 2u : 0u) << 1) | (size << 3);
            out[o] = (uint8_t)h;
            out[o + 1] = (uint8_t)(h >> 8);
            out[o + 2] = (uint8_t)(h >> 16);
        }
        const uint8_t* src = comp ? reinterpret_cast<const uint8_t*>(bp.pp + md.in_off + (td.seg << GPZ_SEG_LOG2))
                                  : bp.in + md.in_off + (td.seg << GPZ_SEG_LOG2) + bp.tile_entry[t];
        for (uint32_t k = tid; k < size; k += kCopyThreads) out[o + 3 + k] = src[k];
    }
}

// FSE encoding table (the same symbol spread as the RFC's decoding table).
void build_tab(ZTab& t, const int16_t* norm, int nsym, int log) {
    const int size = 1 << log, mask = size - 1;
    int high = size - 1, total = 0, next[53];
    uint8_t cell[64];
    for (int s = 0; s < nsym; s++) {
        const int c = norm[s] == -1 ? 1 : norm[s];
        if (norm[s] == -1) cell[high--] = (uint8_t)s;
        next[s] = total;
        if (c == 1) {
            t.nbits[s] = ((uint32_t)log << 16) - (1u << log);
            t.find[s] = total - 1;
        } else {
            const int mb = log - (31 - __builtin_clz((uint32_t)c - 1u));
            t.nbits[s] = ((uint32_t)mb << 16) - ((uint32_t)c << mb);
            t.find[s] = total - c;
        }
        total += c;
    }
    const int step = (size >> 1) + (size >> 3) + 3;
    for (int s = 0, pos = 0; s < nsym; s++)
        for (int i = 0; i < norm[s]; i++) {
            cell[pos] = (uint8_t)s;
            do pos = (pos + step) & mask;
            while (pos > high);
        }
    for (int u = 0; u < size; u++) t.state[next[cell[u]]++] = (uint16_t)(size + u);
    t.log = log;
}

}  // namespace

int gpz_zstd_setup() {
    // RFC 8878 3.1.1.3.2.2: the predefined distributions (-1: one cell)
    static const int16_t ll_norm[36] = {4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 2, 2,
                                        2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1, -1, -1, -1, -1};
    static const int16_t ml_norm[53] = {1, 4, 3, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1,  1,
                                        1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,  1,
                                        1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1};
    static const int16_t of_norm[29] = {1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1,
                                        1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1};
    // RFC 8878 3.1.1.3.2.1.1: code baselines and extra bits
    static const uint32_t ll_base[36] = {0,  1,  2,  3,  4,  5,  6,   7,   8,   9,    10,   11,
                                         12, 13, 14, 15, 16, 18, 20,  22,  24,  28,   32,   40,
                                         48, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536};
    static const uint8_t ll_bits[36] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  1,  1,
                                        1, 1, 2, 2, 3, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
    static const uint32_t ml_base[53] = {3,  4,  5,  6,  7,  8,  9,  10,  11,  12,  13,   14,   15,   16,
                                         17, 18, 19, 20, 21, 22, 23, 24,  25,  26,  27,   28,   29,   30,
                                         31, 32, 33, 34, 35, 37, 39, 41,  43,  47,  51,   59,   67,   83,
                                         99, 131, 259, 515, 1027, 2051, 4099, 8195, 16387, 32771, 65539};
    static const uint8_t ml_bits[53] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                        0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1,
                                        2, 2, 3, 3, 4, 4, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
    ZConst z{};
    build_tab(z.t[0], ll_norm, 36, 6);
    build_tab(z.t[1], ml_norm, 53, 6);
    build_tab(z.t[2], of_norm, 29, 5);
    for (uint32_t v = 0; v < 64; v++) {
        int c = 35;
        while (ll_base[c] > v) c--;
        z.ll_code[v] = (uint8_t)c;
    }
    for (uint32_t m = 0; m < 128; m++) {
        int c = 52;
        while (ml_base[c] > m + 3u) c--;
        z.ml_code[m] = (uint8_t)c;
    }
    for (int i = 0; i < 36; i++) {
        z.ll_base[i] = ll_base[i];
        z.ll_bits[i] = ll_bits[i];
    }
    for (int i = 0; i < 53; i++) {
        z.ml_base[i] = ml_base[i];
        z.ml_bits[i] = ml_bits[i];
    }
    if (cudaMemcpyToSymbol(c_z, &z, sizeof z) != cudaSuccess)
        return -1;
    return 0;
}

int gpz_zstd_occupancy(int* grid_blocks, int* grid_copy) {
    int dev = 0, sms = 0, a = 0, b = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_zblock, kZThreads, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_zcopy, kCopyThreads, 0) != cudaSuccess)
        return -1;
    *grid_blocks = sms * (a > 0 ? a : 1);
    *grid_copy = sms * (b > 0 ? b : 1);
    return 0;
}

int gpz_launch_zstd(const BatchParams& bp, void* stream, void* const* events, int grid_blocks, int grid_copy) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto mark = [&](int i) {
        if (events) cudaEventRecord(static_cast<cudaEvent_t>(events[i]), s);
    };
    const int gb = grid_blocks > 0 ? grid_blocks : (int)(bp.ntiles ? bp.ntiles : 1u);
    const int gc = grid_copy > 0 ? grid_copy : (int)(bp.ntiles ? bp.ntiles : 1u);
    k_zblock<<<gb, kZThreads, 0, s>>>(bp);
    mark(4);
    k_zcopy<<<gc, kCopyThreads, 0, s>>>(bp);
    mark(5);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
