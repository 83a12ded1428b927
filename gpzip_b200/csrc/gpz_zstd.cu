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
//   k_zblock  one warp per tile: literal and match counts (the tile's
//             symbol histogram), the literals scattered by ballots, and the
//             FSE bitstream by one lane walking the tokens backwards.  The
//             block content goes to the tile's slice of `pp` (free after
//             the walk).  The last CTA places every member and tile.
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
__constant__ ZTab c_zt[3];  // literal lengths, match lengths, offsets
__constant__ uint8_t c_ll_code[64];
__constant__ uint8_t c_ml_code[128];
__constant__ uint32_t c_ll_base[36];
__constant__ uint8_t c_ll_bits[36];
__constant__ uint32_t c_ml_base[53];
__constant__ uint8_t c_ml_bits[53];

constexpr int kZWarps = 4;
constexpr int kZThreads = kZWarps * 32;
constexpr int kCopyThreads = 128;
constexpr uint32_t kCompressed = 1u << 31;

// literal-length and match-length codes (RFC 8878 3.1.1.3.2.1.1)
__device__ __forceinline__ uint32_t ll_code(uint32_t ll) {
    return ll < 64u ? c_ll_code[ll] : 31u - __clz(ll) + 19u;
}
__device__ __forceinline__ uint32_t ml_code(uint32_t ml) {
    const uint32_t m = ml - 3u;
    return m < 128u ? c_ml_code[m] : 31u - __clz(m) + 36u;
}

// LSB-first bit writer into a byte buffer bounded by cap (overflow is
// recorded, nothing is written past cap).
struct BitW {
    uint8_t* p;
    uint32_t n, cap;
    unsigned long long acc;
    uint32_t fill;
    bool over;

    __device__ __forceinline__ void add(uint32_t v, uint32_t nb) {
        acc |= (unsigned long long)(v & ((nb >= 32u) ? 0xFFFFFFFFu : ((1u << nb) - 1u))) << fill;
        fill += nb;
        while (fill >= 8u) {
            if (n < cap) p[n] = (uint8_t)acc;
            else over = true;
            n++;
            acc >>= 8;
            fill -= 8u;
        }
    }
};

__device__ __forceinline__ uint32_t fse_init(const ZTab& t, uint32_t s) {
    const uint32_t nb = (t.nbits[s] + (1u << 15)) >> 16;
    const uint32_t v = (nb << 16) - t.nbits[s];
    return t.state[(int32_t)(v >> nb) + t.find[s]];
}

__device__ __forceinline__ void fse_enc(BitW& w, const ZTab& t, uint32_t& state, uint32_t s) {
    const uint32_t nb = (state + t.nbits[s]) >> 16;
    w.add(state, nb);
    state = t.state[(int32_t)(state >> nb) + t.find[s]];
}

// The encoder's state over the sequences of one block, last to first.
struct SeqEnc {
    BitW w;
    uint32_t sll, sml, sof;
    bool started;

    // sequence (literal length ll, match length ml, distance d)
    __device__ __forceinline__ void put(uint32_t ll, uint32_t ml, uint32_t d) {
        const uint32_t llc = ll_code(ll), mlc = ml_code(ml), off = d + 3u, ofc = 31u - __clz(off);
        if (!started) {
            sml = fse_init(c_zt[1], mlc);
            sof = fse_init(c_zt[2], ofc);
            sll = fse_init(c_zt[0], llc);
            started = true;
        } else {
            fse_enc(w, c_zt[2], sof, ofc);
            fse_enc(w, c_zt[1], sml, mlc);
            fse_enc(w, c_zt[0], sll, llc);
        }
        w.add(ll - c_ll_base[llc], c_ll_bits[llc]);
        w.add(ml - c_ml_base[mlc], c_ml_bits[mlc]);
        w.add(off - (1u << ofc), ofc);
    }

    __device__ __forceinline__ void close() {
        w.add(sml, (uint32_t)c_zt[1].log);
        w.add(sof, (uint32_t)c_zt[2].log);
        w.add(sll, (uint32_t)c_zt[0].log);
        w.add(1u, 1u);
        if (w.fill) w.add(0u, 8u - w.fill);
    }
};

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
    __shared__ uint32_t s_tile[kZWarps];
    __shared__ uint32_t s_tok[kZWarps][32];
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t ntiles = bp.dims[0];
    for (;;) {
        if (lane == 0) s_tile[wi] = atomicAdd(&bp.counters[GPZ_CNT_HUFF], 1u);
        __syncwarp();
        const uint32_t t = s_tile[wi];
        __syncwarp();
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
        // literals and matches of the tile, from its symbol histogram
        const uint16_t* hist = bp.tile_hist + (size_t)t * GPZ_NSYM;
        uint32_t nlit = 0, nseq = 0;
        for (uint32_t s = lane; s < 256u; s += 32u) nlit += hist[s];
        if (lane < 29) nseq = hist[257 + lane];
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            nlit += __shfl_xor_sync(0xFFFFFFFFu, nlit, o);
            nseq += __shfl_xor_sync(0xFFFFFFFFu, nseq, o);
        }
        const uint32_t lh = nlit < 32u ? 1u : nlit < 4096u ? 2u : 3u;
        const uint32_t sh = nseq < 128u ? 1u : nseq < 0x7F00u ? 2u : 3u;
        // the content must be smaller than rawlen to be used; the tile's
        // slice of pp (4 bytes per position of the tile) holds it
        uint8_t* dst = reinterpret_cast<uint8_t*>(bp.pp + md.in_off + start);
        const uint32_t cap = rawlen;
        bool comp = lh + nlit + sh + (nseq ? 1u : 0u) < cap;
        uint32_t csize = 0;
        if (comp) {
            if (lane == 0) {
                if (lh == 1u) {
                    dst[0] = (uint8_t)(nlit << 3);
                } else if (lh == 2u) {
                    dst[0] = (uint8_t)(((nlit & 15u) << 4) | 4u);
                    dst[1] = (uint8_t)(nlit >> 4);
                } else {
                    dst[0] = (uint8_t)(((nlit & 15u) << 4) | 12u);
                    dst[1] = (uint8_t)(nlit >> 4);
                    dst[2] = (uint8_t)(nlit >> 12);
                }
            }
            // literals in token order, ranked by ballots
            uint32_t lbase = lh;
            for (uint32_t c = 0; c < ntok; c += 32u) {
                const uint32_t i = c + lane;
                const uint32_t v = i < ntok ? tok[i] : 0xFFFFFFFFu;
                const bool lit = i < ntok && (v >> 16) == 0u;
                const uint32_t m = __ballot_sync(0xFFFFFFFFu, lit);
                if (lit) dst[lbase + __popc(m & lt)] = (uint8_t)v;
                lbase += __popc(m);
            }
            // sequences section header
            const uint32_t q = lh + nlit;
            if (lane == 0) {
                if (sh == 1u) {
                    dst[q] = (uint8_t)nseq;
                } else if (sh == 2u) {
                    dst[q] = (uint8_t)((nseq >> 8) + 0x80u);
                    dst[q + 1] = (uint8_t)nseq;
                } else {
                    dst[q] = 0xFF;
                    dst[q + 1] = (uint8_t)(nseq - 0x7F00u);
                    dst[q + 2] = (uint8_t)((nseq - 0x7F00u) >> 8);
                }
                if (nseq) dst[q + sh] = 0;  // predefined modes
            }
            csize = q + sh;
            if (nseq) {
                // FSE: one lane walks the tokens backwards.  A match waits
                // until the match before it is reached: the literals in
                // between are its literal length.  Tokens come 32 at a
                // time through shared memory.
                SeqEnc e{};
                e.w = BitW{dst + q + sh + 1u, 0u, cap - (q + sh + 1u), 0ull, 0u, false};
                bool pend = false;
                uint32_t pml = 0, pd = 0, run = 0;
                const uint32_t top = (ntok + 31u) & ~31u;
                for (uint32_t c = top; c > 0; c -= 32u) {
                    const uint32_t c0 = c - 32u, i = c0 + lane;
                    const uint32_t v = i < ntok ? tok[i] : 0u;
                    s_tok[wi][lane] = v;
                    const bool valid = i < ntok;
                    const uint32_t mm = __ballot_sync(0xFFFFFFFFu, valid && (v >> 16) != 0u);
                    const uint32_t lm = __ballot_sync(0xFFFFFFFFu, valid && (v >> 16) == 0u);
                    __syncwarp();
                    if (lane == 0) {
                        uint32_t left = mm, upper = 32u;
                        while (left) {
                            // the literals strictly between match j and
                            // the match (or chunk end) above it
                            const uint32_t j = 31u - __clz(left);
                            const uint32_t above_j = j >= 31u ? 0u : ~0u << (j + 1u);
                            const uint32_t below_up = upper >= 32u ? ~0u : (1u << upper) - 1u;
                            run += __popc(lm & above_j & below_up);
                            if (pend) e.put(run, pml, pd);
                            const uint32_t tv = s_tok[wi][j];
                            pend = true;
                            pml = tv >> 16;
                            pd = tv & 0xFFFFu;
                            run = 0;
                            upper = j;
                            left &= ~(1u << j);
                        }
                        run += __popc(lm & (upper >= 32u ? ~0u : ((1u << upper) - 1u)));
                    }
                    __syncwarp();
                }
                if (lane == 0) {
                    if (pend) e.put(run, pml, pd);
                    e.close();
                    csize = q + sh + 1u + e.w.n;
                    if (e.w.over) csize = cap;
                }
                csize = __shfl_sync(0xFFFFFFFFu, csize, 0);
            }
            comp = csize < cap;
        }
        if (lane == 0) bp.tile_zinfo[t] = comp ? (csize | kCompressed) : rawlen;
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
    ZTab tabs[3];
    build_tab(tabs[0], ll_norm, 36, 6);
    build_tab(tabs[1], ml_norm, 53, 6);
    build_tab(tabs[2], of_norm, 29, 5);
    uint8_t llc[64], mlc[128];
    for (uint32_t v = 0; v < 64; v++) {
        int c = 35;
        while (ll_base[c] > v) c--;
        llc[v] = (uint8_t)c;
    }
    for (uint32_t m = 0; m < 128; m++) {
        int c = 52;
        while (ml_base[c] > m + 3u) c--;
        mlc[m] = (uint8_t)c;
    }
    if (cudaMemcpyToSymbol(c_zt, tabs, sizeof tabs) != cudaSuccess ||
        cudaMemcpyToSymbol(c_ll_code, llc, sizeof llc) != cudaSuccess ||
        cudaMemcpyToSymbol(c_ml_code, mlc, sizeof mlc) != cudaSuccess ||
        cudaMemcpyToSymbol(c_ll_base, ll_base, sizeof ll_base) != cudaSuccess ||
        cudaMemcpyToSymbol(c_ll_bits, ll_bits, sizeof ll_bits) != cudaSuccess ||
        cudaMemcpyToSymbol(c_ml_base, ml_base, sizeof ml_base) != cudaSuccess ||
        cudaMemcpyToSymbol(c_ml_bits, ml_bits, sizeof ml_bits) != cudaSuccess)
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
    const int gb = grid_blocks > 0 ? grid_blocks : (int)((bp.ntiles + kZWarps - 1) / kZWarps + 1);
    const int gc = grid_copy > 0 ? grid_copy : (int)(bp.ntiles ? bp.ntiles : 1u);
    k_zblock<<<gb, kZThreads, 0, s>>>(bp);
    mark(4);
    k_zcopy<<<gc, kCopyThreads, 0, s>>>(bp);
    mark(5);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
