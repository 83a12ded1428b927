/*
 * zstd_frame.c -- CPU restatement of the GPU zstd frame encoder (TEST
 * INFRASTRUCTURE).  Only the tests and the CPU-baseline leg of the
 * benchmark load it; the product library never does.
 *
 * The reference compresses `.tar.zst` with one zstd frame per chunk through
 * the zstd crate (ZstdCompressor::chunk_fn,
 * crates/gpzip-codec-cpu/src/compress.rs:76-126, level 5 -> zstd level 3).
 * libzstd's own match finder cannot be reproduced, so the GPU codec defines
 * its frames from the gzip path's tokens (the segmented-hash match finder
 * and lazy walk, lz77_hash_lookup.wgsl:69-119 and lz77.rs:260-284) and this
 * file restates that definition step by step, so that the device output can
 * be compared with it byte for byte.  Every frame is also decoded by
 * libzstd in the tests.  The format is RFC 8878:
 *
 *  - frame header (6 bytes): magic 0xFD2FB528, a descriptor with no content
 *    size, no checksum and no dictionary, and a window descriptor of 64 KiB
 *    (every match of this path is at most 32768 bytes back), as a streaming
 *    encoder writes it;
 *  - one block per 4 KiB tile of each member_bytes piece: the block holds
 *    the walked tokens that start in the tile (a match that runs into the
 *    next tile belongs to the tile it starts in), so every block decodes on
 *    its own and the device encodes all of a member's blocks at once.  The
 *    last block of the frame is flagged; an empty chunk is one empty raw
 *    block;
 *  - a block's tokens become sequences: the literal tokens since the last
 *    match are the sequence's literals, a match ends the sequence with its
 *    length and distance; literals after the last match trail the block;
 *  - literals section: raw (type 0), with a 1-, 2- or 3-byte header;
 *  - sequences section: the count (1, 2 or 3 bytes), then, when there are
 *    sequences, compression modes 0 (the predefined distributions for
 *    literal lengths, offsets and match lengths) and the FSE bitstream;
 *    every offset is sent as distance + 3 (no repeat offsets);
 *  - a block whose compressed content is not smaller than the bytes it
 *    decodes to is written raw (type 0) instead.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gpz_oracle.h"

/* RFC 8878 3.1.1.3.2.2: predefined normalized distributions (-1: a
 * "less than 1" probability, one table cell) and their accuracy logs. */
static const int16_t LL_NORM[36] = {4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 2, 2,
                                    2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1, -1, -1, -1, -1};
static const int16_t ML_NORM[53] = {1, 4, 3, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1,  1,
                                    1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,  1,
                                    1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1};
static const int16_t OF_NORM[29] = {1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1,
                                    1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1};

/* RFC 8878 3.1.1.3.2.1.1: literal-length and match-length codes. */
static const uint32_t LL_BASE[36] = {0,  1,  2,  3,  4,  5,  6,   7,   8,   9,    10,   11,
                                     12, 13, 14, 15, 16, 18, 20,  22,  24,  28,   32,   40,
                                     48, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536};
static const uint8_t LL_BITS[36] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  1,  1,
                                    1, 1, 2, 2, 3, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
static const uint32_t ML_BASE[53] = {3,  4,  5,  6,  7,  8,  9,  10,  11,  12,  13,   14,   15,   16,
                                     17, 18, 19, 20, 21, 22, 23, 24,  25,  26,  27,   28,   29,   30,
                                     31, 32, 33, 34, 35, 37, 39, 41,  43,  47,  51,   59,   67,   83,
                                     99, 131, 259, 515, 1027, 2051, 4099, 8195, 16387, 32771, 65539};
static const uint8_t ML_BITS[53] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                                    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1,
                                    2, 2, 3, 3, 4, 4, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};

static int highbit(uint32_t v) { return 31 - __builtin_clz(v); }

static int ll_code(uint32_t ll) {
    if (ll < 16) return (int)ll;
    int c = 35;
    while (LL_BASE[c] > ll) c--;
    return c;
}

static int ml_code(uint32_t ml) {
    if (ml < 35) return (int)ml - 3;
    int c = 52;
    while (ML_BASE[c] > ml) c--;
    return c;
}

/* FSE encoding table of a normalized distribution: the symbol spread of the
 * RFC's decoding table (less-than-1 symbols in the last cells, the others
 * stepped through the table by (size/2 + size/8 + 3)), each table cell
 * listed under its symbol in cell order as a state size + cell, and per
 * symbol the offset of its states and the bit-count threshold. */
typedef struct {
    int log;
    uint16_t state[64];
    int32_t find[53];     /* first index of the symbol's states in `state`, minus its count */
    uint32_t nbits[53];   /* (max bits << 16) - (count << max bits) */
} fse_ct;

static void fse_build(fse_ct* ct, const int16_t* norm, int nsym, int log) {
    const int size = 1 << log, mask = size - 1;
    int high = size - 1;
    uint8_t cell_sym[64];
    int next[53];
    int total = 0;
    for (int s = 0; s < nsym; s++) {
        const int c = norm[s] == -1 ? 1 : norm[s];
        if (norm[s] == -1) cell_sym[high--] = (uint8_t)s;
        next[s] = total;
        if (c == 1) {
            ct->nbits[s] = ((uint32_t)log << 16) - (1u << log);
            ct->find[s] = total - 1;
        } else {
            const int mb = log - highbit((uint32_t)c - 1);
            ct->nbits[s] = ((uint32_t)mb << 16) - ((uint32_t)c << mb);
            ct->find[s] = total - c;
        }
        total += c;
    }
    int pos = 0;
    const int step = (size >> 1) + (size >> 3) + 3;
    for (int s = 0; s < nsym; s++)
        for (int i = 0; i < norm[s]; i++) {
            cell_sym[pos] = (uint8_t)s;
            do pos = (pos + step) & mask;
            while (pos > high);
        }
    for (int u = 0; u < size; u++) ct->state[next[cell_sym[u]]++] = (uint16_t)(size + u);
    ct->log = log;
}

/* Forward bit writer, least significant bit first (the decoder reads the
 * stream backwards from its final 1 bit). */
typedef struct {
    uint8_t* p;
    size_t n, cap;
    uint64_t acc;
    int fill;
    int over;
} bitw;

static void bw_add(bitw* w, uint32_t v, int nb) {
    if (!nb) return;
    w->acc |= (uint64_t)(v & ((1u << nb) - 1u)) << w->fill;
    w->fill += nb;
    while (w->fill >= 8) {
        if (w->n < w->cap) w->p[w->n] = (uint8_t)w->acc;
        else w->over = 1;
        w->n++;
        w->acc >>= 8;
        w->fill -= 8;
    }
}

static void bw_close(bitw* w) {
    bw_add(w, 1, 1);
    if (w->fill) bw_add(w, 0, 8 - w->fill);
}

static uint32_t fse_init(const fse_ct* ct, int s) {
    const uint32_t nb = (ct->nbits[s] + (1u << 15)) >> 16;
    const uint32_t v = (nb << 16) - ct->nbits[s];
    return ct->state[(int)(v >> nb) + ct->find[s]];
}

static void fse_enc(bitw* w, const fse_ct* ct, uint32_t* state, int s) {
    const uint32_t nb = (*state + ct->nbits[s]) >> 16;
    bw_add(w, *state, (int)nb);
    *state = ct->state[(int)(*state >> nb) + ct->find[s]];
}

typedef struct {
    uint32_t ll, ml, off;
} zseq;

/* One block's compressed content (literals + sequences sections) from its
 * walked tokens; returns its size, or 0 when it does not fit in cap (the
 * number of bytes the block decodes to: such a block is stored raw). */
static size_t block_content(const uint32_t* tok, size_t ntok, uint8_t* out, size_t cap) {
    static fse_ct LLt, MLt, OFt;
    static int built;
    if (!built) {
        fse_build(&LLt, LL_NORM, 36, 6);
        fse_build(&MLt, ML_NORM, 53, 6);
        fse_build(&OFt, OF_NORM, 29, 5);
        built = 1;
    }
    zseq* seq = malloc((ntok + 1) * sizeof(zseq));
    uint8_t* lit = malloc(ntok + 1);
    if (!seq || !lit) {
        free(seq);
        free(lit);
        return 0;
    }
    size_t nseq = 0, nlit = 0;
    uint32_t run = 0;
    for (size_t i = 0; i < ntok; i++) {
        const uint32_t t = tok[i];
        if ((t >> 16) == 0) {
            lit[nlit++] = (uint8_t)t;
            run++;
        } else {
            seq[nseq].ll = run;
            seq[nseq].ml = t >> 16;
            seq[nseq].off = (t & 0xFFFFu) + 3u;
            nseq++;
            run = 0;
        }
    }
    size_t k = 0;
    const size_t lh = nlit < 32 ? 1 : nlit < 4096 ? 2 : 3;
    const size_t sh = nseq < 128 ? 1 : nseq < 0x7F00 ? 2 : 3;
    if (lh + nlit + sh + (nseq ? 1 : 0) >= cap) goto fail;
    /* literals section: raw */
    if (lh == 1) {
        out[k++] = (uint8_t)(nlit << 3);
    } else if (lh == 2) {
        out[k++] = (uint8_t)(((nlit & 15) << 4) | 4);
        out[k++] = (uint8_t)(nlit >> 4);
    } else {
        out[k++] = (uint8_t)(((nlit & 15) << 4) | 12);
        out[k++] = (uint8_t)(nlit >> 4);
        out[k++] = (uint8_t)(nlit >> 12);
    }
    memcpy(out + k, lit, nlit);
    k += nlit;
    /* sequences section */
    if (sh == 1) {
        out[k++] = (uint8_t)nseq;
    } else if (sh == 2) {
        out[k++] = (uint8_t)((nseq >> 8) + 0x80);
        out[k++] = (uint8_t)nseq;
    } else {
        out[k++] = 0xFF;
        out[k++] = (uint8_t)(nseq - 0x7F00);
        out[k++] = (uint8_t)((nseq - 0x7F00) >> 8);
    }
    if (nseq) {
        out[k++] = 0;  /* predefined modes for all three */
        bitw w = {out + k, 0, cap - k, 0, 0, 0};
        /* the last sequence seeds the states; then every earlier one, each
         * with its state transitions (offset, match length, literal length)
         * and its extra bits (literal length, match length, offset) */
        const zseq* z = &seq[nseq - 1];
        int llc = ll_code(z->ll), mlc = ml_code(z->ml), ofc = highbit(z->off);
        uint32_t sml = fse_init(&MLt, mlc), sof = fse_init(&OFt, ofc), sll = fse_init(&LLt, llc);
        bw_add(&w, z->ll - LL_BASE[llc], LL_BITS[llc]);
        bw_add(&w, z->ml - ML_BASE[mlc], ML_BITS[mlc]);
        bw_add(&w, z->off - (1u << ofc), ofc);
        for (size_t i = nseq - 1; i-- > 0;) {
            z = &seq[i];
            llc = ll_code(z->ll);
            mlc = ml_code(z->ml);
            ofc = highbit(z->off);
            fse_enc(&w, &OFt, &sof, ofc);
            fse_enc(&w, &MLt, &sml, mlc);
            fse_enc(&w, &LLt, &sll, llc);
            bw_add(&w, z->ll - LL_BASE[llc], LL_BITS[llc]);
            bw_add(&w, z->ml - ML_BASE[mlc], ML_BITS[mlc]);
            bw_add(&w, z->off - (1u << ofc), ofc);
        }
        bw_add(&w, sml, MLt.log);
        bw_add(&w, sof, OFt.log);
        bw_add(&w, sll, LLt.log);
        bw_close(&w);
        if (w.over) goto fail;
        k += w.n;
    }
    free(seq);
    free(lit);
    return k < cap ? k : 0;
fail:
    free(seq);
    free(lit);
    return 0;
}

size_t gpzo_zstd_bound(size_t n, size_t member_bytes) {
    const size_t nb = n ? (n + 4095) / 4096 : 1;
    (void)member_bytes;
    return 6 + nb * 3 + n;
}

static size_t put_block(uint8_t* out, int last, const uint8_t* raw, size_t rawlen, const uint8_t* body, size_t c) {
    size_t k = 0;
    const int comp = c && c < rawlen;
    const uint32_t hdr = (uint32_t)last | ((comp ? 2u : 0u) << 1) | ((uint32_t)(comp ? c : rawlen) << 3);
    out[k++] = (uint8_t)hdr;
    out[k++] = (uint8_t)(hdr >> 8);
    out[k++] = (uint8_t)(hdr >> 16);
    memcpy(out + k, comp ? body : raw, comp ? c : rawlen);
    return k + (comp ? c : rawlen);
}

size_t gpzo_zstd_chunk(const uint8_t* in, size_t n, size_t member_bytes, uint8_t* out, size_t cap) {
    if (member_bytes == 0 || member_bytes % 4096 || cap < gpzo_zstd_bound(n, member_bytes)) return 0;
    static const uint8_t hdr[6] = {0x28, 0xB5, 0x2F, 0xFD, 0x00, 0x30};
    size_t k = 0;
    memcpy(out, hdr, 6);
    k = 6;
    if (n == 0) {
        out[k++] = 1;  /* last, raw, size 0 */
        out[k++] = 0;
        out[k++] = 0;
        return k;
    }
    uint32_t* pp = malloc(member_bytes * sizeof(uint32_t));
    uint32_t* tok = malloc(member_bytes * sizeof(uint32_t));
    uint8_t* body = malloc(8192);
    if (!pp || !tok || !body) {
        free(pp);
        free(tok);
        free(body);
        return 0;
    }
    for (size_t o = 0; o < n && k; o += member_bytes) {
        const uint32_t len = (uint32_t)(n - o < member_bytes ? n - o : member_bytes);
        const int last_member = o + len >= n;
        if (gpzo_match_find(in + o, len, pp) != 0) {
            k = 0;
            break;
        }
        const size_t nt = gpzo_greedy_walk(pp, in + o, len, tok);
        /* tokens by the tile their first byte lies in */
        const uint32_t ntiles = (len + 4095) / 4096;
        size_t ti = 0;
        uint32_t pos = 0;
        for (uint32_t t = 0; t < ntiles; t++) {
            const size_t t0 = ti;
            const uint32_t p0 = pos;
            while (ti < nt && pos < (t + 1) * 4096u) {
                const uint32_t l = tok[ti] >> 16;
                pos += l ? l : 1;
                ti++;
            }
            const size_t c = block_content(tok + t0, ti - t0, body, pos - p0);
            k += put_block(out + k, last_member && t + 1 == ntiles, in + o + p0, pos - p0, body, c);
        }
    }
    free(pp);
    free(tok);
    free(body);
    return k;
}
