/*
 * gpz_oracle.c -- CPU oracle for the gzip compression path (TEST INFRASTRUCTURE).
 *
 * Plain-C restatement of the reference GPU codec (skmtkytr/gpzip,
 * crates/gpzip-codec-gpu/src/gpu/...).  Each function cites the reference
 * file:line it follows.  Only tests, the smoke check and the CPU-baseline leg
 * of the benchmark use this file; the CUDA product path never does.
 */
#include "gpz_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define HASH_BITS 16u             /* lz77_hash.rs:43 */
#define HASH_BUCKETS (1u << HASH_BITS)
#define MIN_MATCH 3u              /* lz77_hash.rs:46 */
#define MAX_MATCH 258u            /* lz77_hash.rs:47 */
#define WINDOW 32768u             /* lz77_hash.rs:48, passed by gpu.rs:130-133 */
#define SEG_LOG2 12u              /* lz77_hash.rs:68 */
#define SEG_SIZE (1u << SEG_LOG2)

/* ------------------------------------------------------------------ hash3 */

/* lz77_hash_build.wgsl:36-43 (duplicated at lz77_hash_lookup.wgsl:32-39). */
uint32_t gpzo_hash3(const uint8_t* in, uint32_t p) {
    uint32_t x = ((uint32_t)in[p] << 16) | ((uint32_t)in[p + 1] << 8) | (uint32_t)in[p + 2];
    return (x * 0x9E3779B1u) >> (32u - HASH_BITS);
}

/* --------------------------------------------------------- build + lookup */

/* lz77_hash_lookup.wgsl:45-67 (try_candidate).  Returns the match length if
 * it beats cur_best, else 0; *dist receives the distance. */
static uint32_t try_candidate(const uint8_t* in, uint32_t n, uint32_t raw, uint32_t p,
                              uint32_t cur_best, uint32_t* dist) {
    if (raw == 0u || raw == 0xFFFFFFFFu) return 0;
    uint32_t cand = raw - 1u;
    if (cand >= p) return 0;
    uint32_t d = p - cand;
    if (d > WINDOW) return 0;
    if (in[cand] != in[p] || in[cand + 1] != in[p + 1] || in[cand + 2] != in[p + 2]) return 0;
    uint32_t len = 3;
    for (;;) {
        if (len >= MAX_MATCH) break;
        if (p + len >= n) break;
        if (in[cand + len] != in[p + len]) break;
        len++;
    }
    if (len > cur_best) {
        *dist = d;
        return len;
    }
    return 0;
}

/* lz77_hash.rs:306-453 (match_find) with the two shaders it dispatches:
 * the reset (lz77_hash.rs:409-415), build (lz77_hash_build.wgsl:45-54) and
 * lookup (lz77_hash_lookup.wgsl:69-119).  The dense [hash][segment] tables
 * and the walk over every segment back to 0 are kept as the reference has
 * them; the CUDA path bounds the walk at nine segments and must agree. */
int gpzo_match_find(const uint8_t* in, uint32_t n, uint32_t* pp) {
    if (n == 0) return 0;
    uint32_t num_segs = (n + SEG_SIZE - 1) / SEG_SIZE;
    if (num_segs == 0) num_segs = 1;
    size_t entries = (size_t)HASH_BUCKETS * num_segs;
    uint32_t* oldest = (uint32_t*)malloc(entries * sizeof(uint32_t));
    uint32_t* newest = (uint32_t*)calloc(entries, sizeof(uint32_t));
    if (!oldest || !newest) {
        free(oldest);
        free(newest);
        return -1;
    }
    memset(oldest, 0xFF, entries * sizeof(uint32_t));

    /* build */
    for (uint32_t p = 0; p < n; p++) {
        if (p + 2u >= n) break;
        uint32_t h = gpzo_hash3(in, p);
        uint32_t seg = p >> SEG_LOG2;
        size_t idx = (size_t)h * num_segs + seg;
        if (p + 1u < oldest[idx]) oldest[idx] = p + 1u;
        if (p + 1u > newest[idx]) newest[idx] = p + 1u;
    }

    /* lookup */
    for (uint32_t p = 0; p < n; p++) {
        if (p + 2u >= n) {
            pp[p] = in[p];
            continue;
        }
        uint32_t h = gpzo_hash3(in, p);
        uint32_t p_seg = p >> SEG_LOG2;
        uint32_t best_len = 0, best_dist = 0;
        for (uint32_t off = 0; off <= p_seg; off++) {
            uint32_t seg = p_seg - off;
            size_t idx = (size_t)h * num_segs + seg;
            uint32_t d = 0;
            uint32_t l = try_candidate(in, n, newest[idx], p, best_len, &d);
            if (l > 0) {
                best_len = l;
                best_dist = d;
            }
            if (best_len >= MAX_MATCH) break;
            if (best_len < 16u) {
                l = try_candidate(in, n, oldest[idx], p, best_len, &d);
                if (l > 0) {
                    best_len = l;
                    best_dist = d;
                }
                if (best_len >= MAX_MATCH) break;
            }
        }
        pp[p] = best_len == 0 ? (uint32_t)in[p] : ((best_len << 16) | best_dist);
    }
    free(oldest);
    free(newest);
    return 0;
}

/* deflate.rs:992-1016 (cpu_lz77, the reference encoder tests' token source). */
void gpzo_brute_lz77(const uint8_t* in, uint32_t n, uint32_t window, uint32_t* pp) {
    for (uint32_t pos = 0; pos < n; pos++) {
        uint32_t best_len = 0, best_dist = 0;
        uint32_t start = pos > window ? pos - window : 0;
        for (uint32_t prev = start; prev < pos; prev++) {
            uint32_t len = 0;
            while (pos + len < n && len < 258 && in[prev + len] == in[pos + len]) len++;
            if (len > best_len) {
                best_len = len;
                best_dist = pos - prev;
            }
        }
        pp[pos] = best_len >= 3 ? ((best_len << 16) | best_dist) : (uint32_t)in[pos];
    }
}

/* ------------------------------------------------------------- lazy walk */

/* lz77.rs:260-284 */
size_t gpzo_greedy_walk(const uint32_t* pp, const uint8_t* in, uint32_t n, uint32_t* tokens) {
    size_t out = 0;
    uint32_t p = 0;
    while (p < n) {
        uint32_t t = pp[p];
        uint32_t len = t >> 16;
        if (len == 0) {
            tokens[out++] = t;
            p += 1;
            continue;
        }
        if (p + 1 < n) {
            uint32_t nx = pp[p + 1];
            uint32_t nlen = nx >> 16;
            if (nlen != 0 && nlen > len) {
                tokens[out++] = (uint32_t)in[p];
                p += 1;
                continue;
            }
        }
        tokens[out++] = t;
        p += len;
    }
    return out;
}

/* --------------------------------------------------------------- Huffman */

typedef struct {
    uint64_t f;
    uint32_t id;
} hnode;

static int hless(hnode a, hnode b) { return a.f < b.f || (a.f == b.f && a.id < b.id); }

static void heap_push(hnode* h, int* sz, hnode v) {
    int i = (*sz)++;
    h[i] = v;
    while (i > 0) {
        int par = (i - 1) / 2;
        if (!hless(h[i], h[par])) break;
        hnode t = h[i];
        h[i] = h[par];
        h[par] = t;
        i = par;
    }
}

static hnode heap_pop(hnode* h, int* sz) {
    hnode top = h[0];
    h[0] = h[--(*sz)];
    int i = 0;
    for (;;) {
        int l = 2 * i + 1, r = l + 1, m = i;
        if (l < *sz && hless(h[l], h[m])) m = l;
        if (r < *sz && hless(h[r], h[m])) m = r;
        if (m == i) break;
        hnode t = h[i];
        h[i] = h[m];
        h[m] = t;
        i = m;
    }
    return top;
}

/* huffman.rs:63-117 (standard_huffman + walk).  Min-heap on (freq, id);
 * internal node ids count up from nsym; a leaf's length is its depth,
 * at least 1.  At least two used symbols. */
static void standard_huffman(const uint32_t* freq, int nsym, uint8_t* lens) {
    if (nsym <= 0 || nsym > 320) return;
    hnode heap[2 * 320];
    int left[2 * 320], right[2 * 320];
    int sz = 0;
    for (int i = 0; i < nsym; i++)
        if (freq[i] > 0) heap_push(heap, &sz, (hnode){freq[i], (uint32_t)i});
    int next_id = nsym;
    while (sz > 1) {
        hnode a = heap_pop(heap, &sz);
        hnode b = heap_pop(heap, &sz);
        int id = next_id++;
        left[id] = (int)a.id;
        right[id] = (int)b.id;
        heap_push(heap, &sz, (hnode){a.f + b.f, (uint32_t)id});
    }
    int root = (int)heap[0].id;
    memset(lens, 0, (size_t)nsym);
    /* iterative DFS with an explicit stack of (node, depth) */
    int stack_node[2 * 320], stack_depth[2 * 320], sp = 0;
    stack_node[sp] = root;
    stack_depth[sp++] = 0;
    while (sp > 0) {
        sp--;
        int node = stack_node[sp], depth = stack_depth[sp];
        if (node < nsym) {
            lens[node] = (uint8_t)(depth > 1 ? depth : 1);
            continue;
        }
        stack_node[sp] = right[node];
        stack_depth[sp++] = depth + 1;
        stack_node[sp] = left[node];
        stack_depth[sp++] = depth + 1;
    }
}

/* huffman.rs:26-60 (try_build_code_lengths). */
int gpzo_build_code_lengths(const uint32_t* freq, int nsym, int max_bits, uint8_t* lens) {
    if (nsym <= 0 || nsym > 320) return 0;
    int used = 0, only = -1;
    for (int i = 0; i < nsym; i++)
        if (freq[i] > 0) {
            used++;
            only = i;
        }
    memset(lens, 0, (size_t)nsym);
    if (used == 0) return 1;
    if (used == 1) {
        lens[only] = 1;
        return 1;
    }
    /* required_bits = ceil(log2(used)) (huffman.rs:40-43), computed exactly */
    int required = 0;
    while ((1 << required) < used) required++;
    if (required > max_bits) return 0;
    uint32_t work[320];
    memcpy(work, freq, sizeof(uint32_t) * (size_t)nsym);
    for (;;) {
        standard_huffman(work, nsym, lens);
        int mx = 0;
        for (int i = 0; i < nsym; i++)
            if (lens[i] > mx) mx = lens[i];
        if (mx <= max_bits) return 1;
        for (int i = 0; i < nsym; i++)
            if (work[i] > 1) work[i] /= 2;
    }
}

/* huffman.rs:122-152 (canonical_codes, RFC 1951 3.2.2). */
void gpzo_canonical_codes(const uint8_t* lens, int nsym, uint32_t* codes) {
    int max_bits = 0;
    for (int i = 0; i < nsym; i++)
        if (lens[i] > max_bits) max_bits = lens[i];
    memset(codes, 0, sizeof(uint32_t) * (size_t)nsym);
    if (max_bits == 0) return;
    uint32_t bl_count[16] = {0}, next_code[16] = {0};
    for (int i = 0; i < nsym; i++)
        if (lens[i]) bl_count[lens[i]]++;
    uint32_t code = 0;
    for (int bits = 1; bits <= max_bits; bits++) {
        code = (code + bl_count[bits - 1]) << 1;
        next_code[bits] = code;
    }
    for (int s = 0; s < nsym; s++)
        if (lens[s]) codes[s] = next_code[lens[s]]++;
}

/* ------------------------------------------------------------- encoder */

/* deflate.rs:17-19 */
static const int META_ORDER[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

/* RFC 1951 3.2.5 length and distance rows, as in deflate.rs:96-189 and the
 * LUT builders deflate.rs:502-681: (base, extra bits, symbol). */
static const uint16_t LEN_BASE[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                      31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
static const uint8_t LEN_EXTRA[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                      2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
static const uint16_t DIST_BASE[30] = {1,    2,    3,    4,    5,    7,     9,     13,    17,  25,
                                       33,   49,   65,   97,   129,  193,   257,   385,   513, 769,
                                       1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
static const uint8_t DIST_EXTRA[30] = {0, 0, 0, 0, 1, 1, 2, 2,  3,  3,  4,  4,  5,  5,  6,
                                       6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

/* Symbol index into the 29 length rows: largest base <= length
 * (length_code, deflate.rs:130-140). */
static int len_row(uint32_t length) {
    int idx = 0;
    for (int i = 0; i < 29; i++) {
        if (LEN_BASE[i] <= length) idx = i;
        else break;
    }
    return idx;
}

static int dist_row(uint32_t distance) {
    int idx = 0;
    for (int i = 0; i < 30; i++) {
        if (DIST_BASE[i] <= distance) idx = i;
        else break;
    }
    return idx;
}

/* VecBitWriter (deflate.rs:697-745): u64 accumulator, LSB first. */
typedef struct {
    uint8_t* out;
    size_t len, cap;
    uint64_t acc;
    uint32_t nbits;
    int overflow;
} bitw;

static void bw_put(bitw* w, uint32_t value, uint32_t count) {
    w->acc |= (uint64_t)value << w->nbits;
    w->nbits += count;
    while (w->nbits >= 8) {
        if (w->len < w->cap) w->out[w->len] = (uint8_t)w->acc;
        else w->overflow = 1;
        w->len++;
        w->acc >>= 8;
        w->nbits -= 8;
    }
}

static void bw_finish(bitw* w) {
    if (w->nbits > 0) {
        if (w->len < w->cap) w->out[w->len] = (uint8_t)w->acc;
        else w->overflow = 1;
        w->len++;
    }
}

/* deflate.rs:686-692 */
static uint32_t reverse_bits(uint32_t code, uint32_t bits) {
    if (bits == 0) return 0;
    uint32_t r = 0;
    for (uint32_t i = 0; i < bits; i++)
        if (code & (1u << i)) r |= 1u << (bits - 1 - i);
    return r;
}

typedef struct {
    uint8_t code;
    uint8_t extra_bits;
    uint8_t extra_value;
} rle_entry;

/* deflate.rs:254-326 (rle_encode_lengths). */
static int rle_encode_lengths(const uint8_t* lens, int n, rle_entry* out) {
    int k = 0, i = 0;
    while (i < n) {
        uint8_t cur = lens[i];
        int run = 1;
        while (i + run < n && lens[i + run] == cur) run++;
        if (cur == 0) {
            while (run >= 11) {
                int m = run < 138 ? run : 138;
                out[k++] = (rle_entry){18, 7, (uint8_t)(m - 11)};
                run -= m;
                i += m;
            }
            while (run >= 3) {
                int m = run < 10 ? run : 10;
                out[k++] = (rle_entry){17, 3, (uint8_t)(m - 3)};
                run -= m;
                i += m;
            }
            while (run > 0) {
                out[k++] = (rle_entry){0, 0, 0};
                run--;
                i++;
            }
        } else {
            out[k++] = (rle_entry){cur, 0, 0};
            i++;
            run--;
            while (run >= 3) {
                int m = run < 6 ? run : 6;
                out[k++] = (rle_entry){16, 2, (uint8_t)(m - 3)};
                run -= m;
                i += m;
            }
            while (run > 0) {
                out[k++] = (rle_entry){cur, 0, 0};
                run--;
                i++;
            }
        }
    }
    return k;
}

/* deflate.rs:329-335 */
static int trim_to_min(const uint8_t* lens, int n, int min) {
    while (n > min && lens[n - 1] == 0) n--;
    return n;
}

/* deflate.rs:763-799 (write_fixed_block_fast) with fixed_litlen_pre /
 * fixed_dist_pre (deflate.rs:801-828).  Unreachable in practice because the
 * halving loop always converges; restated for completeness. */
static void write_fixed_block(const uint32_t* tokens, size_t count, bitw* w) {
    bw_put(w, 3, 3);
    for (size_t t = 0; t < count; t++) {
        uint32_t tok = tokens[t];
        uint32_t len = tok >> 16, low = tok & 0xFFFF;
        uint32_t sym, code, bits;
        if (len == 0) sym = low;
        else sym = 257 + (uint32_t)len_row(len);
        if (sym <= 143) { code = 0x30 + sym; bits = 8; }
        else if (sym <= 255) { code = 0x190 + (sym - 144); bits = 9; }
        else if (sym <= 279) { code = sym - 256; bits = 7; }
        else { code = 0xC0 + (sym - 280); bits = 8; }
        bw_put(w, reverse_bits(code, bits), bits);
        if (len != 0) {
            int lr = len_row(len);
            if (LEN_EXTRA[lr]) bw_put(w, len - LEN_BASE[lr], LEN_EXTRA[lr]);
            int dr = dist_row(low);
            bw_put(w, reverse_bits((uint32_t)dr, 5), 5);
            if (DIST_EXTRA[dr]) bw_put(w, low - DIST_BASE[dr], DIST_EXTRA[dr]);
        }
    }
    bw_put(w, reverse_bits(0, 7), 7); /* EOB = symbol 256, code 0, 7 bits */
}

/* deflate.rs:830-959 (try_write_dynamic_block_fast).  Returns 0 where the
 * reference returns false. */
static int write_dynamic_block(const uint32_t* tokens, size_t count, bitw* w) {
    uint32_t litlen_freq[286] = {0}, dist_freq[30] = {0};
    for (size_t t = 0; t < count; t++) {
        uint32_t tok = tokens[t];
        uint32_t len = tok >> 16;
        if (len == 0) {
            litlen_freq[tok & 0xFFFF]++;
        } else {
            litlen_freq[257 + len_row(len)]++;
            dist_freq[dist_row(tok & 0xFFFF)]++;
        }
    }
    litlen_freq[256]++;

    uint8_t litlen_lens[286], dist_lens[30];
    if (!gpzo_build_code_lengths(litlen_freq, 286, 15, litlen_lens)) return 0;
    if (!gpzo_build_code_lengths(dist_freq, 30, 15, dist_lens)) return 0;

    int used_dist = 0, only = -1;
    for (int i = 0; i < 30; i++)
        if (dist_lens[i] > 0) {
            if (only < 0) only = i;
            used_dist++;
        }
    if (used_dist == 0) {
        dist_lens[0] = 1;
        dist_lens[1] = 1;
    } else if (used_dist == 1) {
        dist_lens[only] = 1;
        dist_lens[1 - (only < 1 ? only : 1)] = 1;
    }
    int used_lit = 0;
    for (int i = 0; i < 286; i++)
        if (litlen_lens[i] > 0) used_lit++;
    if (used_lit < 2) {
        litlen_lens[0] = 1;
        litlen_lens[256] = 1;
    }

    uint32_t litlen_codes[286], dist_codes[30], litlen_pre[286], dist_pre[30];
    gpzo_canonical_codes(litlen_lens, 286, litlen_codes);
    gpzo_canonical_codes(dist_lens, 30, dist_codes);
    for (int i = 0; i < 286; i++)
        litlen_pre[i] = litlen_lens[i] ? reverse_bits(litlen_codes[i], litlen_lens[i]) : 0;
    for (int i = 0; i < 30; i++) dist_pre[i] = dist_lens[i] ? reverse_bits(dist_codes[i], dist_lens[i]) : 0;

    int nlit = trim_to_min(litlen_lens, 286, 257);
    int ndist = trim_to_min(dist_lens, 30, 1);
    uint8_t combined[316];
    memcpy(combined, litlen_lens, (size_t)nlit);
    memcpy(combined + nlit, dist_lens, (size_t)ndist);
    rle_entry rle[316];
    int nrle = rle_encode_lengths(combined, nlit + ndist, rle);

    uint32_t meta_freq[19] = {0};
    for (int i = 0; i < nrle; i++) meta_freq[rle[i].code]++;
    uint8_t meta_lens[19];
    if (!gpzo_build_code_lengths(meta_freq, 19, 7, meta_lens)) return 0;
    uint32_t meta_codes[19], meta_pre[19];
    gpzo_canonical_codes(meta_lens, 19, meta_codes);
    for (int i = 0; i < 19; i++) meta_pre[i] = meta_lens[i] ? reverse_bits(meta_codes[i], meta_lens[i]) : 0;

    int hclen_count = 19;
    while (hclen_count > 4 && meta_lens[META_ORDER[hclen_count - 1]] == 0) hclen_count--;

    bw_put(w, 5, 3);
    bw_put(w, (uint32_t)(nlit - 257), 5);
    bw_put(w, (uint32_t)(ndist - 1), 5);
    bw_put(w, (uint32_t)(hclen_count - 4), 4);
    for (int i = 0; i < hclen_count; i++) bw_put(w, meta_lens[META_ORDER[i]], 3);
    for (int i = 0; i < nrle; i++) {
        bw_put(w, meta_pre[rle[i].code], meta_lens[rle[i].code]);
        if (rle[i].extra_bits) bw_put(w, rle[i].extra_value, rle[i].extra_bits);
    }
    for (size_t t = 0; t < count; t++) {
        uint32_t tok = tokens[t];
        uint32_t len = tok >> 16, low = tok & 0xFFFF;
        if (len == 0) {
            bw_put(w, litlen_pre[low], litlen_lens[low]);
        } else {
            int lr = len_row(len);
            int sym = 257 + lr;
            bw_put(w, litlen_pre[sym], litlen_lens[sym]);
            if (LEN_EXTRA[lr]) bw_put(w, len - LEN_BASE[lr], LEN_EXTRA[lr]);
            int dr = dist_row(low);
            bw_put(w, dist_pre[dr], dist_lens[dr]);
            if (DIST_EXTRA[dr]) bw_put(w, low - DIST_BASE[dr], DIST_EXTRA[dr]);
        }
    }
    bw_put(w, litlen_pre[256], litlen_lens[256]);
    return 1;
}

/* deflate.rs:752-761 */
/* write_fixed_block_fast alone (deflate.rs:763-799): the block the
 * reference falls back to, for tests of the fixed-block path. */
size_t gpzo_encode_block_fixed(const uint32_t* tokens, size_t count, uint8_t* out, size_t cap) {
    bitw w = {out, 0, cap, 0, 0, 0};
    write_fixed_block(tokens, count, &w);
    bw_finish(&w);
    if (w.overflow) return 0;
    return w.len;
}

size_t gpzo_encode_block_fast(const uint32_t* tokens, size_t count, uint8_t* out, size_t cap) {
    bitw w = {out, 0, cap, 0, 0, 0};
    if (!write_dynamic_block(tokens, count, &w)) {
        w = (bitw){out, 0, cap, 0, 0, 0};
        write_fixed_block(tokens, count, &w);
    }
    bw_finish(&w);
    if (w.overflow) return 0;
    return w.len;
}

/* ----------------------------------------------------------------- CRC-32 */

static uint32_t crc_table[256];
static pthread_once_t crc_once = PTHREAD_ONCE_INIT;

static void crc_init(void) {
    for (uint32_t i = 0; i < 256; i++) {
        uint32_t c = i;
        for (int k = 0; k < 8; k++) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
        crc_table[i] = c;
    }
}

uint32_t gpzo_crc32(const uint8_t* in, size_t n) {
    pthread_once(&crc_once, crc_init);
    uint32_t c = 0xFFFFFFFFu;
    for (size_t i = 0; i < n; i++) c = crc_table[(c ^ in[i]) & 0xFF] ^ (c >> 8);
    return c ^ 0xFFFFFFFFu;
}

/* ------------------------------------------------------------ gzip member */

size_t gpzo_member_bound(size_t n) {
    /* header 10 + trailer 8 + dynamic block header (<= 3+14+57+316*14 bits)
     * + 15 bits per input byte + EOB, rounded up generously */
    return 18 + 1024 + (15 * n + 7) / 8 + 8;
}

/* gpu.rs:271-287 (encode_one) + deflate.rs:962-980 (gzip_wrap). */
size_t gpzo_gzip_member(const uint8_t* in, uint32_t n, uint8_t* out, size_t cap) {
    static const uint8_t header[10] = {0x1f, 0x8b, 0x08, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0xff};
    if (cap < 18) return 0;
    uint32_t* pp = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t* tok = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    if (!pp || !tok) {
        free(pp);
        free(tok);
        return 0;
    }
    size_t ntok = 0;
    if (n > 0) {
        if (gpzo_match_find(in, n, pp) != 0) {
            free(pp);
            free(tok);
            return 0;
        }
        ntok = gpzo_greedy_walk(pp, in, n, tok);
    }
    memcpy(out, header, 10);
    size_t dl = gpzo_encode_block_fast(tok, ntok, out + 10, cap - 18);
    free(pp);
    free(tok);
    if (dl == 0) return 0;
    uint32_t crc = gpzo_crc32(in, n);
    uint8_t* t = out + 10 + dl;
    for (int i = 0; i < 4; i++) t[i] = (uint8_t)(crc >> (8 * i));
    for (int i = 0; i < 4; i++) t[4 + i] = (uint8_t)(n >> (8 * i));
    return 10 + dl + 8;
}

typedef struct {
    const uint8_t* in;
    size_t n, member_bytes, nmem;
    uint8_t** bufs;
    size_t* lens;
    size_t next;
    pthread_mutex_t mu;
    int failed;
} chunk_job;

static void* chunk_worker(void* arg) {
    chunk_job* j = (chunk_job*)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        size_t m = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (m >= j->nmem) break;
        size_t off = m * j->member_bytes;
        size_t len = j->n - off < j->member_bytes ? j->n - off : j->member_bytes;
        size_t cap = gpzo_member_bound(len);
        j->bufs[m] = (uint8_t*)malloc(cap);
        if (!j->bufs[m]) {
            j->failed = 1;
            continue;
        }
        j->lens[m] = gpzo_gzip_member(j->in + off, (uint32_t)len, j->bufs[m], cap);
        if (j->lens[m] == 0) j->failed = 1;
    }
    return NULL;
}

/* gpu.rs:193-208 (gzip_chunk_fn): a chunk of at most member_bytes (an empty
 * one included) is one member; a larger one becomes ceil(n / member_bytes)
 * members. */
size_t gpzo_gzip_chunk(const uint8_t* in, size_t n, size_t member_bytes, uint8_t* out, size_t cap,
                       int threads) {
    if (member_bytes == 0) return 0;
    if (n <= member_bytes) return gpzo_gzip_member(in, (uint32_t)n, out, cap);
    chunk_job j;
    memset(&j, 0, sizeof j);
    j.in = in;
    j.n = n;
    j.member_bytes = member_bytes;
    j.nmem = (n + member_bytes - 1) / member_bytes;
    j.bufs = (uint8_t**)calloc(j.nmem, sizeof(uint8_t*));
    j.lens = (size_t*)calloc(j.nmem, sizeof(size_t));
    pthread_mutex_init(&j.mu, NULL);
    if (threads < 1) threads = 1;
    if ((size_t)threads > j.nmem) threads = (int)j.nmem;
    pthread_t tid[256];
    if (threads > 256) threads = 256;
    for (int t = 1; t < threads; t++) pthread_create(&tid[t], NULL, chunk_worker, &j);
    chunk_worker(&j);
    for (int t = 1; t < threads; t++) pthread_join(tid[t], NULL);
    size_t total = 0;
    for (size_t m = 0; m < j.nmem && !j.failed; m++) {
        if (total + j.lens[m] > cap) {
            j.failed = 1;
            break;
        }
        memcpy(out + total, j.bufs[m], j.lens[m]);
        total += j.lens[m];
    }
    for (size_t m = 0; m < j.nmem; m++) free(j.bufs[m]);
    free(j.bufs);
    free(j.lens);
    pthread_mutex_destroy(&j.mu);
    return j.failed ? 0 : total;
}
