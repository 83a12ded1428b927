// gpz_kernels.cu -- sm_100a kernels of the gzip compression path.
//
// Kernels of one batch, in launch order.  The persistent ones claim work
// items (4 KiB tiles, or members) from a device counter and read the batch's
// member / tile counts from device memory, so one captured launch sequence
// serves every batch of a size bucket:
//
//   k_segtab     per tile: the 4 KiB segment's distinct hashes with their
//                oldest / newest offsets (what lz77_hash_build.wgsl:45-54
//                leaves in table[h][seg]) and a per-position hash id.
//   k_lookup     per tile: window-bounded candidate walk over the tile and
//                the 8 segments before it (lz77_hash_lookup.wgsl:45-119),
//                one packed token per position (pp).
//   k_walk_exit  per tile: exit offset for each of the 258 entry offsets of
//                the lazy walk (lz77.rs:260-284), by pointer jumping.
//                (its last CTA: the entry offset of every tile, by member)
//   k_walk_mark  per tile: walked tokens in order and the tile's symbol
//                histogram.
//   k_huff       per member: CRC-32, length-limited codes (huffman.rs:26-152),
//                dynamic block header (deflate.rs:830-932), exact bit plan
//                per tile (its last CTA: every member's output offset).
//   k_frame      per member: gzip header words, shared boundary words, EOB.
//   k_emit       per tile: per-token codes and bit packing
//                (deflate.rs:934-958) into the batch's gzip stream.
//   k_drain      optional: output and member table into mapped host memory.
//
// All arithmetic is integer and bit-exact with the reference.
#include <cuda_runtime.h>

#include <cstdint>

#include "gpz_internal.h"

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr uint32_t kCrcPoly = 0xEDB88320u;

// x^(8 * 2^k) mod P, reflected, k = 0..31 (filled by gpz_kernel_smem_setup).
__constant__ uint32_t c_x8pow2[32];

// RFC 1951 3.2.5 rows (deflate.rs:99-189).
__constant__ uint16_t c_len_base[29] = {3,  4,  5,  6,  7,  8,  9,  10,  11,  13,  15,  17,  19,  23, 27,
                                        31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
__constant__ uint16_t c_dist_base[30] = {1,    2,    3,    4,    5,    7,    9,    13,    17,    25,
                                         33,   49,   65,   97,   129,  193,  257,  385,   513,   769,
                                         1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
// deflate.rs:17-19
__constant__ uint8_t c_meta_order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ uint32_t len_row(uint32_t len) {  // length 3..258 -> row 0..28
    if (len == 258u) return 28u;
    if (len <= 10u) return len - 3u;
    uint32_t x = len - 3u, k = 31u - __clz(x);
    return 4u * (k - 1u) + ((x >> (k - 2u)) & 3u);
}
__device__ __forceinline__ uint32_t len_extra_bits(uint32_t row) {
    return (row < 8u || row == 28u) ? 0u : (row - 4u) >> 2;
}
__device__ __forceinline__ uint32_t dist_row(uint32_t d) {  // distance 1..32768 -> row 0..29
    if (d <= 4u) return d - 1u;
    uint32_t x = d - 1u, k = 31u - __clz(x);
    return 2u * k + ((x >> (k - 1u)) & 1u);
}
__device__ __forceinline__ uint32_t dist_extra_bits(uint32_t row) { return row < 4u ? 0u : (row - 2u) >> 1; }

// Polynomial product mod P in the reflected CRC-32 domain (bit 31 = x^0).
__device__ uint32_t gf2_mulmod(uint32_t a, uint32_t b) {
    uint32_t m = 1u << 31, p = 0;
    while (m) {
        if (a & m) {
            p ^= b;
            if ((a & (m - 1u)) == 0) break;
        }
        m >>= 1;
        b = (b & 1u) ? (b >> 1) ^ kCrcPoly : b >> 1;
    }
    return p;
}
// x^(8 n) mod P
__device__ uint32_t x8pow(uint32_t n) {
    uint32_t r = 1u << 31;
    for (int k = 0; n; k++, n >>= 1)
        if (n & 1u) r = gf2_mulmod(r, c_x8pow2[k]);
    return r;
}

// Match length at window offsets a < b, capped at limit: 16 bytes per step,
// first difference from the lowest set bit of the XOR (__clz of the
// bit-reversed word).
__device__ __forceinline__ uint32_t match_len(const uint32_t* w, uint32_t a, uint32_t b, uint32_t limit) {
    const uint32_t sa = (a & 3u) * 8u, sb = (b & 3u) * 8u;
    uint32_t ia = a >> 2, ib = b >> 2;
    uint32_t a0 = w[ia], b0 = w[ib];
    for (uint32_t l = 0; l < limit; l += 16u) {
        uint32_t a1 = w[ia + 1], a2 = w[ia + 2], a3 = w[ia + 3], a4 = w[ia + 4];
        uint32_t b1 = w[ib + 1], b2 = w[ib + 2], b3 = w[ib + 3], b4 = w[ib + 4];
        uint32_t x0 = __funnelshift_r(a0, a1, sa) ^ __funnelshift_r(b0, b1, sb);
        uint32_t x1 = __funnelshift_r(a1, a2, sa) ^ __funnelshift_r(b1, b2, sb);
        uint32_t x2 = __funnelshift_r(a2, a3, sa) ^ __funnelshift_r(b2, b3, sb);
        uint32_t x3 = __funnelshift_r(a3, a4, sa) ^ __funnelshift_r(b3, b4, sb);
        uint32_t r = 0xFFFFFFFFu;
        if (x0) r = __clz(__brev(x0)) >> 3;
        else if (x1) r = 4u + (__clz(__brev(x1)) >> 3);
        else if (x2) r = 8u + (__clz(__brev(x2)) >> 3);
        else if (x3) r = 12u + (__clz(__brev(x3)) >> 3);
        if (r != 0xFFFFFFFFu) return min(l + r, limit);
        ia += 4;
        ib += 4;
        a0 = a4;
        b0 = b4;
    }
    return limit;
}

// The first 16 bytes at window offset b as little-endian words: a
// position loads them once and compares every candidate's first 16 bytes
// against registers.
struct Head {
    uint32_t x0, x1, x2, x3;
};

__device__ __forceinline__ Head load_head(const uint32_t* w, uint32_t b) {
    const uint32_t sb = (b & 3u) * 8u, ib = b >> 2;
    const uint32_t b0 = w[ib], b1 = w[ib + 1], b2 = w[ib + 2], b3 = w[ib + 3], b4 = w[ib + 4];
    return Head{__funnelshift_r(b0, b1, sb), __funnelshift_r(b1, b2, sb), __funnelshift_r(b2, b3, sb),
                __funnelshift_r(b3, b4, sb)};
}

// try_candidate (lz77_hash_lookup.wgsl:45-67) on packed best = len<<16|dist,
// for a candidate already known to be valid: it lies before p and at most
// 32768 bytes back (the caller checks what its segment does not imply).
// `a` and `b` are the window offsets of the candidate and of p.  A
// candidate that cannot beat the current best is dropped early: it must
// agree with p at offset best_len, and best_len must be below the cap.  The
// first 16 bytes are compared with p's Head; only a candidate that agrees on
// all of them continues in match_len.
__device__ __forceinline__ void try_win(const uint8_t* win, const uint32_t* w32, const Head& hp, uint32_t a,
                                        uint32_t b, uint32_t dist, uint32_t limit, uint32_t& best) {
    const uint32_t bl = best >> 16;
    if (bl >= limit) return;
    if (bl >= 3u && win[a + bl] != win[b + bl]) return;
    const uint32_t sa = (a & 3u) * 8u, ia = a >> 2;
    const uint32_t a0 = w32[ia], a1 = w32[ia + 1], a2 = w32[ia + 2], a3 = w32[ia + 3], a4 = w32[ia + 4];
    const uint32_t x0 = __funnelshift_r(a0, a1, sa) ^ hp.x0;
    const uint32_t x1 = __funnelshift_r(a1, a2, sa) ^ hp.x1;
    const uint32_t x2 = __funnelshift_r(a2, a3, sa) ^ hp.x2;
    const uint32_t x3 = __funnelshift_r(a3, a4, sa) ^ hp.x3;
    uint32_t len;
    if (x0) len = __clz(__brev(x0)) >> 3;
    else if (x1) len = 4u + (__clz(__brev(x1)) >> 3);
    else if (x2) len = 8u + (__clz(__brev(x2)) >> 3);
    else if (x3) len = 12u + (__clz(__brev(x3)) >> 3);
    else len = limit > 16u ? 16u + match_len(w32, a + 16u, b + 16u, limit - 16u) : 16u;
    len = min(len, limit);
    if (len >= 3u && len > bl) best = (len << 16) | dist;
}

template <int T>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* warp_sums, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < T / 32 ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < T / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    uint32_t before = warp ? warp_sums[warp - 1] : 0u;
    *total = warp_sums[T / 32 - 1];
    uint32_t r = before + x - v;
    __syncthreads();
    return r;
}


// =============================================================== k_segtab

// The reference's dense seg_oldest / seg_newest tables (65536 x num_segs,
// lz77_hash_build.wgsl:45-54) are never materialised.  Instead every 4 KiB
// segment is summarised once: its distinct hashes in ascending order, each
// with its oldest and newest offset -- exactly the two values the
// reference's atomicMin / atomicMax leave in table[h][seg].  A hash's index
// in that order (its id) is its rank in the segment's set of hashes.  The
// set is a 65536-bit bitmap in shared memory, and the rank is the number of
// set bits before it: a prefix count per 32-bit word plus a popcount inside
// the word.  k_lookup rebuilds the same bitmap from the keys, so both
// kernels give a hash the same id without probing a table.  Positions with
// p + 2 >= n have no hash, as in the reference build.
constexpr int kBmWords = 65536 / 32;

struct SegtabSmem {
    static constexpr size_t kBitmap = 0;                       // u32[2048] the segment's hash set
    static constexpr size_t kPrefix = kBitmap + kBmWords * 4;  // u32[2048] set bits before each word
    static constexpr size_t kOld = kPrefix + kBmWords * 4;     // u32[4096] oldest offset per id
    static constexpr size_t kNew = kOld + GPZ_SEG * 4;         // u32[4096] newest offset per id
    static constexpr size_t kKey = kNew + GPZ_SEG * 4;         // u16[4096] hash of each id
    static constexpr size_t kBytes = kKey + GPZ_SEG * 2;
};

// hash3 of the bytes s[0..2] (lz77_hash_build.wgsl:36-43)
__device__ __forceinline__ uint32_t hash3_at(const uint8_t* s) {
    const uint32_t x = ((uint32_t)s[0] << 16) | ((uint32_t)s[1] << 8) | (uint32_t)s[2];
    return (x * 0x9E3779B1u) >> 16;
}

template <int T>
__global__ void __launch_bounds__(T, 3) k_segtab(BatchParams bp) {
    constexpr int PER = GPZ_SEG / T;
    constexpr int WPT = kBmWords / T;
    extern __shared__ __align__(16) uint8_t smem[];
    uint32_t* bm = reinterpret_cast<uint32_t*>(smem + SegtabSmem::kBitmap);
    uint32_t* pre = reinterpret_cast<uint32_t*>(smem + SegtabSmem::kPrefix);
    uint32_t* oldt = reinterpret_cast<uint32_t*>(smem + SegtabSmem::kOld);
    uint32_t* newt = reinterpret_cast<uint32_t*>(smem + SegtabSmem::kNew);
    uint16_t* keyof = reinterpret_cast<uint16_t*>(smem + SegtabSmem::kKey);
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t ntiles = bp.dims[0];
    for (;;) {
        __syncthreads();
        if (tid == 0) s_tile = atomicAdd(&bp.counters[GPZ_CNT_SEGSORT], 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        const uint32_t n = md.len, start = td.seg << GPZ_SEG_LOG2;
        const uint32_t cnt = min(GPZ_SEG, n - start);
        const uint8_t* src = bp.in + md.in_off + start;
        for (int i = tid; i < kBmWords; i += T) bm[i] = 0u;
        for (int i = tid; i < (int)GPZ_SEG; i += T) {
            oldt[i] = kEmpty;
            newt[i] = 0u;
        }
        __syncthreads();
        // the segment's hash set; lanes of a warp hold consecutive positions
        uint32_t hv[PER];
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t i = (uint32_t)(k * T + tid);
            hv[k] = kEmpty;
            if (i < cnt && start + i + 2u < n) {
                hv[k] = hash3_at(src + i);
                atomicOr(&bm[hv[k] >> 5], 1u << (hv[k] & 31u));
            }
        }
        __syncthreads();
        // exclusive prefix count of set bits over the bitmap words
        uint32_t c[WPT], sum = 0, nkeys = 0;
#pragma unroll
        for (int j = 0; j < WPT; j++) {
            c[j] = __popc(bm[tid * WPT + j]);
            sum += c[j];
        }
        uint32_t run = block_excl_scan<T>(sum, wsum, &nkeys);
#pragma unroll
        for (int j = 0; j < WPT; j++) {
            pre[tid * WPT + j] = run;
            run += c[j];
        }
        __syncthreads();
        // oldest / newest per id: one atomic per run of equal ids in a warp,
        // its first lane for the oldest and its last lane for the newest
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t i = (uint32_t)(k * T + tid), h = hv[k];
            uint32_t id = kEmpty;
            if (h != kEmpty) {
                const uint32_t w = h >> 5;
                id = pre[w] + __popc(bm[w] & ((1u << (h & 31u)) - 1u));
                keyof[id] = (uint16_t)h;
            }
            const uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, id, 1);
            const uint32_t next = __shfl_down_sync(0xFFFFFFFFu, id, 1);
            if (id != kEmpty) {
                if (lane == 0 || prev != id) atomicMin(&oldt[id], i);
                if (lane == 31 || next != id) atomicMax(&newt[id], i);
            }
        }
        __syncthreads();
        uint16_t* keys = bp.seg_keys + (size_t)t * GPZ_SEG;
        uint32_t* on = bp.seg_on + (size_t)t * GPZ_SEG;
        for (uint32_t id = tid; id < nkeys; id += T) {
            keys[id] = keyof[id];
            on[id] = newt[id] | (oldt[id] << 16);
        }
        if (tid == 0) bp.seg_nkeys[t] = nkeys;
    }
}

// ================================================================ k_lookup

// Candidate rows: [id][bpp] entries newest | oldest << 16, one per back
// segment of the current pass (kEmpty: the hash does not occur there).  A
// tile with at most 1280 distinct hashes joins all 8 back segments in one
// pass, up to 2560 in two passes of 4, more in four passes of 2.
constexpr uint32_t kRowEntries = 10240;

struct LookupSmem {
    static constexpr size_t kWin = 0;                          // the window's bytes
    static constexpr size_t kBitmap = kWin + GPZ_WIN_BYTES;    // u32[2048] the tile's hash set
    static constexpr size_t kPrefix = kBitmap + kBmWords * 4;  // u16[2048] ids before each word
    static constexpr size_t kOwnOld = kPrefix + kBmWords * 2;  // u16[4096] oldest offset per id
    static constexpr size_t kBest = kOwnOld + GPZ_SEG * 2;     // u32[4096] best so far per position
    static constexpr size_t kRows = kBest + GPZ_SEG * 4;       // u32[kRowEntries]
    static constexpr size_t kBytes = kRows + kRowEntries * 4;
};
static_assert(LookupSmem::kRows % 16 == 0, "candidate rows are cleared with 16-byte stores");
static_assert(kRowEntries % 4 == 0 && kRowEntries / 2 >= GPZ_SEG, "four passes must hold any tile");

// One CTA per 4 KiB tile S of a member (persistent over tiles); two CTAs
// share an SM, so one's barriers and loads overlap the other's candidate
// evaluation.  The launch bound holds every form to two CTAs per SM:
// 56 registers at 512 threads, 40 at 768, 32 at 1024 (48 and 64 warps per
// SM), none of them spilling; the shared memory (115,008 bytes) fits twice.  The window [S-8, S] plus 320 bytes of lookahead is staged in
// shared memory, and the tile's hash set is rebuilt from its keys.  The
// keys of segments S-1 .. S-8 are looked up in that set, which gives, for
// every hash of the tile, the newest and oldest position in each of those
// segments: the reference's table[h][seg] entries, for exactly the hashes
// this tile queries.  Segments more than 8 back are never reachable: their
// nearest position is more than 32768 bytes from any p in S, which
// try_candidate rejects.  Then every position runs the reference's
// candidate sequence (lz77_hash_lookup.wgsl:69-119): own segment (its
// newest is always >= p, so only the oldest), then S-1 .. S-8, newest, then
// oldest while best < 16.  When the rows of all 8 back segments do not fit,
// the back segments are joined and evaluated a few at a time, in order,
// with each position's best carried between passes.
template <int T>
__global__ void __launch_bounds__(T, 2) k_lookup(BatchParams bp) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint8_t* win = smem + LookupSmem::kWin;
    const uint32_t* w32 = reinterpret_cast<const uint32_t*>(win);
    uint32_t* bm = reinterpret_cast<uint32_t*>(smem + LookupSmem::kBitmap);
    uint16_t* pre = reinterpret_cast<uint16_t*>(smem + LookupSmem::kPrefix);
    uint16_t* own_old = reinterpret_cast<uint16_t*>(smem + LookupSmem::kOwnOld);
    uint32_t* bestv = reinterpret_cast<uint32_t*>(smem + LookupSmem::kBest);
    uint32_t* rows = reinterpret_cast<uint32_t*>(smem + LookupSmem::kRows);
    constexpr int PER = (GPZ_SEG + T - 1) / T;  // keys per thread in the join
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x;

    const uint32_t ntiles = bp.dims[0];
    for (;;) {
        __syncthreads();
        if (tid == 0) s_tile = atomicAdd(&bp.counters[GPZ_CNT_LOOKUP], 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        const uint32_t n = md.len, S = td.seg, start = S << GPZ_SEG_LOG2;
        const uint32_t cnt = min(GPZ_SEG, n - start);
        const uint32_t w0 = S >= 8u ? (S - 8u) << GPZ_SEG_LOG2 : 0u;
        const uint32_t wvalid = min(n - w0, (uint32_t)GPZ_WIN_BYTES);
        const uint32_t pl0 = start - w0;
        const uint32_t nback = min(S, 8u);
        const uint32_t nown = min(bp.seg_nkeys[t], GPZ_SEG);
        const uint32_t bpp = nown <= kRowEntries / 8u ? 8u : nown <= kRowEntries / 4u ? 4u : 2u;
        const uint32_t npass = nback ? (nback + bpp - 1u) / bpp : 1u;

        // ---- stage the window [w0, w0 + wvalid) (16-byte vectors; members
        // are 16-byte aligned and padded in the batch input); clear the set
        {
            const uint4* src = reinterpret_cast<const uint4*>(bp.in + md.in_off + w0);
            uint4* dst = reinterpret_cast<uint4*>(win);
            const uint32_t nvec = (wvalid + 15u) >> 4;
            for (uint32_t i = tid; i < nvec; i += T) dst[i] = __ldg(src + i);
            for (uint32_t i = tid; i < (uint32_t)kBmWords; i += T) bm[i] = 0u;
            for (uint32_t i = tid; i < cnt; i += T) bestv[i] = 0u;
            __syncthreads();
            const uint32_t zend = min((uint32_t)GPZ_WIN_BYTES, (nvec << 4) + 32u);
            for (uint32_t i = wvalid + tid; i < zend; i += T) win[i] = 0;
            // the tile's hash set; its keys ascend, so a key's index is its
            // rank, and the first key of each word gives the word's prefix
            const uint16_t* gk = bp.seg_keys + (size_t)t * GPZ_SEG;
            const uint32_t* go = bp.seg_on + (size_t)t * GPZ_SEG;
            for (uint32_t i = tid; i < nown; i += T) {
                const uint32_t h = gk[i];
                atomicOr(&bm[h >> 5], 1u << (h & 31u));
                if (i == 0u || (uint32_t)(gk[i - 1u] >> 5) != (h >> 5)) pre[h >> 5] = (uint16_t)i;
                own_old[i] = (uint16_t)(go[i] >> 16);
            }
        }

        for (uint32_t pass = 0; pass < npass; pass++) {
            const uint32_t b0 = 1u + pass * bpp;
            const uint32_t nb = nback >= b0 ? min(bpp, nback - b0 + 1u) : 0u;
            // ---- this pass's rows: cleared, then the join of its back
            // segments (their keys probe the tile's set; a key found there
            // writes its segment's newest | oldest into the key's row)
            __syncthreads();
            {
                uint4* r4 = reinterpret_cast<uint4*>(rows);
                const uint32_t n4 = (nown * bpp + 3u) >> 2;
                for (uint32_t r = tid; r < n4; r += T) r4[r] = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
            }
            __syncthreads();
            for (uint32_t j = 0; j < nb; j++) {
                const uint32_t ts = t - (b0 + j);
                const uint32_t ns = min(bp.seg_nkeys[ts], GPZ_SEG);
                const uint16_t* gk = bp.seg_keys + (size_t)ts * GPZ_SEG;
                const uint32_t* go = bp.seg_on + (size_t)ts * GPZ_SEG;
                uint32_t hk[PER], ov[PER];
#pragma unroll
                for (int u = 0; u < PER; u++) {
                    const uint32_t q = tid + (uint32_t)u * T;
                    hk[u] = kEmpty;
                    ov[u] = 0u;
                    if (q < ns) {
                        hk[u] = gk[q];
                        ov[u] = go[q];
                    }
                }
#pragma unroll
                for (int u = 0; u < PER; u++) {
                    const uint32_t h = hk[u];
                    if (h == kEmpty) continue;
                    const uint32_t w = h >> 5, word = bm[w], bit = 1u << (h & 31u);
                    if (!(word & bit)) continue;
                    const uint32_t id = pre[w] + __popc(word & (bit - 1u));
                    if (id < nown) rows[id * bpp + j] = ov[u];
                }
            }
            __syncthreads();

            // ---- every position tries this pass's candidates in the
            // reference's order
#pragma unroll 1
            for (uint32_t i = tid; i < cnt; i += T) {
                if (start + i + 2u >= n) continue;  // no hash: a literal
                const uint32_t b = pl0 + i;
                const uint32_t h = hash3_at(win + b);
                const uint32_t w = h >> 5, word = bm[w], bit = 1u << (h & 31u);
                const uint32_t id = pre[w] + __popc(word & (bit - 1u));
                if (!(word & bit) || id >= nown) continue;  // never: the tile's own hash is in its set
                const uint32_t limit = min(GPZ_MAX_MATCH, n - start - i);
                uint32_t best = bestv[i];
                if ((best >> 16) >= limit) continue;
                const Head hp = load_head(w32, b);
                if (pass == 0u) {
                    const uint32_t oo = own_old[id];
                    if (oo < i) try_win(win, w32, hp, pl0 + oo, b, i - oo, limit, best);
                }
                const uint32_t* row = rows + id * bpp;
                for (uint32_t j = 0; j < nb; j++) {
                    const uint32_t on = row[j];
                    if (on == kEmpty) continue;
                    const uint32_t back = b0 + j;
                    const uint32_t qa = pl0 - (back << GPZ_SEG_LOG2);  // segment S - back in the window
                    const uint32_t on_n = on & 0xFFFFu, on_o = on >> 16;
                    // a candidate up to 7 segments back is within 32767
                    // bytes of p; 8 back, only if p's offset is at most its own
                    if (back < 8u || i <= on_n)
                        try_win(win, w32, hp, qa + on_n, b, (back << GPZ_SEG_LOG2) + i - on_n, limit, best);
                    if ((best >> 16) < 16u && on_o != on_n && (back < 8u || i <= on_o))
                        try_win(win, w32, hp, qa + on_o, b, (back << GPZ_SEG_LOG2) + i - on_o, limit, best);
                }
                bestv[i] = best;
            }
        }
        __syncthreads();

        // ---- pp of the tile: the best match, or the literal byte
        uint32_t* dst = bp.pp + md.in_off + start;
        for (uint32_t i = tid; i < cnt; i += T) {
            const uint32_t best = bestv[i];
            dst[i] = (best >> 16) ? best : (uint32_t)win[pl0 + i];
        }
    }
}

// ================================================================== k_walk

// The lazy walk of lz77.rs:260-284 visits p, next(p), next(next(p)), ...
// where next(p) depends only on pp[p] and pp[p+1].  Each 4 KiB tile is walked
// on its own: k_walk_exit computes, for every position a walk can enter the
// tile at (its first 258), where it leaves, and its last CTA strings the
// tiles of a member together (entry of tile b+1 = exit of tile b at its
// entry);
// k_walk_mark walks from the known entry and emits the visited tokens in
// order with the tile's symbol histogram.  Two forms with identical output:
//   warp  one warp per tile, 32 positions at a time, links inside a window
//         resolved by pointer doubling over shuffles: little shared memory,
//         many tiles in flight per SM -- the throughput form;
//   block one CTA per tile, pointer doubling over all 4096 links in shared
//         memory (13 rounds): the lowest latency per tile -- the form for
//         small batches, where a tile's latency is the batch's.

constexpr uint32_t kFull = 0xFFFFFFFFu;

// Defined below: the per-member tile chaining run by the last CTA of
// k_walk_exit, the member placement run by the last CTA of k_huff, and the
// last-CTA test itself.
__device__ void chain_members(const BatchParams& bp);
template <int T>
__device__ void place_members(const BatchParams& bp, unsigned long long* wsum, unsigned long long& carry);
__device__ bool last_cta_done(uint32_t* counter);

// next(p) (lz77.rs:266-282): a literal advances by one; a match advances by
// its length unless pp[p+1] is a longer match (lazy demotion to a literal).
__device__ __forceinline__ uint32_t walk_next(uint32_t i, uint32_t v, uint32_t v1, bool has_next) {
    const uint32_t l = v >> 16;
    if (!l) return i + 1u;
    const uint32_t l1 = v1 >> 16;
    return (has_next && l1 != 0u && l1 > l) ? i + 1u : i + l;
}

// Warp-per-tile exit tables.  For position p of a full tile, exit(p) is
// next(p) - 4096 if next(p) leaves the tile, else exit(next(p)); windows are
// resolved from the top, so every link that leaves a window lands on a
// position whose exit is known.  A link reaches at most 258 ahead, so only
// the last 16 windows of exits are kept (ring of 512 per warp).
template <int T>
__global__ void __launch_bounds__(T) k_walk_exit_warp(BatchParams bp) {
    constexpr int W = T / 32;
    constexpr uint32_t kRing = 512;
    __shared__ uint16_t ring[W][kRing];
    const int lane = threadIdx.x & 31;
    uint16_t* ex = ring[threadIdx.x >> 5];
    const uint32_t ntiles = bp.dims[0];
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&bp.counters[GPZ_CNT_EXIT], 1u);
        t = __shfl_sync(kFull, t, 0);
        if (t >= ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        if (td.seg + 1u == md.ntiles) continue;  // the member's last tile has no successor
        // not the last tile: it is full and pp[4096] (the next tile's first
        // position) exists
        constexpr uint32_t cnt = GPZ_SEG;
        const uint32_t* ppg = bp.pp + md.in_off + (td.seg << GPZ_SEG_LOG2);
        uint32_t above = ppg[cnt];  // pp just above the current window
        // the current window and the next two below it, loaded ahead
        uint32_t q0 = ppg[cnt - 32u + lane], q1 = ppg[cnt - 64u + lane], q2 = ppg[cnt - 96u + lane];
        for (int base = (int)cnt - 32; base >= 0; base -= 32) {
            const uint32_t v = q0;
            q0 = q1;
            q1 = q2;
            if (base >= 96) q2 = ppg[base - 96 + lane];
            uint32_t v1 = __shfl_down_sync(kFull, v, 1);
            if (lane == 31) v1 = above;
            above = __shfl_sync(kFull, v, 0);
            const uint32_t p = (uint32_t)base + lane;
            const uint32_t nx = walk_next(p, v, v1, true);
            uint32_t val = 0u, tgt = 32u;
            if (nx >= cnt) val = nx - cnt;
            else if (nx >= (uint32_t)base + 32u) val = ex[nx & (kRing - 1u)];
            else tgt = nx - (uint32_t)base;
            // at most 5 rounds; done as soon as every lane is resolved
            for (int r = 0; r < 5 && __any_sync(kFull, tgt < 32u); r++) {
                const uint32_t pv = __shfl_sync(kFull, val, tgt & 31u);
                const uint32_t pt = __shfl_sync(kFull, tgt, tgt & 31u);
                if (tgt < 32u) {
                    val = pv;
                    tgt = pt;
                }
            }
            __syncwarp();
            ex[p & (kRing - 1u)] = (uint16_t)val;
            __syncwarp();
        }
        for (int e = lane; e < GPZ_EXITS; e += 32) bp.tile_exit[(size_t)t * GPZ_EXITS + e] = ex[e];
        __syncwarp();
    }
    // the last CTA strings every member's tiles together
    if (last_cta_done(&bp.counters[GPZ_CNT_EXIT_DONE])) chain_members(bp);
}

// ---- block form: one CTA per tile

struct WalkLinks {
    uint32_t pps[GPZ_SEG + 1];              // pp of the tile and one lookahead
    uint16_t nxt[GPZ_SEG];                  // next position, tile-relative
    uint16_t J[2][GPZ_SEG + GPZ_EXITS];     // doubled links, absorbing past the tile
};

template <int T>
__device__ void walk_links(const BatchParams& bp, const MemberDesc& md, uint32_t start, uint32_t cnt, WalkLinks& w) {
    const uint32_t n = md.len;
    const uint32_t* ppg = bp.pp + md.in_off + start;
    for (uint32_t i = threadIdx.x; i < cnt; i += T) w.pps[i] = ppg[i];
    if (threadIdx.x == 0) w.pps[cnt] = (start + cnt < n) ? ppg[cnt] : 0u;
    for (uint32_t i = cnt + threadIdx.x; i < cnt + GPZ_EXITS; i += T) {
        w.J[0][i] = (uint16_t)i;
        w.J[1][i] = (uint16_t)i;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < cnt; i += T) {
        const uint32_t l = w.pps[i] >> 16;
        uint32_t nx = i + 1u;
        if (l) {
            const uint32_t l1 = w.pps[i + 1] >> 16;
            const bool demote = (start + i + 1u < n) && l1 != 0u && l1 > l;  // lz77.rs:273-278
            if (!demote) nx = i + l;
        }
        w.nxt[i] = (uint16_t)nx;
        w.J[0][i] = (uint16_t)nx;
    }
    __syncthreads();
}

template <int T>
__global__ void __launch_bounds__(T) k_walk_exit_blk(BatchParams bp) {
    __shared__ WalkLinks w;
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x;
    const uint32_t ntiles = bp.dims[0];
    for (;;) {
        __syncthreads();
        if (tid == 0) s_tile = atomicAdd(&bp.counters[GPZ_CNT_EXIT], 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        if (td.seg + 1u == md.ntiles) continue;  // the member's last tile has no successor
        const uint32_t start = td.seg << GPZ_SEG_LOG2, cnt = GPZ_SEG;
        walk_links<T>(bp, md, start, cnt, w);
        int cur = 0;
        for (int r = 0; r < 16; r++) {
            int ch = 0;
            for (uint32_t i = tid; i < cnt; i += T) {
                const uint32_t j = w.J[cur][i];
                const uint32_t nj = j < cnt ? w.J[cur][j] : j;
                w.J[cur ^ 1][i] = (uint16_t)nj;
                ch |= nj != j;
            }
            cur ^= 1;
            if (!__syncthreads_or(ch)) break;
        }
        for (int e = tid; e < GPZ_EXITS; e += T)
            bp.tile_exit[(size_t)t * GPZ_EXITS + e] = (uint16_t)(w.J[cur][e] - cnt);
    }
    // the last CTA strings every member's tiles together
    if (last_cta_done(&bp.counters[GPZ_CNT_EXIT_DONE])) chain_members(bp);
}

// Entry offset of every tile: one thread per member follows the exit tables
// (written by other CTAs: read past L1).  Run by the last CTA of k_walk_exit.
__device__ void chain_members(const BatchParams& bp) {
    const uint32_t nmembers = bp.dims[1];
    for (uint32_t m = threadIdx.x; m < nmembers; m += blockDim.x) {
        const MemberDesc md = bp.members[m];
        uint32_t e = 0;
        for (uint32_t b = 0; b < md.ntiles; b++) {
            const uint32_t t = md.tile_base + b;
            bp.tile_entry[t] = e;
            if (b + 1u < md.ntiles) e = __ldcg(&bp.tile_exit[(size_t)t * GPZ_EXITS + min(e, (uint32_t)GPZ_EXITS - 1u)]);
        }
    }
}

struct MarkSmem {
    WalkLinks w;
    uint8_t mark[GPZ_SEG];
    uint32_t hist[GPZ_NSYM];
    uint32_t wsum[32];
    uint32_t tile;
};

template <int T>
__global__ void __launch_bounds__(T) k_walk_mark_blk(BatchParams bp) {
    constexpr int PER = GPZ_SEG / T;
    __shared__ MarkSmem sm;
    const int tid = threadIdx.x;
    const uint32_t ntiles = bp.dims[0];
    for (;;) {
        __syncthreads();
        if (tid == 0) sm.tile = atomicAdd(&bp.counters[GPZ_CNT_MARK], 1u);
        __syncthreads();
        const uint32_t t = sm.tile;
        if (t >= ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        const uint32_t n = md.len, start = td.seg << GPZ_SEG_LOG2;
        const uint32_t cnt = min(GPZ_SEG, n - start);
        for (int i = tid; i < GPZ_NSYM; i += T) sm.hist[i] = 0;
        for (uint32_t i = tid; i < cnt; i += T) sm.mark[i] = 0xFF;
        walk_links<T>(bp, md, start, cnt, sm.w);
        const uint32_t entry = bp.tile_entry[t];
        if (tid == 0 && entry < cnt) sm.mark[entry] = 0;
        __syncthreads();
        // before round r the marked positions are next^k(entry), k < 2^r
        int cur = 0;
        for (int r = 0; r < 16; r++) {
            int add = 0;
            for (uint32_t i = tid; i < cnt; i += T) {
                const uint32_t j = sm.w.J[cur][i];
                if (sm.mark[i] <= (uint32_t)r && j < cnt) {
                    sm.mark[j] = (uint8_t)(r + 1);
                    add = 1;
                }
                sm.w.J[cur ^ 1][i] = (uint16_t)(j < cnt ? sm.w.J[cur][j] : j);
            }
            cur ^= 1;
            if (!__syncthreads_or(add)) break;
        }

        // compact the visited tokens in order, histogram their symbols
        uint32_t vis = 0, c = 0;
        const uint32_t i0 = tid * PER;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t i = i0 + k;
            const bool v = i < cnt && sm.mark[i] != 0xFF;
            vis |= (uint32_t)v << k;
            c += v;
        }
        uint32_t total;
        uint32_t idx = block_excl_scan<T>(c, sm.wsum, &total);
        uint32_t* tg = bp.tok + md.in_off + start;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            if (!((vis >> k) & 1u)) continue;
            const uint32_t i = i0 + k;
            uint32_t tv = sm.w.pps[i];
            const uint32_t l = tv >> 16;
            if (l && sm.w.nxt[i] == i + 1u) tv = bp.in[md.in_off + start + i];  // lazy demotion to a literal
            tg[idx++] = tv;
            if ((tv >> 16) == 0) {
                atomicAdd(&sm.hist[tv & 0xFFu], 1u);
            } else {
                atomicAdd(&sm.hist[257u + len_row(tv >> 16)], 1u);
                atomicAdd(&sm.hist[GPZ_NLIT + dist_row(tv & 0xFFFFu)], 1u);
            }
        }
        __syncthreads();
        uint16_t* hg = bp.tile_hist + (size_t)t * GPZ_NSYM;
        for (int s = tid; s < GPZ_NSYM; s += T) hg[s] = (uint16_t)sm.hist[s];
        if (tid == 0) bp.tile_ntok[t] = total;
    }
}

// Warp-per-tile forward walk from the tile's entry: per window of 32
// positions (aligned), the lanes on the walk are found by doubling the links
// from the entry lane; they emit their tokens in order (a demoted match
// emits its literal byte) and count them in the warp's histogram; the walk
// continues at the last one's next position.  The three windows after the
// current one (pp and input bytes) are loaded ahead, since the walk usually
// moves on to them.
template <int T>
__global__ void __launch_bounds__(T) k_walk_mark_warp(BatchParams bp) {
    constexpr int W = T / 32;
    __shared__ uint32_t hist_all[W][GPZ_NSYM];
    const int lane = threadIdx.x & 31;
    uint32_t* hist = hist_all[threadIdx.x >> 5];
    const uint32_t ntiles = bp.dims[0];
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&bp.counters[GPZ_CNT_MARK], 1u);
        t = __shfl_sync(kFull, t, 0);
        if (t >= ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        const uint32_t n = md.len, start = td.seg << GPZ_SEG_LOG2;
        const uint32_t cnt = min(GPZ_SEG, n - start);
        const uint32_t* ppg = bp.pp + md.in_off + start;
        const uint8_t* ing = bp.in + md.in_off + start;
        uint32_t* tg = bp.tok + md.in_off + start;
        // pp one past the tile: the next tile's first position, if any
        const uint32_t past = (start + cnt < n) ? ppg[cnt] : 0u;
        for (int s = lane; s < GPZ_NSYM; s += 32) hist[s] = 0u;
        __syncwarp();
        uint32_t cur = bp.tile_entry[t];
        uint32_t ntok = 0;
        // the current window (pp v, input byte b) and the next three, loaded
        // ahead; the byte is what a lazily demoted match emits
        struct Win {
            uint32_t v, b;
        };
        auto ld = [&](uint32_t q) {
            return q + lane < cnt ? Win{ppg[q + lane], (uint32_t)ing[q + lane]} : Win{0u, 0u};
        };
        uint32_t wbase = 0xFFFFFFFFu;
        Win w0{0u, 0u}, w1{0u, 0u}, w2{0u, 0u}, w3{0u, 0u};
        while (cur < cnt) {
            const uint32_t base = cur & ~31u;
            if (base != wbase) {
                if (base == wbase + 32u) {
                    w0 = w1;
                    w1 = w2;
                    w2 = w3;
                    w3 = ld(base + 96u);
                } else if (base == wbase + 64u) {
                    w0 = w2;
                    w1 = w3;
                    w2 = ld(base + 64u);
                    w3 = ld(base + 96u);
                } else if (base == wbase + 96u) {
                    w0 = w3;
                    w1 = ld(base + 32u);
                    w2 = ld(base + 64u);
                    w3 = ld(base + 96u);
                } else {
                    w0 = ld(base);
                    w1 = ld(base + 32u);
                    w2 = ld(base + 64u);
                    w3 = ld(base + 96u);
                }
                wbase = base;
            }
            const uint32_t v = w0.v, vn1 = w1.v;
            const uint32_t p = base + lane;
            uint32_t v1 = __shfl_down_sync(kFull, v, 1);
            const uint32_t vn0 = __shfl_sync(kFull, vn1, 0);
            if (lane == 31) v1 = base + 32u < cnt ? vn0 : past;
            const bool inb = p < cnt;
            const uint32_t nx = walk_next(p, v, v1, start + p + 1u < n);
            // lanes on the walk in this window: doubling from the entry lane
            uint32_t S = 1u << (cur - base);
            uint32_t J = (inb && nx < base + 32u && nx < cnt) ? nx - base : 32u;
            // S holds the walk's first 2^r positions in the window after r
            // rounds; a round that adds nothing means the walk has left
            for (int r = 0; r < 5; r++) {
                const bool in = (S >> lane) & 1u;
                const uint32_t add = __reduce_or_sync(kFull, (in && J < 32u) ? (1u << J) : 0u);
                if ((add & ~S) == 0u) break;
                S |= add;
                const uint32_t Jp = __shfl_sync(kFull, J, J & 31u);
                J = J < 32u ? Jp : 32u;
            }
            if ((S >> lane) & 1u) {
                uint32_t tv = v;
                if ((v >> 16) && nx == p + 1u) tv = w0.b;  // lazy demotion to a literal
                tg[ntok + __popc(S & ((1u << lane) - 1u))] = tv;
                if ((tv >> 16) == 0u) {
                    atomicAdd(&hist[tv & 0xFFu], 1u);
                } else {
                    atomicAdd(&hist[257u + len_row(tv >> 16)], 1u);
                    atomicAdd(&hist[GPZ_NLIT + dist_row(tv & 0xFFFFu)], 1u);
                }
            }
            ntok += __popc(S);
            cur = __shfl_sync(kFull, nx, 31 - __clz(S));  // next of the last lane on the walk
        }
        __syncwarp();
        uint16_t* hg = bp.tile_hist + (size_t)t * GPZ_NSYM;
        for (int s = lane; s < GPZ_NSYM; s += 32) hg[s] = (uint16_t)hist[s];
        if (lane == 0) bp.tile_ntok[t] = ntok;
        __syncwarp();
    }
}

// ================================================================== k_huff

constexpr int kHuffThreads = 512;  // two groups of 256: code construction and CRC
constexpr int kCrcSlices = 256;  // threads folding member bytes into the CRC

struct TreeScratch {
    uint32_t key[512];  // (weight << 9 | symbol), sorted; unused = 0xFFFFFFFF
    uint32_t ukey[GPZ_NLIT];  // the same keys in symbol order (block builder)
    uint32_t w[GPZ_NLIT];
    uint32_t ifreq[GPZ_NLIT];
    uint16_t lparent[GPZ_NLIT];
    uint16_t iparent[GPZ_NLIT];
    uint16_t dep[2][GPZ_NLIT];
    uint16_t anc[2][GPZ_NLIT];
};

__device__ __forceinline__ void warp_bitonic_sort(uint32_t* key, int npad) {
    const int lane = threadIdx.x & 31;
    for (int size = 2; size <= npad; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = lane; i < npad / 2; i += 32) {
                const int lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                const bool up = (lo & size) == 0;
                const uint32_t a = key[lo], b = key[hi];
                if ((a > b) == up) {
                    key[lo] = b;
                    key[hi] = a;
                }
            }
            __syncwarp();
        }
    }
}

// try_build_code_lengths (huffman.rs:26-60) for one alphabet, run by one
// warp.  standard_huffman's min-heap on (freq, id) is evaluated as a
// two-queue merge: leaves sorted by (freq, id), internal nodes in creation
// order; a leaf wins a tie with an internal node because its id is smaller.
// Depths (huffman.rs:102-117) come from pointer jumping over parent links.
__device__ bool warp_code_lengths(const uint32_t* freq, int nsym, int max_bits, uint8_t* lens, TreeScratch& s) {
    const int lane = threadIdx.x & 31;
    int used = 0, only = -1;
    for (int i = lane; i < nsym; i += 32) {
        const uint32_t f = freq[i];
        s.w[i] = f;
        lens[i] = 0;
        if (f) {
            used++;
            only = i;
        }
    }
    used = __reduce_add_sync(0xFFFFFFFFu, used);
    only = __reduce_max_sync(0xFFFFFFFFu, only + 1) - 1;
    __syncwarp();
    if (used == 0) return true;
    if (used == 1) {
        if (lane == 0) lens[only] = 1;
        __syncwarp();
        return true;
    }
    int required = 0;
    while ((1 << required) < used) required++;
    if (required > max_bits) return false;
    int npad = 32;
    while (npad < nsym) npad <<= 1;
    const int nint = used - 1, root = nint - 1;
    for (int iter = 0; iter < 64; iter++) {
        for (int i = lane; i < npad; i += 32) s.key[i] = (i < nsym && s.w[i]) ? ((s.w[i] << 9) | (uint32_t)i) : 0xFFFFFFFFu;
        __syncwarp();
        warp_bitonic_sort(s.key, npad);
        if (lane == 0) {
            const uint32_t INF = 0xFFFFFFFFu;
            int li = 0, ii = 0, ni = 0;
            uint32_t lf = s.key[0] >> 9, fi = INF;
            for (int k = 0; k < nint; k++) {
                uint32_t f2[2];
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    if (li < used && lf <= fi) {
                        f2[q] = lf;
                        s.lparent[li++] = (uint16_t)ni;
                        lf = li < used ? (s.key[li] >> 9) : INF;
                    } else {
                        f2[q] = fi;
                        s.iparent[ii++] = (uint16_t)ni;
                        fi = ii < ni ? s.ifreq[ii] : INF;
                    }
                }
                const uint32_t nf = f2[0] + f2[1];
                s.ifreq[ni] = nf;
                if (ii == ni) fi = nf;
                ni++;
            }
        }
        __syncwarp();
        for (int j = lane; j < nint; j += 32) {
            s.anc[0][j] = (uint16_t)(j == root ? root : s.iparent[j]);
            s.dep[0][j] = (uint16_t)(j == root ? 0 : 1);
        }
        __syncwarp();
        int cur = 0;
        for (int r = 0; r < 9; r++) {
            for (int j = lane; j < nint; j += 32) {
                const int a = s.anc[cur][j];
                s.dep[cur ^ 1][j] = (uint16_t)(s.dep[cur][j] + s.dep[cur][a]);
                s.anc[cur ^ 1][j] = s.anc[cur][a];
            }
            cur ^= 1;
            __syncwarp();
        }
        int mx = 0;
        for (int k = lane; k < used; k += 32) {
            const int d = s.dep[cur][s.lparent[k]] + 1;
            lens[s.key[k] & 511u] = (uint8_t)d;
            mx = d > mx ? d : mx;
        }
        mx = __reduce_max_sync(0xFFFFFFFFu, mx);
        __syncwarp();
        if (mx <= max_bits) return true;
        for (int i = lane; i < nsym; i += 32)
            if (s.w[i] > 1u) s.w[i] >>= 1;
        __syncwarp();
    }
    return false;
}

__device__ __forceinline__ uint32_t rev_code(uint32_t code, uint32_t bits) { return bits ? __brev(code) >> (32u - bits) : 0u; }

// canonical_codes (huffman.rs:122-152) by one warp, packed as reversed code
// | len << 16: per-length counts and ranks from ballots over 32 symbols.
__device__ void warp_canonical(const uint8_t* lens, int nsym, uint32_t* out) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t cnt[16];
#pragma unroll
    for (int L = 0; L < 16; L++) cnt[L] = 0;
    for (int base = 0; base < nsym; base += 32) {
        const uint32_t l = base + lane < nsym ? lens[base + lane] : 0u;
#pragma unroll
        for (int L = 1; L < 16; L++) cnt[L] += __popc(__ballot_sync(0xFFFFFFFFu, l == (uint32_t)L));
    }
    uint32_t next[16];
    uint32_t code = 0;
    next[0] = 0;
#pragma unroll
    for (int bits = 1; bits < 16; bits++) {
        code = (code + (bits > 1 ? cnt[bits - 1] : 0u)) << 1;
        next[bits] = code;
    }
    for (int base = 0; base < nsym; base += 32) {
        const uint32_t l = base + lane < nsym ? lens[base + lane] : 0u;
        uint32_t mine = 0;
#pragma unroll
        for (int L = 1; L < 16; L++) {
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, l == (uint32_t)L);
            if (l == (uint32_t)L) mine = next[L] + __popc(m & lt);
            next[L] += __popc(m);
        }
        if (base + lane < nsym) out[base + lane] = l ? (rev_code(mine, l) | (l << 16)) : 0u;
    }
}

struct HuffSmem {
    uint32_t freq[GPZ_NSYM];
    uint8_t lens[GPZ_NSYM];
    uint32_t codes[GPZ_NSYM];
    uint32_t blen[GPZ_NSYM];
    TreeScratch tree[2];
    uint8_t comb[GPZ_NSYM];
    uint8_t rle_code[GPZ_NSYM];
    uint8_t rle_extra[GPZ_NSYM];
    uint32_t meta_freq[19];
    uint8_t meta_lens[19];
    uint32_t meta_codes[19];
    uint32_t hdr[GPZ_HDR_WORDS];
    uint32_t tile_bits[512];
    uint32_t red[32];
    uint32_t crctab[8 * 256];
    uint32_t crcv[kCrcSlices];
    uint32_t crcx[8];
    uint32_t member, hbits, total, nrle, nlit, ndist, ok, crc;
    uint32_t bt_used[2], bt_only[2], bt_max[2], bt_done[2];
};

// Codes one run of L equal code lengths v emits (rle_encode_lengths,
// deflate.rs:254-326): a zero run as 18s (11-138), then 17s (3-10), then
// single zeros; a non-zero run as the value, then 16s (3-6 repeats), then
// single values.  Writes them at out (if not NULL); returns their number.
__device__ int run_codes(uint32_t v, int L, uint8_t* code, uint8_t* extra) {
    int k = 0;
    auto emit = [&](uint32_t c, uint32_t e) {
        if (code) {
            code[k] = (uint8_t)c;
            extra[k] = (uint8_t)e;
        }
        k++;
    };
    int r = L;
    if (v == 0) {
        while (r >= 11) {
            const int q = r < 138 ? r : 138;
            emit(18, (uint32_t)(q - 11));
            r -= q;
        }
        while (r >= 3) {
            const int q = r < 10 ? r : 10;
            emit(17, (uint32_t)(q - 3));
            r -= q;
        }
        while (r > 0) {
            emit(0, 0);
            r--;
        }
    } else {
        emit(v, 0);
        r--;
        while (r >= 3) {
            const int q = r < 6 ? r : 6;
            emit(16, (uint32_t)(q - 3));
            r -= q;
        }
        while (r > 0) {
            emit(v, 0);
            r--;
        }
    }
    return k;
}

// HLIT / HDIST trims (trim_to_min: at least 257 / 1 codes) and the run-length
// coding of the combined code lengths, by one warp: each lane owns 10
// consecutive lengths and codes the runs that start in them; a run's end is
// the next start, in the lane's chunk or the first one above it.
template <class Smem>
__device__ void warp_rle(Smem& sm, int lane) {
    const uint8_t* ll = sm.lens;
    const uint8_t* dl = sm.lens + GPZ_NLIT;
    int lastl = 0;  // 1 + index of the last non-zero length code >= 257
    for (int i = 257 + lane; i < GPZ_NLIT; i += 32)
        if (ll[i]) lastl = i + 1;
    lastl = __reduce_max_sync(0xFFFFFFFFu, lastl);
    const int lastd = __reduce_max_sync(0xFFFFFFFFu, (lane < GPZ_NDIST && dl[lane]) ? lane + 1 : 0);
    const int nlit = lastl > 257 ? lastl : 257;
    const int ndist = lastd > 1 ? lastd : 1;
    const int n = nlit + ndist;
    for (int i = lane; i < n; i += 32) sm.comb[i] = i < nlit ? ll[i] : dl[i - nlit];
    __syncwarp();
    constexpr int C = 10;  // 32 x 10 >= 286 + 30
    const int lo = lane * C, hi = min(n, lo + C);
    auto is_start = [&](int i) { return i == 0 || sm.comb[i] != sm.comb[i - 1]; };
    int first = n;
    for (int i = lo; i < hi; i++)
        if (is_start(i)) {
            first = i;
            break;
        }
    // first run start in the lanes above this one
    int sfx = first;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_down_sync(0xFFFFFFFFu, sfx, o);
        if (lane + o < 32) sfx = y < sfx ? y : sfx;
    }
    int above = __shfl_down_sync(0xFFFFFFFFu, sfx, 1);
    if (lane == 31) above = n;
    auto run_end = [&](int i) {
        int j = i + 1;
        while (j < hi && sm.comb[j] == sm.comb[i]) j++;
        return j < hi ? j : above;
    };
    int mine = 0;
    for (int i = lo; i < hi; i++)
        if (is_start(i)) mine += run_codes(sm.comb[i], run_end(i) - i, nullptr, nullptr);
    int off = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, off, o);
        if (lane >= o) off += y;
    }
    const int total = __shfl_sync(0xFFFFFFFFu, off, 31);
    off -= mine;
    for (int i = lo; i < hi; i++)
        if (is_start(i)) off += run_codes(sm.comb[i], run_end(i) - i, sm.rle_code + off, sm.rle_extra + off);
    __syncwarp();
    // meta symbol counts: each lane holds up to 10 codes, one warp sum per symbol
    uint32_t mc[C];
#pragma unroll
    for (int u = 0; u < C; u++) {
        const int q = lane + 32 * u;
        mc[u] = q < total ? sm.rle_code[q] : 0xFFu;
    }
    for (uint32_t c = 0; c < 19; c++) {
        uint32_t k = 0;
#pragma unroll
        for (int u = 0; u < C; u++) k += mc[u] == c;
        k = __reduce_add_sync(0xFFFFFFFFu, k);
        if (lane == 0) sm.meta_freq[c] = k;
    }
    if (lane == 0) {
        sm.nrle = (uint32_t)total;
        sm.nlit = (uint32_t)nlit;
        sm.ndist = (uint32_t)ndist;
    }
    __syncwarp();
}

// The dynamic block header bits (deflate.rs:911-932) by one warp: 3 + 5 + 5 +
// 4 fixed bits, 3 bits per meta length in META_ORDER, then per RLE entry its
// meta code and extra bits; every field's bit position comes from a scan
// and the fields are ORed into zeroed words, LSB first.
template <class Smem>
__device__ void warp_header(Smem& sm, int lane) {
    int hclen = 0;  // 1 + last non-zero meta length in META_ORDER, at least 4
    if (lane < 19 && sm.meta_lens[c_meta_order[lane]]) hclen = lane + 1;
    hclen = __reduce_max_sync(0xFFFFFFFFu, hclen);
    if (hclen < 4) hclen = 4;
    for (int w = lane; w < GPZ_HDR_WORDS; w += 32) sm.hdr[w] = 0u;
    __syncwarp();
    auto put_at = [&](uint32_t pos, uint32_t v, uint32_t k) {
        if (!k) return;
        const uint32_t w = pos >> 5, sh = pos & 31u;
        atomicOr(&sm.hdr[w], v << sh);
        if (sh + k > 32u) atomicOr(&sm.hdr[w + 1], v >> (32u - sh));
    };
    if (lane == 0) {
        put_at(0, 5u, 3);
        put_at(3, sm.nlit - 257u, 5);
        put_at(8, sm.ndist - 1u, 5);
        put_at(13, (uint32_t)hclen - 4u, 4);
    }
    if (lane < hclen) put_at(17u + 3u * lane, sm.meta_lens[c_meta_order[lane]], 3);
    const uint32_t base = 17u + 3u * (uint32_t)hclen;
    const int nrle = (int)sm.nrle;
    constexpr int C = 10;
    const int lo = lane * C, hi = min(nrle, lo + C);
    auto field = [&](int q, uint32_t& v) {
        const uint32_t c = sm.rle_code[q], mc = sm.meta_codes[c];
        const uint32_t cl = mc >> 16, eb = c == 16 ? 2u : c == 17 ? 3u : c == 18 ? 7u : 0u;
        v = (mc & 0xFFFFu) | ((uint32_t)sm.rle_extra[q] << cl);
        return cl + eb;
    };
    uint32_t mine = 0, v;
    for (int q = lo; q < hi; q++) mine += field(q, v);
    uint32_t off = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, off, o);
        if (lane >= o) off += y;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, off, 31);
    uint32_t pos = base + off - mine;
    for (int q = lo; q < hi; q++) {
        const uint32_t k = field(q, v);
        put_at(pos, v, k);
        pos += k;
    }
    if (lane == 0) sm.hbits = base + total;
    __syncwarp();
}

// try_build_code_lengths (huffman.rs:26-60) for the litlen and distance
// alphabets at once (15-bit limit), by the whole CTA: the same two-queue
// evaluation of standard_huffman's (freq, id) heap as warp_code_lengths, with
// the leaves ranked by all threads (rank = number of smaller keys), one
// thread per alphabet for the merge (the next leaf and the next two internal
// nodes kept in registers), and depths by pointer jumping over all threads.
// Each alphabet halves its weights until its longest code fits, on its own.
// Leaves sm.ok = 0 if an alphabet cannot be coded (never expected).
template <int T, class Smem, class Sync>
__device__ void block_code_lengths(Smem& sm, int tid, Sync sync) {
    constexpr int kMax = 15;
    const int nsym[2] = {GPZ_NLIT, GPZ_NDIST};
    const int nall = GPZ_NLIT + GPZ_NDIST;
    auto alpha = [&](int idx, int& i) {
        const int a = idx < GPZ_NLIT ? 0 : 1;
        i = idx - (a ? GPZ_NLIT : 0);
        return a;
    };
    if (tid < 2) {
        sm.bt_used[tid] = 0;
        sm.bt_only[tid] = 0;
        sm.bt_done[tid] = 0;
    }
    sync();
    for (int idx = tid; idx < nall; idx += T) {
        int i;
        const int a = alpha(idx, i);
        const uint32_t f = sm.freq[idx];
        sm.tree[a].w[i] = f;
        sm.lens[idx] = 0;
        if (f) {
            atomicAdd(&sm.bt_used[a], 1u);
            atomicMax(&sm.bt_only[a], (uint32_t)i);
        }
    }
    sync();
    if (tid < 2) {
        const uint32_t used = sm.bt_used[tid];
        if (used <= 1) {
            if (used == 1) sm.lens[(tid ? GPZ_NLIT : 0) + sm.bt_only[tid]] = 1;
            sm.bt_done[tid] = 1;
        } else if (used > (1u << kMax)) {
            sm.bt_done[tid] = 1;
            sm.ok = 0;
        }
    }
    sync();
    for (int iter = 0; iter < 64 && !(sm.bt_done[0] && sm.bt_done[1]); iter++) {
        for (int idx = tid; idx < nall; idx += T) {
            int i;
            const int a = alpha(idx, i);
            const uint32_t w = sm.tree[a].w[i];
            sm.tree[a].ukey[i] = w ? ((w << 9) | (uint32_t)i) : 0xFFFFFFFFu;
        }
        if (tid < 2) sm.bt_max[tid] = 0;
        sync();
        // leaves in (weight, symbol) order: rank = number of smaller keys
        for (int idx = tid; idx < nall; idx += T) {
            int i;
            const int a = alpha(idx, i);
            if (sm.bt_done[a]) continue;
            const uint32_t k = sm.tree[a].ukey[i];
            if (k == 0xFFFFFFFFu) continue;
            uint32_t r = 0;
            for (int j = 0; j < nsym[a]; j++) r += sm.tree[a].ukey[j] < k;
            sm.tree[a].key[r] = k;
        }
        sync();
        // two-queue merge, one thread per alphabet (warps 0 and 1)
        if ((tid == 0 || tid == 32) && !sm.bt_done[tid >> 5]) {
            TreeScratch& s = sm.tree[tid >> 5];
            const uint32_t used = sm.bt_used[tid >> 5];
            const uint32_t INF = 0xFFFFFFFFu;
            const int nint = (int)used - 1;
            int li = 0, ii = 0, ni = 0;
            uint32_t lf = s.key[0] >> 9, lf2 = used > 1 ? s.key[1] >> 9 : INF;
            uint32_t fi = INF, fi2 = INF;  // front and second of the internal queue [ii, ni)
            for (int k = 0; k < nint; k++) {
                uint32_t f2[2];
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    if (li < (int)used && lf <= fi) {
                        f2[q] = lf;
                        s.lparent[li++] = (uint16_t)ni;
                        lf = lf2;
                        lf2 = li + 1 < (int)used ? s.key[li + 1] >> 9 : INF;
                    } else {
                        f2[q] = fi;
                        s.iparent[ii++] = (uint16_t)ni;
                        fi = fi2;
                        fi2 = ii + 1 < ni ? s.ifreq[ii + 1] : INF;
                    }
                }
                const uint32_t nf = f2[0] + f2[1];
                s.ifreq[ni] = nf;
                if (ii == ni) fi = nf;
                else if (ii + 1 == ni) fi2 = nf;
                ni++;
            }
        }
        sync();
        // depths: pointer jumping over the internal nodes' parent links
        const int nint0 = sm.bt_done[0] ? 0 : (int)sm.bt_used[0] - 1;
        const int nint1 = sm.bt_done[1] ? 0 : (int)sm.bt_used[1] - 1;
        for (int idx = tid; idx < nint0 + nint1; idx += T) {
            const int a = idx < nint0 ? 0 : 1;
            const int j = idx - (a ? nint0 : 0), root = (a ? nint1 : nint0) - 1;
            TreeScratch& s = sm.tree[a];
            s.anc[0][j] = (uint16_t)(j == root ? root : s.iparent[j]);
            s.dep[0][j] = (uint16_t)(j == root ? 0 : 1);
        }
        sync();
        int cur = 0;
        for (int r = 0; r < 9; r++) {
            for (int idx = tid; idx < nint0 + nint1; idx += T) {
                const int a = idx < nint0 ? 0 : 1;
                const int j = idx - (a ? nint0 : 0);
                TreeScratch& s = sm.tree[a];
                const int an = s.anc[cur][j];
                s.dep[cur ^ 1][j] = (uint16_t)(s.dep[cur][j] + s.dep[cur][an]);
                s.anc[cur ^ 1][j] = s.anc[cur][an];
            }
            cur ^= 1;
            sync();
        }
        const int u0 = sm.bt_done[0] ? 0 : (int)sm.bt_used[0];
        const int u1 = sm.bt_done[1] ? 0 : (int)sm.bt_used[1];
        for (int idx = tid; idx < u0 + u1; idx += T) {
            const int a = idx < u0 ? 0 : 1;
            const int k = idx - (a ? u0 : 0);
            TreeScratch& s = sm.tree[a];
            const uint32_t d = s.dep[cur][s.lparent[k]] + 1u;
            sm.lens[(a ? GPZ_NLIT : 0) + (s.key[k] & 511u)] = (uint8_t)d;
            atomicMax(&sm.bt_max[a], d);
        }
        sync();
        // an alphabet whose longest code fits is done; the other halves
        const bool fit0 = sm.bt_done[0] || sm.bt_max[0] <= (uint32_t)kMax;
        const bool fit1 = sm.bt_done[1] || sm.bt_max[1] <= (uint32_t)kMax;
        for (int idx = tid; idx < nall; idx += T) {
            int i;
            const int a = alpha(idx, i);
            if (a == 0 ? fit0 : fit1) continue;
            uint32_t& w = sm.tree[a].w[i];
            if (w > 1u) w >>= 1;
        }
        sync();
        if (tid == 0) {
            if (fit0) sm.bt_done[0] = 1;
            if (fit1) sm.bt_done[1] = 1;
        }
        sync();
    }
    if (tid == 0 && !(sm.bt_done[0] && sm.bt_done[1])) sm.ok = 0;
}

// Per member: code lengths and codes, the dynamic block header
// (deflate.rs:830-932), the exact bit plan of every tile, the member's
// DEFLATE size and its CRC-32.  Members are independent: no waiting.
__global__ void __launch_bounds__(kHuffThreads) k_huff(BatchParams bp) {
    __shared__ HuffSmem sm;
    __shared__ unsigned long long s_wsum[32], s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // threads [0, 256): code construction, header and bit plan (named
    // barrier 1); threads [256, 512): the member's CRC-32 (named barrier 2).
    // The two groups run side by side and meet once per member.
    constexpr int G = kHuffThreads / 2, NW = G / 32;
    const bool hgroup = tid < G;
    auto hsync = [] { asm volatile("bar.sync 1, %0;" ::"n"(G) : "memory"); };
    auto csync = [] { asm volatile("bar.sync 2, %0;" ::"n"(G) : "memory"); };

    // slice-by-8 CRC tables: crctab[k][b] = CRC of byte b followed by k zeros
    for (int i = tid; i < 256; i += kHuffThreads) {
        uint32_t c = (uint32_t)i;
        for (int k = 0; k < 8; k++) c = (c & 1u) ? kCrcPoly ^ (c >> 1) : c >> 1;
        sm.crctab[i] = c;
    }
    __syncthreads();
    for (int i = tid; i < 256; i += kHuffThreads) {
        uint32_t c = sm.crctab[i];
        for (int k = 1; k < 8; k++) {
            c = sm.crctab[c & 0xFFu] ^ (c >> 8);
            sm.crctab[k * 256 + i] = c;
        }
    }

    const uint32_t nmembers = bp.dims[1];
    for (;;) {
        __syncthreads();
        if (tid == 0) sm.member = atomicAdd(&bp.counters[GPZ_CNT_HUFF], 1u);
        __syncthreads();
        const uint32_t m = sm.member;
        if (m >= nmembers) break;
        const MemberDesc md = bp.members[m];

        if (!hgroup) {
            // CRC-32 of the member (crc32fast at deflate.rs:974).  The
            // aligned 8-byte words are cut into kCrcSlices equal slices,
            // front-padded with zero words (which a zero-init CRC ignores);
            // each slice is folded with slice-by-8, then the slices are
            // combined pairwise, crc(A||B) = crc(A) * x^(8|B|) + crc(B), in a
            // tree.
            const int ct = tid - G;
            const uint32_t L = md.len, W = L >> 3;
            const uint32_t per = (W + kCrcSlices - 1) / kCrcSlices;
            const uint32_t padw = per * kCrcSlices - W;
            {
                const uint2* words = reinterpret_cast<const uint2*>(bp.in + md.in_off);
                uint32_t c = 0;
                // eight words loaded ahead of the fold (a padding word is zero)
                constexpr uint32_t kAhead = 8;
                for (uint32_t v0 = ct * per; v0 < (ct + 1) * per; v0 += kAhead) {
                    uint2 wv[kAhead];
#pragma unroll
                    for (uint32_t u = 0; u < kAhead; u++) {
                        const uint32_t v = v0 + u;
                        wv[u] = make_uint2(0u, 0u);
                        if (v < (ct + 1) * per && v >= padw) wv[u] = __ldg(words + (v - padw));
                    }
#pragma unroll
                    for (uint32_t u = 0; u < kAhead; u++) {
                        if (v0 + u >= (ct + 1) * per) break;
                        const uint32_t lo = wv[u].x ^ c, hi = wv[u].y;
                        c = sm.crctab[7 * 256 + (lo & 0xFFu)] ^ sm.crctab[6 * 256 + ((lo >> 8) & 0xFFu)] ^
                            sm.crctab[5 * 256 + ((lo >> 16) & 0xFFu)] ^ sm.crctab[4 * 256 + (lo >> 24)] ^
                            sm.crctab[3 * 256 + (hi & 0xFFu)] ^ sm.crctab[2 * 256 + ((hi >> 8) & 0xFFu)] ^
                            sm.crctab[1 * 256 + ((hi >> 16) & 0xFFu)] ^ sm.crctab[hi >> 24];
                    }
                }
                sm.crcv[ct] = c;
            }
            if (ct == 0) {
                uint32_t x = x8pow(8u * per);
                for (int j = 0; j < 8; j++) {
                    sm.crcx[j] = x;
                    x = gf2_mulmod(x, x);
                }
            }
            csync();
            for (int j = 0; j < 8; j++) {
                const int span = 1 << j;
                if ((ct & (2 * span - 1)) == 0) sm.crcv[ct] = gf2_mulmod(sm.crcv[ct], sm.crcx[j]) ^ sm.crcv[ct + span];
                csync();
            }
            if (ct == 0) {
                uint32_t c = sm.crcv[0];
                for (uint32_t i = W << 3; i < L; i++) c = sm.crctab[(c ^ bp.in[md.in_off + i]) & 0xFFu] ^ (c >> 8);
                sm.crc = ~(gf2_mulmod(0xFFFFFFFFu, x8pow(L)) ^ c);
            }
        } else {
            // member symbol counts = sum of its tiles' histograms, + EOB
            for (int q = tid; q < GPZ_NSYM; q += G) {
                uint32_t f = 0;
                const uint16_t* h = bp.tile_hist + (size_t)md.tile_base * GPZ_NSYM + q;
                for (uint32_t j = 0; j < md.ntiles; j++) f += h[(size_t)j * GPZ_NSYM];
                sm.freq[q] = f + (q == 256 ? 1u : 0u);
            }
            if (tid == 0) sm.ok = 1;
            hsync();

            // litlen and distance code lengths, 15-bit limit (skipped when
            // the batch asks for fixed blocks)
            const bool force_fixed = (bp.flags & GPZ_BATCH_FIXED) != 0u;
            if (force_fixed) {
                for (int q = tid; q < GPZ_NSYM; q += G) sm.lens[q] = 0;
                if (tid == 0) sm.ok = 0;
            } else {
                block_code_lengths<G>(sm, tid, hsync);
            }
            hsync();

            // fix-ups (deflate.rs:854-867)
            if (warp == 0) {
                uint8_t* ll = sm.lens;
                uint8_t* dl = sm.lens + GPZ_NLIT;
                const uint32_t dm = __ballot_sync(0xFFFFFFFFu, lane < GPZ_NDIST && dl[lane] != 0);
                int used_l = 0;
                for (int i = lane; i < GPZ_NLIT; i += 32) used_l += ll[i] != 0;
                used_l = __reduce_add_sync(0xFFFFFFFFu, used_l);
                __syncwarp();
                if (lane == 0) {
                    if (dm == 0) {
                        dl[0] = 1;
                        dl[1] = 1;
                    } else if (__popc(dm) == 1) {
                        const int only = __ffs(dm) - 1;
                        dl[only] = 1;
                        dl[1 - (only < 1 ? only : 1)] = 1;
                    }
                    if (used_l < 2) {
                        ll[0] = 1;
                        ll[256] = 1;
                    }
                }
                __syncwarp();
            }
            hsync();
            // canonical codes (warps 0, 1); trims + RLE (deflate.rs:254-335) on warp 2
            if (warp == 0) warp_canonical(sm.lens, GPZ_NLIT, sm.codes);
            else if (warp == 1) warp_canonical(sm.lens + GPZ_NLIT, GPZ_NDIST, sm.codes + GPZ_NLIT);
            else if (warp == 2) warp_rle(sm, lane);
            hsync();
            // meta code lengths, 7-bit limit (deflate.rs:896-903), and codes
            if (warp == 0) {
                const bool ok = warp_code_lengths(sm.meta_freq, 19, 7, sm.meta_lens, sm.tree[0]);
                if (!ok && lane == 0) sm.ok = 0;
                __syncwarp();
                warp_canonical(sm.meta_lens, 19, sm.meta_codes);
            }
            hsync();
            // header bits (deflate.rs:911-932), LSB first; or, where a code
            // could not be built (encode_block_fast, deflate.rs:752-761) or
            // fixed blocks were asked for, the fixed block's codes and its
            // 3-bit header (write_fixed_block_fast, deflate.rs:763-828)
            if (sm.ok) {
                if (warp == 0) warp_header(sm, lane);
            } else {
                for (int q = tid; q < GPZ_NSYM; q += G) {
                    uint32_t code, bits;
                    if (q >= GPZ_NLIT) {
                        code = (uint32_t)(q - GPZ_NLIT);
                        bits = 5;
                    } else if (q <= 143) {
                        code = 0x30u + q;
                        bits = 8;
                    } else if (q <= 255) {
                        code = 0x190u + (q - 144);
                        bits = 9;
                    } else if (q <= 279) {
                        code = (uint32_t)(q - 256);
                        bits = 7;
                    } else {
                        code = 0xC0u + (q - 280);
                        bits = 8;
                    }
                    sm.codes[q] = rev_code(code, bits) | (bits << 16);
                }
                for (int w = tid; w < GPZ_HDR_WORDS; w += G) sm.hdr[w] = w == 0 ? 3u : 0u;  // BFINAL 1, BTYPE 01
                if (tid == 0) sm.hbits = 3;
            }
            hsync();

            // bits per symbol occurrence (code + extra); total member bits
            uint32_t part = 0;
            for (int q = tid; q < GPZ_NSYM; q += G) {
                const uint32_t cl = sm.codes[q] >> 16;
                uint32_t extra = 0;
                if (q >= 257 && q < GPZ_NLIT) extra = len_extra_bits((uint32_t)q - 257u);
                else if (q >= GPZ_NLIT) extra = dist_extra_bits((uint32_t)q - GPZ_NLIT);
                sm.blen[q] = cl + extra;
                part += sm.freq[q] * (cl + extra);
            }
            part = __reduce_add_sync(0xFFFFFFFFu, part);
            if (lane == 0) sm.red[warp] = part;
            // exact bit plan per tile from the tile histograms
            hsync();
            for (uint32_t j = warp; j < md.ntiles; j += NW) {
                const uint16_t* h = bp.tile_hist + (size_t)(md.tile_base + j) * GPZ_NSYM;
                uint32_t sbits = 0;
                for (int q = lane; q < GPZ_NSYM; q += 32) sbits += (uint32_t)h[q] * sm.blen[q];
                sbits = __reduce_add_sync(0xFFFFFFFFu, sbits);
                if (lane == 0) sm.tile_bits[j] = sbits;
            }
        }
        __syncthreads();  // the CRC and the bit plan are both ready
        if (tid == 0) {
            uint32_t tot = sm.hbits;
            for (int w = 0; w < NW; w++) tot += sm.red[w];
            sm.total = tot;
            uint32_t off = sm.hbits;
            for (uint32_t j = 0; j < md.ntiles; j++) {
                bp.tile_bitoff[md.tile_base + j] = off;
                off += sm.tile_bits[j];
            }
            if (off + (sm.codes[256] >> 16) != tot) atomicOr(bp.err, GPZ_ERRBIT_BITS);
            MemberOut mo;
            mo.gz_off = 0;
            mo.deflate_bytes = (tot + 7u) >> 3;
            mo.crc = sm.crc;
            mo.total_bits = tot;
            mo.header_bits = sm.hbits;
            mo.len = md.len;
            mo.frame_bytes = 18;
            bp.member_out[m] = mo;
        }
        for (int q = tid; q < GPZ_NSYM; q += kHuffThreads) bp.member_codes[(size_t)m * GPZ_NSYM + q] = sm.codes[q];
        for (int q = tid; q < GPZ_HDR_WORDS; q += kHuffThreads) bp.member_hdr[(size_t)m * GPZ_HDR_WORDS + q] = sm.hdr[q];
    }
    // the last CTA places every member in the batch output (a scan of sizes)
    if (last_cta_done(&bp.counters[GPZ_CNT_HUFF_DONE])) place_members<kHuffThreads>(bp, s_wsum, s_carry);
}

// ========================================================== member placement

// Byte offset of every member in the batch output: exclusive scan of
// (framing + payload bytes) in member order, one CTA.

template <int T>
__device__ void place_members(const BatchParams& bp, unsigned long long* wsum, unsigned long long& carry) {
    constexpr int NW = T / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t nmembers = bp.dims[1];
    if (tid == 0) carry = bp.out_base;
    __syncthreads();
    for (uint32_t base = 0; base < nmembers; base += T) {
        const uint32_t m = base + tid;
        // written by other CTAs of the producing kernel: read past L1
        const unsigned long long v =
            m < nmembers ? (unsigned long long)__ldcg(&bp.member_out[m].frame_bytes) + __ldcg(&bp.member_out[m].deflate_bytes)
                         : 0ull;
        unsigned long long x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long s = lane < NW ? wsum[lane] : 0ull;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, s, o);
                if (lane >= o) s += y;
            }
            if (lane < NW) wsum[lane] = s;
        }
        __syncthreads();
        const unsigned long long excl = carry + (warp ? wsum[warp - 1] : 0ull) + x - v;
        if (m < nmembers) bp.member_out[m].gz_off = excl;
        __syncthreads();
        if (tid == 0) carry += wsum[NW - 1];
        __syncthreads();
    }
}

// True in the last CTA of the grid to get here: every CTA's global writes
// are fenced before it counts itself, so the last one sees them all.
__device__ bool last_cta_done(uint32_t* counter) {
    __shared__ bool s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == gridDim.x - 1u;
    __syncthreads();
    if (s_last) __threadfence();
    return s_last;
}

// ================================================================= k_frame

// Per member: zero every output word that several writers share (a word a
// tile boundary, the EOB or the last bit falls in), then store the header
// words and OR in the EOB code.  k_emit then stores whole words and ORs the
// shared ones.
constexpr int kFrameThreads = 128;

__global__ void __launch_bounds__(kFrameThreads) k_frame(BatchParams bp) {
    const int tid = threadIdx.x;
    const uint32_t nmembers = bp.dims[1];
    for (uint32_t m = blockIdx.x; m < nmembers; m += gridDim.x) {
        const MemberDesc md = bp.members[m];
        const MemberOut mo = bp.member_out[m];
        const uint32_t eob = bp.member_codes[(size_t)m * GPZ_NSYM + 256];
        const uint32_t eob_len = eob >> 16;
        const unsigned long long base = (mo.gz_off + 10ull) * 8ull;
        uint32_t* outw = bp.out_words;
        for (uint32_t j = tid; j < md.ntiles; j += kFrameThreads)
            outw[(base + bp.tile_bitoff[md.tile_base + j]) >> 5] = 0u;
        if (tid == 0) {
            outw[(base + mo.total_bits - eob_len) >> 5] = 0u;
            outw[(base + mo.total_bits - 1u) >> 5] = 0u;
        }
        __syncthreads();
        const uint32_t* hdr = bp.member_hdr + (size_t)m * GPZ_HDR_WORDS;
        const unsigned long long w0 = base >> 5, w1 = (base + mo.header_bits - 1u) >> 5;
        const unsigned long long shared = (base + mo.header_bits) >> 5;
        for (unsigned long long w = w0 + tid; w <= w1; w += kFrameThreads) {
            const long long L = (long long)(w * 32ull) - (long long)base;  // header bit at word bit 0
            uint32_t v;
            if (L < 0) {
                v = hdr[0] << (uint32_t)(-L);
            } else {
                const uint32_t q = (uint32_t)L >> 5, s = (uint32_t)L & 31u;
                v = __funnelshift_r(hdr[q], hdr[q + 1], s);
            }
            const long long keep = (long long)mo.header_bits - L;
            if (keep < 32) v &= keep <= 0 ? 0u : ((1u << keep) - 1u);
            if (w == shared) atomicOr(&outw[w], v);
            else outw[w] = v;
        }
        if (tid == 0) {
            const uint32_t code = eob & 0xFFFFu;
            const unsigned long long e0 = base + mo.total_bits - eob_len;
            const uint32_t s = (uint32_t)(e0 & 31u);
            atomicOr(&outw[e0 >> 5], code << s);
            if (s + eob_len > 32u) atomicOr(&outw[(e0 >> 5) + 1], code >> (32u - s));
        }
        __syncthreads();
    }
}

// ================================================================== k_emit

struct EmitSmem {
    uint32_t codes[GPZ_NSYM];
    uint32_t buf[GPZ_SEG * 48 / 32 + 4];
    uint32_t wsum[32];
    uint32_t tile;
};

template <int T>
__global__ void __launch_bounds__(T) k_emit(BatchParams bp) {
    constexpr int PER = GPZ_SEG / T;
    __shared__ EmitSmem sm;
    const int tid = threadIdx.x;

    const uint32_t ntiles = bp.dims[0];
    for (;;) {
        __syncthreads();
        if (tid == 0) sm.tile = atomicAdd(&bp.counters[GPZ_CNT_EMIT], 1u);
        __syncthreads();
        const uint32_t t = sm.tile;
        if (t >= ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        const MemberOut mo = bp.member_out[td.member];
        const uint32_t ntok = bp.tile_ntok[t];
        for (int s = tid; s < GPZ_NSYM; s += T) sm.codes[s] = bp.member_codes[(size_t)td.member * GPZ_NSYM + s];
        __syncthreads();

        const uint32_t* tg = bp.tok + md.in_off + ((size_t)td.seg << GPZ_SEG_LOG2);
        unsigned long long v[PER];
        uint32_t nb[PER];
        uint32_t mine = 0;
        const uint32_t i0 = tid * PER;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            v[k] = 0;
            nb[k] = 0;
            const uint32_t i = i0 + k;
            if (i >= ntok) continue;
            const uint32_t tv = tg[i], l = tv >> 16, lo = tv & 0xFFFFu;
            if (l == 0) {
                const uint32_t c = sm.codes[lo];
                v[k] = c & 0xFFFFu;
                nb[k] = c >> 16;
            } else {
                const uint32_t lr = len_row(l), dr = dist_row(lo);
                const uint32_t lc = sm.codes[257u + lr], dc = sm.codes[GPZ_NLIT + dr];
                const uint32_t le = len_extra_bits(lr), de = dist_extra_bits(dr);
                unsigned long long x = lc & 0xFFFFu;
                uint32_t s = lc >> 16;
                x |= (unsigned long long)(l - c_len_base[lr]) << s;
                s += le;
                x |= (unsigned long long)(dc & 0xFFFFu) << s;
                s += dc >> 16;
                x |= (unsigned long long)(lo - c_dist_base[dr]) << s;
                s += de;
                v[k] = x;
                nb[k] = s;
            }
            mine += nb[k];
        }
        uint32_t total;
        uint32_t off = block_excl_scan<T>(mine, sm.wsum, &total);

        const unsigned long long g0 = (mo.gz_off + 10ull) * 8ull + bp.tile_bitoff[t];
        const uint32_t sh = (uint32_t)(g0 & 31u);
        const uint32_t nwords = total ? (sh + total + 31u) >> 5 : 0u;
        for (uint32_t w = tid; w < nwords; w += T) sm.buf[w] = 0u;
        __syncthreads();
        uint32_t pos = sh + off;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            if (!nb[k]) continue;
            const uint32_t w = pos >> 5, b = pos & 31u;
            atomicOr(&sm.buf[w], (uint32_t)(v[k] << b));
            if (b + nb[k] > 32u) atomicOr(&sm.buf[w + 1], (uint32_t)(v[k] >> (32u - b)));
            if (b + nb[k] > 64u) atomicOr(&sm.buf[w + 2], (uint32_t)(v[k] >> (64u - b)));
            pos += nb[k];
        }
        __syncthreads();
        const unsigned long long gw0 = g0 >> 5, gend = g0 + total;
        uint32_t* outw = bp.out_words;
        for (uint32_t w = tid; w < nwords; w += T) {
            const unsigned long long ws = (gw0 + w) * 32ull;
            const uint32_t val = sm.buf[w];
            if (ws >= g0 && ws + 32ull <= gend) outw[gw0 + w] = val;
            else if (val) atomicOr(&outw[gw0 + w], val);
        }
        if (tid == 0) {
            const uint32_t eob_len = sm.codes[256] >> 16;
            const uint32_t planned = (td.seg + 1u < md.ntiles ? bp.tile_bitoff[t + 1] : mo.total_bits - eob_len) -
                                     bp.tile_bitoff[t];
            if (planned != total) atomicOr(bp.err, GPZ_ERRBIT_BITS);
        }
    }
}

// ================================================================= k_drain

// Streams the packed batch output, the member table and the error word into
// host-mapped pinned memory, so the host needs no size round trip before its
// copy: total = end of the last member.
__global__ void k_drain(BatchParams bp, uint8_t* h_out, MemberOut* h_mout, uint32_t* h_err) {
    const uint32_t nmembers = bp.dims[1];
    const size_t gtid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, gstride = (size_t)gridDim.x * blockDim.x;
    unsigned long long total = 0;
    if (nmembers) {
        const MemberOut last = bp.member_out[nmembers - 1];
        total = last.gz_off + last.frame_bytes + last.deflate_bytes - bp.out_base;
    }
    const uint4* src = reinterpret_cast<const uint4*>(bp.out_words);
    uint4* dst = reinterpret_cast<uint4*>(h_out);
    const size_t nvec = (size_t)((total + 15u) >> 4);
    for (size_t i = gtid; i < nvec; i += gstride) dst[i] = src[i];
    for (size_t m = gtid; m < nmembers; m += gstride) h_mout[m] = bp.member_out[m];
    if (gtid == 0) *h_err = *bp.err;
}

}  // namespace

// ================================================================= k_fetch

constexpr int kFetchBlocksPerSm = 2;  // grid: 2 x 74 x this, one wave on 148 SMs

// Copies a batch's descriptor block and input from mapped host memory into
// the device arenas with SM loads over PCIe.  Sizes come from the block's
// header; a header that asks for more than an arena holds sets the
// descriptor error bit, empties the batch and copies nothing (the batch then
// reports an error).
__global__ void k_fetch(FetchSource f, uint32_t* counters) {
    // the work counters and the error word start at zero (in place of the
    // memset that precedes a batch without k_fetch)
    uint32_t* err = counters + GPZ_NCOUNTERS;
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < GPZ_NCOUNTERS + 16; i += blockDim.x) counters[i] = 0u;
    __syncthreads();
    const uint32_t* hdr = reinterpret_cast<const uint32_t*>(f.h_desc);
    const uint64_t nt = hdr[0], nm = hdr[1];
    const uint64_t in_bytes = reinterpret_cast<const unsigned long long*>(f.h_desc)[1];
    if (nt > f.tiles_cap || nm > f.members_cap || in_bytes > f.in_cap || (in_bytes & 15u)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            f.d_dims[0] = 0u;  // the batch's kernels then find no work
            f.d_dims[1] = 0u;
            *err = GPZ_ERRBIT_DESC;
        }
        return;
    }
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthr = (uint64_t)gridDim.x * blockDim.x;
    // descriptors: 4-byte words (the member records are 24 bytes, the tile
    // block starts 8-byte aligned)
    const uint64_t hw = 16, mw = nm * sizeof(MemberDesc) / 4, tw = nt * sizeof(TileDesc) / 4;
    const uint32_t* src = hdr;
    for (uint64_t i = tid; i < hw + mw + tw; i += nthr) {
        const uint32_t v = src[i];
        if (i < hw) f.d_dims[i] = v;
        else if (i < hw + mw) reinterpret_cast<uint32_t*>(f.d_members)[i - hw] = v;
        else reinterpret_cast<uint32_t*>(f.d_tiles)[i - hw - mw] = v;
    }
    // input: 16-byte vectors, four in flight per thread
    const uint4* si = reinterpret_cast<const uint4*>(f.h_in);
    uint4* di = reinterpret_cast<uint4*>(f.d_in);
    const uint64_t nv = in_bytes / 16;
    for (uint64_t i = tid; i < nv; i += 4 * nthr) {
        uint4 v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t j = i + u * nthr;
            if (j < nv) v[u] = si[j];
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t j = i + u * nthr;
            if (j < nv) di[j] = v[u];
        }
    }
}

// ================================================================ launchers

size_t gpz_lookup_smem_bytes() { return LookupSmem::kBytes; }

int gpz_kernel_smem_setup() {
    // x^(8*2^k) mod P for the CRC combine
    uint32_t tab[32];
    auto mul = [](uint32_t a, uint32_t b) {
        uint32_t m = 1u << 31, p = 0;
        while (m) {
            if (a & m) {
                p ^= b;
                if ((a & (m - 1u)) == 0) break;
            }
            m >>= 1;
            b = (b & 1u) ? (b >> 1) ^ kCrcPoly : b >> 1;
        }
        return p;
    };
    uint32_t x8 = 1u << 31;
    for (int i = 0; i < 8; i++) x8 = (x8 & 1u) ? (x8 >> 1) ^ kCrcPoly : x8 >> 1;
    tab[0] = x8;
    for (int k = 1; k < 32; k++) tab[k] = mul(tab[k - 1], tab[k - 1]);
    if (cudaMemcpyToSymbol(c_x8pow2, tab, sizeof tab) != cudaSuccess) return -1;
    if (gpz_zstd_setup() != 0) return -1;
    if (cudaFuncSetAttribute(k_segtab<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SegtabSmem::kBytes) !=
        cudaSuccess)
        return -1;
    // two lookup CTAs per SM need the largest shared-memory carveout
    const int smem = (int)LookupSmem::kBytes;
    for (const void* f : {(const void*)k_lookup<512>, (const void*)k_lookup<768>, (const void*)k_lookup<1024>})
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
            cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared) !=
                cudaSuccess)
            return -1;
    return 0;
}

int gpz_launch_batch(const BatchParams& bp, const LaunchShape& ls, void* stream, void* const* events,
                     const DrainTarget* drain, const FetchSource* fetch) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (fetch) k_fetch<<<2 * kFetchBlocksPerSm * 74, 256, 0, s>>>(*fetch, bp.counters);
    auto mark = [&](int i) {
        if (events) cudaEventRecord(static_cast<cudaEvent_t>(events[i]), s);
    };
    // grid 0: one CTA per item of this batch (the host knows the counts);
    // otherwise a persistent grid that claims items from the device counters
    auto grid_of = [&](int g, uint32_t items) { return g > 0 ? g : (int)(items ? items : 1u); };
    const int nm = grid_of(0, bp.nmembers);
    mark(0);
    const int gs = grid_of(ls.segtab_grid, bp.ntiles);
    const int gl = grid_of(ls.lookup_grid, bp.ntiles);
    k_segtab<512><<<gs, 512, SegtabSmem::kBytes, s>>>(bp);
    mark(1);
    switch (ls.lookup_threads) {
        case 512: k_lookup<512><<<gl, 512, LookupSmem::kBytes, s>>>(bp); break;
        case 768: k_lookup<768><<<gl, 768, LookupSmem::kBytes, s>>>(bp); break;
        default: k_lookup<1024><<<gl, 1024, LookupSmem::kBytes, s>>>(bp); break;
    }
    mark(2);
    // walk form: 1024 selects the block form (512 threads per tile CTA);
    // 256 / 512 the warp form with that many threads per CTA
    const int gw = grid_of(ls.walk_grid, bp.ntiles);
    switch (ls.walk_threads) {
        case 1024:
            k_walk_exit_blk<512><<<gw, 512, 0, s>>>(bp);
            k_walk_mark_blk<512><<<gw, 512, 0, s>>>(bp);
            break;
        case 256:
            k_walk_exit_warp<256><<<gw, 256, 0, s>>>(bp);
            k_walk_mark_warp<256><<<gw, 256, 0, s>>>(bp);
            break;
        default:
            k_walk_exit_warp<512><<<gw, 512, 0, s>>>(bp);
            k_walk_mark_warp<512><<<gw, 512, 0, s>>>(bp);
            break;
    }
    mark(3);
    if (bp.flags & GPZ_BATCH_ZSTD) {
        // zstd blocks in place of the Huffman stages (gpz_zstd.cu)
        if (gpz_launch_zstd(bp, stream, events, ls.zblock_grid, ls.zcopy_grid) != 0) return -1;
        if (drain) k_drain<<<drain->grid, 256, 0, s>>>(bp, drain->h_out, drain->h_mout, drain->h_err);
        return cudaGetLastError() == cudaSuccess ? 0 : -1;
    }
    const int gh = grid_of(ls.huff_grid, bp.nmembers);
    k_huff<<<gh, kHuffThreads, 0, s>>>(bp);
    k_frame<<<gh, kFrameThreads, 0, s>>>(bp);
    mark(4);
    const int ge = grid_of(ls.emit_grid, bp.ntiles);
    switch (ls.emit_threads) {
        case 256: k_emit<256><<<ge, 256, 0, s>>>(bp); break;
        default: k_emit<512><<<ge, 512, 0, s>>>(bp); break;
    }
    mark(5);
    if (drain) k_drain<<<drain->grid, 256, 0, s>>>(bp, drain->h_out, drain->h_mout, drain->h_err);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int gpz_launch_drain(const BatchParams& bp, const DrainTarget& drain, void* stream) {
    k_drain<<<drain.grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(bp, drain.h_out, drain.h_mout, drain.h_err);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int gpz_occupancy(LaunchShape* persistent) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -1;
    auto occ = [&](const void* f, int threads, size_t smem) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, threads, smem) != cudaSuccess || n < 1) n = 1;
        return n;
    };
    persistent->segtab_grid = sms * occ((const void*)k_segtab<512>, 512, SegtabSmem::kBytes);
    const void* lookup_fn = persistent->lookup_threads == 512   ? (const void*)k_lookup<512>
                            : persistent->lookup_threads == 768 ? (const void*)k_lookup<768>
                                                                : (const void*)k_lookup<1024>;
    persistent->lookup_grid = sms * occ(lookup_fn, persistent->lookup_threads, LookupSmem::kBytes);
    const void* walk_fn = persistent->walk_threads == 1024 ? (const void*)k_walk_mark_blk<512>
                          : persistent->walk_threads == 256  ? (const void*)k_walk_mark_warp<256>
                                                             : (const void*)k_walk_mark_warp<512>;
    persistent->walk_grid = sms * occ(walk_fn, persistent->walk_threads == 1024 ? 512 : persistent->walk_threads, 0);
    persistent->huff_grid = sms * occ((const void*)k_huff, kHuffThreads, 0);
    if (gpz_zstd_occupancy(&persistent->zblock_grid, &persistent->zcopy_grid) != 0)
        persistent->zblock_grid = persistent->zcopy_grid = 0;
    persistent->emit_grid = sms * occ(persistent->emit_threads == 256 ? (const void*)k_emit<256>
                                                                       : (const void*)k_emit<512>,
                                      persistent->emit_threads, 0);
    return sms;
}
