// gpz_kernels.cu -- sm_100a kernels of the gzip compression path.
//
// Four stages per batch, each a persistent kernel that claims work items
// (4 KiB tiles, or members) from a device counter:
//
//   k_lookup  per tile: segmented-hash build + window-bounded lookup
//             (lz77_hash_build.wgsl:45-54 + lz77_hash_lookup.wgsl:99-173),
//             plus the tile's zero-init CRC-32 (slice-by-8).
//   k_walk    per tile: lazy-rule walk (lz77.rs:260-284) by pointer jumping,
//             chained across tiles with a decoupled look-back; emits the
//             walked tokens and the tile's symbol histogram.
//   k_huff    per member: length-limited Huffman code construction
//             (huffman.rs:26-152), dynamic block header (deflate.rs:830-932),
//             exact bit plan per tile, gzip member placement by a decoupled
//             look-back over members, CRC-32 combine.
//   k_emit    per tile: per-token codes, block scan of bit lengths, bit
//             packing into the batch's gzip stream (deflate.rs:934-958).
//
// All arithmetic is integer and bit-exact with the reference.
#include <cuda_runtime.h>

#include <cstdint>

#include "gpz_internal.h"

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr uint32_t kCrcPoly = 0xEDB88320u;
constexpr uint32_t kSpinLimit = 1u << 22;  // x >= 64 ns per try: a few hundred ms, then error

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

__device__ __forceinline__ uint32_t ld32u(const uint32_t* w, uint32_t off) {
    return __funnelshift_r(w[off >> 2], w[(off >> 2) + 1], (off & 3u) * 8u);
}

// hash3 of lz77_hash_build.wgsl:36-43 on bytes at window offset o.
__device__ __forceinline__ uint32_t hash_at(const uint32_t* w, uint32_t o) {
    uint32_t x = __byte_perm(ld32u(w, o), 0u, 0x4012);  // b0<<16 | b1<<8 | b2
    return (x * 0x9E3779B1u) >> 16;
}

__device__ __forceinline__ uint32_t key_slot(uint32_t h) { return (h * 0x85EBCA6Bu) >> 19; }

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

// try_candidate (lz77_hash_lookup.wgsl:99-121) on packed best = len<<16|dist.
// A candidate that cannot beat the current best is dropped early: it must
// agree with p at offset best_len, and best_len must be below the cap.
__device__ __forceinline__ void try_cand(const uint8_t* win, const uint32_t* w32, uint32_t raw, uint32_t p,
                                         uint32_t n, uint32_t w0, uint32_t& best) {
    if (raw == 0u || raw == kEmpty) return;
    uint32_t cand = raw - 1u;
    if (cand >= p) return;
    uint32_t dist = p - cand;
    if (dist > GPZ_WINDOW) return;
    uint32_t limit = min(GPZ_MAX_MATCH, n - p);
    uint32_t bl = best >> 16;
    if (bl >= limit) return;
    uint32_t a = cand - w0, b = p - w0;
    if (bl >= 3u && win[a + bl] != win[b + bl]) return;
    uint32_t len = match_len(w32, a, b, limit);
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

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *(volatile const uint32_t*)p; }
__device__ __forceinline__ unsigned long long ld_volatile64(const unsigned long long* p) {
    return *(volatile const unsigned long long*)p;
}

// ================================================================ k_lookup

struct LookupSmem {
    static constexpr size_t kWin = 0;
    static constexpr size_t kKeys = kWin + GPZ_WIN_BYTES;
    static constexpr size_t kNew = kKeys + GPZ_KEY_SLOTS * 4;
    static constexpr size_t kOld = kNew + GPZ_SEG * 4;
    static constexpr size_t kBits = kOld + GPZ_SEG * 4;
    static constexpr size_t kBytes = kBits + 65536 / 8;
};

// One CTA per 4 KiB tile S of a member (persistent over tiles).  The window
// [S-8, S] plus 320 bytes of lookahead is staged in shared memory.  The
// reference's dense seg_oldest / seg_newest tables (65536 x num_segs each)
// are never materialised: only the hashes the tile itself queries matter, so
// the tile's own keys go into a small open-addressed table (dense ids) and,
// for each segment S-1 .. S-8 in the reference's order, the oldest / newest
// positions of exactly those keys are rebuilt with shared-memory atomics.
// Segments more than 8 back are never reachable: their nearest position is
// more than 32768 bytes from any p in S, which try_candidate rejects.
//
// The per-segment entries are kept with atomicMin only, tagged so that
// stale values from the previous (higher) segment lose and read as absent:
//   oldest:  q + 1                       (valid iff <= qbase + 4096)
//   newest:  2*qbase + 4095 - q          (valid iff <= qbase + 4095)
// which saves clearing the arrays between segments.
template <int T>
__global__ void __launch_bounds__(T, (T >= 1024 ? 1 : 2)) k_lookup(BatchParams bp) {
    constexpr int PER = GPZ_SEG / T;
    extern __shared__ __align__(16) uint8_t smem[];
    uint8_t* win = smem + LookupSmem::kWin;
    uint32_t* w32 = reinterpret_cast<uint32_t*>(win);
    uint32_t* keytab = reinterpret_cast<uint32_t*>(smem + LookupSmem::kKeys);
    uint32_t* cnew = reinterpret_cast<uint32_t*>(smem + LookupSmem::kNew);
    uint32_t* cold = reinterpret_cast<uint32_t*>(smem + LookupSmem::kOld);
    uint32_t* kbits = reinterpret_cast<uint32_t*>(smem + LookupSmem::kBits);  // presence of each hash
    __shared__ uint32_t s_tile, s_nkeys;
    const int tid = threadIdx.x, lane = tid & 31;

    for (;;) {
        __syncthreads();
        if (tid == 0) s_tile = atomicAdd(&bp.counters[GPZ_CNT_LOOKUP], 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= bp.ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        const uint32_t n = md.len, S = td.seg, start = S << GPZ_SEG_LOG2;
        const uint32_t cnt = min(GPZ_SEG, n - start);
        const uint32_t w0 = S >= 8u ? (S - 8u) << GPZ_SEG_LOG2 : 0u;
        const uint32_t wvalid = min(n - w0, (uint32_t)GPZ_WIN_BYTES);
        const uint32_t pl0 = start - w0;

        // ---- stage the window [w0, w0 + wvalid) (16-byte vectors; members
        // are 16-byte aligned and padded in the batch input)
        {
            const uint4* src = reinterpret_cast<const uint4*>(bp.in + md.in_off + w0);
            uint4* dst = reinterpret_cast<uint4*>(win);
            const uint32_t nvec = (wvalid + 15u) >> 4;
            for (uint32_t i = tid; i < nvec; i += T) dst[i] = __ldg(src + i);
            for (int i = tid; i < GPZ_KEY_SLOTS; i += T) keytab[i] = kEmpty;
            for (int i = tid; i < 65536 / 32; i += T) kbits[i] = 0u;
            for (int i = tid; i < GPZ_SEG; i += T) {
                cnew[i] = kEmpty;
                cold[i] = kEmpty;
            }
            if (tid == 0) s_nkeys = 0;
            __syncthreads();
            const uint32_t zend = min((uint32_t)GPZ_WIN_BYTES, (nvec << 4) + 32u);
            for (uint32_t i = wvalid + tid; i < zend; i += T) win[i] = 0;
        }
        __syncthreads();

        // ---- insert the tile's own hash keys (p + 2 < n)
        uint32_t info[PER];  // slot | h << 13, or kEmpty
        uint32_t own = 0;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t i = tid + k * T, p = start + i;
            info[k] = kEmpty;
            if (i < cnt && p + 2u < n) {
                const uint32_t h = hash_at(w32, pl0 + i);
                uint32_t s = key_slot(h);
                for (;;) {
                    uint32_t old = atomicCAS(&keytab[s], kEmpty, h);
                    if (old == kEmpty) {
                        own |= 1u << k;
                        atomicOr(&kbits[h >> 5], 1u << (h & 31u));
                        break;
                    }
                    if (old == h) break;
                    s = (s + 1u) & (GPZ_KEY_SLOTS - 1);
                }
                info[k] = s | (h << 13);
            }
        }
        __syncthreads();
        // dense ids for the distinct keys (warp-aggregated)
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const bool o = (own >> k) & 1u;
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, o);
            uint32_t base = 0;
            if (lane == 0 && m) base = atomicAdd(&s_nkeys, __popc(m));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (o) {
                const uint32_t id = base + __popc(m & ((1u << lane) - 1u));
                keytab[info[k] & (GPZ_KEY_SLOTS - 1)] = (info[k] >> 13) | (id << 16);
            }
        }
        __syncthreads();
        uint32_t myid[PER];
        uint32_t best[PER];
#pragma unroll
        for (int k = 0; k < PER; k++) {
            myid[k] = info[k] == kEmpty ? kEmpty : keytab[info[k] & (GPZ_KEY_SLOTS - 1)] >> 16;
            best[k] = 0;
        }

        // ---- own segment: the newest entry is always >= p (p itself is in
        // the table), so only the oldest can be a candidate
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t id = myid[k];
            if (!__ballot_sync(0xFFFFFFFFu, id != kEmpty)) continue;
            const uint32_t grp = __match_any_sync(0xFFFFFFFFu, id == kEmpty ? 0x10000u + lane : id);
            if (id != kEmpty && lane == __ffs(grp) - 1) atomicMin(&cold[id], start + tid + k * T + 1u);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PER; k++)
            if (myid[k] != kEmpty) try_cand(win, w32, cold[myid[k]], start + tid + k * T, n, w0, best[k]);

        // ---- segments S-1 .. S-8 in the reference's order: newest, then
        // oldest while best < 16 (lz77_hash_lookup.wgsl:138-166)
        for (uint32_t back = 1; back <= 8u && back <= S; back++) {
            const uint32_t qbase = (S - back) << GPZ_SEG_LOG2;
            __syncthreads();  // the previous segment's reads are done
#pragma unroll
            for (int k = 0; k < PER; k++) {
                const uint32_t i = tid + k * T, q = qbase + i;
                uint32_t id = kEmpty;
                if (q + 2u < n) {
                    const uint32_t h = hash_at(w32, q - w0);
                    if ((kbits[h >> 5] >> (h & 31u)) & 1u) {
                        uint32_t s = key_slot(h);
                        for (;;) {
                            const uint32_t wv = keytab[s];
                            if (wv == kEmpty) break;
                            if ((wv & 0xFFFFu) == h) {
                                id = wv >> 16;
                                break;
                            }
                            s = (s + 1u) & (GPZ_KEY_SLOTS - 1);
                        }
                    }
                }
                if (!__ballot_sync(0xFFFFFFFFu, id != kEmpty)) continue;
                const uint32_t grp = __match_any_sync(0xFFFFFFFFu, id == kEmpty ? 0x10000u + lane : id);
                if (id != kEmpty) {
                    if (lane == __ffs(grp) - 1) atomicMin(&cold[id], q + 1u);
                    if (lane == 31 - __clz(grp)) atomicMin(&cnew[id], 2u * qbase + 4095u - q);
                }
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < PER; k++) {
                const uint32_t id = myid[k];
                if (id == kEmpty) continue;
                const uint32_t p = start + tid + k * T;
                const uint32_t en = cnew[id];
                const uint32_t rn = en <= qbase + 4095u ? 2u * qbase + 4096u - en : 0u;  // q + 1, or absent
                try_cand(win, w32, rn, p, n, w0, best[k]);
                if ((best[k] >> 16) < 16u) {
                    const uint32_t ro = cold[id];
                    if (ro <= qbase + GPZ_SEG && ro != rn) try_cand(win, w32, ro, p, n, w0, best[k]);
                }
            }
        }

        // ---- per-position packed tokens
        uint32_t* dst = bp.pp + md.in_off + start;
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const uint32_t i = tid + k * T;
            if (i < cnt) dst[i] = (best[k] >> 16) ? best[k] : (uint32_t)win[pl0 + i];
        }
    }
}

// ================================================================== k_walk

struct WalkSmem {
    uint32_t pps[GPZ_SEG + 1];
    uint16_t nxt[GPZ_SEG];
    uint16_t J[2][GPZ_SEG + GPZ_EXITS];
    uint8_t mark[GPZ_SEG];
    uint32_t hist[GPZ_NSYM];
    uint32_t wsum[32];
    uint32_t tile, entry;
};

template <int T>
__global__ void __launch_bounds__(T) k_walk(BatchParams bp) {
    constexpr int PER = GPZ_SEG / T;
    __shared__ WalkSmem sm;
    const int tid = threadIdx.x;

    for (;;) {
        __syncthreads();
        if (tid == 0) sm.tile = atomicAdd(&bp.counters[GPZ_CNT_WALK], 1u);
        __syncthreads();
        const uint32_t t = sm.tile;
        if (t >= bp.ntiles) break;
        const TileDesc td = bp.tiles[t];
        const MemberDesc md = bp.members[td.member];
        const uint32_t n = md.len, b = td.seg, start = b << GPZ_SEG_LOG2;
        const uint32_t cnt = min(GPZ_SEG, n - start);
        const uint32_t* ppg = bp.pp + md.in_off + start;

        for (uint32_t i = tid; i < cnt; i += T) sm.pps[i] = ppg[i];
        if (tid == 0) sm.pps[cnt] = (start + cnt < n) ? ppg[cnt] : 0u;
        for (int i = tid; i < GPZ_NSYM; i += T) sm.hist[i] = 0;
        for (uint32_t i = cnt + tid; i < cnt + GPZ_EXITS; i += T) {
            sm.J[0][i] = (uint16_t)i;
            sm.J[1][i] = (uint16_t)i;
        }
        __syncthreads();

        // next-position links (lz77.rs:265-281)
        for (uint32_t i = tid; i < cnt; i += T) {
            const uint32_t t0 = sm.pps[i], l = t0 >> 16;
            uint32_t nx = i + 1u;
            if (l) {
                const uint32_t l1 = sm.pps[i + 1] >> 16;
                const bool demote = (start + i + 1u < n) && l1 != 0u && l1 > l;
                if (!demote) nx = i + l;
            }
            sm.nxt[i] = (uint16_t)nx;
            sm.J[0][i] = (uint16_t)nx;
        }
        __syncthreads();

        // pointer jumping: J = next^(2^r), absorbing at >= cnt
        int cur = 0;
        for (int r = 0; r < 16; r++) {
            int ch = 0;
            for (uint32_t i = tid; i < cnt; i += T) {
                const uint32_t j = sm.J[cur][i];
                const uint32_t nj = j < cnt ? sm.J[cur][j] : j;
                sm.J[cur ^ 1][i] = (uint16_t)nj;
                ch |= nj != j;
            }
            cur ^= 1;
            if (!__syncthreads_or(ch)) break;
        }

        // publish the exit table (entry offset -> entry offset into the
        // next tile); the member's last tile has no successor
        const bool last = b + 1u == md.ntiles;
        if (!last)
            for (int e = tid; e < GPZ_EXITS; e += T)
                bp.tile_exit[(size_t)t * GPZ_EXITS + e] = (uint16_t)(sm.J[cur][e] - cnt);
        __threadfence();
        __syncthreads();
        if (tid == 0) {
            uint32_t e = 0;
            if (b > 0) {
                atomicExch(&bp.tile_status[t], GPZ_ST_AGG);
                uint32_t j = t - 1u, spins = 0;
                for (;;) {
                    const uint32_t s = ld_volatile(&bp.tile_status[j]);
                    if (s & GPZ_ST_INCL) {
                        e = s & 0xFFFFu;
                        break;
                    }
                    if ((s & GPZ_ST_AGG) && j > md.tile_base) {
                        j--;
                        continue;
                    }
                    if (++spins > kSpinLimit) {
                        atomicOr(bp.err, GPZ_ERRBIT_SPIN);
                        e = 0;
                        break;
                    }
                    __nanosleep(64);
                }
                __threadfence();
                for (uint32_t k = j + 1u; k < t; k++) {
                    e = bp.tile_exit[(size_t)k * GPZ_EXITS + min(e, (uint32_t)GPZ_EXITS - 1u)];
                }
            }
            sm.entry = e;
            const uint32_t nexte = e < cnt ? (uint32_t)sm.J[cur][e] - cnt : e - cnt;
            __threadfence();
            atomicExch(&bp.tile_status[t], GPZ_ST_INCL | (nexte & 0xFFFFu));
        }
        __syncthreads();
        const uint32_t entry = sm.entry;

        // mark the positions the walk visits, by doubling from the entry:
        // before round r the marks are next^k(entry), k < 2^r
        for (uint32_t i = tid; i < cnt; i += T) {
            sm.mark[i] = 0xFF;
            sm.J[0][i] = sm.nxt[i];
        }
        __syncthreads();
        if (tid == 0 && entry < cnt) sm.mark[entry] = 0;
        __syncthreads();
        cur = 0;
        for (int r = 0; r < 16; r++) {
            int add = 0;
            for (uint32_t i = tid; i < cnt; i += T) {
                const uint32_t j = sm.J[cur][i];
                if (sm.mark[i] <= (uint32_t)r && j < cnt) {
                    sm.mark[j] = (uint8_t)(r + 1);
                    add = 1;
                }
                sm.J[cur ^ 1][i] = (uint16_t)(j < cnt ? sm.J[cur][j] : j);
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
            uint32_t tv = sm.pps[i];
            const uint32_t l = tv >> 16;
            if (l && sm.nxt[i] == i + 1u) tv = bp.in[md.in_off + start + i];  // lazy demotion
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

// ================================================================== k_huff

constexpr int kHuffThreads = 320;
constexpr int kCrcSlices = 256;  // threads folding member bytes into the CRC

struct TreeScratch {
    uint32_t w[GPZ_NLIT];
    uint16_t order[GPZ_NLIT];
    uint16_t lparent[GPZ_NLIT];
    uint32_t ifreq[GPZ_NLIT];
    uint16_t iparent[GPZ_NLIT];
    uint16_t idepth[GPZ_NLIT];
};

// try_build_code_lengths (huffman.rs:26-60) for one alphabet, run by one
// warp.  standard_huffman's min-heap on (freq, id) is evaluated as a
// two-queue merge: leaves sorted by (freq, id), internal nodes in creation
// order; a leaf wins a tie with an internal node because its id is smaller.
__device__ bool warp_code_lengths(const uint32_t* freq, int nsym, int max_bits, uint8_t* lens, TreeScratch& s) {
    const int lane = threadIdx.x & 31;
    int used = 0, only = -1;
    for (int i = lane; i < nsym; i += 32) {
        s.w[i] = freq[i];
        lens[i] = 0;
    }
    __syncwarp();
    for (int i = 0; i < nsym; i++)
        if (s.w[i]) {
            used++;
            only = i;
        }
    if (used == 0) return true;
    if (used == 1) {
        if (lane == 0) lens[only] = 1;
        __syncwarp();
        return true;
    }
    int required = 0;
    while ((1 << required) < used) required++;
    if (required > max_bits) return false;
    for (int iter = 0; iter < 64; iter++) {
        for (int i = lane; i < nsym; i += 32) {
            const uint32_t wi = s.w[i];
            if (!wi) continue;
            int r = 0;
            for (int j = 0; j < nsym; j++) {
                const uint32_t wj = s.w[j];
                r += wj && (wj < wi || (wj == wi && j < i));
            }
            s.order[r] = (uint16_t)i;
        }
        __syncwarp();
        int mx = 0;
        if (lane == 0) {
            int li = 0, ii = 0, nint = 0;
            for (int k = 0; k < used - 1; k++) {
                uint32_t f[2];
                for (int q = 0; q < 2; q++) {
                    if (li < used && (ii >= nint || s.w[s.order[li]] <= s.ifreq[ii])) {
                        f[q] = s.w[s.order[li]];
                        s.lparent[li++] = (uint16_t)nint;
                    } else {
                        f[q] = s.ifreq[ii];
                        s.iparent[ii++] = (uint16_t)nint;
                    }
                }
                s.ifreq[nint++] = f[0] + f[1];
            }
            s.idepth[nint - 1] = 0;
            for (int j = nint - 2; j >= 0; j--) s.idepth[j] = (uint16_t)(s.idepth[s.iparent[j]] + 1);
            for (int k = 0; k < used; k++) {
                int d = s.idepth[s.lparent[k]] + 1;
                lens[s.order[k]] = (uint8_t)d;
                mx = d > mx ? d : mx;
            }
        }
        mx = __shfl_sync(0xFFFFFFFFu, mx, 0);
        __syncwarp();
        if (mx <= max_bits) return true;
        for (int i = lane; i < nsym; i += 32)
            if (s.w[i] > 1u) s.w[i] >>= 1;
        __syncwarp();
    }
    return false;
}

__device__ __forceinline__ uint32_t rev_code(uint32_t code, uint32_t bits) { return bits ? __brev(code) >> (32u - bits) : 0u; }

// canonical_codes (huffman.rs:122-152), packed as reversed code | len << 16.
__device__ void canonical_packed(const uint8_t* lens, int nsym, uint32_t* out) {
    uint32_t bl_count[16] = {0}, next_code[16] = {0};
    int max_bits = 0;
    for (int i = 0; i < nsym; i++) {
        bl_count[lens[i]]++;
        max_bits = lens[i] > max_bits ? lens[i] : max_bits;
    }
    bl_count[0] = 0;
    uint32_t code = 0;
    for (int bits = 1; bits <= max_bits; bits++) {
        code = (code + bl_count[bits - 1]) << 1;
        next_code[bits] = code;
    }
    for (int s = 0; s < nsym; s++) {
        const uint32_t l = lens[s];
        out[s] = l ? (rev_code(next_code[l]++, l) | (l << 16)) : 0u;
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
    uint32_t hdr[GPZ_MAX_HEADER_WORDS + 2];
    uint32_t tile_bits[512];
    uint32_t red[32];
    uint32_t crctab[8 * 256];
    uint32_t crcv[kCrcSlices];
    uint32_t crcx[8];
    unsigned long long gz_off;
    uint32_t member, hbits, total, nrle, nlit, ndist, ok, crc;
};

__global__ void __launch_bounds__(kHuffThreads) k_huff(BatchParams bp) {
    __shared__ HuffSmem sm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kHuffThreads / 32;

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

    for (;;) {
        __syncthreads();
        if (tid == 0) sm.member = atomicAdd(&bp.counters[GPZ_CNT_HUFF], 1u);
        __syncthreads();
        const uint32_t m = sm.member;
        if (m >= bp.nmembers) break;
        const MemberDesc md = bp.members[m];

        // member symbol counts = sum of its tiles' histograms, + EOB
        if (tid < GPZ_NSYM) {
            uint32_t f = 0;
            const uint16_t* h = bp.tile_hist + (size_t)md.tile_base * GPZ_NSYM + tid;
            for (uint32_t j = 0; j < md.ntiles; j++) f += h[(size_t)j * GPZ_NSYM];
            sm.freq[tid] = f + (tid == 256 ? 1u : 0u);
        }
        if (tid == 0) sm.ok = 1;

        // CRC-32 of the member (crc32fast at deflate.rs:974).  The aligned
        // 8-byte words are cut into kCrcSlices equal slices, front-padded
        // with zero words (which a zero-init CRC ignores); each slice is
        // folded with slice-by-8, then the slices are combined pairwise,
        // crc(A||B) = crc(A) * x^(8|B|) + crc(B), in a tree.
        {
            const uint32_t L = md.len, W = L >> 3;
            const uint32_t per = (W + kCrcSlices - 1) / kCrcSlices;
            const uint32_t padw = per * kCrcSlices - W;
            if (tid < kCrcSlices) {
                const uint2* words = reinterpret_cast<const uint2*>(bp.in + md.in_off);
                uint32_t c = 0;
                for (uint32_t v = tid * per; v < (tid + 1) * per; v++) {
                    if (v < padw) continue;
                    const uint2 w = __ldg(words + (v - padw));
                    const uint32_t lo = w.x ^ c, hi = w.y;
                    c = sm.crctab[7 * 256 + (lo & 0xFFu)] ^ sm.crctab[6 * 256 + ((lo >> 8) & 0xFFu)] ^
                        sm.crctab[5 * 256 + ((lo >> 16) & 0xFFu)] ^ sm.crctab[4 * 256 + (lo >> 24)] ^
                        sm.crctab[3 * 256 + (hi & 0xFFu)] ^ sm.crctab[2 * 256 + ((hi >> 8) & 0xFFu)] ^
                        sm.crctab[1 * 256 + ((hi >> 16) & 0xFFu)] ^ sm.crctab[hi >> 24];
                }
                sm.crcv[tid] = c;
            }
            if (tid == 0) {
                uint32_t x = x8pow(8u * per);
                for (int j = 0; j < 8; j++) {
                    sm.crcx[j] = x;
                    x = gf2_mulmod(x, x);
                }
            }
            __syncthreads();
            for (int j = 0; j < 8; j++) {
                const int span = 1 << j;
                if (tid < kCrcSlices && (tid & (2 * span - 1)) == 0)
                    sm.crcv[tid] = gf2_mulmod(sm.crcv[tid], sm.crcx[j]) ^ sm.crcv[tid + span];
                __syncthreads();
            }
            if (tid == 0) {
                uint32_t c = sm.crcv[0];
                for (uint32_t i = W << 3; i < L; i++) c = sm.crctab[(c ^ bp.in[md.in_off + i]) & 0xFFu] ^ (c >> 8);
                sm.crc = ~(gf2_mulmod(0xFFFFFFFFu, x8pow(L)) ^ c);
            }
        }
        __syncthreads();

        // litlen (warp 0) and distance (warp 1) code lengths, 15-bit limit
        if (warp < 2) {
            const bool ok = warp == 0 ? warp_code_lengths(sm.freq, GPZ_NLIT, 15, sm.lens, sm.tree[0])
                                      : warp_code_lengths(sm.freq + GPZ_NLIT, GPZ_NDIST, 15, sm.lens + GPZ_NLIT,
                                                          sm.tree[1]);
            if (!ok && lane == 0) sm.ok = 0;
        }
        __syncthreads();

        // fix-ups (deflate.rs:854-867), codes, trims, RLE (deflate.rs:254-326)
        if (tid == 0) {
            uint8_t* ll = sm.lens;
            uint8_t* dl = sm.lens + GPZ_NLIT;
            int used_d = 0, only = -1, used_l = 0;
            for (int i = 0; i < GPZ_NDIST; i++)
                if (dl[i]) {
                    if (only < 0) only = i;
                    used_d++;
                }
            if (used_d == 0) {
                dl[0] = 1;
                dl[1] = 1;
            } else if (used_d == 1) {
                dl[only] = 1;
                dl[1 - (only < 1 ? only : 1)] = 1;
            }
            for (int i = 0; i < GPZ_NLIT; i++) used_l += ll[i] != 0;
            if (used_l < 2) {
                ll[0] = 1;
                ll[256] = 1;
            }
            canonical_packed(ll, GPZ_NLIT, sm.codes);
            canonical_packed(dl, GPZ_NDIST, sm.codes + GPZ_NLIT);
            int nlit = GPZ_NLIT;
            while (nlit > 257 && ll[nlit - 1] == 0) nlit--;
            int ndist = GPZ_NDIST;
            while (ndist > 1 && dl[ndist - 1] == 0) ndist--;
            for (int i = 0; i < nlit; i++) sm.comb[i] = ll[i];
            for (int i = 0; i < ndist; i++) sm.comb[nlit + i] = dl[i];
            const int n = nlit + ndist;
            int k = 0, i = 0;
            while (i < n) {
                const uint8_t cur = sm.comb[i];
                int run = 1;
                while (i + run < n && sm.comb[i + run] == cur) run++;
                if (cur == 0) {
                    while (run >= 11) {
                        const int q = run < 138 ? run : 138;
                        sm.rle_code[k] = 18;
                        sm.rle_extra[k++] = (uint8_t)(q - 11);
                        run -= q;
                        i += q;
                    }
                    while (run >= 3) {
                        const int q = run < 10 ? run : 10;
                        sm.rle_code[k] = 17;
                        sm.rle_extra[k++] = (uint8_t)(q - 3);
                        run -= q;
                        i += q;
                    }
                    while (run > 0) {
                        sm.rle_code[k] = 0;
                        sm.rle_extra[k++] = 0;
                        run--;
                        i++;
                    }
                } else {
                    sm.rle_code[k] = cur;
                    sm.rle_extra[k++] = 0;
                    i++;
                    run--;
                    while (run >= 3) {
                        const int q = run < 6 ? run : 6;
                        sm.rle_code[k] = 16;
                        sm.rle_extra[k++] = (uint8_t)(q - 3);
                        run -= q;
                        i += q;
                    }
                    while (run > 0) {
                        sm.rle_code[k] = cur;
                        sm.rle_extra[k++] = 0;
                        run--;
                        i++;
                    }
                }
            }
            for (int q = 0; q < 19; q++) sm.meta_freq[q] = 0;
            for (int q = 0; q < k; q++) sm.meta_freq[sm.rle_code[q]]++;
            sm.nrle = (uint32_t)k;
            sm.nlit = (uint32_t)nlit;
            sm.ndist = (uint32_t)ndist;
        }
        __syncthreads();
        // meta code lengths, 7-bit limit (deflate.rs:896-903)
        if (warp == 0) {
            const bool ok = warp_code_lengths(sm.meta_freq, 19, 7, sm.meta_lens, sm.tree[0]);
            if (!ok && lane == 0) sm.ok = 0;
        }
        __syncthreads();
        // header bits (deflate.rs:911-932), LSB first
        if (tid == 0) {
            canonical_packed(sm.meta_lens, 19, sm.meta_codes);
            int hclen = 19;
            while (hclen > 4 && sm.meta_lens[c_meta_order[hclen - 1]] == 0) hclen--;
            for (int q = 0; q < GPZ_MAX_HEADER_WORDS + 2; q++) sm.hdr[q] = 0;
            uint32_t pos = 0;
            auto put = [&](uint32_t v, uint32_t nb) {
                if (!nb) return;
                const uint32_t w = pos >> 5, s = pos & 31u;
                sm.hdr[w] |= v << s;
                if (s + nb > 32u) sm.hdr[w + 1] |= v >> (32u - s);
                pos += nb;
            };
            put(5u, 3);
            put(sm.nlit - 257u, 5);
            put(sm.ndist - 1u, 5);
            put((uint32_t)hclen - 4u, 4);
            for (int q = 0; q < hclen; q++) put(sm.meta_lens[c_meta_order[q]], 3);
            for (uint32_t q = 0; q < sm.nrle; q++) {
                const uint32_t c = sm.rle_code[q], mc = sm.meta_codes[c];
                put(mc & 0xFFFFu, mc >> 16);
                if (c == 16) put(sm.rle_extra[q], 2);
                else if (c == 17) put(sm.rle_extra[q], 3);
                else if (c == 18) put(sm.rle_extra[q], 7);
            }
            sm.hbits = pos;
        }
        __syncthreads();

        // bits per symbol occurrence (code + extra); total member bits
        uint32_t part = 0;
        if (tid < GPZ_NSYM) {
            const uint32_t cl = sm.codes[tid] >> 16;
            uint32_t extra = 0;
            if (tid >= 257 && tid < GPZ_NLIT) extra = len_extra_bits((uint32_t)tid - 257u);
            else if (tid >= GPZ_NLIT) extra = dist_extra_bits((uint32_t)tid - GPZ_NLIT);
            sm.blen[tid] = cl + extra;
            part = sm.freq[tid] * (cl + extra);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
        if (lane == 0) sm.red[warp] = part;
        __syncthreads();
        if (tid == 0) {
            uint32_t tot = sm.hbits;
            for (int w = 0; w < NW; w++) tot += sm.red[w];
            sm.total = tot;
        }
        __syncthreads();
        // place the member in the batch output: decoupled look-back over
        // members on (18 + DEFLATE bytes), 32 predecessors per step
        if (warp == 0) {
            const unsigned long long agg = 18ull + ((sm.total + 7u) >> 3);
            const unsigned long long vmask = (1ull << 62) - 1ull;
            unsigned long long excl = 0;
            if (lane == 0) atomicExch(&bp.member_status[m], ((m == 0 ? 2ull : 1ull) << 62) | agg);
            long long j = (long long)m - 1;
            uint32_t spins = 0;
            while (j >= 0) {
                const long long idx = j - lane;
                const unsigned long long st = idx >= 0 ? ld_volatile64(&bp.member_status[idx]) : (2ull << 62);
                const uint32_t f = (uint32_t)(st >> 62);
                const uint32_t incl = __ballot_sync(0xFFFFFFFFu, f == 2u);
                const uint32_t zero = __ballot_sync(0xFFFFFFFFu, f == 0u);
                const int first = incl ? __ffs(incl) - 1 : 32;
                const uint32_t before = first == 32 ? 0xFFFFFFFFu : ((1u << first) - 1u);
                if (zero & before) {
                    if (++spins > kSpinLimit) {
                        if (lane == 0) atomicOr(bp.err, GPZ_ERRBIT_SPIN);
                        break;
                    }
                    __nanosleep(64);
                    continue;
                }
                unsigned long long v = (lane <= first) ? (st & vmask) : 0ull;
#pragma unroll
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
                excl += v;
                if (first < 32) break;
                j -= 32;
            }
            if (lane == 0) {
                if (m > 0) atomicExch(&bp.member_status[m], (2ull << 62) | (excl + agg));
                sm.gz_off = bp.out_base + excl;
            }
        }
        __syncthreads();

        // exact bit plan per tile from the tile histograms
        for (uint32_t j = warp; j < md.ntiles; j += NW) {
            const uint16_t* h = bp.tile_hist + (size_t)(md.tile_base + j) * GPZ_NSYM;
            uint32_t s = 0;
            for (int q = lane; q < GPZ_NSYM; q += 32) s += (uint32_t)h[q] * sm.blen[q];
#pragma unroll
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
            if (lane == 0) sm.tile_bits[j] = s;
        }
        __syncthreads();
        const uint32_t eob_len = sm.codes[256] >> 16;
        const unsigned long long base = (sm.gz_off + 10ull) * 8ull;
        uint32_t* outw = bp.out_words;
        if (tid == 0) {
            uint32_t off = sm.hbits;
            for (uint32_t j = 0; j < md.ntiles; j++) {
                bp.tile_bitoff[md.tile_base + j] = off;
                off += sm.tile_bits[j];
            }
            if (off + eob_len != sm.total) atomicOr(bp.err, GPZ_ERRBIT_BITS);
            if (!sm.ok) atomicOr(bp.err, GPZ_ERRBIT_HUFF);
        }
        __syncthreads();
        // zero every word a tile boundary, the EOB or the last bit falls in
        for (uint32_t j = tid; j < md.ntiles; j += kHuffThreads)
            outw[(base + bp.tile_bitoff[md.tile_base + j]) >> 5] = 0u;
        if (tid == 0) {
            outw[(base + sm.total - eob_len) >> 5] = 0u;
            outw[(base + sm.total - 1u) >> 5] = 0u;
        }
        __syncthreads();
        // header words: whole words are stored, the word shared with the
        // first token is OR-ed into its zeroed copy
        {
            const unsigned long long w0 = base >> 5, w1 = (base + sm.hbits - 1u) >> 5;
            const unsigned long long shared = (base + sm.hbits) >> 5;
            for (unsigned long long w = w0 + tid; w <= w1; w += kHuffThreads) {
                const long long L = (long long)(w * 32ull) - (long long)base;  // header bit at word bit 0
                uint32_t v;
                if (L < 0) {
                    v = sm.hdr[0] << (uint32_t)(-L);
                } else {
                    const uint32_t q = (uint32_t)L >> 5, s = (uint32_t)L & 31u;
                    v = __funnelshift_r(sm.hdr[q], sm.hdr[q + 1], s);
                }
                const long long keep = (long long)sm.hbits - L;  // header bits in this word above L
                if (keep < 32) v &= keep <= 0 ? 0u : ((1u << keep) - 1u);
                if (w == shared) atomicOr(&outw[w], v);
                else outw[w] = v;
            }
        }
        if (tid == 0) {
            const uint32_t eob = sm.codes[256] & 0xFFFFu;
            const unsigned long long e0 = base + sm.total - eob_len;
            const uint32_t s = (uint32_t)(e0 & 31u);
            atomicOr(&outw[e0 >> 5], eob << s);
            if (s + eob_len > 32u) atomicOr(&outw[(e0 >> 5) + 1], eob >> (32u - s));
            MemberOut mo;
            mo.gz_off = sm.gz_off;
            mo.deflate_bytes = (sm.total + 7u) >> 3;
            mo.crc = sm.crc;
            mo.total_bits = sm.total;
            mo.header_bits = sm.hbits;
            mo.len = md.len;
            mo.pad = 0;
            bp.member_out[m] = mo;
        }
        for (int s = tid; s < GPZ_NSYM; s += kHuffThreads) bp.member_codes[(size_t)m * GPZ_NSYM + s] = sm.codes[s];
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

    for (;;) {
        __syncthreads();
        if (tid == 0) sm.tile = atomicAdd(&bp.counters[GPZ_CNT_EMIT], 1u);
        __syncthreads();
        const uint32_t t = sm.tile;
        if (t >= bp.ntiles) break;
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

}  // namespace

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
    const int smem = (int)LookupSmem::kBytes;
    if (cudaFuncSetAttribute(k_lookup<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return -1;
    if (cudaFuncSetAttribute(k_lookup<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return -1;
    if (cudaFuncSetAttribute(k_lookup<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return -1;
    return 0;
}

template <int T>
static void launch_lookup(const BatchParams& bp, int grid, cudaStream_t s) {
    k_lookup<T><<<grid, T, LookupSmem::kBytes, s>>>(bp);
}

int gpz_launch_batch(const BatchParams& bp, const LaunchShape& ls, void* stream, void* const* events) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto mark = [&](int i) {
        if (events) cudaEventRecord(static_cast<cudaEvent_t>(events[i]), s);
    };
    auto grid_of = [&](int g, uint32_t items) { return g > 0 ? g : (int)(items ? items : 1u); };
    mark(0);
    const int gl = grid_of(ls.lookup_grid, bp.ntiles);
    switch (ls.lookup_threads) {
        case 256: launch_lookup<256>(bp, gl, s); break;
        case 1024: launch_lookup<1024>(bp, gl, s); break;
        default: launch_lookup<512>(bp, gl, s); break;
    }
    mark(1);
    const int gw = grid_of(ls.walk_grid, bp.ntiles);
    switch (ls.walk_threads) {
        case 256: k_walk<256><<<gw, 256, 0, s>>>(bp); break;
        default: k_walk<512><<<gw, 512, 0, s>>>(bp); break;
    }
    mark(2);
    k_huff<<<bp.nmembers ? (int)bp.nmembers : 1, kHuffThreads, 0, s>>>(bp);
    mark(3);
    const int ge = grid_of(ls.emit_grid, bp.ntiles);
    switch (ls.emit_threads) {
        case 256: k_emit<256><<<ge, 256, 0, s>>>(bp); break;
        default: k_emit<512><<<ge, 512, 0, s>>>(bp); break;
    }
    mark(4);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
