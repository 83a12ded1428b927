// gpz_inflate.cu -- device side of gpz_inflate: decompression of gzip
// streams written by gpzip (concatenated members with the fixed 10-byte
// header), the GPU counterpart of parallel_decompress
// (crates/gpzip-codec-cpu/src/parallel_decompress.rs:63-113).
//
// Two phases, so that the serial part of a member's decode does no byte
// copying:
//   k_inflate_par     one CTA of kParThreads per member that is one final
//                     dynamic block (every gpzip member): the lanes decode
//                     spans of its bit stream at once until their starts
//                     settle on symbol boundaries (gpzi::decode_span,
//                     gpz_inflate_core.h), then write the tokens.  Where
//                     starts have not settled after a few rounds (runs of
//                     codes of one length keep a misaligned decode
//                     misaligned), the rest of the block is its tail:
//   k_inflate_cand    every tail's sub-spans of gpzi::kSubBits from each of
//                     their first gpzi::kCands bits, all at once;
//   k_inflate_chain   one CTA per tail: a walk picks the candidate that
//                     starts where the one before ended, then the threads
//                     write the tokens of the chosen ones.  A member these
//                     kernels cannot take (another block type, or anything
//                     invalid) is left to
//   k_inflate_tok     one warp per member: gpzi::inflate_member<32, true>
//                     (gpz_inflate_core.h) decodes the Huffman codes into the
//                     member's tokens (a literal as its byte, a match as
//                     length << 16 | distance), with every check of the
//                     byte-producing decoder; 9.9 KB of shared memory
//                     (staged input, two code tables);
//   k_inflate_expand  256 threads per member: each round of 256 tokens gets
//                     its output offsets from a block scan; literals are
//                     written at once, and a match is copied as soon as every
//                     byte it reads lies below the first byte not yet
//                     written (the earliest unwritten match always
//                     qualifies, so every round of the loop makes progress);
//   k_inflate_crc     256 threads per member: CRC-32 of the member's output
//                     against its trailer (slices folded byte by byte, then
//                     combined pairwise in a tree).
#include <cuda_runtime.h>

#include <cstdint>

#include "gpz_inflate_core.h"
#include "gpz_internal.h"

namespace {

constexpr uint32_t kPoly = 0xEDB88320u;
constexpr int kCrcThreads = 256;

// Product mod P in the reflected CRC-32 domain (bit 31 = x^0), as in
// gpz_kernels.cu.
__device__ uint32_t gf2_mul(uint32_t a, uint32_t b) {
    uint32_t m = 1u << 31, p = 0;
    while (m) {
        if (a & m) {
            p ^= b;
            if ((a & (m - 1u)) == 0) break;
        }
        m >>= 1;
        b = (b & 1u) ? (b >> 1) ^ kPoly : b >> 1;
    }
    return p;
}

// x^(8 n) mod P by square and multiply from x^8 (bit 23).
__device__ uint32_t x8pow_n(uint64_t n) {
    uint32_t r = 1u << 31, b = 1u << 23;
    for (; n; n >>= 1) {
        if (n & 1u) r = gf2_mul(r, b);
        b = gf2_mul(b, b);
    }
    return r;
}

constexpr int kParThreads = 128;
constexpr int kCandThreads = 128;

// A member whose tail (the part of its block where the lanes' starts did
// not settle) k_inflate_cand and k_inflate_chain decode: its tail starts at
// bit t0, a true symbol start, and covers nsub sub-spans of kSubBits taken
// from sub_base in the scratch; tok_base / byte_base tokens and bytes come
// before it; lit / dist are the block's code tables.
struct InflateTail {
    uint32_t m;
    uint32_t nsub;
    uint64_t t0;
    uint32_t sub_base;
    uint32_t tok_base;
    uint32_t byte_base;
    uint32_t pad;
    gpzi::Table lit, dist;
};

// Takes n sub-spans of the scratch for one tail (compare-and-swap, so the
// counter never passes the capacity); false when they do not fit.
__device__ bool take_subs(uint32_t* counter, uint32_t n, uint32_t cap, uint32_t* base) {
    uint32_t old = *reinterpret_cast<volatile uint32_t*>(counter);
    for (int tries = 0; tries < (1 << 20); tries++) {  // each failure is another CTA's success
        if (old > cap || cap - old < n) return false;
        const uint32_t prev = atomicCAS(counter, old, old + n);
        if (prev == old) {
            *base = old;
            return true;
        }
        old = prev;
    }
    return false;
}

// Exclusive prefix sum over the CTA's T threads (64-bit); *total gets the
// sum.  buf holds T values.
template <int T>
__device__ uint64_t excl_scan64(uint64_t v, uint64_t* buf, uint64_t* total) {
    const uint32_t k = threadIdx.x;
    buf[k] = v;
    __syncthreads();
    for (uint32_t o = 1; o < (uint32_t)T; o <<= 1) {
        const uint64_t add = k >= o ? buf[k - o] : 0ull;
        __syncthreads();
        buf[k] += add;
        __syncthreads();
    }
    *total = buf[T - 1];
    const uint64_t incl = buf[k];
    __syncthreads();
    return incl - v;
}

// Tokens of member m go to tok + out_off, as k_inflate_tok writes them;
// done[m] = 1 when this kernel decoded the member (status kOk), else 0.
__global__ void __launch_bounds__(kParThreads) k_inflate_par(const uint8_t* in, uint32_t* toks,
                                                             const InflateMember* members, uint32_t* status,
                                                             uint32_t* ntok, uint32_t* done, InflateScratch sc,
                                                             uint32_t count) {
    extern __shared__ __align__(16) uint8_t smem[];
    gpzi::Shared& s = *reinterpret_cast<gpzi::Shared*>(smem);  // only the bytes before its ring
    __shared__ uint64_t s_exit[kParThreads], s_scan[kParThreads];
    __shared__ uint64_t s_h, s_end;
    __shared__ uint32_t s_ok, s_ended, s_f, s_tail, s_nsub, s_base;
    const uint32_t m = blockIdx.x, k = threadIdx.x;
    if (m >= count) return;
    const InflateMember im = members[m];
    const uint8_t* src = in + im.in_off;
    uint32_t* tok = toks + im.out_off;
    // the block header and its tables, by the first warp
    if (k < 32) {
        const uint64_t h = gpzi::par_header<32>(s, k, src, im.in_len);
        if (k == 0) s_h = h;
    }
    __syncthreads();
    const uint64_t h = s_h, data_bits = 8ull * im.in_len;
    if (h == 0 || h >= data_bits) {  // uniform: another block type, or a bad header
        if (k == 0) done[m] = 0u;
        return;
    }
    const uint64_t bits = data_bits - h;
    const uint32_t R = gpzi::par_lanes(bits, kParThreads);
    const uint64_t span = (bits + R - 1) / R;
    const bool lane = k < R;
    const uint64_t stop = k + 1 < R ? h + (uint64_t)(k + 1) * span : gpzi::kSpanBad - 1;
    uint64_t start = h + (uint64_t)k * span;
    gpzi::Span r{gpzi::kSpanBad, 0ull, 0u, 0u};
    // rounds: each lane starts where its left neighbour left off in the
    // round before, until no start changes (or kParRounds)
    uint64_t next = start;
    for (uint32_t round = 0; round < gpzi::kParRounds; round++) {
        if (lane) {
            r = gpzi::decode_span(s.lit, s.dist, src, im.in_len, start, stop, nullptr, 0u, im.isize);
            s_exit[k] = r.exit;
        }
        __syncthreads();
        next = (k == 0 || !lane) ? start : s_exit[k - 1];
        if (__syncthreads_and(next == start) || round + 1 == gpzi::kParRounds) break;
        start = next;
    }
    // the lanes before the first one whose start moved decoded from true
    // starts (lane 0's is, and so is each exit of a true start); they write
    // their tokens, and one lane decodes the rest from that lane's next
    // start, which is true
    if (k == 0) {
        s_f = R;
        s_ok = 1u;
        s_ended = 0u;
        s_end = 0ull;
    }
    __syncthreads();
    if (lane && next != start) atomicMin(&s_f, k);
    __syncthreads();
    const uint32_t f = s_f;
    const bool keep = k < f;
    uint64_t nkeep = 0, bkeep = 0;
    const uint64_t toff = excl_scan64<kParThreads>(keep ? r.ntok : 0u, s_scan, &nkeep);
    const uint64_t boff = excl_scan64<kParThreads>(keep ? r.nbytes : 0u, s_scan, &bkeep);
    if (keep && boff <= im.isize) {
        const gpzi::Span g = gpzi::decode_span(s.lit, s.dist, src, im.in_len, start, stop, tok + toff, (uint32_t)boff, im.isize);
        if (g.exit != r.exit || g.ntok != r.ntok || g.nbytes != r.nbytes) s_ok = 0u;
        if (start != gpzi::kSpanEnd && g.exit == gpzi::kSpanEnd) {
            s_end = g.end;
            s_ended = 1u;
        }
    } else if (keep) {
        s_ok = 0u;
    }
    __syncthreads();
    if (k == 0) {
        uint64_t ntotal = nkeep, btotal = bkeep, end = s_end;
        bool ok = s_ok != 0u, ended = s_ended != 0u;
        s_tail = 0xFFFFFFFFu;
        if (ok && f < R && !ended && bkeep <= im.isize) {
            const uint64_t from = s_exit[f - 1];  // f >= 1: lane 0's start never moves
            // the tail goes to k_inflate_cand and k_inflate_chain; one lane
            // decodes it here only if the scratch has no room for it
            uint32_t base = 0;
            const uint64_t nsub = from < data_bits ? (data_bits - from + gpzi::kSubBits - 1) / gpzi::kSubBits : 0u;
            if (nsub && nsub < sc.sub_cap && take_subs(sc.counters + 1, (uint32_t)nsub, sc.sub_cap, &base)) {
                const uint32_t w = atomicAdd(sc.counters, 1u);  // below count: one tail per member
                InflateTail& t = static_cast<InflateTail*>(sc.tails)[w];
                t.m = m;
                t.nsub = (uint32_t)nsub;
                t.t0 = from;
                t.sub_base = base;
                t.tok_base = (uint32_t)nkeep;
                t.byte_base = (uint32_t)bkeep;
                s_tail = w;
                s_nsub = (uint32_t)nsub;
                s_base = base;
            } else {
                const gpzi::Span g = gpzi::decode_span(s.lit, s.dist, src, im.in_len, from, gpzi::kSpanBad - 1,
                                                       tok + nkeep, (uint32_t)bkeep, im.isize);
                if (from != gpzi::kSpanEnd && g.exit == gpzi::kSpanEnd) {
                    end = g.end;
                    ended = true;
                }
                ntotal += g.ntok;
                btotal += g.nbytes;
            }
        }
        if (s_tail == 0xFFFFFFFFu) {
            ok = ok && ended && end <= data_bits && (end + 7) / 8 == im.in_len && btotal == im.isize;
            if (ok) {
                status[m] = gpzi::kOk;
                ntok[m] = (uint32_t)ntotal;
            }
            done[m] = ok ? 1u : 0u;  // else k_inflate_tok decodes it and reports the status
        }
    }
    __syncthreads();
    if (s_tail != 0xFFFFFFFFu) {
        // the tail's record: the code tables, and the sub-spans' owner
        InflateTail& t = static_cast<InflateTail*>(sc.tails)[s_tail];
        const uint32_t* a = reinterpret_cast<const uint32_t*>(&s.lit);
        const uint32_t* d = reinterpret_cast<const uint32_t*>(&s.dist);
        uint32_t* ta = reinterpret_cast<uint32_t*>(&t.lit);
        uint32_t* td = reinterpret_cast<uint32_t*>(&t.dist);
        for (uint32_t i = k; i < sizeof(gpzi::Table) / 4; i += kParThreads) {
            ta[i] = a[i];
            td[i] = d[i];
        }
        for (uint32_t i = k; i < s_nsub; i += kParThreads) sc.sub_start[s_base + i] = s_tail;
        if (k == 0) done[m] = 2u;
    }
}

static_assert(sizeof(gpzi::Table) % 4 == 0, "tables are copied as words");

// Every sub-span of every tail from each of its kCands first bits (a grid
// of any size walks the list): the packed result of each candidate.
__global__ void __launch_bounds__(kCandThreads) k_inflate_cand(const uint8_t* in, const InflateMember* members,
                                                               InflateScratch sc) {
    const uint32_t used = min(sc.counters[1], sc.sub_cap);
    const uint64_t items = (uint64_t)used * gpzi::kCands;
    const InflateTail* tails = static_cast<const InflateTail*>(sc.tails);
    for (uint64_t it = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t sub = (uint32_t)(it / gpzi::kCands), j = (uint32_t)(it % gpzi::kCands);
        const InflateTail& t = tails[sc.sub_start[sub]];
        const InflateMember im = members[t.m];
        const uint32_t q = sub - t.sub_base;
        const uint64_t first = t.t0 + (uint64_t)q * gpzi::kSubBits, nf = first + gpzi::kSubBits;
        const uint64_t stop = q + 1 < t.nsub ? nf : gpzi::kSpanBad - 1;
        const gpzi::Span r =
            gpzi::decode_span(t.lit, t.dist, in + im.in_off, im.in_len, first + j, stop, nullptr, 0u, im.isize);
        sc.cands[it] = gpzi::pack_cand(r, first, nf);
    }
}

// One CTA per tail: one thread walks the sub-spans in order, taking the
// candidate that starts where the last one ended (decoding the sub-span
// itself where that start lies kCands or more bits in), and records each
// sub-span's start and token and byte offsets; then every thread takes
// sub-spans and writes their tokens, checking distances, and the member is
// done (or left to k_inflate_tok).
__global__ void __launch_bounds__(kCandThreads) k_inflate_chain(const uint8_t* in, uint32_t* toks,
                                                                const InflateMember* members, uint32_t* status,
                                                                uint32_t* ntok, uint32_t* done, InflateScratch sc,
                                                                uint32_t count) {
    __shared__ uint32_t s_ok, s_nq, s_ntok;
    const uint32_t w = blockIdx.x, k = threadIdx.x;
    if (w >= min(sc.counters[0], count)) return;
    const InflateTail& t = static_cast<const InflateTail*>(sc.tails)[w];
    const InflateMember im = members[t.m];
    const uint8_t* src = in + im.in_off;
    uint32_t* tok = toks + im.out_off;
    const uint64_t data_bits = 8ull * im.in_len;
    if (k == 0) {
        uint64_t e = t.t0, acc_t = t.tok_base, acc_b = t.byte_base, end = 0;
        bool ok = acc_t <= acc_b && acc_b <= im.isize, ended = false;
        uint32_t nq = 0;
        for (uint32_t q = 0; q < t.nsub && ok && !ended; q++) {
            const uint64_t first = t.t0 + (uint64_t)q * gpzi::kSubBits, nf = first + gpzi::kSubBits;
            const uint64_t stop = q + 1 < t.nsub ? nf : gpzi::kSpanBad - 1;
            const uint64_t j = e - first;  // e >= first: the last exit lies at or after this sub-span's first bit
            const uint64_t c =
                j < gpzi::kCands
                    ? sc.cands[(uint64_t)(t.sub_base + q) * gpzi::kCands + j]
                    : gpzi::pack_cand(gpzi::decode_span(t.lit, t.dist, src, im.in_len, e, stop, nullptr, 0u, im.isize),
                                      first, nf);
            const uint32_t code = (uint32_t)(c & 255u);
            const uint64_t nt = (c >> 21) & 8191u, nb = c >> 34;
            if (code == gpzi::kCandBad || nt > nb || j >= gpzi::kMaxSymBits) {
                ok = false;
                break;
            }
            sc.sub_start[t.sub_base + q] = (uint32_t)j;
            sc.sub_tok[t.sub_base + q] = (uint32_t)acc_t;
            sc.sub_byte[t.sub_base + q] = (uint32_t)acc_b;
            acc_t += nt;
            acc_b += nb;
            nq = q + 1;
            if (acc_b > im.isize) ok = false;
            if (code == gpzi::kCandEnd) {
                ended = true;
                end = first + ((c >> 8) & 8191u);
            } else {
                e = nf + code;
            }
        }
        s_ok = ok && ended && end <= data_bits && (end + 7) / 8 == im.in_len && acc_b == im.isize;
        s_nq = nq;
        s_ntok = (uint32_t)acc_t;
    }
    __syncthreads();
    if (s_ok) {
        const uint32_t nq = s_nq;
        for (uint32_t q = k; q < nq; q += kCandThreads) {
            const uint32_t at = t.sub_base + q;
            const uint64_t first = t.t0 + (uint64_t)q * gpzi::kSubBits, nf = first + gpzi::kSubBits;
            const uint64_t stop = q + 1 < t.nsub ? nf : gpzi::kSpanBad - 1;
            const uint32_t tb = sc.sub_tok[at], bb = sc.sub_byte[at];
            // tokens and bytes this sub-span must give, and where it must end
            const uint32_t want_t = (q + 1 < nq ? sc.sub_tok[at + 1] : s_ntok) - tb;
            const uint32_t want_b = (q + 1 < nq ? sc.sub_byte[at + 1] : im.isize) - bb;
            const uint64_t want_exit = q + 1 < nq ? nf + sc.sub_start[at + 1] : gpzi::kSpanEnd;
            const gpzi::Span g =
                gpzi::decode_span(t.lit, t.dist, src, im.in_len, first + sc.sub_start[at], stop, tok + tb, bb, im.isize);
            if (g.ntok != want_t || g.nbytes != want_b || g.exit != want_exit) s_ok = 0u;
        }
    }
    __syncthreads();
    if (k == 0) {
        if (s_ok) {
            status[t.m] = gpzi::kOk;
            ntok[t.m] = s_ntok;
        }
        done[t.m] = s_ok ? 1u : 0u;  // else k_inflate_tok decodes it and reports the status
    }
}

// Tokens of member m go to tok + out_off (a member has at most ISIZE
// tokens); their count to ntok[m].  Members k_inflate_par decoded are
// skipped.
__global__ void __launch_bounds__(32) k_inflate_tok(const uint8_t* in, uint32_t* tok, const InflateMember* members,
                                                    uint32_t* status, uint32_t* ntok, const uint32_t* done,
                                                    uint32_t count) {
    extern __shared__ __align__(16) uint8_t smem[];
    gpzi::Shared& s = *reinterpret_cast<gpzi::Shared*>(smem);  // only the bytes before its ring
    const uint32_t m = blockIdx.x;
    if (m >= count || done[m]) return;
    const InflateMember im = members[m];
    const uint32_t st = gpzi::inflate_member<32, true>(s, threadIdx.x, in + im.in_off, im.in_len, nullptr, im.isize,
                                                       tok + im.out_off, threadIdx.x == 0 ? ntok + m : nullptr);
    if (threadIdx.x == 0) status[m] = st;
}

constexpr int kExpandThreads = 256;

// With host_out (a page-locked host buffer, as the device sees it), each
// member's bytes are copied there as soon as they are all written, so the
// copy over PCIe overlaps the members still being expanded.
__global__ void __launch_bounds__(kExpandThreads) k_inflate_expand(const uint32_t* toks, const uint32_t* ntok,
                                                                   uint8_t* out, const InflateMember* members,
                                                                   const uint32_t* status, uint8_t* host_out,
                                                                   uint32_t count) {
    __shared__ uint32_t s_sum[kExpandThreads / 32];
    __shared__ uint32_t s_first;
    const uint32_t m = blockIdx.x, t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    if (m >= count || status[m] != gpzi::kOk) return;  // uniform per block
    const InflateMember im = members[m];
    const uint32_t* tok = toks + im.out_off;
    uint8_t* dst = out + im.out_off;
    const uint32_t nt = ntok[m];
    uint32_t base = 0;  // output offset of this round's first token
    for (uint32_t c0 = 0; c0 < nt; c0 += kExpandThreads) {
        const uint32_t k = c0 + t;
        const uint32_t v = k < nt ? tok[k] : 0u;
        const uint32_t l = k < nt ? ((v >> 16) ? (v >> 16) : 1u) : 0u;
        uint32_t x = l;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) s_sum[warp] = x;
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t w = 0; w < kExpandThreads / 32; w++) {
            if (w < warp) before += s_sum[w];
            total += s_sum[w];
        }
        const uint32_t off = base + before + x - l;
        bool done = k >= nt;
        if (!done && (v >> 16) == 0u) {
            dst[off] = (uint8_t)v;
            done = true;
        }
        // a match reads [off - d, off - d + min(l, d)): bytes it may copy
        // once everything below that end is written
        const uint32_t d = v & 0xFFFFu;
        const uint32_t need = done ? 0u : off - d + (l < d ? l : d);
        for (;;) {
            __syncthreads();  // the last round's bytes are visible; s_first is free
            if (t == 0) s_first = 0xFFFFFFFFu;
            __syncthreads();
            if (!done) atomicMin(&s_first, off);
            __syncthreads();
            const uint32_t first = s_first;  // every byte below it is written
            if (first == 0xFFFFFFFFu) break;
            if (!done && need <= first) {
                // byte q repeats byte q mod d of [off - d, off) (a copy with
                // d < l reads only bytes written before this match)
                uint32_t r = 0;
                for (uint32_t q = 0; q < l; q++) {
                    dst[off + q] = dst[off - d + r];
                    if (++r == d) r = 0;
                }
                done = true;
            }
        }
        base += total;
    }
    if (host_out) {
        __syncthreads();  // every byte of the member is written
        uint8_t* hd = host_out + im.out_off;
        const uint32_t n = im.isize;
        // 16-byte stores where both sides share an alignment, bytes elsewhere
        const uint32_t head = (uint32_t)((16u - ((uintptr_t)dst & 15u)) & 15u);
        if ((((uintptr_t)dst ^ (uintptr_t)hd) & 15u) == 0u && n >= head + 16u) {
            for (uint32_t i = t; i < head; i += kExpandThreads) hd[i] = dst[i];
            const uint32_t nv = (n - head) >> 4;
            const uint4* s4 = reinterpret_cast<const uint4*>(dst + head);
            uint4* d4 = reinterpret_cast<uint4*>(hd + head);
            for (uint32_t i = t; i < nv; i += kExpandThreads) d4[i] = s4[i];
            for (uint32_t i = head + (nv << 4) + t; i < n; i += kExpandThreads) hd[i] = dst[i];
        } else {
            for (uint32_t i = t; i < n; i += kExpandThreads) hd[i] = dst[i];
        }
    }
}

// The member's output is treated as front-padded with zeros to 256 equal
// slices (leading zeros leave a zero-initialised CRC unchanged); slice CRCs
// combine as crc(A || B) = crc(A) * x^(8|B|) + crc(B).
__global__ void __launch_bounds__(kCrcThreads) k_inflate_crc(const uint8_t* out, const InflateMember* members,
                                                             uint32_t* status, uint32_t count) {
    __shared__ uint32_t tab[256];
    __shared__ uint32_t part[kCrcThreads];
    __shared__ uint32_t pw[8];
    const uint32_t m = blockIdx.x, t = threadIdx.x;
    if (m >= count || status[m] != gpzi::kOk) return;  // uniform per block
    for (uint32_t i = t; i < 256; i += kCrcThreads) {
        uint32_t c = i;
        for (int k = 0; k < 8; k++) c = (c & 1u) ? kPoly ^ (c >> 1) : c >> 1;
        tab[i] = c;
    }
    const InflateMember im = members[m];
    const uint32_t L = im.isize;
    const uint32_t q = (L + kCrcThreads - 1) / kCrcThreads, pad = q * kCrcThreads - L;
    if (t == 0) {
        uint32_t x = x8pow_n(q);
        for (int j = 0; j < 8; j++) {
            pw[j] = x;
            x = gf2_mul(x, x);
        }
    }
    __syncthreads();
    const uint8_t* d = out + im.out_off;
    uint32_t c = 0;
    for (uint32_t p = t * q; p < (t + 1) * q; p++)
        if (p >= pad) c = tab[(c ^ d[p - pad]) & 0xFFu] ^ (c >> 8);
    part[t] = c;
    __syncthreads();
    for (int j = 0; j < 8; j++) {
        const uint32_t span = 1u << j;
        if ((t & (2 * span - 1)) == 0) part[t] = gf2_mul(part[t], pw[j]) ^ part[t + span];
        __syncthreads();
    }
    if (t == 0) {
        const uint32_t crc = ~(gf2_mul(0xFFFFFFFFu, x8pow_n(L)) ^ part[0]);
        if (crc != im.crc) status[m] = gpzi::kErrCrc;
    }
}

}  // namespace

size_t gpz_inflate_smem_bytes() { return gpzi::kSharedTokBytes; }
size_t gpz_inflate_tail_bytes() { return sizeof(InflateTail); }
uint32_t gpz_inflate_cands() { return gpzi::kCands; }

int gpz_launch_inflate(const uint8_t* in, uint8_t* out, uint32_t* tok, const InflateMember* members,
                       uint32_t* status, uint32_t* ntok, uint32_t* done, const InflateScratch& sc, uint8_t* host_out,
                       uint32_t count, void* stream, void* const* events) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!count) return 0;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -1;
    if (events) cudaEventRecord(static_cast<cudaEvent_t>(events[0]), s);
    if (cudaMemsetAsync(sc.counters, 0, 8, s) != cudaSuccess) return -1;
    k_inflate_par<<<count, kParThreads, gpzi::kSharedTokBytes, s>>>(in, tok, members, status, ntok, done, sc, count);
    // the candidates of all tails, on a grid that fills the GPU once
    k_inflate_cand<<<sms * (2048 / kCandThreads), kCandThreads, 0, s>>>(in, members, sc);
    k_inflate_chain<<<count, kCandThreads, 0, s>>>(in, tok, members, status, ntok, done, sc, count);
    k_inflate_tok<<<count, 32, gpzi::kSharedTokBytes, s>>>(in, tok, members, status, ntok, done, count);
    k_inflate_expand<<<count, kExpandThreads, 0, s>>>(tok, ntok, out, members, status, host_out, count);
    k_inflate_crc<<<count, kCrcThreads, 0, s>>>(out, members, status, count);
    if (events) cudaEventRecord(static_cast<cudaEvent_t>(events[1]), s);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
