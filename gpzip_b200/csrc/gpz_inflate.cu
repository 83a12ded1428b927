// gpz_inflate.cu -- device side of gpz_inflate: decompression of gzip
// streams written by gpzip (concatenated members with the fixed 10-byte
// header), the GPU counterpart of parallel_decompress
// (crates/gpzip-codec-cpu/src/parallel_decompress.rs:63-113).
//
// Two phases, so that the serial part of a member's decode does no byte
// copying:
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

// Tokens of member m go to tok + out_off (a member has at most ISIZE
// tokens); their count to ntok[m].
__global__ void __launch_bounds__(32) k_inflate_tok(const uint8_t* in, uint32_t* tok, const InflateMember* members,
                                                    uint32_t* status, uint32_t* ntok, uint32_t count) {
    extern __shared__ __align__(16) uint8_t smem[];
    gpzi::Shared& s = *reinterpret_cast<gpzi::Shared*>(smem);  // only the bytes before its ring
    const uint32_t m = blockIdx.x;
    if (m >= count) return;
    const InflateMember im = members[m];
    const uint32_t st = gpzi::inflate_member<32, true>(s, threadIdx.x, in + im.in_off, im.in_len, nullptr, im.isize,
                                                       tok + im.out_off, threadIdx.x == 0 ? ntok + m : nullptr);
    if (threadIdx.x == 0) status[m] = st;
}

constexpr int kExpandThreads = 256;

__global__ void __launch_bounds__(kExpandThreads) k_inflate_expand(const uint32_t* toks, const uint32_t* ntok,
                                                                   uint8_t* out, const InflateMember* members,
                                                                   const uint32_t* status, uint32_t count) {
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

int gpz_launch_inflate(const uint8_t* in, uint8_t* out, uint32_t* tok, const InflateMember* members,
                       uint32_t* status, uint32_t* ntok, uint32_t count, void* stream, void* const* events) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!count) return 0;
    if (events) cudaEventRecord(static_cast<cudaEvent_t>(events[0]), s);
    k_inflate_tok<<<count, 32, gpzi::kSharedTokBytes, s>>>(in, tok, members, status, ntok, count);
    k_inflate_expand<<<count, kExpandThreads, 0, s>>>(tok, ntok, out, members, status, count);
    k_inflate_crc<<<count, kCrcThreads, 0, s>>>(out, members, status, count);
    if (events) cudaEventRecord(static_cast<cudaEvent_t>(events[1]), s);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
