// gpz_inflate.cu -- device side of gpz_inflate: decompression of gzip
// streams written by gpzip (concatenated members with the fixed 10-byte
// header), the GPU counterpart of parallel_decompress
// (crates/gpzip-codec-cpu/src/parallel_decompress.rs:63-113).
//
//   k_inflate      one warp per member: gpzi::inflate_member<32>
//                  (gpz_inflate_core.h), 40.6 KB of shared memory (the
//                  32 KiB window ring, staged input, two code tables);
//   k_inflate_crc  256 threads per member: CRC-32 of the member's output
//                  against its trailer (slices folded byte by byte, then
//                  combined pairwise in a tree).
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

__global__ void __launch_bounds__(32) k_inflate(const uint8_t* in, uint8_t* out, const InflateMember* members,
                                                uint32_t* status, uint32_t count) {
    extern __shared__ __align__(16) uint8_t smem[];
    gpzi::Shared& s = *reinterpret_cast<gpzi::Shared*>(smem);
    const uint32_t m = blockIdx.x;
    if (m >= count) return;
    const InflateMember im = members[m];
    const uint32_t st =
        gpzi::inflate_member<32>(s, threadIdx.x, in + im.in_off, im.in_len, out + im.out_off, im.isize);
    if (threadIdx.x == 0) status[m] = st;
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

size_t gpz_inflate_smem_bytes() { return sizeof(gpzi::Shared); }

int gpz_launch_inflate(const uint8_t* in, uint8_t* out, const InflateMember* members, uint32_t* status,
                       uint32_t count, void* stream, void* const* events) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!count) return 0;
    if (events) cudaEventRecord(static_cast<cudaEvent_t>(events[0]), s);
    k_inflate<<<count, 32, sizeof(gpzi::Shared), s>>>(in, out, members, status, count);
    k_inflate_crc<<<count, kCrcThreads, 0, s>>>(out, members, status, count);
    if (events) cudaEventRecord(static_cast<cudaEvent_t>(events[1]), s);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
