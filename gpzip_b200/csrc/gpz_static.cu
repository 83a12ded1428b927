// gpz_static.cu -- allocation-free compression of one gzip member.
//
// Some callers cannot allocate GPU memory at the point where they need to
// compress: a process whose device memory is entirely reserved by another
// allocator (a framework's caching pool owns the GPU), a latency-critical
// path that must not take cudaMalloc / cudaFree (both can synchronise the
// whole device), or code that runs where the CUDA runtime's allocator must
// not be entered.  gpz_compress_member_static serves them: it compresses one
// member of at most GPZ_STATIC_MAX_BYTES input bytes with every piece of
// working memory (input and output staging, per-position and walked tokens,
// per-tile and per-member tables, work counters) carved out of one
// file-scope device array of fixed size, so it never calls cudaMalloc,
// cudaFree or any allocating library routine.
//
// The array lives in every GPU that loads this library until the process
// exits.  All calls share it and it keeps the last call's contents; each
// call clears what must start at zero.  Two calls whose device work overlaps
// (for example on two streams, or from two host threads on one device) would
// race on the array; calls on one device are serialised on the host and each
// call waits for its own stream before returning.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/gpz.h"
#include "gpz_internal.h"

namespace {

constexpr size_t kMax = GPZ_STATIC_MAX_BYTES;
constexpr uint32_t kTiles = (uint32_t)((kMax + GPZ_SEG - 1) / GPZ_SEG);
constexpr size_t kOutCap = 18 + 600 + 2 * kMax + 8;  // one member's worst case

constexpr size_t al(size_t v) { return (v + 255) & ~size_t(255); }

// Byte offsets of each region inside the scratch array.
constexpr size_t kIn = 0;
constexpr size_t kPp = kIn + al(kMax + 64);
constexpr size_t kTok = kPp + al(kMax * 4 + 64);
constexpr size_t kOut = kTok + al(kMax * 4 + 64);
constexpr size_t kSkeys = kOut + al(kOutCap + 64);
constexpr size_t kSon = kSkeys + al(kTiles * GPZ_SEG * 2);
constexpr size_t kSnkeys = kSon + al(kTiles * GPZ_SEG * 4);
constexpr size_t kTentry = kSnkeys + al(kTiles * 4);
constexpr size_t kTexit = kTentry + al(kTiles * 4);
constexpr size_t kThist = kTexit + al(kTiles * GPZ_EXITS * 2);
constexpr size_t kTntok = kThist + al(kTiles * GPZ_NSYM * 2);
constexpr size_t kTbit = kTntok + al(kTiles * 4);
constexpr size_t kMcodes = kTbit + al(kTiles * 4);
constexpr size_t kMhdr = kMcodes + al(GPZ_NSYM * 4);
constexpr size_t kMout = kMhdr + al(GPZ_HDR_WORDS * 4);
constexpr size_t kCnt = kMout + al(sizeof(MemberOut));
constexpr size_t kMembers = kCnt + al(GPZ_NCOUNTERS * 4 + 64);
constexpr size_t kTilesOff = kMembers + al(sizeof(MemberDesc));
constexpr size_t kDims = kTilesOff + al(kTiles * sizeof(TileDesc));
constexpr size_t kResult = kDims + al(64);
constexpr size_t kTotal = kResult + al(16);

}  // namespace

// The scratch array.  Host code must not hand this name to a kernel: on the
// host it only stands for the symbol; the device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) uint8_t g_gpz_static_scratch[kTotal];

namespace {

// Clears the state that must start at zero and writes the member / tile
// descriptors for one member of n bytes.
__global__ void k_static_setup(uint8_t* base, uint32_t n) {
    uint32_t* cnt = reinterpret_cast<uint32_t*>(base + kCnt);
    MemberDesc* md = reinterpret_cast<MemberDesc*>(base + kMembers);
    TileDesc* td = reinterpret_cast<TileDesc*>(base + kTilesOff);
    uint32_t* dims = reinterpret_cast<uint32_t*>(base + kDims);
    const uint32_t nt = (n + GPZ_SEG - 1) / GPZ_SEG;
    if (threadIdx.x == 0) {
        dims[0] = nt;
        dims[1] = 1u;
    }
    for (uint32_t i = threadIdx.x; i < GPZ_NCOUNTERS + 16; i += blockDim.x) cnt[i] = 0u;
    for (uint32_t i = threadIdx.x; i < kTiles; i += blockDim.x) td[i] = TileDesc{0u, i};
    if (threadIdx.x == 0) {
        MemberDesc d{};
        d.in_off = 0;
        d.len = n;
        d.tile_base = 0;
        d.ntiles = nt;
        d.frame = GPZ_MEMBER_FIRST | GPZ_MEMBER_LAST;
        d.out_slot = 0;
        md[0] = d;
    }
}

// Copies the staged member into the caller's buffer with its 10-byte header
// and 8-byte trailer (deflate.rs:962-980) and records the length.
__global__ void k_static_finish(const uint8_t* base, uint8_t* dst, size_t cap) {
    const MemberOut mo = *reinterpret_cast<const MemberOut*>(base + kMout);
    const uint32_t err = reinterpret_cast<const uint32_t*>(base + kCnt)[GPZ_NCOUNTERS];
    unsigned long long* result = reinterpret_cast<unsigned long long*>(const_cast<uint8_t*>(base) + kResult);
    const size_t total = 18 + (size_t)mo.deflate_bytes;
    if (total > cap || err) {
        if (threadIdx.x == 0 && blockIdx.x == 0) {
            result[0] = total;
            result[1] = err ? err : 0xFFFFFFFFull;
        }
        return;
    }
    const uint8_t* src = base + kOut;
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        uint8_t b;
        if (i < 10) {
            const uint8_t hdr[10] = {0x1f, 0x8b, 0x08, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0xff};
            b = hdr[i];
        } else if (i < 10 + mo.deflate_bytes) {
            b = src[i];
        } else {
            const size_t k = i - 10 - mo.deflate_bytes;
            b = k < 4 ? (uint8_t)(mo.crc >> (8 * k)) : (uint8_t)(mo.len >> (8 * (k - 4)));
        }
        dst[i] = b;
    }
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        result[0] = total;
        result[1] = 0;
    }
}

// A call that fails after it has queued work on s waits for that work
// before it returns (and releases the array to the next caller), so that
// no kernel of a failed call still uses the array when the next one starts.
int drain_failed(cudaStream_t s) {
    cudaStreamSynchronize(s);
    cudaGetLastError();
    return GPZ_E_CUDA;
}

constexpr int kMaxDevices = 64;
std::mutex g_static_mu[kMaxDevices];
uint8_t* g_static_addr[kMaxDevices];  // device address of the scratch array, per device

}  // namespace

extern "C" int gpz_compress_member_static(const uint8_t* d_in, size_t n, uint8_t* d_out, size_t out_cap,
                                          size_t* out_len, void* stream) {
    if ((!d_in && n) || !d_out || !out_len) return GPZ_E_ARG;
    if (n > kMax) return GPZ_E_ARG;  // above GPZ_STATIC_MAX_BYTES
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return GPZ_E_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_static_mu[dev]);
    if (!g_static_addr[dev]) {
        // first call on this device (the device is current here): resolve
        // the scratch array's device address and set the kernel attributes
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_gpz_static_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return GPZ_E_CUDA;
        }
        if (gpz_kernel_smem_setup() != 0) {
            cudaGetLastError();
            return GPZ_E_CUDA;
        }
        g_static_addr[dev] = static_cast<uint8_t*>(p);
    }
    uint8_t* base = g_static_addr[dev];
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    if (n && cudaMemcpyAsync(base + kIn, d_in, n, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        // the copy may still have been queued: let it finish before the
        // array is released to the next caller
        return drain_failed(s);
    }
    k_static_setup<<<1, 256, 0, s>>>(base, (uint32_t)n);

    BatchParams bp{};
    bp.in = base + kIn;
    bp.members = reinterpret_cast<const MemberDesc*>(base + kMembers);
    bp.tiles = reinterpret_cast<const TileDesc*>(base + kTilesOff);
    bp.pp = reinterpret_cast<uint32_t*>(base + kPp);
    bp.tok = reinterpret_cast<uint32_t*>(base + kTok);
    bp.out_words = reinterpret_cast<uint32_t*>(base + kOut);
    bp.seg_keys = reinterpret_cast<uint16_t*>(base + kSkeys);
    bp.seg_on = reinterpret_cast<uint32_t*>(base + kSon);
    bp.seg_nkeys = reinterpret_cast<uint32_t*>(base + kSnkeys);
    bp.tile_entry = reinterpret_cast<uint32_t*>(base + kTentry);
    bp.tile_exit = reinterpret_cast<uint16_t*>(base + kTexit);
    bp.tile_hist = reinterpret_cast<uint16_t*>(base + kThist);
    bp.tile_ntok = reinterpret_cast<uint32_t*>(base + kTntok);
    bp.tile_bitoff = reinterpret_cast<uint32_t*>(base + kTbit);
    bp.member_codes = reinterpret_cast<uint32_t*>(base + kMcodes);
    bp.member_out = reinterpret_cast<MemberOut*>(base + kMout);
    bp.member_hdr = reinterpret_cast<uint32_t*>(base + kMhdr);
    bp.counters = reinterpret_cast<uint32_t*>(base + kCnt);
    bp.err = bp.counters + GPZ_NCOUNTERS;
    bp.dims = reinterpret_cast<const uint32_t*>(base + kDims);
    bp.nmembers = 1;
    bp.ntiles = (uint32_t)((n + GPZ_SEG - 1) / GPZ_SEG);
    bp.out_base = 0;
    const LaunchShape shape{1024, 0, 512, 0, 512, 0, 0, 0};
    // the stages launched before a failing launch still run on s
    if (gpz_launch_batch(bp, shape, s, nullptr, nullptr) != 0) return drain_failed(s);
    k_static_finish<<<8, 256, 0, s>>>(base, d_out, out_cap);

    unsigned long long result[2] = {0, 0};
    if (cudaMemcpyAsync(result, base + kResult, sizeof result, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return drain_failed(s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return GPZ_E_CUDA;
    }
    *out_len = (size_t)result[0];
    if (result[1] == 0xFFFFFFFFull) return GPZ_E_SPACE;
    if (result[1]) return GPZ_E_INTERNAL;
    return GPZ_OK;
}
