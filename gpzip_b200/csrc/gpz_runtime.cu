// gpz_runtime.cu -- host runtime and C ABI of the gzip compression path.
//
// Replaces the reference's wgpu plumbing (GpuContext, Lz77HashPipeline's
// BufferSet pool, BatchedLz77's submitter / completer threads; gpu.rs:125-167,
// lz77_hash.rs:98-297, batch.rs:48-141) with:
//
//  * pipeline slots: each has a CUDA stream for its uploads, device arenas
//    sized for a batch, pinned input staging (skipped for page-locked
//    inputs) and host-mapped output; the synchronous path runs the kernels
//    of all slots in pass order on one stream, so one pass uploads while
//    the previous one computes and drains, and the passes ramp up in size
//    so that only a small first upload is exposed;
//  * a batch planner that cuts every input into members (member_bytes each,
//    gpu.rs:193-208) and members into 4 KiB tiles, written as one descriptor
//    block (batch dimensions, members, tiles) that the persistent kernels
//    read on the device;
//  * one CUDA graph per (slot, size bucket): the memset of the work counters,
//    the stage kernels with the bucket's autotuned launch shape, and the
//    drain into mapped host memory;
//  * a continuous-batching serving engine (gpz_submit / gpz_poll).
#include <cuda.h>
#include <cuda_runtime.h>

#include <emmintrin.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gpz.h"
#include "gpz_inflate_core.h"
#include "gpz_internal.h"
#include "gpz_stream.h"

namespace {

constexpr size_t kDefaultMember = 131072;
constexpr size_t kMaxMember = 2u << 20;
constexpr size_t kDefaultBatch = 64u << 20;
constexpr size_t kDefaultPool = 40ull << 30;
constexpr int kDefaultWaitMs = 60000;
// pipeline slots of the synchronous path: while one pass computes, the
// next two can be staged and uploaded
constexpr int kSyncSlots = 3;
constexpr int kBuckets = 5;
constexpr size_t kDescHeader = 64;  // batch dimensions at the start of a descriptor block
// kernels of one batch without k_fetch / k_drain: segtab, lookup, walk exit
// (+ chaining), walk mark, huff (+ placement), frame, emit
constexpr uint64_t kStageKernels = 7;

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Worst case of one member of n bytes: 18 framing bytes, a dynamic header of
// at most 4498 bits, at most 16 bits per input byte (a length-3 match costs
// at most 15 + 5 + 15 + 13 bits), the EOB, and word slack.
size_t member_bound(size_t n) { return 18 + 600 + 2 * n + 8; }

// Size bucket of a batch by its tile count.
int bucket_of(size_t ntiles) {
    if (ntiles <= 64) return 0;
    if (ntiles <= 512) return 1;
    if (ntiles <= 4096) return 2;
    if (ntiles <= 32768) return 3;
    return 4;
}

struct DevArena {
    void* p = nullptr;
    size_t cap = 0;
};

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// memcpy with non-temporal stores: the copy engine reads staged inputs at
// full rate only when they are not left dirty in the CPU caches (measured
// on a 44 MiB upload: 15 GB/s after a cached copy, 53 GB/s after this one).
void copy_streaming(void* dst, const void* src, size_t n) {
    auto* d = static_cast<uint8_t*>(dst);
    auto* s = static_cast<const uint8_t*>(src);
    const size_t head = std::min(n, (size_t)((16u - (reinterpret_cast<uintptr_t>(d) & 15u)) & 15u));
    std::memcpy(d, s, head);
    d += head;
    s += head;
    n -= head;
    size_t i = 0;
    for (; i + 64 <= n; i += 64) {
        const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i));
        const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i + 16));
        const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i + 32));
        const __m128i e = _mm_loadu_si128(reinterpret_cast<const __m128i*>(s + i + 48));
        _mm_stream_si128(reinterpret_cast<__m128i*>(d + i), a);
        _mm_stream_si128(reinterpret_cast<__m128i*>(d + i + 16), b);
        _mm_stream_si128(reinterpret_cast<__m128i*>(d + i + 32), c);
        _mm_stream_si128(reinterpret_cast<__m128i*>(d + i + 48), e);
    }
    std::memcpy(d + i, s + i, n - i);
    _mm_sfence();
}

// A small pool of host threads for the staging copies (inputs into pinned
// memory, gzip streams out of it): a batch's copies are cut into pieces and
// spread over the workers and the calling thread.  Each run publishes an
// immutable job; a worker that wakes late only finds it drained.  Inputs
// are staged with non-temporal stores (streaming = true).
class CopyPool {
  public:
    struct Copy {
        void* dst;
        const void* src;
        size_t n;
    };

    // Half the host's cores (at most 8 copiers with the caller): the copies
    // are memory-bound, and the other half stays free for the application.
    // With every core taken, a copier that the scheduler preempted held up
    // its whole batch of pieces while the application kept running.
    CopyPool() {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const unsigned nw = std::max(1u, std::min(hw / 2, 8u)) - 1;
        for (unsigned i = 0; i < nw; i++) th_.emplace_back([this] { work(); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
            stop_flag_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }

    void run(const std::vector<Copy>& copies, bool streaming = false) {
        size_t total = 0;
        for (auto& c : copies) total += c.n;
        // 1 MiB pieces; 256 KiB ones for copies under 4 MiB (a writer's
        // 1 MiB writes), which then take four copiers instead of one
        const size_t kPiece = total < (4u << 20) ? (256u << 10) : (1u << 20);
        if (total < 2 * kPiece || th_.empty()) {
            for (auto& c : copies) (streaming ? copy_streaming : copy_cached)(c.dst, c.src, c.n);
            return;
        }
        auto job = std::make_shared<Job>();
        job->streaming = streaming;
        for (auto& c : copies)
            for (size_t o = 0; o < c.n; o += kPiece)
                job->pieces.push_back(Copy{static_cast<char*>(c.dst) + o, static_cast<const char*>(c.src) + o,
                                           std::min(kPiece, c.n - o)});
        job->left = job->pieces.size();
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = job;
            gen_.fetch_add(1);
        }
        cv_.notify_all();
        drain(*job);
        std::unique_lock<std::mutex> lk(job->mu);
        job->cv.wait(lk, [&] { return job->left.load() == 0; });
    }

  private:
    static void copy_cached(void* d, const void* s, size_t n) { std::memcpy(d, s, n); }
    struct Job {
        bool streaming = false;
        std::vector<Copy> pieces;
        std::atomic<size_t> next{0}, left{0};
        std::mutex mu;
        std::condition_variable cv;
    };
    static void drain(Job& j) {
        for (;;) {
            const size_t i = j.next.fetch_add(1);
            if (i >= j.pieces.size()) return;
            (j.streaming ? copy_streaming : copy_cached)(j.pieces[i].dst, j.pieces[i].src, j.pieces[i].n);
            if (j.left.fetch_sub(1) == 1) {
                std::lock_guard<std::mutex> lk(j.mu);
                j.cv.notify_all();
            }
        }
    }
    // A worker polls for the next job for up to kSpinUs after each one
    // before it sleeps: back-to-back copies (a writer's) then skip the
    // wake-up latency of the condition variable.
    static constexpr int64_t kSpinUs = 200;
    void work() {
        uint64_t seen = 0;
        for (;;) {
            const auto t0 = std::chrono::steady_clock::now();
            while (gen_.load() == seen && !stop_flag_.load() &&
                   std::chrono::steady_clock::now() - t0 < std::chrono::microseconds(kSpinUs))
                _mm_pause();
            std::shared_ptr<Job> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_.load() != seen; });
                if (stop_) return;
                seen = gen_.load();
                job = job_;
            }
            if (job) drain(*job);
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::shared_ptr<Job> job_;
    std::atomic<uint64_t> gen_{0};
    std::atomic<bool> stop_flag_{false};
    bool stop_ = false;
};

CopyPool& copy_pool() {
    static CopyPool pool;
    return pool;
}

struct Span {
    size_t n = 0;
    uint64_t dev_off = 0;     // where the input sits in the batch input
    size_t first_member = 0;  // index into the slot's member list
    size_t nmembers = 0;
};

struct Slot {
    DevArena d_in, d_pp, d_tok, d_out, d_skeys, d_son, d_snkeys, d_tentry, d_texit, d_thist, d_tntok,
        d_tbit, d_mcodes, d_mhdr, d_mout, d_cnt, d_members, d_tiles, d_dims;
    DevArena d_itail, d_icand, d_isub;  // inflate: the parallel decode's tail scratch
    uint8_t* h_in = nullptr;
    size_t h_in_cap = 0;
    uint8_t* h_desc = nullptr;
    size_t h_desc_cap = 0;
    uint8_t* h_out = nullptr;  // mapped
    size_t h_out_cap = 0;
    MemberOut* h_mout = nullptr;  // mapped
    size_t h_mout_cap = 0;
    uint32_t* h_err = nullptr;  // mapped
    size_t h_err_cap = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t tv[3] = {nullptr, nullptr, nullptr};  // before the upload, after it, after the kernels
    float last_h2d_ms = 0, last_kernel_ms = 0;          // of the last batch waited for
    cudaEvent_t ev[GPZ_STAGES + 1] = {};
    uint64_t gen = 1;  // bumps whenever a buffer the graphs capture moves
    struct Graph {
        uint64_t gen = 0;
        cudaGraphExec_t exec = nullptr;
    } graphs[kBuckets];
    // the batch in flight
    std::vector<MemberDesc> members;
    std::vector<TileDesc> tiles;
    std::vector<Span> spans;
    size_t in_bytes = 0;
    bool busy = false;
    // a call stopped waiting for this slot's last work (GPZ_E_TIMEOUT): the
    // work may still run, so the slot is not reused until `done` completes
    bool stale = false;
    int bucket = 0;
};

}  // namespace

struct ServeEngine;

struct gpz_ctx {
    int device = 0;
    size_t member_bytes = kDefaultMember;
    size_t pool_cap = kDefaultPool;
    size_t batch_bytes = kDefaultBatch;
    int flags = 0;
    int codec = GPZ_CODEC_GZIP;
    int sms = 0;
    // bound of every host wait for the device in the calling thread, ms
    std::atomic<int> wait_ms{kDefaultWaitMs};
    std::mutex mu;  // the synchronous entry points (and their slots)
    // gpz_compress_chunk callers waiting to be batched (see there)
    struct ChunkCall {
        gpz_desc d;
        gpz_out o;
        int rc = GPZ_OK;
        bool done = false;
    };
    // gpz_inflate's device buffers (d_in, d_out, d_members: the member
    // descriptors, d_cnt: their statuses) and pinned staging
    Slot inf;
    cudaEvent_t inf_ev[2] = {nullptr, nullptr};
    float inf_ms = 0;
    std::mutex comb_mu;
    std::condition_variable comb_cv;
    std::deque<ChunkCall*> comb_q;
    bool comb_busy = false;
    std::string last_err;
    std::atomic<uint64_t> launches{0};
    std::atomic<size_t> pool_used{0};
    LaunchShape fixed{0, 0, 0, 0, 0, 0, 0, 0};  // set by gpz_set_shape (threads > 0 overrides)
    LaunchShape shape[kBuckets];
    bool tuned[kBuckets] = {false, false, false, false, false};
    std::mutex tune_mu;
    Slot slots[kSyncSlots];
    // kernels of the synchronous path, in pass order; each slot uploads on
    // its own stream, so the next pass's copy overlaps this pass's kernels
    cudaStream_t kstream = nullptr;
    // upload-done event of the pass submitted last on kstream: the next
    // pass's upload starts after it, so the first pass gets the whole link
    cudaEvent_t last_upload = nullptr;
    int next_slot = 0;
    float stage_ms[GPZ_STAGES] = {};
    // host-side time per pipeline step, ms, accumulated (gpz_host_times)
    std::mutex times_mu;
    double host_ms[6] = {0, 0, 0, 0, 0, 0};  // plan, copy in, enqueue, wait, frame + copy out, batches
    std::vector<MemberOut> mout;  // member table of the last synchronous pass
    std::unique_ptr<ServeEngine> serve;
    std::mutex serve_mu;
};

namespace {

int fail(gpz_ctx* c, int code, const char* what, cudaError_t e = cudaSuccess) {
    if (c) {
        c->last_err = what;
        if (e != cudaSuccess) {
            c->last_err += ": ";
            c->last_err += cudaGetErrorString(e);
        }
    }
    return code;
}

#define CU(ctx, call)                                                     \
    do {                                                                  \
        cudaError_t _e = (call);                                          \
        if (_e != cudaSuccess) return fail((ctx), GPZ_E_CUDA, #call, _e); \
    } while (0)

// Waits for event e at most the context's wait_ms (GPZ_E_TIMEOUT when that
// passes first; a limit of 0 gives up at once unless e is already done).
// The first 2 ms poll without sleeping, as a spinning synchronisation would;
// after that the thread sleeps 50 us between polls.  A device error ends the
// wait with GPZ_E_CUDA.
int wait_event(gpz_ctx* c, cudaEvent_t e, const char* what) {
    const double t0 = now_ms();
    const int limit = c->wait_ms.load();
    for (;;) {
        const cudaError_t q = cudaEventQuery(e);
        if (q == cudaSuccess) return GPZ_OK;
        if (q != cudaErrorNotReady) {
            cudaGetLastError();
            return fail(c, GPZ_E_CUDA, what, q);
        }
        const double el = now_ms() - t0;
        if (el >= (double)limit) return fail(c, GPZ_E_TIMEOUT, what);
        if (el < 2.0) _mm_pause();
        else std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

// capped: the growth counts against the context's pool cap (the serving
// engine's fixed arenas, sized once at start, do not).
int ensure_dev(gpz_ctx* c, Slot& sl, DevArena& a, size_t bytes, bool capped = true) {
    bytes = round_up(std::max<size_t>(bytes, 256), 256);
    if (a.cap >= bytes) return GPZ_OK;
    size_t grow = std::max(bytes, a.cap + a.cap / 2);
    if (capped && c->pool_used - a.cap + grow > c->pool_cap) {
        grow = bytes;
        if (c->pool_used - a.cap + grow > c->pool_cap) return fail(c, GPZ_E_ADMISSION, "device pool cap exceeded");
    }
    if (a.p) cudaFree(a.p);
    c->pool_used -= a.cap;
    a.p = nullptr;
    a.cap = 0;
    sl.gen++;
    cudaError_t e = cudaMalloc(&a.p, grow);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GPZ_E_NOMEM, "cudaMalloc", e);
    }
    a.cap = grow;
    c->pool_used += grow;
    return GPZ_OK;
}

template <class T>
int ensure_host(gpz_ctx* c, Slot& sl, T*& p, size_t& cap, size_t count, bool mapped) {
    if (cap >= count) return GPZ_OK;
    size_t grow = std::max(count, cap + cap / 2);
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    if (mapped) sl.gen++;
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&p), grow * sizeof(T),
                                  mapped ? cudaHostAllocMapped : cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GPZ_E_NOMEM, "cudaHostAlloc", e);
    }
    cap = grow;
    return GPZ_OK;
}

template <class T>
T* mapped_dev(T* host) {
    void* d = nullptr;
    if (cudaHostGetDevicePointer(&d, host, 0) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return static_cast<T*>(d);
}

// Cut inputs into members (gpu.rs:193-208: an input of at most member_bytes,
// empty included, is one member) and members into tiles.
void plan(const gpz_ctx* c, Slot& sl) {
    sl.members.clear();
    sl.tiles.clear();
    for (auto& s : sl.spans) {
        s.first_member = sl.members.size();
        const size_t nm = s.n == 0 ? 1 : (s.n + c->member_bytes - 1) / c->member_bytes;
        s.nmembers = nm;
        for (size_t j = 0; j < nm; j++) {
            MemberDesc md{};
            md.in_off = s.dev_off + j * c->member_bytes;
            md.len = (uint32_t)std::min(c->member_bytes, s.n - std::min(s.n, j * c->member_bytes));
            md.tile_base = (uint32_t)sl.tiles.size();
            md.ntiles = (md.len + GPZ_SEG - 1) / GPZ_SEG;
            md.frame = (j == 0 ? GPZ_MEMBER_FIRST : 0u) | (j + 1 == nm ? GPZ_MEMBER_LAST : 0u);
            md.out_slot = sl.members.size();
            for (uint32_t t = 0; t < md.ntiles; t++) sl.tiles.push_back(TileDesc{(uint32_t)sl.members.size(), t});
            sl.members.push_back(md);
        }
    }
}

size_t out_bound_of_plan(const Slot& sl) {
    size_t b = 0;
    for (auto& m : sl.members) b += member_bound(m.len);
    return b;
}

size_t desc_bytes(size_t nm, size_t nt) { return kDescHeader + nm * sizeof(MemberDesc) + nt * sizeof(TileDesc); }

// The descriptor arenas have fixed addresses between reallocations (which
// bump the slot's generation), so a captured graph stays valid for any batch
// that fits them.

// Sizes every device array (and the pinned descriptor / member-table
// staging) for a batch of in_bytes input, nm members and nt tiles.  Arrays
// only grow; a growth frees the old array (cudaFree synchronises the device)
// and bumps the slot's generation.
int reserve_counts(gpz_ctx* c, Slot& sl, size_t in_bytes, size_t nm, size_t nt, bool own_in, bool own_out,
                   size_t out_bytes, bool capped = true) {
    nm = std::max<size_t>(nm, 1);
    nt = std::max<size_t>(nt, 1);
    int rc;
    if (own_in && (rc = ensure_dev(c, sl, sl.d_in, in_bytes + 64, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_pp, in_bytes * 4 + 64, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_tok, in_bytes * 4 + 64, capped))) return rc;
    if (own_out && (rc = ensure_dev(c, sl, sl.d_out, out_bytes + 64, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_skeys, nt * GPZ_SEG * 2, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_son, nt * GPZ_SEG * 4, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_snkeys, nt * 4, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_tentry, nt * 4, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_texit, nt * GPZ_EXITS * 2, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_thist, nt * GPZ_NSYM * 2, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_tntok, nt * 4, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_tbit, nt * 4, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_mcodes, nm * GPZ_NSYM * 4, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_mhdr, nm * GPZ_HDR_WORDS * 4, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_mout, nm * sizeof(MemberOut), capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_cnt, GPZ_NCOUNTERS * 4 + 64, capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_members, nm * sizeof(MemberDesc), capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_tiles, nt * sizeof(TileDesc), capped))) return rc;
    if ((rc = ensure_dev(c, sl, sl.d_dims, kDescHeader, capped))) return rc;
    if ((rc = ensure_host(c, sl, sl.h_desc, sl.h_desc_cap, desc_bytes(nm, nt), true))) return rc;
    if ((rc = ensure_host(c, sl, sl.h_mout, sl.h_mout_cap, nm, true))) return rc;
    if ((rc = ensure_host(c, sl, sl.h_err, sl.h_err_cap, 16, true))) return rc;
    return GPZ_OK;
}

// Sizes the slot for its planned batch.
int reserve(gpz_ctx* c, Slot& sl, size_t in_bytes, bool own_in, bool own_out, size_t out_bytes) {
    return reserve_counts(c, sl, in_bytes, sl.members.size(), sl.tiles.size(), own_in, own_out, out_bytes);
}

// Sizes the slot once for every batch of at most max_bytes input in at most
// max_items items (all arrays, pinned input staging and mapped output), so
// that no batch within those limits allocates or frees anything.
int reserve_limits(gpz_ctx* c, Slot& sl, size_t max_bytes, size_t max_items) {
    const size_t in_bytes = max_bytes + 16 * max_items + 64;
    const size_t nm = max_bytes / c->member_bytes + max_items;
    const size_t nt = max_bytes / GPZ_SEG + max_items;
    const size_t out_bytes = nm * member_bound(0) + 2 * max_bytes;
    int rc;
    if ((rc = reserve_counts(c, sl, in_bytes, nm, nt, true, true, out_bytes, false))) return rc;
    if ((rc = ensure_host(c, sl, sl.h_in, sl.h_in_cap, in_bytes + 64, true))) return rc;
    return ensure_host(c, sl, sl.h_out, sl.h_out_cap, out_bytes + 64, true);
}

BatchParams params_of(const gpz_ctx* c, Slot& sl, const uint8_t* d_in, uint8_t* d_out) {
    BatchParams bp{};
    bp.in = d_in;
    bp.dims = static_cast<const uint32_t*>(sl.d_dims.p);
    bp.members = static_cast<const MemberDesc*>(sl.d_members.p);
    bp.tiles = static_cast<const TileDesc*>(sl.d_tiles.p);
    bp.pp = static_cast<uint32_t*>(sl.d_pp.p);
    bp.seg_keys = static_cast<uint16_t*>(sl.d_skeys.p);
    bp.seg_on = static_cast<uint32_t*>(sl.d_son.p);
    bp.seg_nkeys = static_cast<uint32_t*>(sl.d_snkeys.p);
    bp.tok = static_cast<uint32_t*>(sl.d_tok.p);
    bp.out_words = reinterpret_cast<uint32_t*>(d_out);
    bp.tile_entry = static_cast<uint32_t*>(sl.d_tentry.p);
    bp.tile_exit = static_cast<uint16_t*>(sl.d_texit.p);
    bp.tile_hist = static_cast<uint16_t*>(sl.d_thist.p);
    bp.tile_ntok = static_cast<uint32_t*>(sl.d_tntok.p);
    bp.tile_bitoff = static_cast<uint32_t*>(sl.d_tbit.p);
    bp.member_codes = static_cast<uint32_t*>(sl.d_mcodes.p);
    bp.member_hdr = static_cast<uint32_t*>(sl.d_mhdr.p);
    bp.member_out = static_cast<MemberOut*>(sl.d_mout.p);
    bp.counters = static_cast<uint32_t*>(sl.d_cnt.p);
    bp.err = bp.counters + GPZ_NCOUNTERS;
    bp.nmembers = (uint32_t)sl.members.size();
    bp.ntiles = (uint32_t)sl.tiles.size();
    bp.out_base = 0;
    bp.flags = (c->flags & GPZ_FLAG_FIXED_BLOCKS) ? GPZ_BATCH_FIXED : 0u;
    if (c->codec == GPZ_CODEC_ZSTD) {
        bp.flags = GPZ_BATCH_ZSTD;
        // 4 bytes per tile inside the exit tables (516 bytes per tile)
        bp.tile_zinfo = static_cast<uint32_t*>(sl.d_texit.p);
    }
    return bp;
}

// Descriptors staged as [dims][members][tiles] in pinned memory: the
// 64-byte header holds the tile and member counts (u32 at bytes 0 and 4) and
// the batch's input bytes (u64 at byte 8).
void write_desc(Slot& sl) {
    const size_t nm = sl.members.size(), nt = sl.tiles.size();
    uint32_t* dims = reinterpret_cast<uint32_t*>(sl.h_desc);
    std::memset(dims, 0, kDescHeader);
    dims[0] = (uint32_t)nt;
    dims[1] = (uint32_t)nm;
    const uint64_t in_bytes = sl.in_bytes;
    std::memcpy(sl.h_desc + 8, &in_bytes, 8);
    uint8_t* hm = sl.h_desc + kDescHeader;
    std::memcpy(hm, sl.members.data(), nm * sizeof(MemberDesc));
    if (nt) std::memcpy(hm + nm * sizeof(MemberDesc), sl.tiles.data(), nt * sizeof(TileDesc));
}

// ... uploaded into their three arenas by copies on stream s.
int upload_desc(gpz_ctx* c, Slot& sl, cudaStream_t s) {
    const size_t nm = sl.members.size(), nt = sl.tiles.size();
    write_desc(sl);
    uint8_t* hm = sl.h_desc + kDescHeader;
    uint8_t* ht = hm + nm * sizeof(MemberDesc);
    CU(c, cudaMemcpyAsync(sl.d_dims.p, sl.h_desc, kDescHeader, cudaMemcpyHostToDevice, s));
    CU(c, cudaMemcpyAsync(sl.d_members.p, hm, nm * sizeof(MemberDesc), cudaMemcpyHostToDevice, s));
    if (nt) CU(c, cudaMemcpyAsync(sl.d_tiles.p, ht, nt * sizeof(TileDesc), cudaMemcpyHostToDevice, s));
    return GPZ_OK;
}

LaunchShape shape_for(gpz_ctx* c, int bucket) {
    LaunchShape s;
    {
        std::lock_guard<std::mutex> lk(c->tune_mu);
        s = c->shape[bucket];
    }
    if (c->fixed.lookup_threads) {
        LaunchShape f{c->fixed.lookup_threads, 0, c->fixed.walk_threads, 0, c->fixed.emit_threads, 0, 0, 0};
        gpz_occupancy(&f);
        if (c->fixed.lookup_grid) f.lookup_grid = c->fixed.lookup_grid;
        if (c->fixed.walk_grid) f.walk_grid = c->fixed.walk_grid;
        if (c->fixed.emit_grid) f.emit_grid = c->fixed.emit_grid;
        s = f;
    }
    return s;
}

// Stage kernels (+ drain) for the slot's planned batch, as a CUDA graph per
// (slot, bucket) or as direct launches on stream s.
int launch(gpz_ctx* c, Slot& sl, const BatchParams& bp, const LaunchShape& shape, bool use_graph,
           const DrainTarget* drain, bool timing, cudaStream_t s, const FetchSource* fetch = nullptr) {
    if (!use_graph) {
        // with k_fetch, the fetch kernel zeroes the counters itself
        if (!fetch) CU(c, cudaMemsetAsync(sl.d_cnt.p, 0, GPZ_NCOUNTERS * 4 + 64, s));
        if (gpz_launch_batch(bp, shape, s, timing ? reinterpret_cast<void* const*>(sl.ev) : nullptr, drain,
                             fetch) != 0)
            return fail(c, GPZ_E_CUDA, "kernel launch", cudaGetLastError());
        c->launches = kStageKernels + (drain ? 1 : 0) + (fetch ? 1 : 0);
        return GPZ_OK;
    }
    Slot::Graph& g = sl.graphs[sl.bucket];
    if (g.exec && g.gen != sl.gen) {
        cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
    if (!g.exec) {
        cudaGraph_t graph = nullptr;
        CU(c, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        if (!fetch) cudaMemsetAsync(sl.d_cnt.p, 0, GPZ_NCOUNTERS * 4 + 64, s);
        gpz_launch_batch(bp, shape, s, nullptr, drain, fetch);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (e != cudaSuccess) return fail(c, GPZ_E_CUDA, "graph capture", e);
        e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            g.exec = nullptr;
            return fail(c, GPZ_E_CUDA, "graph instantiate", e);
        }
        g.gen = sl.gen;
    }
    CU(c, cudaGraphLaunch(g.exec, s));
    c->launches = kStageKernels + (drain ? 1 : 0) + (fetch ? 1 : 0);
    return GPZ_OK;
}

// Persistent default shape for every bucket; tuned lazily on first use.
// Small batches (up to 512 tiles) walk in the block form, whose latency per
// tile is lowest; larger ones in the warp form, whose throughput is highest.
void default_shapes(gpz_ctx* c) {
    for (int b = 0; b < kBuckets; b++) {
        LaunchShape s{1024, 0, b <= 1 ? 1024 : 512, 0, 512, 0, 0, 0};
        gpz_occupancy(&s);
        c->shape[b] = s;
    }
}

// Autotuner: each candidate (threads per lookup CTA, per walk CTA, per emit
// CTA, with persistent grids from occupancy) runs the batch -- every shape
// gives the same output -- and the fastest becomes the bucket's shape.  All
// candidates run once untimed first: a kernel's first launch in a process
// also loads its module, which would otherwise count against whichever
// candidate uses it first.
int autotune(gpz_ctx* c, Slot& sl, const BatchParams& bp, const DrainTarget* dt, cudaStream_t s) {
    const int lt[3] = {1024, 768, 512}, wt[2] = {512, 1024}, et[2] = {512, 256};
    constexpr int kCands = 12;
    float best = 1e30f;
    LaunchShape best_s = c->shape[sl.bucket];
    cudaEvent_t a, b;
    CU(c, cudaEventCreate(&a));
    CU(c, cudaEventCreate(&b));
    int rc = GPZ_OK;
    for (int i = 0; i < 2 * kCands && rc == GPZ_OK; i++) {
        const int k = i % kCands;
        LaunchShape cand{lt[k % 3], 0, wt[(k / 3) & 1], 0, et[(k / 6) & 1], 0, 0, 0};
        gpz_occupancy(&cand);
        cudaEventRecord(a, s);
        rc = launch(c, sl, bp, cand, false, dt, false, s);
        cudaEventRecord(b, s);
        if (rc == GPZ_OK) rc = wait_event(c, b, "autotune");
        if (rc == GPZ_E_TIMEOUT && cudaEventRecord(sl.done, s) == cudaSuccess) sl.stale = true;
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (rc == GPZ_OK && i >= kCands && ms < best) {
            best = ms;
            best_s = cand;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->tune_mu);
    c->shape[sl.bucket] = best_s;
    c->tuned[sl.bucket] = true;
    return GPZ_OK;
}

void add_time(gpz_ctx* c, int k, double ms) {
    std::lock_guard<std::mutex> lk(c->times_mu);
    c->host_ms[k] += ms;
}

// How a batch is launched.
struct LaunchPolicy {
    bool exact = false;     // grids sized to this batch (one CTA per item), no graph
    bool autotune = true;   // tune the bucket's shape on its first use
    bool graphs = true;     // per-(slot, bucket) CUDA graph
    bool fetch = false;     // SMs fetch input and descriptors from mapped memory (k_fetch)
    int grid_pct = 100;     // persistent grids at this percentage of full occupancy
};
constexpr LaunchPolicy kPolicyBatched{false, true, true, false, 100};
constexpr LaunchPolicy kPolicyPlain{true, false, false, false, 100};
// The streaming pass loop never stops to tune: its passes change size as
// chunks arrive, and tuning a new bucket (every shape run twice) held a
// writer's stream for 60-120 ms.  It uses the tuned shape where a bucket
// has one and the default shape otherwise.
constexpr LaunchPolicy kPolicyStream{false, false, true, false, 100};

// True when every non-empty input of the batch starts in page-locked host
// memory (cudaHostAlloc or cudaHostRegister), so the copy engine can read
// it directly.  Whether a whole range is page-locked is the driver's to
// decide: cudaMemcpyAsync handles any host range correctly and only loses
// its asynchrony on pageable memory.
bool all_page_locked(const gpz_desc* d, size_t count) {
    size_t nonempty = 0;
    for (size_t i = 0; i < count; i++) {
        if (!d[i].n) continue;
        nonempty++;
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, d[i].in) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (a.type != cudaMemoryTypeHost) return false;
    }
    return nonempty > 0;
}

// Plans, uploads and launches one batch of host items on a slot (no wait).
// Uploads go on the slot's stream; kernels on ks when given (after the
// upload), else on the slot's stream too.
int submit_slot(gpz_ctx* c, Slot& sl, const gpz_desc* d, size_t count, const LaunchPolicy& pol,
                cudaStream_t ks = nullptr) {
    double t0 = now_ms();
    sl.spans.assign(count, Span{});
    size_t in_bytes = 0;
    for (size_t i = 0; i < count; i++) {
        sl.spans[i].n = d[i].n;
        sl.spans[i].dev_off = in_bytes;
        in_bytes += round_up(std::max<size_t>(d[i].n, 1), 16);
    }
    sl.in_bytes = in_bytes;
    plan(c, sl);
    const size_t obound = out_bound_of_plan(sl);
    int rc;
    if ((rc = reserve(c, sl, in_bytes, true, true, obound))) return rc;
    if ((rc = ensure_host(c, sl, sl.h_in, sl.h_in_cap, in_bytes + 64, true))) return rc;
    if ((rc = ensure_host(c, sl, sl.h_out, sl.h_out_cap, obound + 64, true))) return rc;
    double t1 = now_ms();
    add_time(c, 0, t1 - t0);
    // Inputs the caller already holds in page-locked memory are uploaded
    // from where they are; the others are first staged into the slot's
    // pinned buffer by the copy threads.
    const bool direct = !pol.fetch && all_page_locked(d, count);
    if (!direct) {
        std::vector<CopyPool::Copy> copies;
        for (size_t i = 0; i < count; i++)
            if (d[i].n) copies.push_back(CopyPool::Copy{sl.h_in + sl.spans[i].dev_off, d[i].in, d[i].n});
        copy_pool().run(copies, true);
    }
    t0 = now_ms();
    add_time(c, 1, t0 - t1);
    cudaStream_t s = sl.stream;
    if (ks && c->last_upload) CU(c, cudaStreamWaitEvent(s, c->last_upload, 0));
    CU(c, cudaEventRecord(sl.tv[0], s));
    FetchSource fs{};
    if (pol.fetch) {
        write_desc(sl);
        fs.h_desc = mapped_dev(sl.h_desc);
        fs.h_in = mapped_dev(sl.h_in);
        if (!fs.h_desc || !fs.h_in) return fail(c, GPZ_E_CUDA, "mapped host memory");
        fs.d_dims = static_cast<uint32_t*>(sl.d_dims.p);
        fs.d_members = static_cast<MemberDesc*>(sl.d_members.p);
        fs.d_tiles = static_cast<TileDesc*>(sl.d_tiles.p);
        fs.d_in = static_cast<uint8_t*>(sl.d_in.p);
        fs.members_cap = sl.d_members.cap / sizeof(MemberDesc);
        fs.tiles_cap = sl.d_tiles.cap / sizeof(TileDesc);
        fs.in_cap = sl.d_in.cap;
    } else {
        if (direct) {
            uint8_t* din = static_cast<uint8_t*>(sl.d_in.p);
            for (size_t i = 0; i < count; i++)
                if (d[i].n) CU(c, cudaMemcpyAsync(din + sl.spans[i].dev_off, d[i].in, d[i].n, cudaMemcpyHostToDevice, s));
        } else {
            CU(c, cudaMemcpyAsync(sl.d_in.p, sl.h_in, in_bytes, cudaMemcpyHostToDevice, s));
        }
        if ((rc = upload_desc(c, sl, s))) return rc;
    }
    CU(c, cudaEventRecord(sl.tv[1], s));
    // with a separate kernel stream, the drain runs on the slot's stream:
    // the next pass's kernels need not wait for it
    const bool split_drain = ks && ks != s && !pol.fetch;
    if (ks && ks != s) {
        CU(c, cudaStreamWaitEvent(ks, sl.tv[1], 0));
        c->last_upload = sl.tv[1];
        s = ks;
    }
    BatchParams bp = params_of(c, sl, static_cast<const uint8_t*>(sl.d_in.p), static_cast<uint8_t*>(sl.d_out.p));
    DrainTarget dt{mapped_dev(sl.h_out), mapped_dev(sl.h_mout), mapped_dev(sl.h_err), c->sms * 4};
    if (!dt.h_out || !dt.h_mout || !dt.h_err) return fail(c, GPZ_E_CUDA, "mapped host memory");
    sl.bucket = bucket_of(sl.tiles.size());
    const bool timing = (c->flags & GPZ_FLAG_STAGE_TIMING) != 0;
    if (pol.exact) {
        // one launch per kernel, grids sized to this batch, no graph
        const LaunchShape exact{1024, 0, 1024, 0, 512, 0, 0, 0};
        rc = launch(c, sl, bp, exact, false, split_drain ? nullptr : &dt, timing, s);
    } else {
        bool tuned;
        {
            std::lock_guard<std::mutex> lk(c->tune_mu);
            tuned = c->tuned[sl.bucket];
        }
        if (pol.autotune && !tuned && !(c->flags & GPZ_FLAG_NO_AUTOTUNE) && !c->fixed.lookup_threads &&
            (rc = autotune(c, sl, bp, &dt, s)))
            return rc;
        const bool graphs = pol.graphs && !(c->flags & GPZ_FLAG_NO_GRAPHS) && !timing;
        LaunchShape shape = shape_for(c, sl.bucket);
        if (pol.grid_pct < 100) {
            for (int* g : {&shape.lookup_grid, &shape.walk_grid, &shape.emit_grid, &shape.segtab_grid,
                           &shape.huff_grid})
                *g = std::max(1, *g * pol.grid_pct / 100);
        }
        rc = launch(c, sl, bp, shape, graphs, split_drain ? nullptr : &dt, timing, s, pol.fetch ? &fs : nullptr);
    }
    if (rc) return rc;
    CU(c, cudaEventRecord(sl.tv[2], s));
    if (split_drain) {
        CU(c, cudaStreamWaitEvent(sl.stream, sl.tv[2], 0));
        if (gpz_launch_drain(bp, dt, sl.stream) != 0) return fail(c, GPZ_E_CUDA, "drain launch", cudaGetLastError());
        c->launches++;
        CU(c, cudaEventRecord(sl.done, sl.stream));
    } else {
        CU(c, cudaEventRecord(sl.done, s));
    }
    sl.busy = true;
    add_time(c, 2, now_ms() - t0);
    {
        std::lock_guard<std::mutex> lk(c->times_mu);
        c->host_ms[5] += 1;
    }
    return GPZ_OK;
}

// 10-byte header and 8-byte trailer of every member (deflate.rs:962-980),
// written into a host copy of the batch output that starts at `base`.
void frame_members(const MemberOut* mo, size_t first, size_t count, uint8_t* dst, uint64_t base) {
    static const uint8_t hdr[10] = {0x1f, 0x8b, 0x08, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0xff};
    for (size_t m = first; m < first + count; m++) {
        if (mo[m].frame_bytes != 18) continue;  // zstd frames are complete on the device
        uint8_t* p = dst + (mo[m].gz_off - base);
        std::memcpy(p, hdr, 10);
        uint8_t* t = p + 10 + mo[m].deflate_bytes;
        for (int i = 0; i < 4; i++) t[i] = (uint8_t)(mo[m].crc >> (8 * i));
        for (int i = 0; i < 4; i++) t[4 + i] = (uint8_t)(mo[m].len >> (8 * i));
    }
}

// Waits for the slot's batch; returns the device status.
int wait_slot(gpz_ctx* c, Slot& sl) {
    sl.busy = false;
    const double t0 = now_ms();
    const int w = wait_event(c, sl.done, "waiting for a device pass");
    add_time(c, 3, now_ms() - t0);
    if (w == GPZ_E_TIMEOUT) sl.stale = true;
    if (w) return w;
    cudaEventElapsedTime(&sl.last_h2d_ms, sl.tv[0], sl.tv[1]);
    cudaEventElapsedTime(&sl.last_kernel_ms, sl.tv[1], sl.tv[2]);
    if (c->flags & GPZ_FLAG_STAGE_TIMING)
        for (int i = 0; i < GPZ_STAGES; i++) cudaEventElapsedTime(&c->stage_ms[i], sl.ev[i], sl.ev[i + 1]);
    if (*sl.h_err) return fail(c, GPZ_E_INTERNAL, "device self-check failed");
    return GPZ_OK;
}

// Waits for the slot's batch, frames it and copies each item's gzip stream
// into its caller buffer.
int finish_slot(gpz_ctx* c, Slot& sl, gpz_out* outs, size_t first_item) {
    int rc = wait_slot(c, sl);
    const double t0 = now_ms();
    const size_t nm = sl.members.size();
    c->mout.assign(sl.h_mout, sl.h_mout + nm);
    if (rc) return rc;
    frame_members(sl.h_mout, 0, nm, sl.h_out, 0);
    int first_bad = GPZ_OK;
    std::vector<CopyPool::Copy> copies;
    for (size_t i = 0; i < sl.spans.size(); i++) {
        const Span& sp = sl.spans[i];
        const MemberOut& a = sl.h_mout[sp.first_member];
        const MemberOut& z = sl.h_mout[sp.first_member + sp.nmembers - 1];
        const uint64_t beg = a.gz_off, end = z.gz_off + z.frame_bytes + z.deflate_bytes;
        gpz_out& o = outs[first_item + i];
        o.out_len = end - beg;
        if (!o.out || o.out_cap < end - beg) {
            o.status = GPZ_E_SPACE;
            if (first_bad == GPZ_OK) first_bad = GPZ_E_SPACE;
            continue;
        }
        copies.push_back(CopyPool::Copy{o.out, sl.h_out + beg, end - beg});
        o.status = GPZ_OK;
    }
    copy_pool().run(copies);
    add_time(c, 4, now_ms() - t0);
    if (first_bad != GPZ_OK) fail(c, first_bad, "output buffer too small");
    return first_bad;
}

// Before a synchronous call reuses the context's slots: the work of every
// slot a timed-out call left behind must have finished (bounded again).
int settle_stale(gpz_ctx* c) {
    for (int k = 0; k <= kSyncSlots; k++) {
        Slot* sl = k < kSyncSlots ? &c->slots[k] : &c->inf;
        if (!sl->stale) continue;
        const int rc = wait_event(c, sl->done, "work of an earlier call that timed out");
        if (rc) return rc;
        sl->stale = false;
    }
    return GPZ_OK;
}

// Items -> device passes of at most batch_bytes, pipelined over the slots
// (plain: one item per pass, waited for before the next).
int run_host_items(gpz_ctx* c, const gpz_desc* d, size_t count, gpz_out* outs, bool plain) {
    if (const int rc = settle_stale(c)) {
        for (size_t q = 0; q < count; q++) outs[q].status = rc;
        return rc;
    }
    int first_bad = GPZ_OK, fatal = GPZ_OK;
    size_t pending_first[kSyncSlots] = {};
    auto settle = [&](int k) {
        Slot& sl = c->slots[k];
        if (!sl.busy) return;
        int rc = finish_slot(c, sl, outs, pending_first[k]);
        if (rc != GPZ_OK && rc != GPZ_E_SPACE) {
            for (size_t q = 0; q < sl.spans.size(); q++) outs[pending_first[k] + q].status = rc;
            if (fatal == GPZ_OK) fatal = rc;
        } else if (rc != GPZ_OK && first_bad == GPZ_OK) {
            first_bad = rc;
        }
    };
    size_t i = 0;
    int pass = 0;
    while (i < count && fatal == GPZ_OK) {
        size_t j = i, bytes = 0;
        if (plain) {
            j = i + 1;
        } else {
            // ramp up: the first passes are 1/16 and 1/4 of the pass size.
            // Only the first upload is exposed, and each later one is at
            // most 4x the pass before it, while uploads run ~4x faster
            // than the kernels, so it is done before the device needs it.
            const size_t cap = c->batch_bytes >> (pass < 2 ? 4 - 2 * pass : 0);
            while (j < count && (j == i || bytes + d[j].n <= cap)) bytes += d[j++].n;
        }
        pass++;
        const int k = plain ? 0 : c->next_slot;
        settle(k);
        if (fatal) break;
        int rc = submit_slot(c, c->slots[k], d + i, j - i, plain ? kPolicyPlain : kPolicyBatched, c->kstream);
        if (rc) {
            for (size_t q = i; q < j; q++) outs[q].status = rc;
            fatal = rc;
            break;
        }
        pending_first[k] = i;
        if (plain) settle(0);
        else c->next_slot = (c->next_slot + 1) % kSyncSlots;
        i = j;
    }
    for (int q = 0; q < kSyncSlots; q++) settle((c->next_slot + q) % kSyncSlots);
    return fatal != GPZ_OK ? fatal : first_bad;
}

}  // namespace

// The device writer's pass loop (gpz_stream.h).  Slots are used round robin
// and settled in submission order, as run_host_items does, but the passes
// are formed from whatever chunks the writer has ready, so consecutive
// passes of a stream overlap on the device without a call boundary between
// them; results go to the feed straight from the slot's mapped output.
int gpz_stream_run(gpz_ctx* c, GpzStreamFeed& feed) {
    if (!c) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    int fatal = settle_stale(c);
    if (fatal) return fatal;
    std::deque<int> pend;  // slots in submission order
    auto settle = [&]() {
        const int k = pend.front();
        pend.pop_front();
        Slot& sl = c->slots[k];
        int r = wait_slot(c, sl);
        const double t0 = now_ms();
        if (r == GPZ_OK && fatal == GPZ_OK) {
            frame_members(sl.h_mout, 0, sl.members.size(), sl.h_out, 0);
            for (size_t i = 0; i < sl.spans.size() && r == GPZ_OK; i++) {
                const Span& sp = sl.spans[i];
                const MemberOut& a = sl.h_mout[sp.first_member];
                const MemberOut& z = sl.h_mout[sp.first_member + sp.nmembers - 1];
                const uint64_t end = z.gz_off + z.frame_bytes + z.deflate_bytes;
                if (feed.deliver(sl.h_out + a.gz_off, end - a.gz_off) != 0) r = fail(c, GPZ_E_SINK, "sink");
            }
            feed.pass_done();
        }
        add_time(c, 4, now_ms() - t0);
        if (r != GPZ_OK && fatal == GPZ_OK) fatal = r;
    };
    std::vector<gpz_desc> items;
    for (int pass = 0; fatal == GPZ_OK;) {
        if ((int)pend.size() == kSyncSlots) {
            settle();
            continue;
        }
        const size_t cap = c->batch_bytes >> (pass < 2 ? 4 - 2 * pass : 0);
        const bool busy = !pend.empty();
        items.clear();
        // an idle device takes whatever is queued, empty inputs included
        feed.take(items, cap, busy ? std::min<size_t>(cap, 8u << 20) : 0, false);
        if (items.empty()) {
            if (!busy) break;  // nothing ready and nothing on the device
            settle();
            continue;
        }
        const int k = c->next_slot;  // not pending: fewer than kSyncSlots are, in round-robin order
        const int rc = submit_slot(c, c->slots[k], items.data(), items.size(), kPolicyStream, c->kstream);
        if (rc) {
            fatal = rc;
            break;
        }
        pend.push_back(k);
        c->next_slot = (k + 1) % kSyncSlots;
        pass++;
    }
    while (!pend.empty()) settle();
    return fatal;
}

uint8_t* gpz_pinned_alloc(size_t n) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, std::max<size_t>(n, 1), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return static_cast<uint8_t*>(p);
}

void gpz_pinned_free(uint8_t* p) {
    if (p) cudaFreeHost(p);
}

void gpz_parallel_copy(void* dst, const void* src, size_t n) { copy_pool().run({CopyPool::Copy{dst, src, n}}, true); }

namespace {

// priority: a CUDA stream priority (lower is more urgent; 0 is the default)
int init_slot(gpz_ctx* c, Slot& sl, int priority = 0) {
    CU(c, cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, priority));
    CU(c, cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    for (auto& e : sl.tv) CU(c, cudaEventCreate(&e));
    if (c->flags & GPZ_FLAG_STAGE_TIMING)
        for (auto& e : sl.ev) CU(c, cudaEventCreate(&e));
    return ensure_host(c, sl, sl.h_err, sl.h_err_cap, 16, true);
}

void free_slot(gpz_ctx* c, Slot& sl) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    for (auto& g : sl.graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (DevArena* a : {&sl.d_in, &sl.d_pp, &sl.d_tok, &sl.d_out, &sl.d_skeys, &sl.d_son, &sl.d_snkeys,
                        &sl.d_tentry, &sl.d_texit, &sl.d_thist, &sl.d_tntok, &sl.d_tbit, &sl.d_mcodes, &sl.d_mhdr,
                        &sl.d_mout, &sl.d_cnt, &sl.d_members, &sl.d_tiles, &sl.d_dims, &sl.d_itail, &sl.d_icand,
                        &sl.d_isub})
        if (a->p) {
            cudaFree(a->p);
            c->pool_used -= a->cap;
            a->p = nullptr;
            a->cap = 0;
        }
    for (void* h : {(void*)sl.h_in, (void*)sl.h_desc, (void*)sl.h_out, (void*)sl.h_mout, (void*)sl.h_err})
        if (h) cudaFreeHost(h);
    for (auto& e : sl.ev)
        if (e) cudaEventDestroy(e);
    if (sl.done) cudaEventDestroy(sl.done);
    for (auto& e : sl.tv)
        if (e) cudaEventDestroy(e);
    if (sl.stream) cudaStreamDestroy(sl.stream);
}

}  // namespace

// ================================================================ serving

namespace {

struct Request {
    uint64_t id = 0;
    std::vector<uint8_t> in;  // owned copy (gpz_submit), or empty (gpz_submit_ref)
    const uint8_t* src = nullptr;
    size_t n = 0;
    size_t units = 0, units_done = 0;
    std::vector<std::vector<uint8_t>> pieces;  // gzip members of each unit
    double t_arrive = 0, t_done = 0;
    int status = GPZ_OK;
    bool done = false;
    bool small = false;
};

struct Unit {
    std::shared_ptr<Request> req;
    size_t index = 0, off = 0, n = 0;
};

}  // namespace

// SM partitions (green contexts) for the serving lanes.  The driver entry
// points are resolved at run time through the CUDA runtime, so the library
// does not link libcuda.  A partition is a CUcontext restricted to a set of
// SMs; memory, streams, events and graphs made while it is current belong to
// it, and kernels launched on its streams run only on its SMs.
struct GreenApi {
    CUresult (*dev_get)(CUdevice*, int) = nullptr;
    CUresult (*get_res)(CUdevice, CUdevResource*, CUdevResourceType) = nullptr;
    CUresult (*split)(CUdevResource*, unsigned*, const CUdevResource*, CUdevResource*, unsigned, unsigned) = nullptr;
    CUresult (*gen_desc)(CUdevResourceDesc*, CUdevResource*, unsigned) = nullptr;
    CUresult (*create)(CUgreenCtx*, CUdevResourceDesc, CUdevice, unsigned) = nullptr;
    CUresult (*destroy)(CUgreenCtx) = nullptr;
    CUresult (*to_ctx)(CUcontext*, CUgreenCtx) = nullptr;
    CUresult (*set_cur)(CUcontext) = nullptr;
    CUresult (*get_cur)(CUcontext*) = nullptr;
    bool ok = false;

    GreenApi() {
        auto get = [](const char* name, auto& fn) {
            void* p = nullptr;
            cudaDriverEntryPointQueryResult q;
            if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess ||
                q != cudaDriverEntryPointSuccess) {
                cudaGetLastError();
                return false;
            }
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(p);
            return true;
        };
        ok = get("cuDeviceGet", dev_get) && get("cuDeviceGetDevResource", get_res) &&
             get("cuDevSmResourceSplitByCount", split) && get("cuDevResourceGenerateDesc", gen_desc) &&
             get("cuGreenCtxCreate", create) && get("cuGreenCtxDestroy", destroy) &&
             get("cuCtxFromGreenCtx", to_ctx) && get("cuCtxSetCurrent", set_cur) && get("cuCtxGetCurrent", get_cur);
    }
};

GreenApi& green_api() {
    static GreenApi api;
    return api;
}

struct SmPartition {
    CUgreenCtx green = nullptr;
    CUcontext ctx = nullptr;
    int sms = 0;
};

// Splits the device's SMs into `first` SMs (rounded as the driver requires)
// and the rest.  Returns false (and leaves nothing behind) if the driver
// cannot.
bool make_partitions(int device, int first, SmPartition out[2]) {
    GreenApi& g = green_api();
    if (!g.ok) return false;
    CUdevice dev;
    CUdevResource all, part[1], rest;
    unsigned nb = 1;
    CUdevResourceDesc d[2];
    if (g.dev_get(&dev, device) != CUDA_SUCCESS || g.get_res(dev, &all, CU_DEV_RESOURCE_TYPE_SM) != CUDA_SUCCESS ||
        g.split(part, &nb, &all, &rest, 0, (unsigned)first) != CUDA_SUCCESS || nb != 1 || rest.sm.smCount == 0 ||
        g.gen_desc(&d[0], &part[0], 1) != CUDA_SUCCESS || g.gen_desc(&d[1], &rest, 1) != CUDA_SUCCESS)
        return false;
    for (int i = 0; i < 2; i++) {
        if (g.create(&out[i].green, d[i], dev, CU_GREEN_CTX_DEFAULT_STREAM) != CUDA_SUCCESS ||
            g.to_ctx(&out[i].ctx, out[i].green) != CUDA_SUCCESS) {
            for (int j = 0; j <= i; j++)
                if (out[j].green) g.destroy(out[j].green);
            out[0] = out[1] = SmPartition{};
            return false;
        }
    }
    out[0].sms = (int)part[0].sm.smCount;
    out[1].sms = (int)rest.sm.smCount;
    return true;
}

// Continuous batching over two lanes.  Requests of at most 1 MiB go to the
// small lane, larger ones (cut into 2 MiB units, whole members) to the large
// lane.  Each lane has pipeline slots (three small, two large), a launcher
// thread that forms a batch from the lane's queue (arrival order, up to the
// lane's batch cap) whenever one of its slots is free and launches it while
// the other slots' batches are still on the device, and a completer thread
// that retires the lane's batches in launch order (framing, copies into the
// requests).
//
// The lanes share the GPU through stream priorities and grid sizes: the
// small lane's streams are the most urgent and the large lane's persistent
// grids cover three quarters of the GPU's resident CTAs, so the small lane's
// CTAs find SMs as the large lane's CTAs retire.  With GPZ_FLAG_SM_PARTITION
// the lanes run on two SM partitions instead (green contexts: 32 SMs for the
// small lane, the rest for the large one): strict isolation, at the price of
// the small lane's peak throughput.  The small
// lane fetches its input and descriptors with SM loads from mapped memory
// (k_fetch), so it never queues behind the large lane's uploads on a copy
// engine.  Every slot is sized once at start for its lane's batch limits,
// so serving never allocates or frees device memory (cudaFree would
// synchronise the device).
//
// A request completes when its last unit does; its gzip stream is its
// units' members in order: byte for byte what gpz_compress_chunk returns for
// it alone.  Admission: a request is rejected with GPZ_E_ADMISSION while the
// bytes queued or on the device would exceed the pool cap, and with
// GPZ_E_BUSY while kMaxRequests requests are submitted and not yet polled.
struct ServeEngine {
    static constexpr size_t kUnit = 2u << 20;
    static constexpr size_t kSmall = 1u << 20;
    static constexpr int kLaneSlots = 3;
    // requests submitted and not yet polled: beyond this, submit says busy
    static constexpr size_t kMaxRequests = 1u << 20;
    // Overload.  Small requests are kept within a few ms of work: a small
    // request is admitted while the small lane's queue (not yet launched)
    // holds at most kSmallBacklog bytes (about 2 ms of the small lane's
    // measured rate).  Large requests yield first: one is admitted only while
    // the pool has kSmallReserve bytes to spare for the small lane and the
    // small lane's queue is below half its limit, and while more than one
    // small batch waits, a large batch is launched only after that backlog
    // clears (for at most kLargeHoldMs, so the large lane always moves).
    // Measured over 60 s at 50k req/s with a 24 MiB limit and a hold on any
    // waiting small work: p99 of small requests 6.6 ms, and the large lane
    // lost throughput at 10k req/s.
    static constexpr size_t kSmallBacklog = 12u << 20;
    static constexpr size_t kSmallReserve = 1ull << 30;
    static constexpr double kLargeHoldMs = 20.0;

    struct Lane {
        int nslots = 2;         // pipeline slots in use (at most kLaneSlots)
        size_t batch_cap = 0;   // input bytes per batch
        size_t batch_cap_busy = 0;  // input bytes per batch while more than one batch waits
        size_t backlog = 0;     // bytes queued and not yet launched
        size_t max_units = 0;   // units per batch
        LaunchPolicy pol;
        Slot slots[kLaneSlots];
        bool slot_free[kLaneSlots] = {true, true, true};
        std::vector<Unit> inflight[kLaneSlots];
        int launch_rc[kLaneSlots] = {0, 0, 0};
        std::deque<Unit> q;
        std::deque<int> inflight_q;  // slots in launch order
        std::condition_variable cv_work, cv_inflight;
        std::thread launcher, completer;
        double t_launch[kLaneSlots] = {0, 0, 0}, t_submitted[kLaneSlots] = {0, 0, 0};
        gpz_lane_stats st{};  // guarded by the engine mutex
    };

    gpz_ctx* c = nullptr;
    Lane lanes[2];  // 0: requests <= 1 MiB, 1: larger
    SmPartition part[2];  // per lane, when the GPU is partitioned
    bool partitioned = false;
    static constexpr int kSmallLaneSms = 32;
    std::mutex mu;
    std::condition_variable cv_done;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    size_t queued_bytes = 0;
    std::vector<double> lat_all, lat_small;
    uint64_t rejected = 0, batches = 0, bytes_in = 0, bytes_out = 0;
    double max_queue_ms = 0;

    // Makes lane l's partition (or the device's primary context) current on
    // the calling thread.
    void bind(int l) {
        if (partitioned) green_api().set_cur(part[l].ctx);
        else cudaSetDevice(c->device);
    }

    int start(gpz_ctx* ctx) {
        c = ctx;
        cudaSetDevice(c->device);
        cudaFree(nullptr);  // the primary context exists before partitioning
        CUcontext primary = nullptr;
        if ((c->flags & GPZ_FLAG_SM_PARTITION) && c->sms >= 4 * kSmallLaneSms && green_api().ok &&
            green_api().get_cur(&primary) == CUDA_SUCCESS)
            partitioned = make_partitions(c->device, kSmallLaneSms, part);
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        Lane& sm = lanes[0];
        sm.nslots = 3;
        sm.batch_cap = 1u << 20;  // <= 256 tiles + one per unit: the low-latency buckets
        // a backlog is worked off in 4 MiB batches: more bytes per launch
        // while the queue, not the batch, sets the small requests' latency
        sm.batch_cap_busy = 4u << 20;
        sm.max_units = 1024;
        sm.pol = LaunchPolicy{false, false, true, true, 100};  // persistent default shape, graphs, k_fetch
        Lane& lg = lanes[1];
        lg.nslots = 2;
        lg.batch_cap = 16u << 20;
        lg.batch_cap_busy = lg.batch_cap;
        lg.max_units = 16;
        // without partitions: persistent grids on 60 % of the GPU, the rest
        // stays free for the small lane's CTAs; copy-engine upload.  Against
        // 75 % grids and 2 MiB small batches this took the small lane's p99
        // at 10k req/s from 2.2-2.5 ms to 1.7-1.9 ms for 2 % less throughput.
        lg.pol = LaunchPolicy{false, false, true, false, 60};
        if (partitioned) {
            // each lane's persistent grids cover its own SMs
            sm.pol.grid_pct = std::max(1, 100 * part[0].sms / c->sms);
            lg.pol.grid_pct = std::max(1, 100 * part[1].sms / c->sms);
        }
        int rc = GPZ_OK;
        for (int l = 0; l < 2 && !rc; l++) {
            bind(l);
            if (partitioned && gpz_kernel_smem_setup() != 0) rc = fail(c, GPZ_E_CUDA, "partition setup");
            for (int k = 0; k < lanes[l].nslots && !rc; k++) {
                Slot& s = lanes[l].slots[k];
                rc = init_slot(c, s, l == 0 ? greatest : least);
                if (!rc) rc = reserve_limits(c, s, lanes[l].batch_cap_busy, lanes[l].max_units);
            }
        }
        if (partitioned) green_api().set_cur(primary);
        if (rc) {
            shutdown();  // frees what was made; no thread runs yet
            return rc;
        }
        for (auto& L : lanes) {
            L.launcher = std::thread([this, &L] { launch_loop(L); });
            L.completer = std::thread([this, &L] { complete_loop(L); });
        }
        return GPZ_OK;
    }

    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        for (auto& L : lanes) {
            L.cv_work.notify_all();
            L.cv_inflight.notify_all();
        }
        for (auto& L : lanes) {
            if (L.launcher.joinable()) L.launcher.join();
            if (L.completer.joinable()) L.completer.join();
        }
        CUcontext primary = nullptr;
        if (partitioned) green_api().get_cur(&primary);
        for (int l = 0; l < 2; l++) {
            bind(l);
            for (auto& s : lanes[l].slots) free_slot(c, s);
        }
        if (partitioned) {
            green_api().set_cur(primary);
            for (auto& p : part) green_api().destroy(p.green);
            partitioned = false;
        }
    }

    int submit(const gpz_desc* d, uint64_t* ticket, bool copy) {
        auto r = std::make_shared<Request>();
        r->t_arrive = now_ms();
        r->small = d->n <= kSmall;
        r->units = d->n == 0 ? 1 : (d->n + kUnit - 1) / kUnit;
        r->pieces.resize(r->units);
        {
            std::lock_guard<std::mutex> lk(mu);
            const size_t reserve = r->small ? 0 : std::min(kSmallReserve, c->pool_cap / 4);
            const bool small_full = r->small ? lanes[0].backlog + d->n > kSmallBacklog
                                             : lanes[0].backlog > kSmallBacklog / 2;
            if (queued_bytes + d->n + reserve > c->pool_cap || small_full) {
                rejected++;
                return GPZ_E_ADMISSION;
            }
            if (reqs.size() >= kMaxRequests) {
                rejected++;
                return GPZ_E_BUSY;
            }
            queued_bytes += d->n;
        }
        if (copy) {
            r->in.assign(d->in, d->in + d->n);
            r->src = r->in.data();
        } else {
            r->src = d->in;  // the caller keeps it alive until the result is polled
        }
        r->n = d->n;
        Lane& L = lanes[r->small ? 0 : 1];
        std::lock_guard<std::mutex> lk(mu);
        r->id = next_id++;
        for (size_t u = 0; u < r->units; u++)
            L.q.push_back(Unit{r, u, u * kUnit, std::min(kUnit, d->n - std::min(d->n, u * kUnit))});
        L.backlog += d->n;
        reqs[r->id] = r;
        *ticket = r->id;
        L.cv_work.notify_one();
        return GPZ_OK;
    }

    int poll(uint64_t ticket, gpz_out* o, int wait_ms) {
        std::unique_lock<std::mutex> lk(mu);
        auto it = reqs.find(ticket);
        if (it == reqs.end()) return GPZ_E_ARG;
        auto r = it->second;
        if (!r->done && wait_ms > 0)
            cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return r->done; });
        if (!r->done) return GPZ_E_PENDING;
        size_t total = 0;
        for (auto& p : r->pieces) total += p.size();
        o->out_len = total;
        if (r->status != GPZ_OK) {
            o->status = r->status;
            reqs.erase(it);
            return o->status;
        }
        if (!o->out || o->out_cap < total) {
            o->status = GPZ_E_SPACE;
            return GPZ_E_SPACE;  // the result stays available for a larger buffer
        }
        lk.unlock();
        size_t k = 0;
        for (auto& p : r->pieces) {
            std::memcpy(o->out + k, p.data(), p.size());
            k += p.size();
        }
        o->status = GPZ_OK;
        lk.lock();
        reqs.erase(ticket);
        return GPZ_OK;
    }

    // The lane's next batch, in arrival order (caller holds mu).
    static std::vector<Unit> take_batch(Lane& L) {
        std::vector<Unit> b;
        size_t bytes = 0;
        const size_t cap = L.backlog > L.batch_cap ? L.batch_cap_busy : L.batch_cap;
        while (!L.q.empty() && b.size() < L.max_units && (b.empty() || bytes + L.q.front().n <= cap)) {
            bytes += L.q.front().n;
            b.push_back(L.q.front());
            L.q.pop_front();
        }
        L.backlog -= std::min(L.backlog, bytes);
        return b;
    }

    static int free_slot_of(const Lane& L) {
        for (int i = 0; i < L.nslots; i++)
            if (L.slot_free[i]) return i;
        return -1;
    }

    void launch_loop(Lane& L) {
        bind(&L == &lanes[0] ? 0 : 1);
        for (;;) {
            int k = -1;
            std::vector<Unit> batch;
            {
                std::unique_lock<std::mutex> lk(mu);
                L.cv_work.wait(lk, [&] { return stop || (!L.q.empty() && free_slot_of(L) >= 0); });
                if (stop) return;
                if (&L == &lanes[1]) {
                    // small work first: a large batch waits while small
                    // requests are queued, up to kLargeHoldMs
                    const double t_hold = now_ms();
                    while (!stop && lanes[0].backlog > lanes[0].batch_cap && now_ms() - t_hold < kLargeHoldMs)
                        L.cv_work.wait_for(lk, std::chrono::microseconds(200));
                    if (stop) return;
                    if (L.q.empty() || free_slot_of(L) < 0) continue;
                }
                k = free_slot_of(L);
                batch = take_batch(L);
                if (&L == &lanes[0] && lanes[0].backlog <= lanes[0].batch_cap) lanes[1].cv_work.notify_one();
                L.slot_free[k] = false;
                const double tl = now_ms(), q = tl - batch.front().req->t_arrive;
                max_queue_ms = std::max(max_queue_ms, q);
                L.st.queue_ms += q;
                L.st.max_queue_ms = std::max(L.st.max_queue_ms, q);
                L.t_launch[k] = tl;
            }
            std::vector<gpz_desc> ds(batch.size());
            for (size_t i = 0; i < batch.size(); i++)
                ds[i] = gpz_desc{batch[i].req->src + batch[i].off, batch[i].n, 0};
            L.inflight[k] = std::move(batch);
            const int rc = submit_slot(c, L.slots[k], ds.data(), ds.size(), L.pol);
            std::lock_guard<std::mutex> lk(mu);
            L.t_submitted[k] = now_ms();
            L.st.submit_ms += L.t_submitted[k] - L.t_launch[k];
            if (rc == GPZ_OK) batches++;
            else L.slots[k].busy = false;
            L.launch_rc[k] = rc;
            L.inflight_q.push_back(k);
            L.cv_inflight.notify_one();
        }
    }

    void complete_loop(Lane& L) {
        bind(&L == &lanes[0] ? 0 : 1);
        for (;;) {
            int k;
            {
                std::unique_lock<std::mutex> lk(mu);
                L.cv_inflight.wait(lk, [&] { return stop || !L.inflight_q.empty(); });
                if (L.inflight_q.empty()) return;
                k = L.inflight_q.front();
                L.inflight_q.pop_front();
            }
            int rc = L.launch_rc[k];
            if (rc == GPZ_OK) rc = wait_slot(c, L.slots[k]);
            {
                std::lock_guard<std::mutex> lk(mu);
                L.st.wait_ms += now_ms() - L.t_submitted[k];
                L.st.h2d_ms += L.slots[k].last_h2d_ms;
                L.st.kernel_ms += L.slots[k].last_kernel_ms;
            }
            complete(L, k, rc);
            // the batch's requests have their status; a batch that outlived
            // the wait still runs, so its slot is reused only once it is done
            if (L.slots[k].stale) {
                cudaEventSynchronize(L.slots[k].done);
                cudaGetLastError();
                L.slots[k].stale = false;
            }
            std::lock_guard<std::mutex> lk(mu);
            L.slot_free[k] = true;
            L.cv_work.notify_one();
        }
    }

    void complete(Lane& L, int k, int rc) {
        Slot& sl = L.slots[k];
        std::vector<Unit>& units = L.inflight[k];
        const double t0 = now_ms();
        std::vector<std::vector<uint8_t>> outs(units.size());
        if (rc == GPZ_OK) {
            frame_members(sl.h_mout, 0, sl.members.size(), sl.h_out, 0);
            for (size_t i = 0; i < units.size(); i++) {
                const Span& sp = sl.spans[i];
                const MemberOut& a = sl.h_mout[sp.first_member];
                const MemberOut& z = sl.h_mout[sp.first_member + sp.nmembers - 1];
                outs[i].assign(sl.h_out + a.gz_off, sl.h_out + z.gz_off + z.frame_bytes + z.deflate_bytes);
            }
        }
        const double t = now_ms();
        add_time(c, 4, t - t0);
        std::lock_guard<std::mutex> lk(mu);
        L.st.complete_ms += t - t0;
        L.st.batches++;
        L.st.units += units.size();
        for (auto& u : units) L.st.bytes += u.n;
        L.st.max_batch_ms = std::max(L.st.max_batch_ms, t - L.t_launch[k]);
        for (size_t i = 0; i < units.size(); i++) {
            auto& r = units[i].req;
            queued_bytes -= units[i].n;
            if (rc != GPZ_OK) r->status = rc;
            else {
                bytes_out += outs[i].size();
                r->pieces[units[i].index] = std::move(outs[i]);
            }
            if (++r->units_done == r->units) {
                r->done = true;
                r->t_done = t;
                const double lat = t - r->t_arrive;
                lat_all.push_back(lat);
                if (r->small) lat_small.push_back(lat);
                bytes_in += r->n;
                std::vector<uint8_t>().swap(r->in);
                r->src = nullptr;
            }
        }
        units.clear();
        cv_done.notify_all();
    }

    static double pct(std::vector<double> v, double q) {
        if (v.empty()) return 0;
        std::sort(v.begin(), v.end());
        const size_t i = (size_t)std::min<double>((double)(v.size() - 1), q * (double)(v.size() - 1) + 0.5);
        return v[i];
    }
};

// ====================================================================== ABI

extern "C" {

void gpz_config_default(gpz_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof *cfg);
    cfg->device = 0;
    cfg->member_bytes = kDefaultMember;
}

int gpz_create(const gpz_config* cfg, gpz_ctx** out) {
    if (!out) return GPZ_E_ARG;
    *out = nullptr;
    gpz_config def;
    gpz_config_default(&def);
    if (!cfg) cfg = &def;
    const size_t mb = cfg->member_bytes ? cfg->member_bytes : kDefaultMember;
    if (mb % GPZ_SEG != 0 || mb > kMaxMember) return GPZ_E_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return GPZ_E_CUDA;
    }
    if (cfg->device < 0 || cfg->device >= ndev) return GPZ_E_ARG;
    auto* c = new (std::nothrow) gpz_ctx();
    if (!c) return GPZ_E_NOMEM;
    c->device = cfg->device;
    c->member_bytes = mb;
    c->pool_cap = cfg->pool_bytes ? cfg->pool_bytes : kDefaultPool;
    c->batch_bytes = cfg->batch_bytes ? cfg->batch_bytes : kDefaultBatch;
    c->flags = cfg->flags;
    if (cfg->wait_ms < 0 || (cfg->codec != GPZ_CODEC_GZIP && cfg->codec != GPZ_CODEC_ZSTD) ||
        (cfg->codec == GPZ_CODEC_ZSTD && (cfg->flags & GPZ_FLAG_FIXED_BLOCKS))) {
        delete c;
        return GPZ_E_ARG;
    }
    c->codec = cfg->codec;
    c->wait_ms = cfg->wait_ms ? cfg->wait_ms : kDefaultWaitMs;
    if (cudaSetDevice(c->device) != cudaSuccess || gpz_kernel_smem_setup() != 0) {
        cudaGetLastError();
        delete c;
        return GPZ_E_CUDA;
    }
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
    default_shapes(c);
    // slot streams carry the uploads and the drains: the highest priority,
    // so a drain's CTAs are placed ahead of the next pass's waiting CTAs
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    for (auto& s : c->slots)
        if (init_slot(c, s, greatest) != GPZ_OK) {
            gpz_destroy(c);
            return GPZ_E_CUDA;
        }
    if (cudaStreamCreateWithFlags(&c->kstream, cudaStreamNonBlocking) != cudaSuccess) {
        c->kstream = nullptr;
        gpz_destroy(c);
        return GPZ_E_CUDA;
    }
    *out = c;
    return GPZ_OK;
}

void gpz_destroy(gpz_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->serve) {
        c->serve->shutdown();
        c->serve.reset();
    }
    if (c->kstream) cudaStreamSynchronize(c->kstream);
    for (auto& s : c->slots) free_slot(c, s);
    free_slot(c, c->inf);
    for (auto& e : c->inf_ev)
        if (e) cudaEventDestroy(e);
    if (c->kstream) cudaStreamDestroy(c->kstream);
    delete c;
}

size_t gpz_bound(size_t n) {
    const size_t nm = n == 0 ? 1 : (n + kDefaultMember - 1) / kDefaultMember;
    return nm * member_bound(kDefaultMember);
}

size_t gpz_bound_ctx(const gpz_ctx* c, size_t n) {
    if (!c) return gpz_bound(n);
    const size_t nm = n == 0 ? 1 : (n + c->member_bytes - 1) / c->member_bytes;
    return nm * member_bound(c->member_bytes);
}

// Concurrent callers are combined into one batch: each call queues itself;
// whichever caller finds no batch running takes everything queued (up to
// batch_bytes), runs it as one gpz_compress_batch and hands every caller
// its result.  A lone caller runs its chunk at once.  This takes the place
// of BatchedLz77's submitter thread (batch.rs:48-141), which batches the
// chunks that ParallelChunkedWriter's workers submit concurrently.
namespace {

// The queue of waiting gpz_compress_chunk calls as a stream feed: the
// leader's pass loop takes queued calls into passes and hands each call its
// result; one pass's results are copied out on the copy threads together.
struct CombineFeed : GpzStreamFeed {
    gpz_ctx* c;
    std::deque<gpz_ctx::ChunkCall*> taken;
    std::vector<CopyPool::Copy> copies;
    std::vector<gpz_ctx::ChunkCall*> finished;
    explicit CombineFeed(gpz_ctx* ctx) : c(ctx) {}
    bool take(std::vector<gpz_desc>& out, size_t max_bytes, size_t min_bytes, bool) override {
        std::lock_guard<std::mutex> lk(c->comb_mu);
        size_t have = 0;
        for (auto* q : c->comb_q) have += q->d.n;
        if (c->comb_q.empty() || have < min_bytes) return true;
        size_t bytes = 0;
        while (!c->comb_q.empty() && (out.empty() || bytes + c->comb_q.front()->d.n <= max_bytes)) {
            gpz_ctx::ChunkCall* q = c->comb_q.front();
            c->comb_q.pop_front();
            bytes += q->d.n;
            out.push_back(q->d);
            taken.push_back(q);
        }
        return true;
    }
    int deliver(const uint8_t* data, size_t n) override {
        gpz_ctx::ChunkCall* q = taken.front();
        taken.pop_front();
        q->o.out_len = n;
        if (!q->o.out || q->o.out_cap < n) {
            q->rc = GPZ_E_SPACE;  // this caller's buffer; the others go on
        } else {
            q->rc = GPZ_OK;
            copies.push_back(CopyPool::Copy{q->o.out, data, n});
        }
        finished.push_back(q);
        return GPZ_OK;
    }
    void pass_done() override {
        copy_pool().run(copies);
        copies.clear();
        std::lock_guard<std::mutex> lk(c->comb_mu);
        for (auto* q : finished) q->done = true;
        finished.clear();
        c->comb_cv.notify_all();
    }
};

}  // namespace

// Concurrent calls are combined: each call queues itself; a caller that
// finds no leader becomes one and runs the pass loop over the queue until
// it is empty and nothing is on the device, so the calls that arrive while
// passes run join later passes without the pipeline draining in between
// (BatchedLz77's submitter and completer threads, batch.rs:48-141).
int gpz_compress_chunk(gpz_ctx* c, const uint8_t* in, size_t n, int level, uint8_t* out, size_t out_cap,
                       size_t* out_len) {
    if (!c || (!in && n) || !out_len) return GPZ_E_ARG;
    gpz_ctx::ChunkCall me;
    me.d = gpz_desc{in, n, level};
    me.o = gpz_out{out, out_cap, 0, 0};
    std::unique_lock<std::mutex> q(c->comb_mu);
    c->comb_q.push_back(&me);
    while (!me.done) {
        if (c->comb_busy) {
            c->comb_cv.wait(q);
            continue;
        }
        c->comb_busy = true;
        q.unlock();
        CombineFeed feed(c);
        const int rc = gpz_stream_run(c, feed);
        q.lock();
        // calls taken by a failed loop get its status; queued ones wait for
        // the next leader
        for (auto* t : feed.taken) {
            t->rc = rc != GPZ_OK ? rc : GPZ_E_INTERNAL;
            t->done = true;
        }
        for (auto* t : feed.finished) t->done = true;
        if (rc != GPZ_OK) {
            // the calls still queued would meet the same failure (a wait
            // that timed out, an allocation): they return it too
            for (auto* t : c->comb_q) {
                t->rc = rc;
                t->done = true;
            }
            c->comb_q.clear();
        }
        c->comb_busy = false;
        c->comb_cv.notify_all();
    }
    *out_len = me.o.out_len;
    return me.rc;
}

int gpz_compress_batch(gpz_ctx* c, const gpz_desc* d, size_t count, gpz_out* outs) {
    if (!c || (!d && count) || (!outs && count)) return GPZ_E_ARG;
    for (size_t i = 0; i < count; i++)
        if (!d[i].in && d[i].n) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    return run_host_items(c, d, count, outs, false);
}

int gpz_compress_batch_plain(gpz_ctx* c, const gpz_desc* d, size_t count, gpz_out* outs) {
    if (!c || (!d && count) || (!outs && count)) return GPZ_E_ARG;
    for (size_t i = 0; i < count; i++)
        if (!d[i].in && d[i].n) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    return run_host_items(c, d, count, outs, true);
}

int gpz_compress_device(gpz_ctx* c, const void* d_in, const uint64_t* in_off, const uint64_t* in_len, size_t count,
                        void* d_out, size_t out_cap, uint64_t* out_off, void* stream) {
    if (!c || !d_in || !d_out || !in_off || !in_len || !out_off || !count) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    int rc;
    if ((rc = settle_stale(c))) return rc;
    Slot& sl = c->slots[0];
    sl.spans.assign(count, Span{});
    size_t in_end = 0;
    for (size_t i = 0; i < count; i++) {
        if (in_off[i] % 16) return fail(c, GPZ_E_ARG, "device inputs must start 16-byte aligned");
        sl.spans[i].n = in_len[i];
        sl.spans[i].dev_off = in_off[i];
        in_end = std::max<size_t>(in_end, in_off[i] + round_up(std::max<uint64_t>(in_len[i], 1), 16));
    }
    plan(c, sl);
    if (out_bound_of_plan(sl) > out_cap) return fail(c, GPZ_E_SPACE, "device output buffer below bound");
    if ((rc = reserve(c, sl, in_end, false, false, 0))) return rc;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : sl.stream;
    if ((rc = upload_desc(c, sl, s))) return rc;
    BatchParams bp = params_of(c, sl, static_cast<const uint8_t*>(d_in), static_cast<uint8_t*>(d_out));
    sl.bucket = bucket_of(sl.tiles.size());
    const bool timing = (c->flags & GPZ_FLAG_STAGE_TIMING) != 0;
    if ((rc = launch(c, sl, bp, shape_for(c, sl.bucket), false, nullptr, timing, s))) return rc;
    CU(c, cudaMemcpyAsync(sl.h_mout, sl.d_mout.p, sl.members.size() * sizeof(MemberOut), cudaMemcpyDeviceToHost, s));
    CU(c, cudaMemcpyAsync(sl.h_err, static_cast<uint32_t*>(sl.d_cnt.p) + GPZ_NCOUNTERS, 4, cudaMemcpyDeviceToHost, s));
    CU(c, cudaEventRecord(sl.done, s));
    if ((rc = wait_event(c, sl.done, "waiting for a device pass"))) {
        if (rc == GPZ_E_TIMEOUT) sl.stale = true;
        return rc;
    }
    if (timing)
        for (int i = 0; i < GPZ_STAGES; i++) cudaEventElapsedTime(&c->stage_ms[i], sl.ev[i], sl.ev[i + 1]);
    c->mout.assign(sl.h_mout, sl.h_mout + sl.members.size());
    if (*sl.h_err) return fail(c, GPZ_E_INTERNAL, "device self-check");
    for (size_t i = 0; i < count; i++) out_off[i] = c->mout[sl.spans[i].first_member].gz_off;
    const MemberOut& l = c->mout.back();
    out_off[count] = l.gz_off + l.frame_bytes + l.deflate_bytes;
    return GPZ_OK;
}

namespace {

const uint8_t kGzipHeader[10] = {0x1f, 0x8b, 0x08, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0xff};

uint32_t le32(const uint8_t* p) { return p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }

// Member boundaries as find_member_starts (parallel_decompress.rs:36-58):
// every occurrence of the header, scanning on 10 bytes past each one.
// Every offset at or after byte 10 where the 10-byte header starts, in
// order.  A long stream is cut into pieces of at least 1 MiB of start
// offsets, searched on half the host's threads (a search by one thread ran
// at about 5.7 GB/s, most of an inflate call's host time).
std::vector<size_t> header_hits(const uint8_t* in, size_t n) {
    constexpr size_t kPiece = 1u << 20;
    const size_t span = n - 10;  // start offsets [10, n)
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t pieces = span < 2 * kPiece ? 1 : std::min<size_t>(std::max(1u, hw / 2), span / kPiece);
    std::vector<std::vector<size_t>> hits(pieces);
    auto search = [&](size_t k) {
        // starts in [b, e): the haystack ends 9 bytes past e
        const size_t b = 10 + span * k / pieces, e = 10 + span * (k + 1) / pieces, end = std::min(n, e + 9);
        for (size_t p = b; p < e && p + 10 <= end;) {
            const void* q = memmem(in + p, end - p, kGzipHeader, 10);
            if (!q) break;
            const size_t at = static_cast<const uint8_t*>(q) - in;
            hits[k].push_back(at);
            p = at + 1;
        }
    };
    if (pieces == 1) {
        search(0);
    } else {
        std::vector<std::thread> th;
        for (size_t k = 1; k < pieces; k++) th.emplace_back(search, k);
        search(0);
        for (auto& t : th) t.join();
    }
    std::vector<size_t> all;
    for (auto& h : hits) all.insert(all.end(), h.begin(), h.end());
    return all;
}

int split_members(const uint8_t* in, size_t n, std::vector<InflateMember>* ms, size_t* total, std::string* why) {
    if (ms) ms->clear();
    *total = 0;
    if (n == 0) return GPZ_OK;
    if (n < 18 || std::memcmp(in, kGzipHeader, 10) != 0) {
        *why = "the stream does not start with gpzip's gzip header";
        return GPZ_E_DATA;
    }
    // scanning on 10 bytes past each match: of all header occurrences at or
    // after byte 10, in order, those at least 10 bytes past the last taken
    std::vector<size_t> starts{0};
    size_t p = 10;
    for (const size_t at : header_hits(in, n))
        if (at >= p) {
            starts.push_back(at);
            p = at + 10;
        }
    uint64_t out = 0;
    for (size_t i = 0; i < starts.size(); i++) {
        const size_t b = starts[i], e = i + 1 < starts.size() ? starts[i + 1] : n;
        if (e - b < 18 || e - b - 18 > 0xFFFFFFFFull) {
            *why = "member " + std::to_string(i) + " at byte " + std::to_string(b) + " has an impossible length";
            return GPZ_E_DATA;
        }
        InflateMember m{};
        m.in_off = b + 10;
        m.in_len = (uint32_t)(e - b - 18);
        m.crc = le32(in + e - 8);
        m.isize = le32(in + e - 4);
        // DEFLATE expands at most 1032:1 (a 258-byte match in 2 bits)
        if (m.isize > 1032ull * (m.in_len + 1ull)) {
            *why = "member " + std::to_string(i) + " at byte " + std::to_string(b) + " claims more output than its data can hold";
            return GPZ_E_DATA;
        }
        m.out_off = out;
        out += m.isize;
        if (ms) ms->push_back(m);
    }
    *total = out;
    return GPZ_OK;
}

const char* inflate_reason(uint32_t st) {
    switch (st) {
        case gpzi::kErrBlockType: return "invalid block type";
        case gpzi::kErrStoredLen: return "stored block length check";
        case gpzi::kErrCodeLens: return "invalid code lengths";
        case gpzi::kErrCodeSet: return "over-subscribed or incomplete code";
        case gpzi::kErrSymbol: return "invalid code";
        case gpzi::kErrDistance: return "distance too far back";
        case gpzi::kErrOutput: return "output longer than ISIZE";
        case gpzi::kErrInput: return "ran past the end of the member";
        case gpzi::kErrLength: return "output shorter than ISIZE";
        case gpzi::kErrTrailing: return "data between the last block and the trailer";
        case gpzi::kErrCrc: return "CRC-32 mismatch";
        case gpzi::kErrEmptyLen: return "distance code used but none defined";
        default: return "decode error";
    }
}

}  // namespace

int gpz_inflate_size(const uint8_t* in, size_t n, size_t* members, size_t* out_bytes) {
    if ((!in && n) || !out_bytes) return GPZ_E_ARG;
    std::vector<InflateMember> ms;
    std::string why;
    size_t total = 0;
    const int rc = split_members(in, n, &ms, &total, &why);
    if (members) *members = rc == GPZ_OK ? ms.size() : 0;
    *out_bytes = rc == GPZ_OK ? total : 0;
    return rc;
}

float gpz_inflate_device_ms(const gpz_ctx* c) { return c ? c->inf_ms : 0.0f; }

int gpz_inflate(gpz_ctx* c, const uint8_t* in, size_t n, uint8_t* out, size_t out_cap, size_t* out_len) {
    if (!c || (!in && n) || !out_len) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    int rc;
    if ((rc = settle_stale(c))) return rc;
    Slot& sl = c->inf;
    cudaStream_t s = c->kstream;
    if (!sl.done) CU(c, cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    // a page-locked stream starts uploading before the host cuts it into
    // members; a call that ends early waits for that copy first (bounded),
    // since it reads the caller's buffer
    cudaPointerAttributes a{};
    const bool in_locked = n && cudaPointerGetAttributes(&a, in) == cudaSuccess && a.type == cudaMemoryTypeHost;
    cudaGetLastError();
    bool uploading = false;
    auto end_early = [&](int r) {
        if (uploading && cudaEventRecord(sl.done, s) == cudaSuccess &&
            wait_event(c, sl.done, "the upload of a stream that was refused") == GPZ_E_TIMEOUT)
            sl.stale = true;
        return r;
    };
    if (in_locked) {
        if ((rc = ensure_dev(c, sl, sl.d_in, n + 16))) return rc;
        CU(c, cudaMemcpyAsync(sl.d_in.p, in, n, cudaMemcpyHostToDevice, s));
        uploading = true;
    }
    std::vector<InflateMember> ms;
    std::string why;
    size_t total = 0;
    rc = split_members(in, n, &ms, &total, &why);
    *out_len = total;
    if (rc) return end_early(fail(c, rc, why.c_str()));
    if (total > out_cap || (!out && total)) return end_early(fail(c, GPZ_E_SPACE, "output buffer too small"));
    if (ms.empty()) return end_early(GPZ_OK);
    const size_t nm = ms.size();
    // tokens: at most one per output byte, 4 bytes each; d_cnt holds the
    // members' statuses, their token counts and which members the parallel
    // decode took
    if ((rc = ensure_dev(c, sl, sl.d_in, n + 16)) || (rc = ensure_dev(c, sl, sl.d_out, total + 16)) ||
        (rc = ensure_dev(c, sl, sl.d_tok, (total + 16) * 4)) ||
        (rc = ensure_dev(c, sl, sl.d_members, nm * sizeof(InflateMember))) ||
        (rc = ensure_dev(c, sl, sl.d_cnt, nm * 12)))
        return end_early(rc);
    // a tail of b deflate bytes has at most 8 b / kSubBits + 1 sub-spans
    const size_t sub_cap = n * 8 / gpzi::kSubBits + nm + 1;
    if (sub_cap > 0xFFFFFFFFull / gpz_inflate_cands()) return end_early(fail(c, GPZ_E_ARG, "stream too large"));
    if ((rc = ensure_dev(c, sl, sl.d_itail, nm * gpz_inflate_tail_bytes())) ||
        (rc = ensure_dev(c, sl, sl.d_icand, sub_cap * gpz_inflate_cands() * 8)) ||
        (rc = ensure_dev(c, sl, sl.d_isub, sub_cap * 12 + 16)))
        return end_early(rc);
    InflateScratch sc{};
    sc.tails = sl.d_itail.p;
    sc.cands = static_cast<uint64_t*>(sl.d_icand.p);
    sc.sub_start = static_cast<uint32_t*>(sl.d_isub.p);
    sc.sub_tok = sc.sub_start + sub_cap;
    sc.sub_byte = sc.sub_tok + sub_cap;
    sc.counters = sc.sub_byte + sub_cap;
    sc.sub_cap = (uint32_t)sub_cap;
    for (auto& e : c->inf_ev)
        if (!e) CU(c, cudaEventCreate(&e));
    // member statuses come back through page-locked memory, so the wait for
    // them is the bounded event wait below
    if ((rc = ensure_host(c, sl, sl.h_err, sl.h_err_cap, nm, false))) return end_early(rc);
    if (!in_locked) {
        if ((rc = ensure_host(c, sl, sl.h_in, sl.h_in_cap, n, false))) return rc;
        copy_pool().run({CopyPool::Copy{sl.h_in, in, n}}, true);
        CU(c, cudaMemcpyAsync(sl.d_in.p, sl.h_in, n, cudaMemcpyHostToDevice, s));
    }
    CU(c, cudaMemcpyAsync(sl.d_members.p, ms.data(), nm * sizeof(InflateMember), cudaMemcpyHostToDevice, s));
    // a page-locked output buffer receives each member from the expansion
    // kernel as soon as it is done
    const bool out_locked = cudaPointerGetAttributes(&a, out) == cudaSuccess && a.type == cudaMemoryTypeHost;
    cudaGetLastError();
    uint8_t* host_out = out_locked ? mapped_dev(out) : nullptr;
    if (gpz_launch_inflate(static_cast<const uint8_t*>(sl.d_in.p), static_cast<uint8_t*>(sl.d_out.p),
                           static_cast<uint32_t*>(sl.d_tok.p), static_cast<const InflateMember*>(sl.d_members.p),
                           static_cast<uint32_t*>(sl.d_cnt.p), static_cast<uint32_t*>(sl.d_cnt.p) + nm,
                           static_cast<uint32_t*>(sl.d_cnt.p) + 2 * nm, sc, host_out, (uint32_t)nm, s,
                           reinterpret_cast<void* const*>(c->inf_ev)) != 0)
        return fail(c, GPZ_E_CUDA, "inflate launch", cudaGetLastError());
    const uint32_t* status = sl.h_err;
    CU(c, cudaMemcpyAsync(sl.h_err, sl.d_cnt.p, nm * 4, cudaMemcpyDeviceToHost, s));
    if (!host_out) {
        if ((rc = ensure_host(c, sl, sl.h_out, sl.h_out_cap, total, false))) return rc;
        CU(c, cudaMemcpyAsync(sl.h_out, sl.d_out.p, total, cudaMemcpyDeviceToHost, s));
    }
    CU(c, cudaEventRecord(sl.done, s));
    if ((rc = wait_event(c, sl.done, "waiting for the inflate kernels"))) {
        if (rc == GPZ_E_TIMEOUT) sl.stale = true;
        return rc;
    }
    cudaEventElapsedTime(&c->inf_ms, c->inf_ev[0], c->inf_ev[1]);
    for (size_t i = 0; i < nm; i++)
        if (status[i] != gpzi::kOk) {
            why = "member " + std::to_string(i) + " at byte " + std::to_string(ms[i].in_off - 10) + ": " +
                  inflate_reason(status[i]);
            return fail(c, GPZ_E_DATA, why.c_str());
        }
    if (!host_out) copy_pool().run({CopyPool::Copy{out, sl.h_out, total}});
    return GPZ_OK;
}

int gpz_set_wait_ms(gpz_ctx* c, int wait_ms) {
    if (!c || wait_ms < 0) return GPZ_E_ARG;
    c->wait_ms = wait_ms;
    return GPZ_OK;
}

int gpz_frame_host(gpz_ctx* c, uint8_t* host_out, size_t cap) {
    if (!c || !host_out) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    if (c->mout.empty()) return GPZ_E_ARG;
    const MemberOut& l = c->mout.back();
    if (l.gz_off + l.frame_bytes + l.deflate_bytes > cap) return GPZ_E_SPACE;
    frame_members(c->mout.data(), 0, c->mout.size(), host_out, 0);
    return GPZ_OK;
}

int gpz_debug_chunk(gpz_ctx* c, const uint8_t* in, size_t n, uint32_t* pp, uint32_t* tokens, size_t* ntok,
                    uint8_t* out, size_t out_cap, size_t* out_len) {
    if (!c || (!in && n)) return GPZ_E_ARG;
    if (pp && c->codec == GPZ_CODEC_ZSTD) return GPZ_E_ARG;  // the zstd stages reuse pp as block scratch
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    gpz_desc d{in, n, 0};
    std::vector<uint8_t> tmp;
    gpz_out o{out, out_cap, 0, 0};
    if (!out) {
        tmp.resize(gpz_bound_ctx(c, n));
        o.out = tmp.data();
        o.out_cap = tmp.size();
    }
    const int rc = run_host_items(c, &d, 1, &o, true);
    if (out_len) *out_len = o.out_len;
    if (rc) return rc;
    Slot& sl = c->slots[0];
    if (pp && n) CU(c, cudaMemcpy(pp, sl.d_pp.p, n * 4, cudaMemcpyDeviceToHost));
    if (tokens && ntok) {
        std::vector<uint32_t> tok_all(std::max<size_t>(n, 1)), tntok(std::max<size_t>(sl.tiles.size(), 1));
        if (n) CU(c, cudaMemcpy(tok_all.data(), sl.d_tok.p, n * 4, cudaMemcpyDeviceToHost));
        if (!sl.tiles.empty())
            CU(c, cudaMemcpy(tntok.data(), sl.d_tntok.p, sl.tiles.size() * 4, cudaMemcpyDeviceToHost));
        size_t k = 0;
        for (size_t t = 0; t < sl.tiles.size(); t++) {
            const TileDesc& td = sl.tiles[t];
            const MemberDesc& md = sl.members[td.member];
            std::memcpy(tokens + k, tok_all.data() + md.in_off + ((size_t)td.seg << GPZ_SEG_LOG2), tntok[t] * 4);
            k += tntok[t];
        }
        *ntok = k;
    }
    return o.status;
}

int gpz_submit(gpz_ctx* c, const gpz_desc* d, uint64_t* ticket) {
    if (!c || !d || !ticket || (!d->in && d->n)) return GPZ_E_ARG;
    {
        std::lock_guard<std::mutex> lk(c->serve_mu);
        if (!c->serve) {
            auto e = std::make_unique<ServeEngine>();
            const int rc = e->start(c);
            if (rc) return rc;
            c->serve = std::move(e);
        }
    }
    return c->serve->submit(d, ticket, true);
}

int gpz_submit_ref(gpz_ctx* c, const gpz_desc* d, uint64_t* ticket) {
    if (!c || !d || !ticket || (!d->in && d->n)) return GPZ_E_ARG;
    {
        std::lock_guard<std::mutex> lk(c->serve_mu);
        if (!c->serve) {
            auto e = std::make_unique<ServeEngine>();
            const int rc = e->start(c);
            if (rc) return rc;
            c->serve = std::move(e);
        }
    }
    return c->serve->submit(d, ticket, false);
}

int gpz_host_times(gpz_ctx* c, double* ms6, int reset) {
    if (!c || !ms6) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->times_mu);
    for (int i = 0; i < 6; i++) ms6[i] = c->host_ms[i];
    if (reset)
        for (double& x : c->host_ms) x = 0;
    return GPZ_OK;
}

int gpz_poll(gpz_ctx* c, uint64_t ticket, gpz_out* o, int wait_ms) {
    if (!c || !o || !c->serve) return GPZ_E_ARG;
    return c->serve->poll(ticket, o, wait_ms);
}

int gpz_serve_stats_get(gpz_ctx* c, gpz_serve_stats* st) {
    if (!c || !st) return GPZ_E_ARG;
    std::memset(st, 0, sizeof *st);
    if (!c->serve) return GPZ_OK;
    ServeEngine& e = *c->serve;
    std::lock_guard<std::mutex> lk(e.mu);
    st->completed = e.lat_all.size();
    st->rejected = e.rejected;
    st->batches = e.batches;
    st->p50_ms = ServeEngine::pct(e.lat_all, 0.50);
    st->p99_ms = ServeEngine::pct(e.lat_all, 0.99);
    st->p999_ms = ServeEngine::pct(e.lat_all, 0.999);
    st->max_queue_ms = e.max_queue_ms;
    st->bytes_in = e.bytes_in;
    st->bytes_out = e.bytes_out;
    st->completed_small = e.lat_small.size();
    st->p50_small_ms = ServeEngine::pct(e.lat_small, 0.50);
    st->p99_small_ms = ServeEngine::pct(e.lat_small, 0.99);
    st->p999_small_ms = ServeEngine::pct(e.lat_small, 0.999);
    st->queued_bytes = e.queued_bytes;
    return GPZ_OK;
}

int gpz_serve_lane_stats(gpz_ctx* c, int lane, gpz_lane_stats* st) {
    if (!c || !st || lane < 0 || lane > 1) return GPZ_E_ARG;
    std::memset(st, 0, sizeof *st);
    if (!c->serve) return GPZ_OK;
    std::lock_guard<std::mutex> lk(c->serve->mu);
    *st = c->serve->lanes[lane].st;
    return GPZ_OK;
}

int gpz_serve_reset_stats(gpz_ctx* c) {
    if (!c) return GPZ_E_ARG;
    if (!c->serve) return GPZ_OK;
    std::lock_guard<std::mutex> lk(c->serve->mu);
    for (auto& L : c->serve->lanes) L.st = gpz_lane_stats{};
    c->serve->lat_all.clear();
    c->serve->lat_small.clear();
    c->serve->rejected = c->serve->batches = c->serve->bytes_in = c->serve->bytes_out = 0;
    c->serve->max_queue_ms = 0;
    return GPZ_OK;
}

const char* gpz_strerror(int s) {
    switch (s) {
        case GPZ_OK: return "ok";
        case GPZ_E_NOMEM: return "out of device or pinned memory";
        case GPZ_E_ADMISSION: return "request exceeds the device pool cap";
        case GPZ_E_TIMEOUT: return "the device did not finish within the context's wait limit";
        case GPZ_E_CUDA: return "CUDA runtime error";
        case GPZ_E_ARG: return "invalid argument";
        case GPZ_E_SPACE: return "output buffer too small";
        case GPZ_E_INTERNAL: return "device self-check failed";
        case GPZ_E_BUSY: return "too many requests outstanding; poll some first";
        case GPZ_E_PENDING: return "result not ready";
        case GPZ_E_DATA: return "gzip data this path cannot split or decode";
        case GPZ_E_SINK: return "the writer's sink or chunk function failed";
        default: return "unknown status";
    }
}

const char* gpz_last_error(gpz_ctx* c) { return c ? c->last_err.c_str() : "no context"; }

int gpz_get_shape(gpz_ctx* c, gpz_shape* s) {
    if (!c || !s) return GPZ_E_ARG;
    const LaunchShape x = shape_for(c, bucket_of(64 * 1024));
    s->lookup_threads = x.lookup_threads;
    s->lookup_grid = x.lookup_grid;
    s->walk_threads = x.walk_threads;
    s->walk_grid = x.walk_grid;
    s->emit_threads = x.emit_threads;
    s->emit_grid = x.emit_grid;
    return GPZ_OK;
}

int gpz_set_shape(gpz_ctx* c, const gpz_shape* s) {
    if (!c || !s) return GPZ_E_ARG;
    auto ok_t = [](int t) { return t == 256 || t == 512; };
    if (!(s->lookup_threads == 512 || s->lookup_threads == 768 || s->lookup_threads == 1024) ||
        !(s->walk_threads == 256 || s->walk_threads == 512 || s->walk_threads == 1024) || !ok_t(s->emit_threads) || s->lookup_grid < 0 || s->walk_grid < 0 || s->emit_grid < 0)
        return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    c->fixed = LaunchShape{s->lookup_threads, s->lookup_grid, s->walk_threads, s->walk_grid, s->emit_threads,
                           s->emit_grid, 0, 0};
    for (auto& sl : c->slots) sl.gen++;
    return GPZ_OK;
}

uint64_t gpz_last_launches(gpz_ctx* c) { return c ? c->launches.load() : 0; }

int gpz_stage_times(gpz_ctx* c, float* ms) {
    if (!c || !ms || !(c->flags & GPZ_FLAG_STAGE_TIMING)) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    for (int i = 0; i < GPZ_STAGES; i++) ms[i] = c->stage_ms[i];
    return GPZ_OK;
}

}  // extern "C"
