// gpz_writer.cu -- the callers of the compression path in the reference,
// rebuilt behind the C ABI of include/gpz.h:
//
//  * the streaming chunked writer (gpz_writer_*): ParallelChunkedWriter
//    (crates/gpzip-codec-cpu/src/parallel.rs:28-229);
//  * the hybrid CPU + GPU chunk function (gpz_hybrid_*): the permit
//    scheduler of `--backend auto` (crates/gpzip-cli/src/hybrid.rs:103-147);
//  * the CPU gzip chunk function the hybrid falls through to
//    (GzipCompressor::chunk_fn, crates/gpzip-codec-cpu/src/compress.rs:52-59),
//    here zlib with the same level and framing.
//
// Writer.  Written bytes are cut into chunk_size chunks; the first error is
// sticky (parallel.rs:70-89): every later call returns it, and nothing after
// the failed chunk reaches the sink.
//  - With a device context, chunks live in page-locked buffers (pooled), so
//    the device reads them without a staging copy, and large writes are
//    copied in by the host copy threads.  Every full chunk joins a queue
//    that the writer's thread feeds to the context's pass loop
//    (gpz_stream_run): passes of whatever is ready, overlapped on the
//    device across the whole stream, the members going to the sink in
//    input order straight from the pass's output.  At most
//    max(max_in_flight, 128 MiB / chunk_size) chunks are queued, on the
//    device or waiting for the sink; the caller waits beyond that.
//  - With a chunk function, every full chunk is handed to a pool of
//    max_in_flight worker threads at once, as the reference spawns one rayon
//    task per chunk (parallel.rs:91-129); up to max_in_flight chunks are
//    compressed or waiting for their turn at the sink.  The worker that
//    finishes the oldest chunk writes it and every finished chunk behind it,
//    in input order, one sink call at a time.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <utility>
#include <vector>

#include "gpz.h"
#include "gpz_stream.h"

// An allocator whose resize leaves new bytes uninitialised: a chunk is
// filled by copies right after it grows, so zeroing it first is wasted.
template <class T>
struct UninitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <class U>
    UninitAlloc(const UninitAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
using Chunk = std::vector<uint8_t, UninitAlloc<uint8_t>>;
using Batch = std::vector<Chunk>;

namespace {

// Chunk buffers outlive their writer here, so that a new writer does not
// page-fault its way through fresh memory (a 64 MiB stream would otherwise
// take 16 K page faults).  Bounded: at most kPoolChunks buffers are kept.
constexpr size_t kPoolChunks = 64;
std::mutex g_pool_mu;
std::vector<Chunk> g_pool;

bool pool_take(size_t chunk_size, Chunk& into) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (size_t i = g_pool.size(); i-- > 0;)
        if (g_pool[i].capacity() == chunk_size) {
            into = std::move(g_pool[i]);
            g_pool.erase(g_pool.begin() + (std::ptrdiff_t)i);
            return true;
        }
    return false;
}

// Output buffers, kept across writers for the same reason: the first
// touch of a fresh 64 MiB buffer (page faults, huge-page compaction) cost a
// writer's first batch 50-260 ms instead of 4 ms.  Chunk-function writers
// keep one per chunk in flight.
constexpr size_t kPoolOuts = 40;
std::vector<std::pair<std::unique_ptr<uint8_t[]>, size_t>> g_outs;

std::pair<std::unique_ptr<uint8_t[]>, size_t> out_take(size_t cap) {
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        for (size_t i = 0; i < g_outs.size(); i++)
            if (g_outs[i].second >= cap) {
                auto o = std::move(g_outs[i]);
                g_outs.erase(g_outs.begin() + (std::ptrdiff_t)i);
                return o;
            }
    }
    return {std::unique_ptr<uint8_t[]>(new (std::nothrow) uint8_t[cap]), cap};
}

void out_give(std::unique_ptr<uint8_t[]>& p, size_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (g_outs.size() < kPoolOuts) g_outs.emplace_back(std::move(p), cap);
    p.reset();
}

// Page-locked chunk buffers, kept across writers: cudaHostAlloc takes about
// a millisecond per 2 MiB buffer.  Bounded at kPoolPinned buffers.
constexpr size_t kPoolPinned = 160;
std::vector<std::pair<uint8_t*, size_t>> g_pinned;

uint8_t* pinned_take(size_t n) {
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        for (size_t i = g_pinned.size(); i-- > 0;)
            if (g_pinned[i].second == n) {
                uint8_t* p = g_pinned[i].first;
                g_pinned.erase(g_pinned.begin() + (std::ptrdiff_t)i);
                return p;
            }
    }
    return gpz_pinned_alloc(n);
}

void pinned_give(uint8_t* p, size_t n) {
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (g_pinned.size() < kPoolPinned) {
            g_pinned.emplace_back(p, n);
            return;
        }
    }
    gpz_pinned_free(p);
}

void pool_give(std::vector<Chunk>& chunks) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (Chunk& ch : chunks)
        if (g_pool.size() < kPoolChunks && ch.capacity()) {
            ch.clear();
            g_pool.push_back(std::move(ch));
        }
    chunks.clear();
}

}  // namespace

struct gpz_writer {
    gpz_ctx* ctx = nullptr;
    gpz_chunk_fn fn = nullptr;
    void* fn_user = nullptr;
    gpz_sink_fn sink = nullptr;
    void* sink_user = nullptr;
    size_t chunk_size = 0, max_in_flight = 0;
    Chunk current;  // the chunk being filled (caller's thread only)
    bool finished = false;

    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    int sticky = GPZ_OK;
    std::vector<Chunk> spare;  // chunk buffers of finished chunks, reused (no page faults)

    // ---- device mode: page-locked chunks fed to the context's pass loop
    struct PChunk {
        uint8_t* p = nullptr;
        size_t n = 0;
    };
    PChunk pcur;                 // the chunk being filled (caller's thread only)
    std::deque<PChunk> ready;    // full chunks not yet taken by the pass loop
    std::deque<PChunk> taken;    // taken, not yet delivered (in input order)
    std::vector<uint8_t*> pfree; // this writer's spare chunk buffers
    size_t outstanding = 0;      // ready + taken
    size_t max_outstanding = 0;
    bool ending = false;         // finish: the partial chunk is queued, nothing more comes
    bool running = false;        // the streamer is inside a pass loop
    std::thread streamer;

    struct Feed : GpzStreamFeed {
        gpz_writer* w;
        explicit Feed(gpz_writer* wr) : w(wr) {}
        bool take(std::vector<gpz_desc>& out, size_t max_bytes, size_t min_bytes, bool) override {
            std::lock_guard<std::mutex> lk(w->mu);
            size_t have = 0;
            for (const PChunk& c : w->ready) have += c.n;
            if (w->ready.empty() || (have < min_bytes && !w->ending)) return !(w->ending && w->ready.empty());
            size_t bytes = 0;
            while (!w->ready.empty() && (out.empty() || bytes + w->ready.front().n <= max_bytes)) {
                PChunk c = w->ready.front();
                w->ready.pop_front();
                bytes += c.n;
                out.push_back(gpz_desc{c.p, c.n, 5});
                w->taken.push_back(c);
            }
            return true;
        }
        int deliver(const uint8_t* data, size_t n) override {
            const int rc = w->sink(w->sink_user, data, n);
            std::lock_guard<std::mutex> lk(w->mu);
            PChunk c = w->taken.front();
            w->taken.pop_front();
            w->pfree.push_back(c.p);
            w->outstanding--;
            w->cv.notify_all();
            return rc;
        }
    };

    // ---- chunk-function mode: one job per chunk, workers in a pool
    struct Job {
        Chunk in;
        std::unique_ptr<uint8_t[]> out;
        size_t out_cap = 0, out_len = 0;
        int rc = GPZ_OK;
        bool done = false;
    };
    std::deque<std::unique_ptr<Job>> jobs;  // input order; the front is the next for the sink
    size_t started = 0;                     // jobs[0 .. started) have been taken by a worker
    bool sinking = false;                   // a worker is writing finished jobs to the sink
    bool broken = false;                    // a job failed or the sink did: nothing more is written
    std::vector<std::thread> pool;

    void recycle(Chunk& ch) {
        if (spare.size() < 2 * max_in_flight && ch.capacity() == chunk_size) {
            ch.clear();
            spare.push_back(std::move(ch));
        }
    }

    // The device mode's thread: whenever chunks are ready, runs the pass
    // loop until nothing is ready and nothing is on the device.  After an
    // error, queued chunks are dropped, not written.
    void run_stream() {
        Feed feed(this);
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !ready.empty(); });
                if (ready.empty()) return;
                if (sticky != GPZ_OK) {
                    drop_queued();
                    continue;
                }
                running = true;
            }
            const int rc = gpz_stream_run(ctx, feed);
            std::lock_guard<std::mutex> lk(mu);
            running = false;
            if (rc != GPZ_OK && sticky == GPZ_OK) sticky = rc;
            if (sticky != GPZ_OK) drop_queued();
            cv.notify_all();
        }
    }

    // (mu held) returns every queued or undelivered chunk buffer
    void drop_queued() {
        for (auto* q : {&ready, &taken}) {
            for (PChunk& c : *q) {
                pfree.push_back(c.p);
                outstanding--;
            }
            q->clear();
        }
        cv.notify_all();
    }

    // One worker of the chunk-function pool: takes the oldest job nobody
    // has started, compresses it, then writes every finished job at the
    // front of the queue unless another worker is already doing so.
    void run_jobs() {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv.wait(lk, [&] { return stop || started < jobs.size(); });
            if (started >= jobs.size()) return;
            Job* j = jobs[started++].get();
            const int failed = sticky;
            lk.unlock();
            int rc = failed;
            if (rc == GPZ_OK) {
                const size_t cap = gpz_bound(j->in.size());
                if (j->out_cap < cap) {
                    auto o = out_take(cap);
                    j->out = std::move(o.first);
                    j->out_cap = j->out ? o.second : 0;
                }
                size_t n = 0;
                if (!j->out) rc = GPZ_E_NOMEM;
                else if (fn(fn_user, j->in.data(), j->in.size(), j->out.get(), cap, &n) != 0 || n > cap) rc = GPZ_E_SINK;
                j->out_len = n;
            }
            lk.lock();
            j->rc = rc;
            j->done = true;
            if (rc != GPZ_OK && sticky == GPZ_OK) sticky = rc;
            if (!sinking) {
                sinking = true;
                while (!jobs.empty() && jobs.front()->done) {
                    std::unique_ptr<Job> f = std::move(jobs.front());
                    jobs.pop_front();
                    started--;
                    // the stream ends before the first failed job (in
                    // input order): the jobs ahead of it are written, it
                    // and everything after it are dropped (parallel.rs:
                    // 144-150 writes results in order up to the gap)
                    if (f->rc != GPZ_OK) broken = true;
                    const bool write = !broken;
                    lk.unlock();
                    int src = GPZ_OK;
                    if (write && sink(sink_user, f->out.get(), f->out_len) != 0) src = GPZ_E_SINK;
                    out_give(f->out, f->out_cap);
                    lk.lock();
                    if (src != GPZ_OK) {
                        broken = true;
                        if (sticky == GPZ_OK) sticky = src;
                    }
                    recycle(f->in);
                }
                sinking = false;
            }
            cv.notify_all();
        }
    }

    // device mode: queues the full (or last) chunk for the streamer once
    // fewer than max_outstanding are queued
    void dispatch_pinned() {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return outstanding < max_outstanding || sticky != GPZ_OK; });
        if (sticky != GPZ_OK) {
            pfree.push_back(pcur.p);
        } else {
            ready.push_back(pcur);
            outstanding++;
        }
        pcur = PChunk{};
        cv.notify_all();
    }

    // a page-locked chunk buffer, from this writer's spares or the pool
    bool fresh_pinned() {
        {
            std::lock_guard<std::mutex> lk(mu);
            if (!pfree.empty()) {
                pcur.p = pfree.back();
                pfree.pop_back();
                pcur.n = 0;
                return true;
            }
        }
        pcur.p = pinned_take(chunk_size);
        pcur.n = 0;
        return pcur.p != nullptr;
    }

    // chunk-function mode: queues a full chunk for the pool once fewer than
    // max_in_flight are outstanding
    void dispatch(Chunk&& ch) {
        auto j = std::unique_ptr<Job>(new (std::nothrow) Job());
        std::unique_lock<std::mutex> lk(mu);
        if (!j) {
            if (sticky == GPZ_OK) sticky = GPZ_E_NOMEM;
            return;
        }
        cv.wait(lk, [&] { return jobs.size() < max_in_flight; });
        j->in = std::move(ch);
        jobs.push_back(std::move(j));
        cv.notify_all();
    }

    // waits until every chunk handed over has been written or dropped
    void drain() {
        std::unique_lock<std::mutex> lk(mu);
        ending = true;
        cv.notify_all();
        cv.wait(lk, [&] { return jobs.empty() && outstanding == 0 && !running; });
    }

    int status() {
        std::lock_guard<std::mutex> lk(mu);
        return sticky;
    }

    // an empty chunk buffer of chunk_size capacity, from a finished chunk if
    // one is free
    void fresh_chunk() {
        {
            std::lock_guard<std::mutex> lk(mu);
            if (!spare.empty()) {
                current = std::move(spare.back());
                spare.pop_back();
                return;
            }
        }
        if (pool_take(chunk_size, current)) return;
        current = Chunk{};
        current.reserve(chunk_size);
    }
};

namespace {

int open_writer(gpz_ctx* ctx, gpz_chunk_fn fn, void* fn_user, size_t chunk_size, size_t max_in_flight,
                gpz_sink_fn sink, void* sink_user, gpz_writer** out) {
    if (!out) return GPZ_E_ARG;
    *out = nullptr;
    if ((!ctx && !fn) || !sink || chunk_size == 0 || max_in_flight == 0 || max_in_flight > 1024) return GPZ_E_ARG;
    auto* w = new (std::nothrow) gpz_writer();
    if (!w) return GPZ_E_NOMEM;
    w->ctx = ctx;
    w->fn = fn;
    w->fn_user = fn_user;
    w->sink = sink;
    w->sink_user = sink_user;
    w->chunk_size = chunk_size;
    w->max_in_flight = max_in_flight;
    w->max_outstanding = std::max(max_in_flight, (size_t)(128u << 20) / chunk_size + 1);
    try {
        if (ctx) {
            w->streamer = std::thread([w] { w->run_stream(); });
        } else {
            for (size_t i = 0; i < max_in_flight; i++) w->pool.emplace_back([w] { w->run_jobs(); });
        }
    } catch (...) {
        {
            std::lock_guard<std::mutex> lk(w->mu);
            w->stop = true;
        }
        w->cv.notify_all();
        for (auto& t : w->pool) t.join();
        delete w;
        return GPZ_E_NOMEM;
    }
    *out = w;
    return GPZ_OK;
}

}  // namespace

int gpz_writer_open(gpz_ctx* ctx, size_t chunk_size, size_t max_in_flight, gpz_sink_fn sink, void* sink_user,
                    gpz_writer** out) {
    if (!ctx) {
        if (out) *out = nullptr;
        return GPZ_E_ARG;
    }
    return open_writer(ctx, nullptr, nullptr, chunk_size, max_in_flight, sink, sink_user, out);
}

int gpz_writer_open_fn(gpz_chunk_fn fn, void* fn_user, size_t chunk_size, size_t max_in_flight, gpz_sink_fn sink,
                       void* sink_user, gpz_writer** out) {
    if (!fn) {
        if (out) *out = nullptr;
        return GPZ_E_ARG;
    }
    return open_writer(nullptr, fn, fn_user, chunk_size, max_in_flight, sink, sink_user, out);
}

int gpz_writer_write(gpz_writer* w, const uint8_t* buf, size_t n) {
    if (!w || (!buf && n) || w->finished) return GPZ_E_ARG;
    int rc = w->status();
    if (rc != GPZ_OK) return rc;
    if (w->ctx) {
        while (n) {
            if (!w->pcur.p && !w->fresh_pinned()) {
                std::lock_guard<std::mutex> lk(w->mu);
                if (w->sticky == GPZ_OK) w->sticky = GPZ_E_NOMEM;
                return w->sticky;
            }
            const size_t take = std::min(n, w->chunk_size - w->pcur.n);
            if (take >= (256u << 10)) gpz_parallel_copy(w->pcur.p + w->pcur.n, buf, take);
            else std::memcpy(w->pcur.p + w->pcur.n, buf, take);
            w->pcur.n += take;
            buf += take;
            n -= take;
            if (w->pcur.n == w->chunk_size) w->dispatch_pinned();
        }
        return w->status();
    }
    while (n) {
        if (w->current.capacity() < w->chunk_size) w->fresh_chunk();
        const size_t take = std::min(n, w->chunk_size - w->current.size());
        const size_t at = w->current.size();
        w->current.resize(at + take);  // within its capacity: no reallocation
        std::memcpy(w->current.data() + at, buf, take);
        buf += take;
        n -= take;
        if (w->current.size() == w->chunk_size) {
            w->dispatch(std::move(w->current));
            w->current = Chunk{};  // capacity 0: the next byte takes a fresh buffer
        }
    }
    return w->status();
}

int gpz_writer_flush(gpz_writer* w) {
    if (!w) return GPZ_E_ARG;
    return w->status();
}

int gpz_writer_finish(gpz_writer* w) {
    if (!w) return GPZ_E_ARG;
    if (!w->finished) {
        w->finished = true;
        if (w->ctx) {
            if (w->pcur.p && w->pcur.n) w->dispatch_pinned();
        } else {
            if (!w->current.empty()) w->dispatch(std::move(w->current));
            w->current = Chunk{};
        }
        w->drain();
    }
    return w->status();
}

void gpz_writer_close(gpz_writer* w) {
    if (!w) return;
    gpz_writer_finish(w);
    {
        std::lock_guard<std::mutex> lk(w->mu);
        w->stop = true;
    }
    w->cv.notify_all();
    if (w->streamer.joinable()) w->streamer.join();
    for (auto& t : w->pool) t.join();
    pool_give(w->spare);
    if (w->pcur.p) w->pfree.push_back(w->pcur.p);
    for (uint8_t* p : w->pfree) pinned_give(p, w->chunk_size);
    delete w;
}

// ================================================================ hybrid

// The CPU chunk function: one gzip member of the whole chunk at a zlib
// level, as GzipCompressor::chunk_fn writes with flate2's GzEncoder
// (compress.rs:52-59: header with no name or time, the DEFLATE stream, the
// CRC-32 / ISIZE trailer).  zlib writes OS = 3 (Unix) where flate2 writes
// 255 (unknown); a gzip reader ignores the byte.
int gpz_cpu_gzip_chunk(void* level, const uint8_t* in, size_t n, uint8_t* out, size_t out_cap, size_t* out_len) {
    if ((!in && n) || !out || !out_len) return GPZ_E_ARG;
    const int lvl = level ? *static_cast<const int*>(level) : 5;
    if (lvl < 0 || lvl > 9) return GPZ_E_ARG;
    z_stream z{};
    if (deflateInit2(&z, lvl, Z_DEFLATED, 15 + 16, 8, Z_DEFAULT_STRATEGY) != Z_OK) return GPZ_E_NOMEM;
    z.next_out = out;
    z.avail_out = (uInt)std::min<size_t>(out_cap, 0xFFFFFFFFu);
    static const uint8_t kEmpty = 0;
    z.next_in = const_cast<Bytef*>(n ? in : &kEmpty);
    int zr = Z_OK;
    size_t left = n;
    while (zr == Z_OK) {
        const uInt take = (uInt)std::min<size_t>(left, 1u << 30);
        z.avail_in = take;
        left -= take;
        zr = deflate(&z, left ? Z_NO_FLUSH : Z_FINISH);
        if (zr == Z_OK && z.avail_out == 0) break;  // out of space
    }
    *out_len = out_cap - z.avail_out;
    deflateEnd(&z);
    return zr == Z_STREAM_END ? GPZ_OK : GPZ_E_SPACE;
}

struct gpz_hybrid {
    gpz_hybrid_config cfg{};
    int level = 5;
    std::atomic<size_t> permits{0};
    std::atomic<uint64_t> counter{0}, cpu_chunks{0}, gpu_chunks{0};
    // the device context: the caller's, or one made on the first chunk
    // that may use the GPU (so a small input never pays for it); a context
    // that cannot be made leaves every chunk to the CPU
    std::once_flag once;
    gpz_ctx* ctx = nullptr;
    bool own_ctx = false;

    gpz_ctx* gpu() {
        std::call_once(once, [this] {
            if (cfg.ctx) {
                ctx = cfg.ctx;
                return;
            }
            gpz_config c;
            gpz_config_default(&c);
            c.device = cfg.device;
            if (gpz_create(&c, &ctx) == GPZ_OK) own_ctx = true;
            else ctx = nullptr;
        });
        return ctx;
    }

    // decrement-if-positive (hybrid.rs:150-163)
    bool try_acquire() {
        size_t cur = permits.load(std::memory_order_acquire);
        while (cur) {
            if (permits.compare_exchange_weak(cur, cur - 1, std::memory_order_acq_rel, std::memory_order_acquire))
                return true;
        }
        return false;
    }
};

void gpz_hybrid_config_default(gpz_hybrid_config* cfg) {
    if (!cfg) return;
    *cfg = gpz_hybrid_config{};
    cfg->ctx = nullptr;
    cfg->device = 0;
    cfg->level = 5;
    cfg->gpu_permits = 1;
    cfg->warmup_chunks = 4;
    cfg->cpu_fn = nullptr;
    cfg->cpu_user = nullptr;
    cfg->gpu_fn = nullptr;
    cfg->gpu_user = nullptr;
}

int gpz_hybrid_create(const gpz_hybrid_config* cfg, gpz_hybrid** out) {
    if (!out) return GPZ_E_ARG;
    *out = nullptr;
    gpz_hybrid_config def;
    gpz_hybrid_config_default(&def);
    if (!cfg) cfg = &def;
    if (cfg->level < 0 || cfg->level > 9 || cfg->gpu_permits > 4096) return GPZ_E_ARG;
    auto* h = new (std::nothrow) gpz_hybrid();
    if (!h) return GPZ_E_NOMEM;
    h->cfg = *cfg;
    h->level = cfg->level;
    h->permits = cfg->gpu_permits;
    *out = h;
    return GPZ_OK;
}

int gpz_hybrid_chunk(void* hp, const uint8_t* in, size_t n, uint8_t* out, size_t out_cap, size_t* out_len) {
    auto* h = static_cast<gpz_hybrid*>(hp);
    if (!h || (!in && n) || !out || !out_len) return GPZ_E_ARG;
    // the composed ChunkFn of hybrid.rs:123-138: the first warmup_chunks
    // chunks, and every chunk while no GPU permit is free, go to the CPU
    const uint64_t k = h->counter.fetch_add(1, std::memory_order_relaxed);
    if (h->cfg.gpu_permits > 0 && k >= h->cfg.warmup_chunks) {
        gpz_ctx* g = h->cfg.gpu_fn ? nullptr : h->gpu();
        if ((g || h->cfg.gpu_fn) && h->try_acquire()) {
            const int rc = h->cfg.gpu_fn ? h->cfg.gpu_fn(h->cfg.gpu_user, in, n, out, out_cap, out_len)
                                         : gpz_compress_chunk(g, in, n, h->level, out, out_cap, out_len);
            h->permits.fetch_add(1, std::memory_order_release);
            h->gpu_chunks.fetch_add(1, std::memory_order_relaxed);
            return rc;
        }
    }
    h->cpu_chunks.fetch_add(1, std::memory_order_relaxed);
    if (h->cfg.cpu_fn) return h->cfg.cpu_fn(h->cfg.cpu_user, in, n, out, out_cap, out_len);
    return gpz_cpu_gzip_chunk(&h->level, in, n, out, out_cap, out_len);
}

int gpz_hybrid_stats(const gpz_hybrid* h, uint64_t* cpu_chunks, uint64_t* gpu_chunks) {
    if (!h) return GPZ_E_ARG;
    if (cpu_chunks) *cpu_chunks = h->cpu_chunks.load();
    if (gpu_chunks) *gpu_chunks = h->gpu_chunks.load();
    return GPZ_OK;
}

void gpz_hybrid_destroy(gpz_hybrid* h) {
    if (!h) return;
    if (h->own_ctx) gpz_destroy(h->ctx);
    delete h;
}
