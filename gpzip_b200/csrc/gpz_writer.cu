// gpz_writer.cu -- the streaming chunked writer of include/gpz.h: the
// caller of ChunkFn in the reference, ParallelChunkedWriter
// (crates/gpzip-codec-cpu/src/parallel.rs:28-229).
//
// Written bytes are cut into chunk_size chunks.  Full chunks collect into
// a batch of up to max_in_flight chunks; a full batch goes to the writer's
// thread, which compresses it (one gpz_compress_batch call, or the caller's
// chunk function per chunk) and hands the members to the sink in input
// order, while the caller fills the next batch.  At most one batch waits
// behind the one being compressed, so memory stays bounded.  The first
// error is sticky (parallel.rs:70-89): every later call returns it.
#include <algorithm>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <utility>
#include <vector>

#include "gpz.h"

using Chunk = std::vector<uint8_t>;
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
// writer's first batch 50-260 ms instead of 4 ms.
constexpr size_t kPoolOuts = 4;
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
    Batch filling;  // full chunks of the open batch (caller's thread only)
    bool finished = false;

    std::mutex mu;
    std::condition_variable cv;
    std::deque<Batch> queue;  // batches handed over, not yet taken
    bool busy = false;        // the thread is compressing a batch
    bool stop = false;
    int sticky = GPZ_OK;
    std::thread worker;
    std::unique_ptr<uint8_t[]> out;  // the thread's output buffer, from and back to the pool
    size_t out_cap = 0;
    std::vector<Chunk> spare;  // chunk buffers of finished batches, reused (no page faults)

    int compress(Batch& b) {
        size_t cap = 0;
        for (const Chunk& ch : b) cap += ctx ? gpz_bound_ctx(ctx, ch.size()) : gpz_bound(ch.size());
        if (out_cap < cap) {
            out_give(out, out_cap);
            auto o = out_take(cap);
            out = std::move(o.first);
            out_cap = out ? o.second : 0;
            if (!out) return GPZ_E_NOMEM;
        }
        std::vector<gpz_out> outs(b.size());
        size_t off = 0;
        for (size_t i = 0; i < b.size(); i++) {
            const size_t c = ctx ? gpz_bound_ctx(ctx, b[i].size()) : gpz_bound(b[i].size());
            outs[i] = gpz_out{out.get() + off, c, 0, 0};
            off += c;
        }
        if (ctx) {
            std::vector<gpz_desc> ds(b.size());
            for (size_t i = 0; i < b.size(); i++) ds[i] = gpz_desc{b[i].data(), b[i].size(), 5};
            const int rc = gpz_compress_batch(ctx, ds.data(), ds.size(), outs.data());
            if (rc != GPZ_OK) return rc;
        } else {
            for (size_t i = 0; i < b.size(); i++) {
                size_t n = 0;
                if (fn(fn_user, b[i].data(), b[i].size(), outs[i].out, outs[i].out_cap, &n) != 0 || n > outs[i].out_cap)
                    return GPZ_E_SINK;
                outs[i].out_len = n;
            }
        }
        for (size_t i = 0; i < b.size(); i++)
            if (sink(sink_user, outs[i].out, outs[i].out_len) != 0) return GPZ_E_SINK;
        return GPZ_OK;
    }

    void run() {
        for (;;) {
            Batch b;
            int failed;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (queue.empty()) return;
                b = std::move(queue.front());
                queue.pop_front();
                busy = true;
                failed = sticky;
                cv.notify_all();
            }
            // after an error the remaining batches are dropped, not written
            const int rc = failed != GPZ_OK ? failed : compress(b);
            std::lock_guard<std::mutex> lk(mu);
            if (rc != GPZ_OK && sticky == GPZ_OK) sticky = rc;
            for (Chunk& ch : b)
                if (spare.size() < 2 * max_in_flight && ch.capacity() == chunk_size) {
                    ch.clear();
                    spare.push_back(std::move(ch));
                }
            busy = false;
            cv.notify_all();
        }
    }

    // hands the open batch to the thread once fewer than one batch waits
    void submit() {
        if (filling.empty()) return;
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return queue.empty(); });
        queue.push_back(std::move(filling));
        filling = Batch{};
        cv.notify_all();
    }

    int status() {
        std::lock_guard<std::mutex> lk(mu);
        return sticky;
    }

    // an empty chunk buffer of chunk_size capacity, from a finished batch if
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
    if ((!ctx && !fn) || !sink || chunk_size == 0 || max_in_flight == 0) return GPZ_E_ARG;
    auto* w = new (std::nothrow) gpz_writer();
    if (!w) return GPZ_E_NOMEM;
    w->ctx = ctx;
    w->fn = fn;
    w->fn_user = fn_user;
    w->sink = sink;
    w->sink_user = sink_user;
    w->chunk_size = chunk_size;
    w->max_in_flight = max_in_flight;
    w->worker = std::thread([w] { w->run(); });
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
    while (n) {
        if (w->current.capacity() < w->chunk_size) w->fresh_chunk();
        const size_t take = std::min(n, w->chunk_size - w->current.size());
        w->current.insert(w->current.end(), buf, buf + take);
        buf += take;
        n -= take;
        if (w->current.size() == w->chunk_size) {
            w->filling.push_back(std::move(w->current));
            w->current = Chunk{};  // capacity 0: the next byte takes a fresh buffer
            if (w->filling.size() >= w->max_in_flight) w->submit();
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
        if (!w->current.empty()) w->filling.push_back(std::move(w->current));
        w->current = Chunk{};
        w->submit();
        std::unique_lock<std::mutex> lk(w->mu);
        w->cv.wait(lk, [&] { return w->queue.empty() && !w->busy; });
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
    w->worker.join();
    pool_give(w->spare);
    out_give(w->out, w->out_cap);
    delete w;
}
