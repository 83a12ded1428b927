// gpz_stream.h -- the streaming pass loop that the device writer runs
// (gpz_runtime.cu), and the host helpers it shares with the writer.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/gpz.h"

// What a stream of chunks looks like to the pass loop.  take() appends the
// chunks that are ready (their bytes stay valid and unchanged until they
// are delivered): at most max_bytes of them (at least one chunk, however
// large), and only when at least min_bytes are ready or the stream has
// ended; with `block` set it waits until that holds.  It returns false once
// the stream has ended and every chunk has been taken.  With min_bytes 0
// any queued chunk is ready, an empty one included.  deliver() gets each
// taken chunk's compressed stream, in take order, from memory that stays
// valid until pass_done() returns (after the deliveries of that pass); a
// nonzero return stops the stream.
struct GpzStreamFeed {
    virtual bool take(std::vector<gpz_desc>& out, size_t max_bytes, size_t min_bytes, bool block) = 0;
    virtual int deliver(const uint8_t* data, size_t n) = 0;
    // after the deliveries of one pass, before its memory is reused
    virtual void pass_done() {}
    virtual ~GpzStreamFeed() {}
};

// Runs the chunks of `feed` through the context's pipeline slots until the
// feed ends or nothing is ready and nothing is in flight (then it returns
// GPZ_OK and the caller may call again when more chunks are ready).  Passes
// grow from 1/16 of the pass size to the whole of it, every pass holds
// whatever is ready up to that size, and a pass is started while others are
// on the device only when at least 8 MiB (or the rest of the stream) is
// ready; with nothing on the device, any ready chunk starts one.  Holds the context for as long as it runs.  The first failure is
// returned; chunks after it are not delivered.
int gpz_stream_run(gpz_ctx* ctx, GpzStreamFeed& feed);

// Page-locked host buffers (cudaHostAlloc) for chunks the device reads
// directly; nullptr when the allocation fails.
uint8_t* gpz_pinned_alloc(size_t n);
void gpz_pinned_free(uint8_t* p);

// memcpy on the host copy threads, with non-temporal stores (for buffers
// the copy engine reads next).
void gpz_parallel_copy(void* dst, const void* src, size_t n);
