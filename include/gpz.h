/*
 * gpz.h -- C ABI of the B200 (sm_100a) gzip compression path.
 *
 * Drop-in boundary for the reference's chunk-codec interface
 * (skmtkytr/gpzip):
 *   - ChunkFn = Arc<dyn Fn(&[u8]) -> io::Result<Vec<u8>>>
 *       crates/gpzip-codec-cpu/src/parallel.rs:21
 *   - GpuBackend::gzip_chunk_fn / encode_one
 *       crates/gpzip-codec-gpu/src/gpu.rs:193-208, 271-287
 *   - BatchedLz77::submit (the batching channel this replaces)
 *       crates/gpzip-codec-gpu/src/gpu/batch.rs:74-85
 * Plain pointers and sizes only; no CUDA or torch types cross the boundary.
 *
 * Output of every compress call is a concatenation of RFC 1952 gzip members,
 * one per `member_bytes` slice of the input (131072 by default, matching
 * GpuBackend's chunk_size at gpu.rs:160), each carrying one dynamic-Huffman
 * RFC 1951 block whose bytes equal the reference's encode_block_fast output
 * for the reference's segmented-hash + lazy-walk tokens.
 *
 * Errors are status codes, never aborts.  All entry points are thread safe.
 * There is no CPU fallback: without a usable CUDA device gpz_create fails.
 */
#ifndef GPZ_H
#define GPZ_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GPZ_API __attribute__((visibility("default")))
#else
#define GPZ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define GPZ_OK 0
#define GPZ_E_NOMEM 1       /* device or pinned allocation failed */
#define GPZ_E_ADMISSION 2   /* request does not fit the device pool cap (now, or at all) */
#define GPZ_E_TIMEOUT 3     /* the device did not finish within the context's wait limit */
#define GPZ_E_CUDA 4        /* CUDA runtime error */
#define GPZ_E_ARG 5         /* invalid argument */
#define GPZ_E_SPACE 6       /* output buffer too small */
#define GPZ_E_INTERNAL 7    /* device self-check failed (bit plan mismatch) */
#define GPZ_E_BUSY 8        /* too many serving requests outstanding: poll some, then retry */
#define GPZ_E_PENDING 9     /* ticket not finished yet */
#define GPZ_E_DATA 10       /* gzip input this path cannot split or decode (use a serial decoder) */
#define GPZ_E_SINK 11       /* a writer's sink or chunk function reported an error */

typedef struct gpz_ctx gpz_ctx;

typedef struct gpz_config {
    int device;            /* CUDA device ordinal */
    size_t member_bytes;   /* input bytes per gzip member: 131072 (default, the reference's
                              sub-chunk) up to 2097152 (whole-chunk mode); multiple of 4096 */
    size_t pool_bytes;     /* device pool cap in bytes (0: 40 GiB) */
    size_t batch_bytes;    /* input bytes per device pass (0: 64 MiB); larger calls are split into
                              passes that overlap upload, compute and download */
    int streams;           /* reserved (0) */
    int flags;             /* GPZ_FLAG_* */
    int wait_ms;           /* bound of every wait of a calling thread for the device, ms (0: 60000) */
    int codec;             /* GPZ_CODEC_GZIP (0) or GPZ_CODEC_ZSTD */
} gpz_config;

/* Codecs.  GZIP: the reference GPU path's gzip members (everything above).
 * ZSTD: the chunk-parallel zstd codec of the reference
 * (ZstdCompressor::chunk_fn, crates/gpzip-codec-cpu/src/compress.rs:76-126):
 * every input becomes one RFC 8878 zstd frame (no content size, no
 * checksum, 64 KiB window), from the same segmented-hash matches and lazy
 * walk as the gzip path; one block per 4 KiB of input, raw literals, the
 * predefined FSE distributions for the sequences, raw blocks where that is
 * not smaller.  Concatenated frames decode as one stream, as the reference's
 * .tar.zst does.  The compress calls, the writer and serving work the same;
 * gpz_debug_chunk cannot return pp, and GPZ_FLAG_FIXED_BLOCKS does not apply. */
#define GPZ_CODEC_GZIP 0
#define GPZ_CODEC_ZSTD 1

#define GPZ_FLAG_NO_GRAPHS 1    /* launch kernels directly instead of per-bucket CUDA graphs */
#define GPZ_FLAG_NO_AUTOTUNE 2  /* keep the default launch shapes */
#define GPZ_FLAG_STAGE_TIMING 4 /* record CUDA events around each stage (gpz_stage_times) */
#define GPZ_FLAG_SM_PARTITION 8 /* serving: run the small- and large-request lanes on separate SM partitions */
#define GPZ_FLAG_FIXED_BLOCKS 16 /* every member as one fixed-Huffman block (RFC 1951 BTYPE 01), the block
                                  encode_block_fast falls back to (deflate.rs:752-799) */

typedef struct gpz_desc {
    const uint8_t* in;   /* one chunk or file */
    size_t n;
    int level;           /* accepted and ignored, as the reference GPU codec does (gpu.rs:223) */
} gpz_desc;

typedef struct gpz_out {
    uint8_t* out;        /* caller-owned */
    size_t out_cap;
    size_t out_len;      /* written bytes */
    int status;          /* GPZ_OK or an error for this item */
} gpz_out;

/* Waits.  A call that waits for the device (every compress and inflate
 * call, and the completion of serving batches) polls for at most the
 * context's wait limit and then returns GPZ_E_TIMEOUT instead of blocking
 * without end.  The work it gave up on may still run and still write the
 * call's output buffers; the context's next call first waits (again within
 * the limit) for that work, and only then reuses the buffers.  Serving
 * requests of a timed-out batch complete with GPZ_E_TIMEOUT. */

/* Fill *cfg with defaults (device 0, 131072-byte members). */
GPZ_API void gpz_config_default(gpz_config* cfg);

/* Create a context on cfg->device (NULL: defaults).  Replaces
 * GpuBackend::try_init (gpu.rs:125-167). */
GPZ_API int gpz_create(const gpz_config* cfg, gpz_ctx** out);
GPZ_API void gpz_destroy(gpz_ctx* ctx);

/* Change the context's wait limit (ms, >= 0).  0 gives up at once unless
 * the device has already finished: a call then returns GPZ_E_TIMEOUT
 * whenever its work is still running when it first checks. */
GPZ_API int gpz_set_wait_ms(gpz_ctx* ctx, int wait_ms);

/* Worst-case output size of one compress call on n input bytes with
 * 131072-byte members; gpz_bound_ctx uses the context's member size. */
GPZ_API size_t gpz_bound(size_t n);
GPZ_API size_t gpz_bound_ctx(const gpz_ctx* ctx, size_t n);

/* One chunk -> concatenated gzip members.  Blocking.  The ChunkFn of
 * gpu.rs:193-208: n <= member_bytes (including 0) gives one member. */
GPZ_API int gpz_compress_chunk(gpz_ctx* ctx, const uint8_t* in, size_t n, int level, uint8_t* out,
                       size_t out_cap, size_t* out_len);

/* Many chunks or files of uneven size in one batched device pass (the
 * persistent kernels fed by the device descriptor queue).  outs[i] receives
 * the gzip stream of d[i].  Returns GPZ_OK if every item succeeded, else the
 * first failing item's status (each item's status is also set). */
GPZ_API int gpz_compress_batch(gpz_ctx* ctx, const gpz_desc* d, size_t count, gpz_out* outs);

/* Same, one device pass per chunk with a host synchronisation in between:
 * the plain one-launch-per-chunk path the batched path is measured against. */
GPZ_API int gpz_compress_batch_plain(gpz_ctx* ctx, const gpz_desc* d, size_t count, gpz_out* outs);

/* Device-resident batch.  d_in holds `count` inputs at 16-byte aligned device
 * offsets in_off[i] with lengths in_len[i] (host arrays).  The gzip streams
 * are written back to back into d_out (device, out_cap >= the bound) with the
 * 10-byte member headers and 8-byte trailers left as gaps for the host
 * (gpz_frame_host fills them in a host copy).  out_off (host, count+1
 * entries) receives each input's start offset and, last, the total length.
 * stream: a cudaStream_t (NULL: the context's stream).  Blocks until the
 * device pass finishes. */
GPZ_API int gpz_compress_device(gpz_ctx* ctx, const void* d_in, const uint64_t* in_off, const uint64_t* in_len,
                        size_t count, void* d_out, size_t out_cap, uint64_t* out_off, void* stream);

/* After gpz_compress_device: write the 10-byte headers and 8-byte trailers of
 * the last device batch into host_out, a host copy of d_out. */
GPZ_API int gpz_frame_host(gpz_ctx* ctx, uint8_t* host_out, size_t cap);

/* Parity hooks.  Run one chunk and also return the per-position packed
 * tokens (pp, n entries, length<<16 | distance-or-byte; lz77_hash.rs:54-62)
 * and the walked token stream of all members back to back (tokens, up to n
 * entries, *ntok set).  Any of pp / tokens / out may be NULL. */
GPZ_API int gpz_debug_chunk(gpz_ctx* ctx, const uint8_t* in, size_t n, uint32_t* pp, uint32_t* tokens,
                    size_t* ntok, uint8_t* out, size_t out_cap, size_t* out_len);

/* Serving (continuous batching): submit a request -- one gzip stream, the
 * input is copied before return -- and poll for its result.  Requests that
 * arrive while others are on the device join the next batch as soon as a
 * pipeline slot frees; requests of at most 1 MiB go first.  A request whose
 * bytes would push the queued and in-flight total past the pool cap is
 * rejected with GPZ_E_ADMISSION; while 1,048,576 requests are submitted and
 * not yet polled, gpz_submit returns GPZ_E_BUSY.  gpz_poll returns
 * GPZ_E_PENDING until the stream is ready (wait_ms > 0 blocks up to that
 * long), GPZ_E_SPACE (result kept) if o->out_cap is short; the result is
 * copied into o->out. */
GPZ_API int gpz_submit(gpz_ctx* ctx, const gpz_desc* d, uint64_t* ticket);
/* As gpz_submit, without the copy: the caller keeps d->in unchanged and
 * alive until gpz_poll has returned the result. */
GPZ_API int gpz_submit_ref(gpz_ctx* ctx, const gpz_desc* d, uint64_t* ticket);
GPZ_API int gpz_poll(gpz_ctx* ctx, uint64_t ticket, gpz_out* o, int wait_ms);

/* Serving statistics since the engine started or was last reset (latencies
 * in ms, arrival at gpz_submit to result ready; "small" = requests of at most
 * 1 MiB). */
typedef struct gpz_serve_stats {
    uint64_t completed;
    uint64_t rejected;
    uint64_t batches;
    double p50_ms, p99_ms, p999_ms;
    double max_queue_ms;
    uint64_t bytes_in, bytes_out;
    uint64_t completed_small;
    double p50_small_ms, p99_small_ms, p999_small_ms;
    uint64_t queued_bytes;
} gpz_serve_stats;
GPZ_API int gpz_serve_stats_get(gpz_ctx* ctx, gpz_serve_stats* st);
GPZ_API int gpz_serve_reset_stats(gpz_ctx* ctx);

/* Where a serving lane's time goes, since the engine started or its
 * statistics were last reset.  Lane 0 serves requests of at most 1 MiB,
 * lane 1 the larger ones.  Times are ms summed over the lane's batches
 * (divide by batches for means); the maxima are per batch. */
typedef struct gpz_lane_stats {
    uint64_t batches, units, bytes;
    double queue_ms;     /* oldest unit: arrival to its batch's launch */
    double submit_ms;    /* host: plan, staging copy, enqueue */
    double h2d_ms;       /* device: input and descriptor upload */
    double kernel_ms;    /* device: kernels and drain */
    double wait_ms;      /* host: enqueue done to batch done */
    double complete_ms;  /* host: framing and copies into the requests */
    double max_queue_ms, max_batch_ms;  /* max_batch_ms: launch to completion */
} gpz_lane_stats;
GPZ_API int gpz_serve_lane_stats(gpz_ctx* ctx, int lane, gpz_lane_stats* st);

GPZ_API const char* gpz_strerror(int status);

/* Last CUDA / device diagnostic of this context (static storage). */
GPZ_API const char* gpz_last_error(gpz_ctx* ctx);

/* Launch geometry in use: threads per CTA for lookup (512, 768, 1024) and emit
 * (256, 512) and the persistent grid sizes (0 = one CTA per tile).  The walk
 * has two forms with identical output: walk_threads 256 or 512 walks one
 * tile per warp (throughput), 1024 walks one tile per 512-thread CTA by
 * pointer doubling (lowest latency, the default for batches of up to 512
 * tiles).  Set by the autotuner per size bucket; may be overridden. */
typedef struct gpz_shape {
    int lookup_threads, lookup_grid;
    int walk_threads, walk_grid;
    int emit_threads, emit_grid;
} gpz_shape;
GPZ_API int gpz_get_shape(gpz_ctx* ctx, gpz_shape* s);
GPZ_API int gpz_set_shape(gpz_ctx* ctx, const gpz_shape* s);

/* Number of kernel launches the last compress call issued. */
GPZ_API uint64_t gpz_last_launches(gpz_ctx* ctx);

/* ---- Decompression of gpzip-written archives (the `gpzip x` path) ----
 *
 * The GPU counterpart of parallel_decompress
 * (crates/gpzip-codec-cpu/src/parallel_decompress.rs:63-113): the stream is
 * cut into members at every occurrence of the fixed 10-byte header that
 * gpzip writes (1f 8b 08 00 00 00 00 00 00 ff, parallel_decompress.rs:29-58),
 * and every member is decoded on the device into its place in the output
 * (offsets from the members' ISIZE trailers): a member that is one dynamic
 * block (every gpzip member) by many threads at once, any other by one warp.
 * Page-locked input starts uploading while the stream is cut; a page-locked
 * output buffer receives each member from the device as soon as it is
 * decoded.
 *
 * gpz_inflate_size: host only, no context.  Scans in[0, n) and returns the
 * member count and the total output size.  GPZ_E_DATA when the stream does
 * not start with the header or a member is shorter than 18 bytes.
 *
 * gpz_inflate: *out_len receives the total output size; GPZ_E_SPACE when
 * out_cap is smaller (out may then be NULL).  GPZ_E_DATA when the stream
 * cannot be cut as above, or when any member fails to decode, does not end
 * exactly at its trailer, or does not match its CRC-32 or ISIZE: the caller
 * then decodes serially, as parallel_decompress falls back to
 * MultiGzDecoder.  gpz_last_error names the member and the reason.  An
 * empty input gives an empty output. */
GPZ_API int gpz_inflate_size(const uint8_t* in, size_t n, size_t* members, size_t* out_bytes);
GPZ_API int gpz_inflate(gpz_ctx* ctx, const uint8_t* in, size_t n, uint8_t* out, size_t out_cap,
                        size_t* out_len);
/* Device time of the last gpz_inflate's kernels (decode and CRC, and, with
 * a page-locked output buffer, the members' copies to it), in ms. */
GPZ_API float gpz_inflate_device_ms(const gpz_ctx* ctx);

/* Largest input gpz_compress_member_static accepts (one 128 KiB member). */
#define GPZ_STATIC_MAX_BYTES 131072

/* Allocation-free compression of one member.  No counterpart in the
 * reference: it exists for callers that cannot allocate GPU memory when they
 * compress (their device memory is fully reserved by another allocator, or
 * the path must not take cudaMalloc / cudaFree, which can synchronise the
 * device).  All working memory is one fixed device array of about 2.5 MB
 * inside this library, held by every GPU that loads it until process exit.
 * d_in (n <= GPZ_STATIC_MAX_BYTES bytes, any alignment) and d_out (out_cap
 * bytes; gpz_bound(n) always suffices) are device memory on the calling
 * thread's current device; d_out receives one complete gzip member, byte for
 * byte what gpz_compress_chunk returns for the same input, and *out_len its
 * length.  Larger n returns GPZ_E_ARG; a short d_out returns GPZ_E_SPACE.
 * The first call on a device resolves the array's address and sets kernel
 * attributes, so make that first call before any stream capture begins.  The
 * call runs on `stream` (a cudaStream_t, NULL for the legacy default stream)
 * and returns after that stream has finished it.  Calls share the array:
 * calls whose device work overlaps race, so callers on one device are
 * serialised here and should not overlap it with their own device-side
 * reuse of d_out. */
GPZ_API int gpz_compress_member_static(const uint8_t* d_in, size_t n, uint8_t* d_out, size_t out_cap,
                                       size_t* out_len, void* stream);

/* Host time spent in each pipeline step since the last reset, in ms: batch
 * planning and buffer sizing, copying inputs into pinned staging, enqueueing
 * uploads and kernels, waiting for the device, framing and copying results
 * out; ms6[5] counts the device passes.  reset != 0 clears the counters. */
GPZ_API int gpz_host_times(gpz_ctx* ctx, double* ms6, int reset);

/* Device time of each stage of the last device pass, in ms, GPZ_STAGES
 * values: segment summaries (k_segtab), lookup (k_lookup), walk (k_walk_exit
 * with the member chaining in its last CTA, k_walk_mark), Huffman plan and
 * placement (k_huff with the placement in its last CTA, k_frame), emit
 * (k_emit).  Needs GPZ_FLAG_STAGE_TIMING at gpz_create. */
#define GPZ_STAGES 5
GPZ_API int gpz_stage_times(gpz_ctx* ctx, float* ms);

/* ---- Streaming chunked writer (ParallelChunkedWriter) ----
 *
 * The caller of ChunkFn in the reference, ParallelChunkedWriter
 * (crates/gpzip-codec-cpu/src/parallel.rs:28-229), which pack_tar wraps
 * around the archive file (crates/gpzip-core/src/archive/pack.rs:144-176):
 * bytes written are cut into chunk_size chunks, the chunks are compressed
 * into independent gzip members, and the members reach `sink` in input
 * order.  With a device context the chunks are page-locked buffers that an
 * internal thread streams through the context's pipeline as they fill
 * (passes of whatever is ready, overlapped on the device), while the caller
 * fills the next ones; up to max(max_in_flight, 128 MiB / chunk_size)
 * chunks are queued before gpz_writer_write waits.  The writer holds its
 * context while it has chunks on the device: the sink must not call into
 * that context.
 *
 *  - sink(user, buf, n) returns 0 on success; it is called from the
 *    writer's internal threads, never concurrently, and with members in
 *    order.
 *  - gpz_writer_flush does not cut the current partial chunk (tar calls
 *    flush between entries; parallel.rs:207-213) and waits for nothing.
 *  - gpz_writer_finish compresses the partial chunk, waits for every batch
 *    and returns the first error of the writer's life; errors are sticky,
 *    as in the reference (parallel.rs:70-89).  It may be called again.
 *  - gpz_writer_close finishes (if not yet) and frees the writer.
 *  - One writer is driven by one caller thread at a time (like the
 *    reference's &mut self methods); separate writers are independent.
 *
 * gpz_writer_open compresses with ctx (gpz_compress_batch).
 * gpz_writer_open_fn compresses each chunk with fn(fn_user, in, n, out,
 * out_cap, &out_len) instead (out_cap = gpz_bound(n); nonzero return is an
 * error): a caller-supplied ChunkFn, as the reference's writer takes any.
 * Each full chunk is handed at once to one of max_in_flight worker threads
 * (at most 1024), so up to max_in_flight calls of fn run concurrently, as
 * the reference runs one rayon task per chunk (parallel.rs:91-129); fn must
 * be safe to call from several threads.  A failed chunk ends the stream:
 * the chunks before it (in input order) are written, it and the chunks
 * after it are not. */
typedef struct gpz_writer gpz_writer;
typedef int (*gpz_sink_fn)(void* user, const uint8_t* buf, size_t n);
typedef int (*gpz_chunk_fn)(void* user, const uint8_t* in, size_t n, uint8_t* out, size_t out_cap,
                            size_t* out_len);
GPZ_API int gpz_writer_open(gpz_ctx* ctx, size_t chunk_size, size_t max_in_flight, gpz_sink_fn sink,
                            void* sink_user, gpz_writer** out);
GPZ_API int gpz_writer_open_fn(gpz_chunk_fn fn, void* fn_user, size_t chunk_size, size_t max_in_flight,
                               gpz_sink_fn sink, void* sink_user, gpz_writer** out);
GPZ_API int gpz_writer_write(gpz_writer* w, const uint8_t* buf, size_t n);
GPZ_API int gpz_writer_flush(gpz_writer* w);
GPZ_API int gpz_writer_finish(gpz_writer* w);
GPZ_API void gpz_writer_close(gpz_writer* w);

/* ---- Hybrid CPU + GPU chunk function (`--backend auto`) ----
 *
 * The reference's HybridGzipCompressor (crates/gpzip-cli/src/hybrid.rs:
 * 103-147), the default backend's caller of the GPU path: a composed chunk
 * function under which every chunk goes to whichever device is free.
 *  - The first warmup_chunks chunks (the reference: 4) always go to the CPU,
 *    so a small input never pays for the device context, which is made on
 *    the first chunk that may use the GPU (unless cfg.ctx supplies one).
 *    If it cannot be made, every chunk goes to the CPU.
 *  - After that a chunk takes one of gpu_permits GPU permits if one is free
 *    (decrement-if-positive, hybrid.rs:150-163) and runs gpz_compress_chunk
 *    on the context; otherwise it runs the CPU chunk function.  A GPU
 *    chunk's error is returned as is, with no CPU retry (hybrid.rs:131-135).
 *  - The CPU chunk function is cfg.cpu_fn, or gpz_cpu_gzip_chunk at
 *    cfg.level: one zlib gzip member per chunk, as GzipCompressor::chunk_fn
 *    (crates/gpzip-codec-cpu/src/compress.rs:52-59) writes with flate2.
 * Use gpz_hybrid_chunk as a writer's chunk function (gpz_writer_open_fn
 * with fn_user = the gpz_hybrid), with max_in_flight = the CPU workers +
 * gpu_permits, as the reference sizes its writer (hybrid.rs:139-146).  It is
 * safe to call from many threads.  gpz_hybrid_stats counts the chunks each
 * device took.  Destroy the hybrid after every writer using it is closed. */
typedef struct gpz_hybrid gpz_hybrid;
typedef struct gpz_hybrid_config {
    gpz_ctx* ctx;          /* device context to use (NULL: made on the first GPU chunk on `device`) */
    int device;
    int level;             /* zlib level of CPU chunks, 0-9 (default 5) */
    size_t gpu_permits;    /* concurrent GPU chunk calls (default 1, the reference's; 0: CPU only) */
    size_t warmup_chunks;  /* leading chunks kept on the CPU (default 4) */
    gpz_chunk_fn cpu_fn;   /* NULL: gpz_cpu_gzip_chunk at `level` */
    void* cpu_user;
    gpz_chunk_fn gpu_fn;   /* NULL: gpz_compress_chunk on the context; else this function runs the
                              chunks that hold a GPU permit (no context is made) */
    void* gpu_user;
} gpz_hybrid_config;
GPZ_API void gpz_hybrid_config_default(gpz_hybrid_config* cfg);
GPZ_API int gpz_hybrid_create(const gpz_hybrid_config* cfg, gpz_hybrid** out);
/* A gpz_chunk_fn; user is the gpz_hybrid. */
GPZ_API int gpz_hybrid_chunk(void* user, const uint8_t* in, size_t n, uint8_t* out, size_t out_cap,
                             size_t* out_len);
GPZ_API int gpz_hybrid_stats(const gpz_hybrid* h, uint64_t* cpu_chunks, uint64_t* gpu_chunks);
GPZ_API void gpz_hybrid_destroy(gpz_hybrid* h);

/* The CPU chunk function: one gzip member of the whole chunk, zlib at the
 * level *(const int*)level (NULL: 5), the gzip-cpu path of the reference
 * (compress.rs:52-59).  GPZ_E_SPACE when out_cap is too small
 * (gpz_bound(n) always suffices). */
GPZ_API int gpz_cpu_gzip_chunk(void* level, const uint8_t* in, size_t n, uint8_t* out, size_t out_cap,
                               size_t* out_len);

#ifdef __cplusplus
}
#endif
#endif
