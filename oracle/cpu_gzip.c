/*
 * cpu_gzip.c -- "gpzip-cpu-equivalent" timed CPU baseline (TEST/BENCH INFRASTRUCTURE).
 *
 * Restates the reference CPU chunk codec GzipCompressor::chunk_fn
 * (crates/gpzip-codec-cpu/src/compress.rs:52-59): one gzip member per chunk
 * at the given level, chunks compressed on a thread pool of all host cores
 * (backend.rs:31-36) and concatenated in input order
 * (parallel.rs:144-150).  The reference links flate2 1.1.9 over zlib-rs
 * 0.6.3, which cannot be built here; this uses system zlib 1.3
 * (deflateInit2(level, Z_DEFLATED, 31, 8, Z_DEFAULT_STRATEGY)).  Output bytes
 * therefore differ from zlib-rs; throughput and ratio are comparable.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

typedef struct {
    const uint8_t* in;
    size_t n, chunk, nchunks;
    int level;
    uint8_t** bufs;
    size_t* lens;
    size_t next;
    pthread_mutex_t mu;
    int failed;
} job_t;

static size_t gzip_one(const uint8_t* in, size_t n, int level, uint8_t** outp) {
    z_stream s;
    memset(&s, 0, sizeof s);
    if (deflateInit2(&s, level, Z_DEFLATED, 31, 8, Z_DEFAULT_STRATEGY) != Z_OK) return 0;
    uLong cap = deflateBound(&s, (uLong)n) + 32;
    uint8_t* out = (uint8_t*)malloc(cap);
    if (!out) {
        deflateEnd(&s);
        return 0;
    }
    s.next_in = (Bytef*)in;
    s.avail_in = (uInt)n;
    s.next_out = out;
    s.avail_out = (uInt)cap;
    int rc = deflate(&s, Z_FINISH);
    size_t len = cap - s.avail_out;
    deflateEnd(&s);
    if (rc != Z_STREAM_END) {
        free(out);
        return 0;
    }
    *outp = out;
    return len;
}

static void* worker(void* arg) {
    job_t* j = (job_t*)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        size_t c = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (c >= j->nchunks) break;
        size_t off = c * j->chunk;
        size_t len = j->n - off < j->chunk ? j->n - off : j->chunk;
        j->lens[c] = gzip_one(j->in + off, len, j->level, &j->bufs[c]);
        if (j->lens[c] == 0) j->failed = 1;
    }
    return NULL;
}

/* Compress `in` as ceil(n/chunk) gzip members.  Writes the concatenation to
 * out (cap bytes); returns its length, or 0 on failure / overflow. */
size_t gpzcpu_gzip_chunks(const uint8_t* in, size_t n, size_t chunk, int level, int threads,
                          uint8_t* out, size_t cap) {
    if (n == 0 || chunk == 0) return 0;
    job_t j;
    memset(&j, 0, sizeof j);
    j.in = in;
    j.n = n;
    j.chunk = chunk;
    j.level = level;
    j.nchunks = (n + chunk - 1) / chunk;
    j.bufs = (uint8_t**)calloc(j.nchunks, sizeof(uint8_t*));
    j.lens = (size_t*)calloc(j.nchunks, sizeof(size_t));
    pthread_mutex_init(&j.mu, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    for (int t = 1; t < threads; t++) pthread_create(&tid[t], NULL, worker, &j);
    worker(&j);
    for (int t = 1; t < threads; t++) pthread_join(tid[t], NULL);
    size_t total = 0;
    for (size_t c = 0; c < j.nchunks && !j.failed; c++) {
        if (total + j.lens[c] > cap) {
            j.failed = 1;
            break;
        }
        memcpy(out + total, j.bufs[c], j.lens[c]);
        total += j.lens[c];
    }
    for (size_t c = 0; c < j.nchunks; c++) free(j.bufs[c]);
    free(j.bufs);
    free(j.lens);
    pthread_mutex_destroy(&j.mu);
    return j.failed ? 0 : total;
}
