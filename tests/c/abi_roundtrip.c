/* A plain C caller of the library, the way a Rust / C++ host binds it:
 * create a context, compress chunks through gpz_compress_chunk and
 * gpz_compress_batch, and check each result against zlib inflate.
 * Prints "ok" and returns 0 on success. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

#include "gpz.h"

static int inflate_all(const uint8_t* gz, size_t n, uint8_t* out, size_t cap, size_t* out_len) {
    /* concatenated gzip members */
    size_t pos = 0, w = 0;
    while (pos < n) {
        z_stream s;
        memset(&s, 0, sizeof s);
        if (inflateInit2(&s, 31) != Z_OK) return -1;
        s.next_in = (Bytef*)(gz + pos);
        s.avail_in = (uInt)(n - pos);
        s.next_out = out + w;
        s.avail_out = (uInt)(cap - w);
        int rc = inflate(&s, Z_FINISH);
        if (rc != Z_STREAM_END) {
            inflateEnd(&s);
            return -1;
        }
        pos += s.total_in;
        w += s.total_out;
        inflateEnd(&s);
    }
    *out_len = w;
    return 0;
}

int main(void) {
    gpz_config cfg;
    gpz_config_default(&cfg);
    gpz_ctx* ctx = NULL;
    int rc = gpz_create(&cfg, &ctx);
    if (rc != GPZ_OK) {
        fprintf(stderr, "gpz_create: %s\n", gpz_strerror(rc));
        return 1;
    }
    const size_t sizes[4] = {0, 1, 300000, 2u << 20};
    uint8_t* in[4];
    for (int i = 0; i < 4; i++) {
        in[i] = (uint8_t*)malloc(sizes[i] ? sizes[i] : 1);
        uint32_t x = 12345u + (uint32_t)i;
        for (size_t k = 0; k < sizes[i]; k++) {
            x = x * 1103515245u + 12345u;
            /* text-like: a small alphabet with repeats */
            in[i][k] = (uint8_t)("the quick brown fox jumps over the lazy dog\n"[(x >> 16) % 44]);
        }
    }
    uint8_t* back = (uint8_t*)malloc((2u << 20) + 64);
    /* one chunk at a time (the ChunkFn shape) */
    for (int i = 0; i < 4; i++) {
        size_t cap = gpz_bound_ctx(ctx, sizes[i]), len = 0, got = 0;
        uint8_t* out = (uint8_t*)malloc(cap);
        rc = gpz_compress_chunk(ctx, in[i], sizes[i], 5, out, cap, &len);
        if (rc != GPZ_OK || inflate_all(out, len, back, (2u << 20) + 64, &got) != 0 || got != sizes[i] ||
            (got && memcmp(back, in[i], got) != 0)) {
            fprintf(stderr, "chunk %d failed: %s (%s)\n", i, gpz_strerror(rc), gpz_last_error(ctx));
            return 1;
        }
        free(out);
    }
    /* all four in one batched call */
    gpz_desc d[4];
    gpz_out o[4];
    for (int i = 0; i < 4; i++) {
        d[i].in = in[i];
        d[i].n = sizes[i];
        d[i].level = 5;
        o[i].out_cap = gpz_bound_ctx(ctx, sizes[i]);
        o[i].out = (uint8_t*)malloc(o[i].out_cap);
    }
    rc = gpz_compress_batch(ctx, d, 4, o);
    if (rc != GPZ_OK) {
        fprintf(stderr, "batch failed: %s\n", gpz_strerror(rc));
        return 1;
    }
    for (int i = 0; i < 4; i++) {
        size_t got = 0;
        if (o[i].status != GPZ_OK || inflate_all(o[i].out, o[i].out_len, back, (2u << 20) + 64, &got) != 0 ||
            got != sizes[i] || (got && memcmp(back, in[i], got) != 0)) {
            fprintf(stderr, "batch item %d failed\n", i);
            return 1;
        }
    }
    gpz_destroy(ctx);
    printf("ok\n");
    return 0;
}
