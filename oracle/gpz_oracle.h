/*
 * gpz_oracle.h -- CPU oracle for the gzip compression path (TEST INFRASTRUCTURE).
 *
 * This is a plain-C restatement of the reference GPU codec's arithmetic
 * (skmtkytr/gpzip, crate gpzip-codec-gpu).  It exists only to check the CUDA
 * path and to serve as the timed CPU port of that path.  Nothing in the
 * product library links or calls it.
 *
 * Parity status: the reference ships no golden vectors for tokens or DEFLATE
 * bytes, so token- and byte-level parity is pinned by this restatement plus an
 * independent pure-Python restatement (oracle/pyref.py) that must agree with
 * it, by the reference's own property tests (Huffman lengths, round trips, the
 * fixed 10-byte member header) and by zlib inflate / gzip -t on every member.
 *
 * Packed token format (lz77_hash.rs:50-62): length<<16 | (distance or byte).
 */
#ifndef GPZ_ORACLE_H
#define GPZ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* lz77_hash_build.wgsl:36-43 */
uint32_t gpzo_hash3(const uint8_t* in, uint32_t p);

/* Per-position packed tokens for one member of n bytes.  Restates the dense
 * seg_oldest/seg_newest build (lz77_hash_build.wgsl:45-54, reset at
 * lz77_hash.rs:584-587) and the unbounded backward segment walk of
 * lz77_hash_lookup.wgsl:69-119.  pp must hold n entries.  Returns 0, or -1 on
 * allocation failure. */
int gpzo_match_find(const uint8_t* in, uint32_t n, uint32_t* pp);

/* lz77.rs:260-284 (lazy one-step walk).  tokens must hold n entries.
 * Returns the number of tokens written. */
size_t gpzo_greedy_walk(const uint32_t* pp, const uint8_t* in, uint32_t n, uint32_t* tokens);

/* huffman.rs:26-60: length-limited code lengths by halve-and-rebuild.
 * Returns 1 on success, 0 when max_bits is too small for the alphabet. */
int gpzo_build_code_lengths(const uint32_t* freq, int nsym, int max_bits, uint8_t* lens);

/* huffman.rs:122-152 */
void gpzo_canonical_codes(const uint8_t* lens, int nsym, uint32_t* codes);

/* deflate.rs:752-761 (encode_block_fast).  Returns the byte count written to
 * out, or 0 if cap is too small. */
size_t gpzo_encode_block_fast(const uint32_t* tokens, size_t count, uint8_t* out, size_t cap);
size_t gpzo_encode_block_fixed(const uint32_t* tokens, size_t count, uint8_t* out, size_t cap);

/* CRC-32 (IEEE 802.3, reflected, init/xorout 0xFFFFFFFF) as crc32fast 1.5.0
 * computes it at deflate.rs:974. */
uint32_t gpzo_crc32(const uint8_t* in, size_t n);

/* One whole member: match_find -> greedy_walk -> encode_block_fast ->
 * gzip_wrap (gpu.rs:271-287, deflate.rs:962-980).  Returns bytes written or 0
 * when cap is too small / allocation fails. */
size_t gpzo_gzip_member(const uint8_t* in, uint32_t n, uint8_t* out, size_t cap);

/* gzip_chunk_fn (gpu.rs:193-208): split into member_bytes pieces, one member
 * each, concatenated.  threads > 1 runs members on a pthread pool (the
 * result is identical).  Returns bytes written or 0 on failure. */
size_t gpzo_gzip_chunk(const uint8_t* in, size_t n, size_t member_bytes, uint8_t* out,
                       size_t cap, int threads);

/* Worst-case member size bound used by the oracle for buffer sizing. */
size_t gpzo_member_bound(size_t n);

/* zstd frame of one chunk as the GPU zstd codec defines it from this
 * path's tokens (oracle/zstd_frame.c): a 6-byte header, one block per 4 KiB
 * tile of each member_bytes piece, raw literals, predefined FSE sequences,
 * raw blocks where those are not smaller.  Returns bytes written, or 0 when
 * cap < gpzo_zstd_bound or on failure. */
size_t gpzo_zstd_chunk(const uint8_t* in, size_t n, size_t member_bytes, uint8_t* out, size_t cap);
size_t gpzo_zstd_bound(size_t n, size_t member_bytes);

/* Reference brute-force matcher used by the reference's encoder tests
 * (deflate.rs:992-1016); window given in bytes. */
void gpzo_brute_lz77(const uint8_t* in, uint32_t n, uint32_t window, uint32_t* pp);

#ifdef __cplusplus
}
#endif
#endif
