// gpz_internal.h -- layouts shared by the sm_100a kernels and the host runtime.
//
// A batch is a list of members (independent gzip members, 128 KiB each in
// parity mode, as gpu.rs:150-160 and gpu.rs:193-208 of the reference cut
// them).  Every member is split into 4 KiB tiles, which are both the
// reference's hash segments (lz77_hash.rs:64-69, SEG_LOG2 = 12) and the unit
// of the walk / encode stages.
#pragma once
#include <cstdint>

#define GPZ_SEG_LOG2 12
#define GPZ_SEG (1u << GPZ_SEG_LOG2)
#define GPZ_WIN_SEGS 9                      // own segment + 8 back (window-bound proof)
#define GPZ_WIN_BYTES (GPZ_WIN_SEGS * GPZ_SEG + 320)
#define GPZ_MAX_MATCH 258u
#define GPZ_WINDOW 32768u
#define GPZ_NLIT 286
#define GPZ_NDIST 30
#define GPZ_NSYM (GPZ_NLIT + GPZ_NDIST)
#define GPZ_EXITS 258                       // entry offsets a walk can have into a tile
#define GPZ_HDR_WORDS 144                   // dynamic block header <= 4498 bits, + slack

// Error bits reported through BatchParams::err.
#define GPZ_ERRBIT_BITS 2u      // emitted bit count disagreed with the plan
#define GPZ_ERRBIT_HUFF 4u      // code construction failed (never expected)
#define GPZ_ERRBIT_DESC 8u      // a fetched descriptor block exceeded the arenas

// BatchParams.flags
#define GPZ_BATCH_FIXED 1u      // every member as one fixed-Huffman block (RFC 1951 BTYPE 01)
#define GPZ_BATCH_ZSTD 2u       // zstd frames (RFC 8878) instead of gzip members

// MemberDesc.frame
#define GPZ_MEMBER_FIRST 1u     // the first member of its input (a zstd frame starts here)
#define GPZ_MEMBER_LAST 2u      // the last member of its input (its last block ends the frame)
#define GPZ_ZSTD_FRAME_HDR 6u   // bytes of the zstd frame header

struct MemberDesc {
    uint64_t in_off;     // first input byte of the member in the batch input (16-byte aligned)
    uint32_t len;        // member length in bytes
    uint32_t tile_base;  // index of the member's first tile
    uint32_t ntiles;     // ceil(len / 4096)
    uint32_t frame;      // GPZ_MEMBER_* (the level is accepted and ignored, as gpu.rs:223 does)
    uint64_t out_slot;   // caller-visible ordinal (used by the serving queue)
};

struct TileDesc {
    uint32_t member;
    uint32_t seg;
};

struct MemberOut {
    uint64_t gz_off;         // byte offset of this member's output in the batch output
    uint32_t deflate_bytes;  // payload bytes: the DEFLATE block (gzip), everything (zstd)
    uint32_t crc;            // CRC-32 of the member input (gzip)
    uint32_t total_bits;     // DEFLATE bits incl. header and EOB (gzip)
    uint32_t header_bits;
    uint32_t len;            // ISIZE (member input length)
    uint32_t frame_bytes;    // bytes around the payload: 18 (gzip header and trailer), 0 (zstd)
};

// Everything a batch launch needs; passed by value to every kernel.
struct BatchParams {
    const uint8_t* in;
    const MemberDesc* members;
    const TileDesc* tiles;
    uint32_t* pp;             // per-position packed tokens, indexed like `in`
    uint16_t* seg_keys;       // [tile][4096] distinct hashes of the segment, ascending (id = rank)
    uint32_t* seg_on;         // [tile][4096] newest offset | oldest offset << 16, per distinct hash
    uint32_t* seg_nkeys;      // [tile] distinct hashes in the segment
    uint32_t* tok;            // walked tokens, tile-sparse, indexed like `in`
    uint32_t* out_words;      // gzip stream of the batch, as 32-bit words
    uint32_t* tile_entry;     // walk entry offset into each tile
    uint16_t* tile_exit;      // [tile][GPZ_EXITS] exit offset into the next tile
    uint32_t* tile_zinfo;     // zstd: per tile, the block's size | compressed << 31 (in the exit tables'
                              // space, free once the walk is done)
    uint16_t* tile_hist;      // [tile][GPZ_NSYM] symbol counts of the tile's tokens
    uint32_t* tile_ntok;      // tokens per tile
    uint32_t* tile_bitoff;    // tile's first token bit within its member's DEFLATE stream
    uint32_t* member_codes;   // [member][GPZ_NSYM] reversed code | len << 16
    uint32_t* member_hdr;     // [member][GPZ_HDR_WORDS] dynamic block header bits
    MemberOut* member_out;
    uint32_t* counters;       // work-claim counters per stage (zeroed per batch)
    uint32_t* err;
    const uint32_t* dims;     // device: [0] tiles, [1] members of this batch
    uint32_t nmembers;        // host-side copies, used only to size exact grids
    uint32_t ntiles;
    uint64_t out_base;        // byte offset added to every member's gz_off
    uint32_t flags;           // GPZ_BATCH_* below
};

enum {
    GPZ_CNT_LOOKUP = 0,
    GPZ_CNT_EXIT = 1,
    GPZ_CNT_MARK = 2,
    GPZ_CNT_HUFF = 3,
    GPZ_CNT_EMIT = 4,
    GPZ_CNT_SEGSORT = 5,
    GPZ_CNT_EXIT_DONE = 6,  // CTAs of k_walk_exit that finished (the last one chains)
    GPZ_CNT_HUFF_DONE = 7,  // CTAs of k_huff that finished (the last one places)
    GPZ_NCOUNTERS = 8
};

// Per-stage launch geometry chosen by the autotuner: threads per CTA, and
// CTAs per grid (0 = one CTA per item of the batch; > 0 = a persistent grid
// that claims items from the device counters).
struct LaunchShape {
    int lookup_threads;
    int lookup_grid;
    int walk_threads;
    int walk_grid;
    int emit_threads;
    int emit_grid;
    int segtab_grid;
    int huff_grid;
    int zblock_grid;  // zstd stages (0: one CTA per item)
    int zcopy_grid;
};

// Host-mapped pinned destinations of k_drain.
struct DrainTarget {
    uint8_t* h_out;
    MemberOut* h_mout;
    uint32_t* h_err;
    int grid;
};

// Host-mapped pinned sources of k_fetch: the descriptor block (64-byte
// header: tiles, members, input bytes as u64 at byte 8; then the members and
// the tiles) and the batch input, copied by the SMs into the device arenas
// (no copy-engine transfer on the batch's path).  The capacities bound what
// the header may ask for.
struct FetchSource {
    const uint8_t* h_desc;
    const uint8_t* h_in;
    uint32_t* d_dims;
    MemberDesc* d_members;
    TileDesc* d_tiles;
    uint8_t* d_in;
    uint64_t members_cap, tiles_cap, in_cap;
};

// Kernel launchers (gpz_kernels.cu).
// events: NULL or GPZ_STAGES + 1 cudaEvent_t recorded at the stage boundaries.
// drain: NULL, or where k_drain streams the output, member table and error.
// fetch: NULL, or the mapped sources k_fetch copies in before the first stage.
int gpz_launch_batch(const BatchParams& bp, const LaunchShape& ls, void* stream, void* const* events,
                     const DrainTarget* drain, const FetchSource* fetch = nullptr);
// k_drain alone, for a batch whose stage kernels ran on another stream.
int gpz_launch_drain(const BatchParams& bp, const DrainTarget& drain, void* stream);
// One gzip member of a stream to decompress (gpz_inflate).
struct InflateMember {
    uint64_t in_off;   // first DEFLATE byte (after the 10-byte header)
    uint64_t out_off;  // first output byte
    uint32_t in_len;   // DEFLATE bytes (member bytes - 18)
    uint32_t isize;    // ISIZE of the trailer
    uint32_t crc;      // CRC-32 of the trailer
    uint32_t pad;
};
// Device scratch of the parallel decode's tails (gpz_inflate.cu): one
// record of gpz_inflate_tail_bytes() per member, gpz_inflate_cands() packed
// candidate results per sub-span, three u32 per sub-span (sub_start: the
// owning tail, until k_inflate_chain puts the chosen start offset there;
// the token and byte offsets), two counters (tails, sub-spans taken).
// sub_cap = 8 x deflate bytes / gpzi::kSubBits + members + 1 sub-spans
// always suffice.
struct InflateScratch {
    void* tails;
    uint64_t* cands;
    uint32_t* sub_start;
    uint32_t* sub_tok;
    uint32_t* sub_byte;
    uint32_t* counters;
    uint32_t sub_cap;
};
// k_inflate_par (the parallel decode of single-block members; done[m] = 1
// for the members it decoded, 2 for those whose tail it left to
// k_inflate_cand and k_inflate_chain), k_inflate_tok (one warp per
// remaining member: tokens into tok, indexed like out, and their count into
// ntok), k_inflate_expand (tokens to bytes), then k_inflate_crc
// (gpz_inflate.cu); status[m] = 0 or the member's gpzi status code.
// host_out: NULL, or a page-locked host buffer (its device address) that
// receives each member's output as soon as it is expanded.  events: NULL or
// two cudaEvent_t recorded before and after.
int gpz_launch_inflate(const uint8_t* in, uint8_t* out, uint32_t* tok, const InflateMember* members,
                       uint32_t* status, uint32_t* ntok, uint32_t* done, const InflateScratch& sc, uint8_t* host_out,
                       uint32_t count, void* stream, void* const* events);
size_t gpz_inflate_tail_bytes();
uint32_t gpz_inflate_cands();
size_t gpz_inflate_smem_bytes();
// Persistent grid sizes (SMs x resident CTAs) for the shape's thread counts.
int gpz_occupancy(LaunchShape* persistent);
int gpz_kernel_smem_setup();
size_t gpz_lookup_smem_bytes();
// zstd stages after the walk (gpz_zstd.cu): k_zblock (blocks, placement in
// its last CTA) and k_zcopy; events[4..5] as in gpz_launch_batch.
int gpz_launch_zstd(const BatchParams& bp, void* stream, void* const* events, int grid_blocks, int grid_copy);
int gpz_zstd_setup();
int gpz_zstd_occupancy(int* grid_blocks, int* grid_copy);
