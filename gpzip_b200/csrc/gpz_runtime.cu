// gpz_runtime.cu -- host runtime and C ABI of the gzip compression path.
//
// Replaces the reference's wgpu plumbing (GpuContext, Lz77HashPipeline's
// BufferSet pool, BatchedLz77's submitter/completer threads; gpu.rs:125-167,
// lz77_hash.rs:98-297, batch.rs:48-141) with one CUDA context per gpz_ctx:
// a device pool sized for a batch, pinned staging, and a batch planner that
// cuts every input into members and 4 KiB tiles for the persistent kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gpz.h"
#include "gpz_internal.h"

namespace {

constexpr size_t kDefaultMember = 131072;
constexpr size_t kMaxMember = 2u << 20;
constexpr size_t kDefaultBatch = 256u << 20;
constexpr size_t kDefaultPool = 40ull << 30;

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Worst case of one member of n bytes: 18 framing bytes, a dynamic header of
// at most 4498 bits, at most 16 bits per input byte (a length-3 match costs
// at most 15 + 5 + 15 + 13 bits), the EOB, and word slack.
size_t member_bound(size_t n) { return 18 + 600 + 2 * n + 8; }

struct DevArena {
    void* p = nullptr;
    size_t cap = 0;
};

}  // namespace

struct gpz_ctx {
    int device = 0;
    size_t member_bytes = kDefaultMember;
    size_t pool_cap = kDefaultPool;
    size_t batch_bytes = kDefaultBatch;
    int flags = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;  // one device pass at a time per context
    std::string last_err;
    uint64_t launches = 0;
    LaunchShape shape{1024, 0, 512, 0, 512, 0};

    // device pool (one batch in flight)
    DevArena d_in, d_pp, d_tok, d_out, d_skeys, d_son, d_sposid, d_snkeys, d_tentry, d_texit, d_thist, d_tntok, d_tbit, d_mcodes, d_mhdr, d_mout,
        d_cnt, d_members, d_tiles;
    size_t pool_used = 0;
    // pinned staging
    uint8_t* h_in = nullptr;
    size_t h_in_cap = 0;
    uint8_t* h_out = nullptr;
    size_t h_out_cap = 0;
    std::vector<MemberDesc> members;
    std::vector<TileDesc> tiles;
    std::vector<MemberOut> mout;
    MemberDesc* h_members = nullptr;
    size_t h_members_cap = 0;
    TileDesc* h_tiles = nullptr;
    size_t h_tiles_cap = 0;
    MemberOut* h_mout = nullptr;
    size_t h_mout_cap = 0;
    uint32_t* h_err = nullptr;
    // per-stage CUDA events of the last pass (GPZ_FLAG_STAGE_TIMING)
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    float stage_ms[4] = {0, 0, 0, 0};
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

#define CU(ctx, call)                                                       \
    do {                                                                    \
        cudaError_t _e = (call);                                            \
        if (_e != cudaSuccess) return fail((ctx), GPZ_E_CUDA, #call, _e);   \
    } while (0)

int ensure_dev(gpz_ctx* c, DevArena& a, size_t bytes) {
    bytes = round_up(std::max<size_t>(bytes, 256), 256);
    if (a.cap >= bytes) return GPZ_OK;
    size_t grow = std::max(bytes, a.cap + a.cap / 2);
    if (c->pool_used - a.cap + grow > c->pool_cap) {
        grow = bytes;
        if (c->pool_used - a.cap + grow > c->pool_cap) return fail(c, GPZ_E_ADMISSION, "device pool cap exceeded");
    }
    if (a.p) cudaFree(a.p);
    c->pool_used -= a.cap;
    a.p = nullptr;
    a.cap = 0;
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
int ensure_host(gpz_ctx* c, T*& p, size_t& cap, size_t count) {
    if (cap >= count) return GPZ_OK;
    size_t grow = std::max(count, cap + cap / 2);
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&p), grow * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, GPZ_E_NOMEM, "cudaMallocHost", e);
    }
    cap = grow;
    return GPZ_OK;
}

struct Span {
    size_t n;
    uint64_t dev_off;      // where the input sits in the device input buffer
    size_t first_member;   // index into ctx->members
    size_t nmembers;
};

// Cut inputs into members (member_bytes each, gpu.rs:193-208: an input of at
// most member_bytes, empty included, is one member) and members into tiles.
void plan(gpz_ctx* c, std::vector<Span>& spans) {
    c->members.clear();
    c->tiles.clear();
    for (auto& s : spans) {
        s.first_member = c->members.size();
        size_t nm = s.n == 0 ? 1 : (s.n + c->member_bytes - 1) / c->member_bytes;
        s.nmembers = nm;
        for (size_t j = 0; j < nm; j++) {
            MemberDesc md{};
            md.in_off = s.dev_off + j * c->member_bytes;
            md.len = (uint32_t)std::min(c->member_bytes, s.n - std::min(s.n, j * c->member_bytes));
            md.tile_base = (uint32_t)c->tiles.size();
            md.ntiles = (md.len + GPZ_SEG - 1) / GPZ_SEG;
            md.level = 0;
            md.out_slot = c->members.size();
            for (uint32_t t = 0; t < md.ntiles; t++) c->tiles.push_back(TileDesc{(uint32_t)c->members.size(), t});
            c->members.push_back(md);
        }
    }
}

// Sizes every device array for the planned batch.
int reserve(gpz_ctx* c, size_t in_bytes, bool own_in, bool own_out, size_t out_bytes) {
    const size_t nm = c->members.size(), nt = std::max<size_t>(c->tiles.size(), 1);
    int rc;
    if (own_in && (rc = ensure_dev(c, c->d_in, in_bytes + 64))) return rc;
    if ((rc = ensure_dev(c, c->d_pp, in_bytes * 4 + 64))) return rc;
    if ((rc = ensure_dev(c, c->d_tok, in_bytes * 4 + 64))) return rc;
    if (own_out && (rc = ensure_dev(c, c->d_out, out_bytes + 64))) return rc;
    if ((rc = ensure_dev(c, c->d_skeys, nt * GPZ_SEG * 2))) return rc;
    if ((rc = ensure_dev(c, c->d_son, nt * GPZ_SEG * 4))) return rc;
    if ((rc = ensure_dev(c, c->d_sposid, nt * GPZ_SEG * 2))) return rc;
    if ((rc = ensure_dev(c, c->d_snkeys, nt * 4))) return rc;
    if ((rc = ensure_dev(c, c->d_tentry, nt * 4))) return rc;
    if ((rc = ensure_dev(c, c->d_texit, nt * GPZ_EXITS * 2))) return rc;
    if ((rc = ensure_dev(c, c->d_thist, nt * GPZ_NSYM * 2))) return rc;
    if ((rc = ensure_dev(c, c->d_tntok, nt * 4))) return rc;
    if ((rc = ensure_dev(c, c->d_tbit, nt * 4))) return rc;
    if ((rc = ensure_dev(c, c->d_mcodes, nm * GPZ_NSYM * 4))) return rc;
    if ((rc = ensure_dev(c, c->d_mout, nm * sizeof(MemberOut)))) return rc;
    if ((rc = ensure_dev(c, c->d_mhdr, nm * GPZ_HDR_WORDS * 4))) return rc;
    if ((rc = ensure_dev(c, c->d_cnt, GPZ_NCOUNTERS * 4 + 64))) return rc;
    if ((rc = ensure_dev(c, c->d_members, nm * sizeof(MemberDesc)))) return rc;
    if ((rc = ensure_dev(c, c->d_tiles, nt * sizeof(TileDesc)))) return rc;
    if ((rc = ensure_host(c, c->h_members, c->h_members_cap, nm))) return rc;
    if ((rc = ensure_host(c, c->h_tiles, c->h_tiles_cap, nt))) return rc;
    if ((rc = ensure_host(c, c->h_mout, c->h_mout_cap, nm))) return rc;
    return GPZ_OK;
}

size_t out_bound_of_plan(const gpz_ctx* c) {
    size_t b = 0;
    for (auto& m : c->members) b += member_bound(m.len);
    return b;
}

// Upload descriptors, clear the look-back state, launch the four stages and
// read back the member table.  in/out are device pointers.
int run_device(gpz_ctx* c, const uint8_t* d_in, uint8_t* d_out, cudaStream_t s) {
    const size_t nm = c->members.size(), nt = c->tiles.size();
    std::memcpy(c->h_members, c->members.data(), nm * sizeof(MemberDesc));
    if (nt) std::memcpy(c->h_tiles, c->tiles.data(), nt * sizeof(TileDesc));
    CU(c, cudaMemcpyAsync(c->d_members.p, c->h_members, nm * sizeof(MemberDesc), cudaMemcpyHostToDevice, s));
    if (nt) CU(c, cudaMemcpyAsync(c->d_tiles.p, c->h_tiles, nt * sizeof(TileDesc), cudaMemcpyHostToDevice, s));
    CU(c, cudaMemsetAsync(c->d_cnt.p, 0, GPZ_NCOUNTERS * 4 + 64, s));

    BatchParams bp{};
    bp.in = d_in;
    bp.members = static_cast<const MemberDesc*>(c->d_members.p);
    bp.tiles = static_cast<const TileDesc*>(c->d_tiles.p);
    bp.pp = static_cast<uint32_t*>(c->d_pp.p);
    bp.tok = static_cast<uint32_t*>(c->d_tok.p);
    bp.out_words = reinterpret_cast<uint32_t*>(d_out);
    bp.seg_keys = static_cast<uint16_t*>(c->d_skeys.p);
    bp.seg_on = static_cast<uint32_t*>(c->d_son.p);
    bp.seg_posid = static_cast<uint16_t*>(c->d_sposid.p);
    bp.seg_nkeys = static_cast<uint32_t*>(c->d_snkeys.p);
    bp.tile_entry = static_cast<uint32_t*>(c->d_tentry.p);
    bp.tile_exit = static_cast<uint16_t*>(c->d_texit.p);
    bp.tile_hist = static_cast<uint16_t*>(c->d_thist.p);
    bp.tile_ntok = static_cast<uint32_t*>(c->d_tntok.p);
    bp.tile_bitoff = static_cast<uint32_t*>(c->d_tbit.p);
    bp.member_codes = static_cast<uint32_t*>(c->d_mcodes.p);
    bp.member_out = static_cast<MemberOut*>(c->d_mout.p);
    bp.member_hdr = static_cast<uint32_t*>(c->d_mhdr.p);
    bp.counters = static_cast<uint32_t*>(c->d_cnt.p);
    bp.err = bp.counters + GPZ_NCOUNTERS;
    bp.nmembers = (uint32_t)nm;
    bp.ntiles = (uint32_t)nt;
    bp.out_base = 0;
    const bool timing = (c->flags & GPZ_FLAG_STAGE_TIMING) && c->ev[0];
    if (gpz_launch_batch(bp, c->shape, s, timing ? reinterpret_cast<void* const*>(c->ev) : nullptr) != 0)
        return fail(c, GPZ_E_CUDA, "kernel launch", cudaGetLastError());
    c->launches = 9;
    CU(c, cudaMemcpyAsync(c->h_mout, c->d_mout.p, nm * sizeof(MemberOut), cudaMemcpyDeviceToHost, s));
    CU(c, cudaMemcpyAsync(c->h_err, bp.err, 4, cudaMemcpyDeviceToHost, s));
    CU(c, cudaStreamSynchronize(s));
    c->mout.assign(c->h_mout, c->h_mout + nm);
    if (timing)
        for (int i = 0; i < 4; i++) cudaEventElapsedTime(&c->stage_ms[i], c->ev[i], c->ev[i + 1]);
    const uint32_t err = *c->h_err;
    if (err & GPZ_ERRBIT_SPIN) return fail(c, GPZ_E_TIMEOUT, "bounded device wait expired");
    if (err) return fail(c, GPZ_E_INTERNAL, "device self-check failed");
    return GPZ_OK;
}

uint64_t batch_out_bytes(const gpz_ctx* c) {
    if (c->mout.empty()) return 0;
    const MemberOut& l = c->mout.back();
    return l.gz_off + 18 + l.deflate_bytes;
}

// 10-byte header and 8-byte trailer of every member (deflate.rs:962-980),
// written into a host copy of the batch output that starts at `base`.
void frame_members(const gpz_ctx* c, size_t first, size_t count, uint8_t* dst, uint64_t base) {
    static const uint8_t hdr[10] = {0x1f, 0x8b, 0x08, 0x00, 0x00, 0x00, 0x00, 0x00, 0x00, 0xff};
    for (size_t m = first; m < first + count; m++) {
        const MemberOut& mo = c->mout[m];
        uint8_t* p = dst + (mo.gz_off - base);
        std::memcpy(p, hdr, 10);
        uint8_t* t = p + 10 + mo.deflate_bytes;
        for (int i = 0; i < 4; i++) t[i] = (uint8_t)(mo.crc >> (8 * i));
        for (int i = 0; i < 4; i++) t[4 + i] = (uint8_t)(mo.len >> (8 * i));
    }
}

// Host inputs -> one device pass -> host outputs.  Items must fit one batch.
int run_host_batch(gpz_ctx* c, const gpz_desc* d, size_t count, gpz_out* outs, uint32_t* pp_out = nullptr,
                   uint32_t* tok_out = nullptr, size_t* ntok = nullptr) {
    std::vector<Span> spans(count);
    size_t in_bytes = 0;
    for (size_t i = 0; i < count; i++) {
        spans[i].n = d[i].n;
        spans[i].dev_off = in_bytes;
        in_bytes += round_up(std::max<size_t>(d[i].n, 1), 16);
    }
    plan(c, spans);
    const size_t obound = out_bound_of_plan(c);
    int rc;
    if ((rc = reserve(c, in_bytes, true, true, obound))) return rc;
    if ((rc = ensure_host(c, c->h_in, c->h_in_cap, in_bytes + 64))) return rc;
    for (size_t i = 0; i < count; i++)
        if (d[i].n) std::memcpy(c->h_in + spans[i].dev_off, d[i].in, d[i].n);
    cudaStream_t s = c->stream;
    CU(c, cudaMemcpyAsync(c->d_in.p, c->h_in, in_bytes, cudaMemcpyHostToDevice, s));
    if ((rc = run_device(c, static_cast<const uint8_t*>(c->d_in.p), static_cast<uint8_t*>(c->d_out.p), s)))
        return rc;
    const uint64_t total = batch_out_bytes(c);
    if ((rc = ensure_host(c, c->h_out, c->h_out_cap, total + 64))) return rc;
    CU(c, cudaMemcpyAsync(c->h_out, c->d_out.p, total, cudaMemcpyDeviceToHost, s));
    if (pp_out && in_bytes) {
        // per-position tokens of input 0 (debug path: one input)
        CU(c, cudaMemcpyAsync(pp_out, c->d_pp.p, d[0].n * 4, cudaMemcpyDeviceToHost, s));
    }
    std::vector<uint32_t> tok_all, tntok;
    if (tok_out && ntok) {
        tok_all.resize(std::max<size_t>(d[0].n, 1));
        tntok.resize(std::max<size_t>(c->tiles.size(), 1));
        if (d[0].n) CU(c, cudaMemcpyAsync(tok_all.data(), c->d_tok.p, d[0].n * 4, cudaMemcpyDeviceToHost, s));
        if (!c->tiles.empty())
            CU(c, cudaMemcpyAsync(tntok.data(), c->d_tntok.p, c->tiles.size() * 4, cudaMemcpyDeviceToHost, s));
    }
    CU(c, cudaStreamSynchronize(s));
    frame_members(c, 0, c->members.size(), c->h_out, 0);
    int first_bad = GPZ_OK;
    for (size_t i = 0; i < count; i++) {
        const Span& sp = spans[i];
        const MemberOut& a = c->mout[sp.first_member];
        const MemberOut& z = c->mout[sp.first_member + sp.nmembers - 1];
        const uint64_t beg = a.gz_off, end = z.gz_off + 18 + z.deflate_bytes;
        outs[i].out_len = end - beg;
        if (!outs[i].out || outs[i].out_cap < end - beg) {
            outs[i].status = GPZ_E_SPACE;
            if (first_bad == GPZ_OK) first_bad = GPZ_E_SPACE;
            continue;
        }
        std::memcpy(outs[i].out, c->h_out + beg, end - beg);
        outs[i].status = GPZ_OK;
    }
    if (tok_out && ntok) {
        size_t k = 0;
        for (size_t t = 0; t < c->tiles.size(); t++) {
            const TileDesc& td = c->tiles[t];
            const MemberDesc& md = c->members[td.member];
            const uint32_t* src = tok_all.data() + md.in_off + ((size_t)td.seg << GPZ_SEG_LOG2);
            std::memcpy(tok_out + k, src, tntok[t] * 4);
            k += tntok[t];
        }
        *ntok = k;
    }
    if (first_bad != GPZ_OK) fail(c, first_bad, "output buffer too small");
    return first_bad;
}

// Split a list of items into device passes of at most batch_bytes input.
int run_host_items(gpz_ctx* c, const gpz_desc* d, size_t count, gpz_out* outs, bool plain) {
    int first_bad = GPZ_OK;
    size_t i = 0;
    while (i < count) {
        size_t j = i, bytes = 0;
        if (plain) {
            j = i + 1;
        } else {
            while (j < count && (j == i || bytes + d[j].n <= c->batch_bytes)) bytes += d[j++].n;
        }
        int rc = run_host_batch(c, d + i, j - i, outs + i);
        if (rc != GPZ_OK && rc != GPZ_E_SPACE) {
            for (size_t k = i; k < j; k++) outs[k].status = rc;
            return rc;
        }
        if (rc != GPZ_OK && first_bad == GPZ_OK) first_bad = rc;
        i = j;
    }
    return first_bad;
}

}  // namespace

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
    size_t mb = cfg->member_bytes ? cfg->member_bytes : kDefaultMember;
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
    if (cudaSetDevice(c->device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        gpz_kernel_smem_setup() != 0 || cudaMallocHost(reinterpret_cast<void**>(&c->h_err), 64) != cudaSuccess) {
        cudaGetLastError();
        gpz_destroy(c);
        return GPZ_E_CUDA;
    }
    if (c->flags & GPZ_FLAG_STAGE_TIMING)
        for (auto& e : c->ev)
            if (cudaEventCreate(&e) != cudaSuccess) {
                cudaGetLastError();
                gpz_destroy(c);
                return GPZ_E_CUDA;
            }
    *out = c;
    return GPZ_OK;
}

void gpz_destroy(gpz_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (DevArena* a : {&c->d_in, &c->d_pp, &c->d_tok, &c->d_out, &c->d_skeys, &c->d_son, &c->d_sposid,
                        &c->d_snkeys, &c->d_tentry, &c->d_texit, &c->d_thist,
                        &c->d_tntok, &c->d_tbit, &c->d_mcodes, &c->d_mhdr, &c->d_mout, &c->d_cnt, &c->d_members,
                        &c->d_tiles})
        if (a->p) cudaFree(a->p);
    if (c->h_in) cudaFreeHost(c->h_in);
    if (c->h_out) cudaFreeHost(c->h_out);
    if (c->h_members) cudaFreeHost(c->h_members);
    if (c->h_tiles) cudaFreeHost(c->h_tiles);
    if (c->h_mout) cudaFreeHost(c->h_mout);
    if (c->h_err) cudaFreeHost(c->h_err);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

size_t gpz_bound(size_t n) {
    size_t nm = n == 0 ? 1 : (n + kDefaultMember - 1) / kDefaultMember;
    return nm * member_bound(kDefaultMember);
}

size_t gpz_bound_ctx(const gpz_ctx* c, size_t n) {
    if (!c) return gpz_bound(n);
    size_t nm = n == 0 ? 1 : (n + c->member_bytes - 1) / c->member_bytes;
    return nm * member_bound(c->member_bytes);
}

int gpz_compress_chunk(gpz_ctx* c, const uint8_t* in, size_t n, int level, uint8_t* out, size_t out_cap,
                       size_t* out_len) {
    if (!c || (!in && n) || !out_len) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    gpz_desc d{in, n, level};
    gpz_out o{out, out_cap, 0, 0};
    int rc = run_host_batch(c, &d, 1, &o);
    *out_len = o.out_len;
    return rc;
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
    std::vector<Span> spans(count);
    size_t in_end = 0;
    for (size_t i = 0; i < count; i++) {
        if (in_off[i] % 16) return fail(c, GPZ_E_ARG, "device inputs must start 16-byte aligned");
        spans[i].n = in_len[i];
        spans[i].dev_off = in_off[i];
        in_end = std::max<size_t>(in_end, in_off[i] + round_up(std::max<uint64_t>(in_len[i], 1), 16));
    }
    plan(c, spans);
    if (out_bound_of_plan(c) > out_cap) return fail(c, GPZ_E_SPACE, "device output buffer below bound");
    int rc;
    if ((rc = reserve(c, in_end, false, false, 0))) return rc;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    if ((rc = run_device(c, static_cast<const uint8_t*>(d_in), static_cast<uint8_t*>(d_out), s))) return rc;
    for (size_t i = 0; i < count; i++) out_off[i] = c->mout[spans[i].first_member].gz_off;
    out_off[count] = batch_out_bytes(c);
    return GPZ_OK;
}

int gpz_frame_host(gpz_ctx* c, uint8_t* host_out, size_t cap) {
    if (!c || !host_out) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    if (batch_out_bytes(c) > cap) return GPZ_E_SPACE;
    frame_members(c, 0, c->mout.size(), host_out, 0);
    return GPZ_OK;
}

int gpz_debug_chunk(gpz_ctx* c, const uint8_t* in, size_t n, uint32_t* pp, uint32_t* tokens, size_t* ntok,
                    uint8_t* out, size_t out_cap, size_t* out_len) {
    if (!c || (!in && n)) return GPZ_E_ARG;
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
    int rc = run_host_batch(c, &d, 1, &o, pp, tokens, ntok);
    if (out_len) *out_len = o.out_len;
    return rc;
}

const char* gpz_strerror(int s) {
    switch (s) {
        case GPZ_OK: return "ok";
        case GPZ_E_NOMEM: return "out of device or pinned memory";
        case GPZ_E_ADMISSION: return "request exceeds the device pool cap";
        case GPZ_E_TIMEOUT: return "bounded device wait expired";
        case GPZ_E_CUDA: return "CUDA runtime error";
        case GPZ_E_ARG: return "invalid argument";
        case GPZ_E_SPACE: return "output buffer too small";
        case GPZ_E_INTERNAL: return "device self-check failed";
        case GPZ_E_BUSY: return "serving queue full";
        case GPZ_E_PENDING: return "result not ready";
        default: return "unknown status";
    }
}

const char* gpz_last_error(gpz_ctx* c) { return c ? c->last_err.c_str() : "no context"; }

int gpz_get_shape(gpz_ctx* c, gpz_shape* s) {
    if (!c || !s) return GPZ_E_ARG;
    s->lookup_threads = c->shape.lookup_threads;
    s->lookup_grid = c->shape.lookup_grid;
    s->walk_threads = c->shape.walk_threads;
    s->walk_grid = c->shape.walk_grid;
    s->emit_threads = c->shape.emit_threads;
    s->emit_grid = c->shape.emit_grid;
    return GPZ_OK;
}

int gpz_set_shape(gpz_ctx* c, const gpz_shape* s) {
    if (!c || !s) return GPZ_E_ARG;
    auto ok_t = [](int t) { return t == 256 || t == 512; };
    if (!(s->lookup_threads == 512 || s->lookup_threads == 1024) || !ok_t(s->walk_threads) || !ok_t(s->emit_threads) ||
        s->lookup_grid < 0 || s->walk_grid < 0 || s->emit_grid < 0)
        return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    c->shape = LaunchShape{s->lookup_threads, s->lookup_grid, s->walk_threads, s->walk_grid, s->emit_threads,
                           s->emit_grid};
    return GPZ_OK;
}

uint64_t gpz_last_launches(gpz_ctx* c) { return c ? c->launches : 0; }

int gpz_stage_times(gpz_ctx* c, float* ms4) {
    if (!c || !ms4 || !(c->flags & GPZ_FLAG_STAGE_TIMING)) return GPZ_E_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    for (int i = 0; i < 4; i++) ms4[i] = c->stage_ms[i];
    return GPZ_OK;
}

int gpz_submit(gpz_ctx*, const gpz_desc*, uint64_t*) { return GPZ_E_ARG; }
int gpz_poll(gpz_ctx*, uint64_t, gpz_out*, int) { return GPZ_E_ARG; }
int gpz_serve_stats_get(gpz_ctx*, gpz_serve_stats*) { return GPZ_E_ARG; }

}  // extern "C"
