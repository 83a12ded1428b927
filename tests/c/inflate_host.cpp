// Host build of the member decoder in gpzip_b200/csrc/gpz_inflate_core.h
// (one lane), for the CPU tests: reads records [u32 deflate bytes][u32
// ISIZE][bytes] from argv[1] and writes [u32 status][u32 bytes][output] per
// record to argv[2].  Every record is also decoded in the token form, which
// must agree (exit code 4: status, 5: bytes), and by the parallel decode of
// single-block members with 1, 7 and 128 lanes, which may leave a member to
// the serial decoder but must never take a member the serial decoder
// rejects, nor give other tokens (exit code 6).  stderr gets
// "parallel: <taken> of <records>".
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gpz_inflate_core.h"

static gpzi::Shared g_shared;
static gpzi::Shared g_par;

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    FILE* g = std::fopen(argv[2], "wb");
    if (!f || !g) return 2;
    unsigned long taken = 0, records = 0;
    for (;;) {
        uint32_t hdr[2];
        if (std::fread(hdr, 4, 2, f) != 2) break;
        std::vector<uint8_t> in(hdr[0]), out(hdr[1]);
        if (hdr[0] && std::fread(in.data(), 1, hdr[0], f) != hdr[0]) return 3;
        const uint32_t st = gpzi::inflate_member<1>(g_shared, 0, in.data(), hdr[0], out.data(), hdr[1]);
        // the token form must return the same status, and its tokens must
        // expand to the same bytes
        std::vector<uint32_t> tok(hdr[1] + 1u);
        uint32_t nt = 0;
        const uint32_t st2 =
            gpzi::inflate_member<1, true>(g_shared, 0, in.data(), hdr[0], nullptr, hdr[1], tok.data(), &nt);
        if (st2 != st) return 4;
        if (st == gpzi::kOk) {
            if (nt > hdr[1]) return 5;
            std::vector<uint8_t> again(hdr[1]);
            gpzi::expand_tokens(tok.data(), nt, again.data());
            if (again != out) return 5;
        }
        for (uint32_t lanes : {1u, 7u, 128u}) {
            std::vector<uint32_t> ptok(hdr[1] + 1u);
            uint32_t pn = 0;
            if (!gpzi::inflate_member_par(g_par, in.data(), hdr[0], hdr[1], lanes, ptok.data(), &pn)) continue;
            if (st != gpzi::kOk || pn != nt) return 6;
            for (uint32_t i = 0; i < nt; i++)
                if (ptok[i] != tok[i]) return 6;
            if (lanes == 128u) taken++;
        }
        records++;
        const uint32_t n = st == gpzi::kOk ? hdr[1] : 0u;
        std::fwrite(&st, 4, 1, g);
        std::fwrite(&n, 4, 1, g);
        if (n) std::fwrite(out.data(), 1, n, g);
    }
    std::fclose(f);
    std::fclose(g);
    std::fprintf(stderr, "parallel: %lu of %lu\n", taken, records);
    return 0;
}
