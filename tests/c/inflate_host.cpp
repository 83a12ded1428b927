// Host build of the member decoder in gpzip_b200/csrc/gpz_inflate_core.h
// (one lane), for the CPU tests: reads records [u32 deflate bytes][u32
// ISIZE][bytes] from argv[1] and writes [u32 status][u32 bytes][output] per
// record to argv[2].  Every record is also decoded in the token form, which
// must agree (exit code 4: status, 5: bytes).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gpz_inflate_core.h"

static gpzi::Shared g_shared;

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    FILE* g = std::fopen(argv[2], "wb");
    if (!f || !g) return 2;
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
        const uint32_t n = st == gpzi::kOk ? hdr[1] : 0u;
        std::fwrite(&st, 4, 1, g);
        std::fwrite(&n, 4, 1, g);
        if (n) std::fwrite(out.data(), 1, n, g);
    }
    std::fclose(f);
    std::fclose(g);
    return 0;
}
