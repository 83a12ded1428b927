// Host build of the member decoder in gpzip_b200/csrc/gpz_inflate_core.h
// with 32 host threads as the 32 lanes of a warp (lane_sync = a barrier), so
// that the lane-cooperative code of the device build (strided staging,
// table fills, match copies with distances below 32, flushes) runs and is
// checked on the CPU.  Same record format as inflate_host.cpp; every lane
// must return the same status.
#include <barrier>
#include <cstdio>
#include <thread>
#include <vector>

#define GPZI_HOST_LANES 1
#include "gpz_inflate_core.h"

static gpzi::Shared g_shared;

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    FILE* g = std::fopen(argv[2], "wb");
    if (!f || !g) return 2;
    constexpr int NL = 32;
    for (;;) {
        uint32_t hdr[2];
        if (std::fread(hdr, 4, 2, f) != 2) break;
        std::vector<uint8_t> in(hdr[0]), out(hdr[1]);
        if (hdr[0] && std::fread(in.data(), 1, hdr[0], f) != hdr[0]) return 3;
        std::barrier<> bar(NL);
        gpzi::g_lanes = &bar;
        uint32_t st[NL];
        std::vector<std::thread> th;
        for (int l = 0; l < NL; l++)
            th.emplace_back([&, l] {
                st[l] = gpzi::inflate_member<NL>(g_shared, (uint32_t)l, in.data(), hdr[0], out.data(), hdr[1]);
            });
        for (auto& t : th) t.join();
        for (int l = 1; l < NL; l++)
            if (st[l] != st[0]) return 4;  // lanes disagree
        // the token form on the same lanes: same status, same bytes
        std::vector<uint32_t> tok(hdr[1] + 1u);
        uint32_t nt = 0, st2[NL];
        std::vector<std::thread> th2;
        for (int l = 0; l < NL; l++)
            th2.emplace_back([&, l] {
                st2[l] = gpzi::inflate_member<NL, true>(g_shared, (uint32_t)l, in.data(), hdr[0], nullptr, hdr[1],
                                                        tok.data(), l == 0 ? &nt : nullptr);
            });
        for (auto& t : th2) t.join();
        for (int l = 0; l < NL; l++)
            if (st2[l] != st[0]) return 4;
        if (st[0] == gpzi::kOk) {
            std::vector<uint8_t> again(hdr[1]);
            gpzi::expand_tokens(tok.data(), nt, again.data());
            if (again != out) return 5;
        }
        const uint32_t n = st[0] == gpzi::kOk ? hdr[1] : 0u;
        std::fwrite(&st[0], 4, 1, g);
        std::fwrite(&n, 4, 1, g);
        if (n) std::fwrite(out.data(), 1, n, g);
    }
    std::fclose(f);
    std::fclose(g);
    return 0;
}
