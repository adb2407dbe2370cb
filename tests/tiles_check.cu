// Host-only checks (no GPU) of the bitmap x bitmap engine's planning:
//  * sb200::build_tiles -- for each tiling (128 x 256 tcgen05, 128 x 192
//    double-buffered tcgen05, 128 x 128 POPC) every pair i <= j < n lies in
//    exactly one tile, tiles are ordered by A block and every A block has one;
//  * sb200::host_panels -- the panels partition the tile list from its end,
//    whole waves but the last, one launch for short lists;
//  * the host-output plan built on them (the rule DenseEngine::panels_to_host
//    follows): after each panel the rows whose A blocks are complete are
//    copied, the copies tile the packed triangle from its end exactly once,
//    and each panel's tiles read only rows already uploaded when rows arrive
//    in chunks last-first.
// Built and run by test_tiles_cpu.py.
#include <cstdio>
#include <vector>

#include "dense.cuh"

static int g_fail = 0;
#define CHECK(c, ...)                      \
    do {                                   \
        if (!(c)) {                        \
            std::printf(__VA_ARGS__);      \
            std::printf("\n");             \
            ++g_fail;                      \
            return;                        \
        }                                  \
    } while (0)

static uint32_t tile_bn(int kind) {
    return kind == STORM_B200_KERNEL_POPC ? 128u : kind == STORM_B200_KERNEL_MMA_DB ? 192u : 256u;
}

static void check_cover(int kind, uint64_t n) {
    std::vector<uint2> t;
    sb200::build_tiles(t, n, kind);
    const uint64_t bm = 128, bn = tile_bn(kind);
    std::vector<uint8_t> seen(n * n, 0);
    uint32_t prev_bi = 0;
    std::vector<uint8_t> has_block((n + bm - 1) / bm, 0);
    for (size_t k = 0; k < t.size(); ++k) {
        CHECK(k == 0 || t[k].x >= prev_bi, "kind %d n %llu: tiles not ordered by A block", kind,
              (unsigned long long)n);
        prev_bi = t[k].x;
        CHECK(t[k].x < has_block.size(), "kind %d: A block out of range", kind);
        has_block[t[k].x] = 1;
        bool any = false;
        for (uint64_t i = t[k].x * bm; i < (t[k].x + 1) * bm && i < n; ++i)
            for (uint64_t j = t[k].y * bn; j < (t[k].y + 1) * bn && j < n; ++j)
                if (i <= j) {
                    ++seen[i * n + j];
                    any = true;
                }
        CHECK(any, "kind %d n %llu: tile (%u, %u) holds no pair", kind, (unsigned long long)n, t[k].x, t[k].y);
    }
    for (uint64_t i = 0; i < n; ++i)
        for (uint64_t j = i; j < n; ++j)
            CHECK(seen[i * n + j] == 1, "kind %d n %llu: pair (%llu, %llu) covered %d times", kind,
                  (unsigned long long)n, (unsigned long long)i, (unsigned long long)j, seen[i * n + j]);
    for (size_t b = 0; b < has_block.size(); ++b) CHECK(has_block[b], "kind %d: A block %zu has no tile", kind, b);
}

static void check_plan(int kind, uint64_t n, uint32_t wave) {
    std::vector<uint2> t;
    sb200::build_tiles(t, n, kind);
    const uint64_t bm = 128, bn = tile_bn(kind);
    const auto panels = sb200::host_panels((uint32_t)t.size(), wave);
    std::vector<uint32_t> first_tile(t.back().x + 1, 0);
    for (uint32_t k = (uint32_t)t.size(); k-- > 0;) first_tile[t[k].x] = k;
    const uint64_t chunk = (std::max<uint64_t>(1, (n + 31) / 32) + 127) / 128 * 128;
    uint64_t expect_hi = t.size(), copied_from = n, uploaded_from = n;
    auto tri = [n](uint64_t r) { return r * n - (r * (r - 1)) / 2; };
    uint64_t copied_entries = 0;
    for (size_t p = 0; p < panels.size(); ++p) {
        const uint32_t t0 = panels[p].first, t1 = panels[p].second;
        CHECK(t1 == expect_hi && t0 < t1, "plan kind %d n %llu: panel %zu does not continue the list", kind,
              (unsigned long long)n, p);
        CHECK(p + 1 == panels.size() || (t1 - t0) % wave == 0, "plan: panel %zu is not whole waves", p);
        expect_hi = t0;
        uint64_t need = n;
        for (uint32_t k = t0; k < t1; ++k) need = std::min<uint64_t>(need, std::min(t[k].x * bm, t[k].y * bn));
        const uint64_t c = need / chunk;
        uploaded_from = std::min(uploaded_from, c * chunk);   // chunks c .. last are resident
        for (uint32_t k = t0; k < t1; ++k)
            CHECK(t[k].x * bm >= uploaded_from && t[k].y * bn >= uploaded_from,
                  "plan: tile %u reads rows not yet uploaded", k);
        uint64_t b = t[t0].x;
        if (first_tile[b] != t0) ++b;
        const uint64_t r = std::min<uint64_t>(n, b * bm);
        if (r < copied_from) {
            for (uint64_t k = 0; k < t.size(); ++k)
                if (t[k].x >= b) CHECK(k >= t0, "plan: rows copied before tile %llu ran", (unsigned long long)k);
            copied_entries += tri(copied_from) - tri(r);
            copied_from = r;
        }
    }
    CHECK(expect_hi == 0 && copied_from == 0, "plan kind %d n %llu: list or triangle not covered", kind,
          (unsigned long long)n);
    CHECK(copied_entries == n * (n + 1) / 2, "plan: copies do not add up to the triangle");
}

int main() {
    const int kinds[3] = {STORM_B200_KERNEL_MMA, STORM_B200_KERNEL_MMA_DB, STORM_B200_KERNEL_POPC};
    const uint64_t sizes[] = {1, 2, 127, 128, 129, 191, 192, 193, 255, 256, 257, 383, 384, 385, 640, 1000, 2049};
    for (int kind : kinds)
        for (uint64_t n : sizes) check_cover(kind, n);
    // panel partition alone, over list lengths around the wave multiples
    for (uint32_t wave : {1u, 7u, 148u, 296u})
        for (uint32_t nt : {1u, 5u, 148u, 591u, 592u, 593u, 1331u, 6319u, 65792u, 88064u}) {
            const auto p = sb200::host_panels(nt, wave);
            uint64_t hi = nt;
            for (size_t k = 0; k < p.size(); ++k) {
                if (p[k].second != hi || p[k].first >= p[k].second) {
                    std::printf("panels wave %u tiles %u: not a partition\n", wave, nt);
                    ++g_fail;
                    break;
                }
                hi = p[k].first;
            }
            if (hi != 0) {
                std::printf("panels wave %u tiles %u: list not covered\n", wave, nt);
                ++g_fail;
            }
            if (nt <= 4ull * wave && p.size() != 1) {
                std::printf("panels wave %u tiles %u: short list split\n", wave, nt);
                ++g_fail;
            }
        }
    // the whole host-output plan, at sizes that give one to forty panels
    for (int kind : kinds)
        for (uint64_t n : {1ull, 300ull, 4096ull, 9000ull, 20000ull, 65536ull})
            check_plan(kind, n, kind == STORM_B200_KERNEL_POPC ? 296u : 148u);
    if (g_fail) {
        std::printf("FAIL (%d)\n", g_fail);
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
