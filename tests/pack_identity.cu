// Host-only check (no GPU) that the threaded bulk packer of STORM_t rows,
// sb200::ChunkPack::add_rows, lays out exactly what add_row produces one row
// at a time: CSR offsets, chunk ids, kinds and lengths, offsets, the bitmap
// pool, the list pool (including its 8-entry alignment padding), the per-row
// facts and the largest chunk id. Rows come from the library's own STORM_add
// and STORM_bitmap_cont_add, plus hand-made chunks the public layout allows
// (short bitmaps, NULL data, NULL lists). Built and run by test_pack_cpu.py.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "chunk_engine.cuh"

using sb200::ChunkPack;

static int g_fail = 0;

template <class V1, class V2>
static void same(const char* what, const V1& a, const V2& b) {
    if (a.size() != b.size()) {
        std::printf("%s: size %zu vs %zu\n", what, (size_t)a.size(), (size_t)b.size());
        ++g_fail;
        return;
    }
    for (size_t i = 0; i < a.size(); ++i)
        if (a[i] != b[i]) {
            std::printf("%s: entry %zu differs\n", what, i);
            ++g_fail;
            return;
        }
}

static void compare(const char* name, const ChunkPack& a, const ChunkPack& b) {
    same("row_off", a.row_off, b.row_off);
    same("cid", a.cid, b.cid);
    same("ckl", a.ckl, b.ckl);
    same("coff", a.coff, b.coff);
    same("bm", a.bm, b.bm);
    same("lst", a.lst, b.lst);
    if (a.facts.size() != b.facts.size()) {
        std::printf("facts: size\n");
        ++g_fail;
    } else {
        for (size_t r = 0; r < a.facts.size(); ++r) {
            const auto &x = a.facts[r], &y = b.facts[r];
            if (x.card != y.card || x.list_entries != y.list_entries || x.chunks != y.chunks ||
                x.bitmap_chunks != y.bitmap_chunks || x.plain != y.plain || x.runs != y.runs) {
                std::printf("facts: row %zu differs\n", r);
                ++g_fail;
                break;
            }
        }
    }
    if (a.max_cid != b.max_cid) {
        std::printf("max_cid differs\n");
        ++g_fail;
    }
    std::printf("%s: %zu rows, %zu chunks, %zu bitmap words, %zu list entries%s\n", name, (size_t)a.rows(),
                a.cid.size(), a.bm.size(), a.lst.size(), g_fail ? "  MISMATCH" : "");
}

static void check(const char* name, const STORM_t* s, uint32_t split) {
    ChunkPack one, bulk;
    for (uint32_t r = 0; r < s->n_conts; ++r) one.add_row(&s->conts[r]);
    // the first `split` rows row by row (leaves the list pool unaligned), the rest in bulk
    for (uint32_t r = 0; r < split && r < s->n_conts; ++r) bulk.add_row(&s->conts[r]);
    if (split < s->n_conts) bulk.add_rows(s->conts + split, s->n_conts - split);
    compare(name, one, bulk);
}

int main() {
    std::mt19937_64 g(20261204);
    // 1. a mixed corpus large enough for several packing threads
    STORM_t* s = STORM_new();
    std::vector<uint32_t> v;
    for (uint32_t r = 0; r < 3000; ++r) {
        v.clear();
        const uint32_t kind = r % 5;
        const uint32_t universe = 1u << 22;
        if (kind == 0) {                      // empty row
        } else if (kind == 1) {               // sparse: list chunks
            for (uint32_t k = 0; k < 1 + g() % 300; ++k) v.push_back((uint32_t)(g() % universe));
        } else if (kind == 2) {               // dense in a few chunks: bitmap chunks
            const uint32_t base = (uint32_t)(g() % 60) << 16;
            for (uint32_t x = base; x < base + (3u << 16); x += 1 + g() % 9) v.push_back(x);
        } else if (kind == 3) {               // repeated values inside list chunks
            for (uint32_t k = 0; k < 50; ++k) {
                const uint32_t x = (uint32_t)(g() % universe);
                v.push_back(x);
                if (k % 7 == 0) v.push_back(x);
            }
        } else {                              // around the 4096-value list/bitmap cut
            const uint32_t base = (uint32_t)(g() % 60) << 16;
            const uint32_t cnt = 4090 + (uint32_t)(g() % 12);
            for (uint32_t k = 0; k < cnt; ++k) v.push_back(base + k * 16);
        }
        std::sort(v.begin(), v.end());
        STORM_add(s, v.data(), (uint32_t)v.size());
    }
    // appends through the public struct: a repeated chunk id in some rows
    for (uint32_t r = 1; r < 3000; r += 97) {
        uint32_t x[3] = {s->conts[r].prev_inserted_value + 1, s->conts[r].prev_inserted_value + 5,
                         s->conts[r].prev_inserted_value + 9};
        STORM_bitmap_cont_add(&s->conts[r], x, 3);
    }
    check("mixed", s, 0);
    check("mixed, 7 rows first", s, 7);
    check("mixed, all but 1 row first", s, 2999);

    // 2. hand-made chunks the public layout allows
    static uint64_t words[1024];
    for (uint32_t i = 0; i < 1024; ++i) words[i] = g();
    static uint16_t list[5] = {1, 2, 2, 9, 70};
    STORM_bitmap_t ch[5];
    std::memset(ch, 0, sizeof(ch));
    ch[0].data = words; ch[0].n_bitmap = 10; ch[0].n_bits_set = 77;          // short bitmap
    ch[1].data = nullptr; ch[1].n_bitmap = 1024; ch[1].n_bits_set = 5;       // bitmap without data
    ch[2].scalar = nullptr; ch[2].n_scalar = 5;                              // list without entries
    ch[3].scalar = list; ch[3].n_scalar = 5;                                 // list with a repeat
    ch[4].data = words; ch[4].n_bitmap = 1024; ch[4].n_bits_set = 1000;     // full bitmap
    uint32_t ids[5] = {0, 3, 3, 4, 9};
    STORM_bitmap_cont_t conts[3];
    std::memset(conts, 0, sizeof(conts));
    conts[0].bitmaps = ch; conts[0].block_ids = ids; conts[0].n_bitmaps = 5;
    conts[2].bitmaps = ch + 2; conts[2].block_ids = ids + 2; conts[2].n_bitmaps = 2;
    STORM_t hand;
    hand.conts = conts; hand.n_conts = 3; hand.m_conts = 3;
    check("hand-made", &hand, 0);
    check("hand-made, 1 row first", &hand, 1);
    STORM_free(s);
    if (g_fail) {
        std::printf("FAIL\n");
        return 1;
    }
    std::printf("identical\n");
    return 0;
}
