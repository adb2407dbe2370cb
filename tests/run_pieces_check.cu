// Host-only check (no GPU) of the run postings' piece rules
// (stormbitmaps-internal_b200/csrc/run_pieces.cuh), the same functions the
// kernels call:
//  * list chunks (entries) and bitmap chunks (words, with the bits of the
//    neighbouring words as the kernels pass them) give the same pieces for
//    the same set, for every bin width 2^4 .. 2^15;
//  * the pieces are disjoint, lie inside one bin each, cover the set, and
//    are maximal (no two pieces of one bin touch);
//  * for pairs of random rows, the sum over bins of the overlaps of their
//    pieces equals |A & B|.
// Built and run by test_run_pieces_cpu.py.
#include <algorithm>
#include <cstdio>
#include <random>
#include <utility>
#include <vector>

#include "run_pieces.cuh"

using Piece = std::pair<uint32_t, uint32_t>;   // [first value, end)
static int g_fail = 0;

static std::vector<Piece> pieces_of_list(const std::vector<uint16_t>& l, uint32_t base, uint32_t wlog) {
    const uint32_t wmask = (1u << wlog) - 1u, nl = (uint32_t)l.size();
    std::vector<uint32_t> st, la;
    for (uint32_t e = 0; e < nl; ++e) {
        if (sb200::run_piece_start(l.data(), e, wmask)) st.push_back(base + l[e]);
        if (sb200::run_piece_last(l.data(), e, nl, wmask)) la.push_back(base + l[e] + 1);
    }
    std::vector<Piece> out;
    if (st.size() != la.size()) {
        std::printf("list: %zu starts, %zu ends\n", st.size(), la.size());
        ++g_fail;
        return out;
    }
    for (size_t k = 0; k < st.size(); ++k) out.push_back({st[k], la[k]});
    return out;
}

static std::vector<Piece> pieces_of_bitmap(const std::vector<uint64_t>& w, uint32_t base, uint32_t wlog) {
    std::vector<uint32_t> st, la;
    for (uint32_t k = 0; k < 1024; ++k) {
        const uint64_t cin = k ? w[k - 1] >> 63 : 0, nin = k + 1 < 1024 ? w[k + 1] & 1 : 0;
        uint64_t s, l;
        sb200::run_word_masks(w[k], cin, nin, k, wlog, s, l);
        for (int b = 0; b < 64; ++b) {
            if (s >> b & 1) st.push_back(base + k * 64 + b);
            if (l >> b & 1) la.push_back(base + k * 64 + b + 1);
        }
    }
    std::vector<Piece> out;
    if (st.size() != la.size()) {
        std::printf("bitmap: %zu starts, %zu ends\n", st.size(), la.size());
        ++g_fail;
        return out;
    }
    for (size_t k = 0; k < st.size(); ++k) out.push_back({st[k], la[k]});
    return out;
}

// A chunk's set (sorted chunk-local values) with runs, scattered values or both.
static std::vector<uint16_t> random_chunk(std::mt19937_64& g) {
    std::vector<uint8_t> bit(65536, 0);
    const int kind = (int)(g() % 4);
    const int runs = (int)(g() % 40);
    for (int r = 0; r < runs; ++r) {
        const uint32_t s = (uint32_t)(g() % 65536), len = 1 + (uint32_t)(g() % (kind == 0 ? 9000 : 300));
        for (uint32_t x = s; x < s + len && x < 65536; ++x) bit[x] = 1;
    }
    if (kind >= 2) {
        const uint32_t thr = (uint32_t)(g() % 1000);
        for (uint32_t x = 0; x < 65536; ++x)
            if (g() % 1000 < thr) bit[x] = 1;
    }
    if (kind == 3) bit[0] = bit[65535] = 1;
    std::vector<uint16_t> l;
    for (uint32_t x = 0; x < 65536; ++x)
        if (bit[x]) l.push_back((uint16_t)x);
    return l;
}

static void check_pieces(const std::vector<Piece>& p, const std::vector<uint16_t>& l, uint32_t base, uint32_t wlog,
                         const char* what) {
    std::vector<uint8_t> seen(65536, 0);
    for (size_t k = 0; k < p.size(); ++k) {
        const uint32_t s = p[k].first, e = p[k].second;
        if (!(s < e) || (s >> wlog) != ((e - 1) >> wlog) || s < base || e > base + 65536) {
            std::printf("%s: piece [%u, %u) not inside one bin of 2^%u\n", what, s, e, wlog);
            ++g_fail;
            return;
        }
        if (k && p[k - 1].second == s && (s & ((1u << wlog) - 1u)) != 0) {
            std::printf("%s: pieces [.., %u) and [%u, ..) touch inside a bin\n", what, s, s);
            ++g_fail;
            return;
        }
        for (uint32_t x = s; x < e; ++x) {
            if (seen[x - base]) {
                std::printf("%s: value %u in two pieces\n", what, x);
                ++g_fail;
                return;
            }
            seen[x - base] = 1;
        }
    }
    size_t covered = 0;
    for (uint16_t v : l) covered += seen[v];
    size_t total = 0;
    for (uint8_t b : seen) total += b;
    if (covered != l.size() || total != l.size()) {
        std::printf("%s: pieces cover %zu values, the set has %zu\n", what, total, l.size());
        ++g_fail;
    }
}

int main() {
    std::mt19937_64 g(20261204);
    const uint32_t base = 3u << 16;
    std::vector<std::vector<uint16_t>> chunks;
    for (int t = 0; t < 40; ++t) chunks.push_back(random_chunk(g));
    for (uint32_t wlog = 4; wlog <= 15; ++wlog) {
        std::vector<std::vector<Piece>> ps;
        for (const auto& l : chunks) {
            std::vector<uint64_t> w(1024, 0);
            for (uint16_t v : l) w[v >> 6] |= 1ull << (v & 63);
            const auto a = pieces_of_list(l, base, wlog), b = pieces_of_bitmap(w, base, wlog);
            if (a != b) {
                std::printf("wlog %u: list and bitmap pieces differ (%zu vs %zu)\n", wlog, a.size(), b.size());
                ++g_fail;
            }
            check_pieces(a, l, base, wlog, "list");
            ps.push_back(a);
        }
        // overlaps summed over bins against the intersection
        for (size_t i = 0; i + 1 < chunks.size(); i += 3) {
            const size_t j = i + 1;
            uint64_t ov = 0;
            for (const Piece& p : ps[i])
                for (const Piece& q : ps[j]) {
                    if ((p.first >> wlog) != (q.first >> wlog)) continue;
                    const uint32_t s = std::max(p.first, q.first), e = std::min(p.second, q.second);
                    if (e > s) ov += e - s;
                }
            std::vector<uint16_t> both;
            std::set_intersection(chunks[i].begin(), chunks[i].end(), chunks[j].begin(), chunks[j].end(),
                                  std::back_inserter(both));
            if (ov != both.size()) {
                std::printf("wlog %u: overlaps %llu, intersection %zu\n", wlog, (unsigned long long)ov, both.size());
                ++g_fail;
            }
        }
    }
    if (g_fail) {
        std::printf("FAIL\n");
        return 1;
    }
    std::printf("%zu chunks x 12 bin widths: pieces agree and are exact\nok\n", chunks.size());
    return 0;
}
