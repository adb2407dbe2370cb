/*
 * ref_harness.cpp -- C entry points into the StormBitmaps reference itself.
 *
 * TEST AND BASELINE INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file
 * together with the reference's own sources (storm.cpp, kernels/*.cpp) into
 * oracle/_ref/libstorm_ref.so.  It is used for two things and nothing else:
 *   1. generating the golden vectors in tests/golden/ that pin the oracle
 *      (tests/golden/make_golden.py), and
 *   2. bench.py's reference arm: the reference's own CPU code, timed on the
 *      host cores.
 * It adds no algorithm of its own: every count comes out of a reference
 * function (named in each comment).  The multi-threaded loop in
 * ref_contig_matrix_mt is a harness that splits the pair loop over threads and
 * calls the reference's AND+popcount kernel per pair, the kernel
 * STORM_contig_pairw_intersect_cardinality dispatches to (storm.cpp:1155,
 * selected by STORM_get_intersect_count_func, libalgebra.h:3105).
 */
#include "storm.h"
#include "kernels/storm_repr.h"
#include "kernels/storm_cells.h"
#include "kernels/storm_cost.h"
#include "kernels/storm_allpairs.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

extern "C" {

/* Reference STORM_contiguous_t end to end: add each row by its set positions
 * and return STORM_contig_pairw_intersect_cardinality (storm.cpp:1232).
 * blocked > 0 uses the _blocked variant (storm.cpp:1248). */
uint64_t ref_contig_sum(const uint64_t* words, uint64_t n, uint64_t nw, uint64_t vector_length,
                        uint32_t blocked) {
    STORM_contiguous_t* c = STORM_contig_new(vector_length);
    std::vector<uint32_t> pos;
    for (uint64_t r = 0; r < n; ++r) {
        pos.clear();
        for (uint64_t k = 0; k < nw; ++k) {
            uint64_t w = words[r * nw + k];
            while (w) {
                pos.push_back((uint32_t)(k * 64 + __builtin_ctzll(w)));
                w &= w - 1;
            }
        }
        STORM_contig_add(c, pos.data(), (uint32_t)pos.size());
    }
    const uint64_t s = blocked ? STORM_contig_pairw_intersect_cardinality_blocked(c, blocked)
                               : STORM_contig_pairw_intersect_cardinality(c);
    STORM_contig_free(c);
    return s;
}

/* Per-pair counts with the reference's bitmap kernel, rows [r0, r1) of the
 * packed upper triangle, split over `threads` host threads.  Returns the sum
 * over i < j of the processed rows.  The traversal is the reference's cache
 * blocking (STORM_contig_pairw_intersect_cardinality_blocked,
 * storm.cpp:1248-1281): a thread takes a block of REF_BLOCK rows i and walks
 * every row j >= the block's first row once, pairing it with each row of the
 * block, so the block's rows stay in cache and each j row is read once per
 * block instead of once per row. */
static const uint64_t REF_BLOCK = 16;

uint64_t ref_contig_matrix_mt(const uint64_t* words, uint64_t n, uint64_t nw, uint64_t r0,
                              uint64_t r1, uint32_t* out, uint32_t threads) {
    const STORM_compute_func f = STORM_get_intersect_count_func(nw);
    if (threads == 0) threads = 1;
    if (r1 > n) r1 = n;
    std::atomic<uint64_t> next(r0), total(0);
    auto work = [&]() {
        uint64_t local = 0;
        for (;;) {
            const uint64_t i0 = next.fetch_add(REF_BLOCK);
            if (i0 >= r1) break;
            const uint64_t i1 = std::min(r1, i0 + REF_BLOCK);
            for (uint64_t j = i0; j < n; ++j) {
                const uint64_t* wj = words + j * nw;
                const uint64_t ie = std::min(i1, j + 1);   // rows i <= j of the block
                for (uint64_t i = i0; i < ie; ++i) {
                    const uint64_t c = (*f)(words + i * nw, wj, nw);
                    if (out) out[i * n - (i * (i - 1)) / 2 - i + j] = (uint32_t)c;
                    if (j > i) local += c;
                }
            }
        }
        total.fetch_add(local);
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return total.load();
}

/* Reference STORM_t end to end: STORM_add per row, then
 * STORM_pairw_intersect_cardinality (storm.cpp:927) or the blocked form
 * (storm.cpp:947). */
uint64_t ref_storm_sum(const uint32_t* values, const uint64_t* offsets, uint64_t n, uint32_t blocked) {
    STORM_t* s = STORM_new();
    for (uint64_t r = 0; r < n; ++r)
        STORM_add(s, values + offsets[r], (uint32_t)(offsets[r + 1] - offsets[r]));
    const uint64_t v = blocked ? STORM_pairw_intersect_cardinality_blocked(s, blocked)
                               : STORM_pairw_intersect_cardinality(s);
    STORM_free(s);
    return v;
}

/* The same, with the wall time of the all-pairs call alone (ingest not
 * counted) in *seconds: the CPU baseline of the STORM_t forms. */
uint64_t ref_storm_sum_timed(const uint32_t* values, const uint64_t* offsets, uint64_t n, double* seconds) {
    STORM_t* s = STORM_new();
    for (uint64_t r = 0; r < n; ++r)
        STORM_add(s, values + offsets[r], (uint32_t)(offsets[r + 1] - offsets[r]));
    const auto t0 = std::chrono::steady_clock::now();
    const uint64_t v = STORM_pairw_intersect_cardinality(s);
    const auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    STORM_free(s);
    return v;
}

/* A harness over the reference's own per-pair STORM_t call: the pair loop of
 * STORM_pairw_intersect_cardinality (storm.cpp:927-945) split over threads
 * (rows handed out one at a time from a shared counter), each thread with
 * its own scratch buffer, calling STORM_bitmap_cont_intersect_cardinality_
 * premade with the kernel STORM_get_intersect_count_func selects. Returns
 * the same sum; *seconds = wall time of the pair loop alone. */
uint64_t ref_storm_sum_mt(const uint32_t* values, const uint64_t* offsets, uint64_t n, uint32_t threads,
                          double* seconds) {
    STORM_t* s = STORM_new();
    for (uint64_t r = 0; r < n; ++r)
        STORM_add(s, values + offsets[r], (uint32_t)(offsets[r + 1] - offsets[r]));
    if (threads == 0) threads = 1;
    const STORM_compute_func f = STORM_get_intersect_count_func((uint32_t)(STORM_DEFAULT_BLOCK_SIZE / 64));
    std::atomic<uint64_t> next(0), total(0);
    const auto t0 = std::chrono::steady_clock::now();
    auto work = [&]() {
        std::vector<uint32_t> out(2 * STORM_DEFAULT_SCALAR_THRESHOLD);
        uint64_t local = 0;
        for (;;) {
            const uint64_t i = next.fetch_add(1);
            if (i >= s->n_conts) break;
            for (uint64_t j = i + 1; j < s->n_conts; ++j)
                local += STORM_bitmap_cont_intersect_cardinality_premade(&s->conts[i], &s->conts[j], f, out.data());
        }
        total += local;
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < threads; ++t) pool.emplace_back(work);
    for (auto& th : pool) th.join();
    const auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    STORM_free(s);
    return total.load();
}

/* Reference rectangular form (storm.cpp:1027). */
uint64_t ref_storm_square(const uint32_t* xv, const uint64_t* xo, uint64_t nx,
                          const uint32_t* yv, const uint64_t* yo, uint64_t ny) {
    STORM_t* a = STORM_new();
    STORM_t* b = STORM_new();
    for (uint64_t r = 0; r < nx; ++r) STORM_add(a, xv + xo[r], (uint32_t)(xo[r + 1] - xo[r]));
    for (uint64_t r = 0; r < ny; ++r) STORM_add(b, yv + yo[r], (uint32_t)(yo[r + 1] - yo[r]));
    const uint64_t v = STORM_intersect_cardinality_square(a, b);
    STORM_free(a);
    STORM_free(b);
    return v;
}

/* Per-pair counts of one STORM_t pair via STORM_bitmap_cont_intersect_cardinality
 * (storm.cpp:804), packed upper triangle including the diagonal. */
uint64_t ref_storm_matrix(const uint32_t* values, const uint64_t* offsets, uint64_t n, uint32_t* out) {
    STORM_t* s = STORM_new();
    for (uint64_t r = 0; r < n; ++r)
        STORM_add(s, values + offsets[r], (uint32_t)(offsets[r + 1] - offsets[r]));
    uint64_t sum = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t base = i * n - (i * (i - 1)) / 2 - i;
        for (uint64_t j = i; j < n; ++j) {
            const uint64_t c = STORM_bitmap_cont_intersect_cardinality(&s->conts[i], &s->conts[j]);
            out[base + j] = (uint32_t)c;
            if (j > i) sum += c;
        }
    }
    STORM_free(s);
    return sum;
}

/* The chunk layout STORM_add builds for one row (storm.cpp:737-803):
 * ids, kind (1 = bitmap chunk, 0 = list chunk) and n_bits_set per chunk. */
uint32_t ref_storm_layout(const uint32_t* values, uint32_t n, uint32_t* ids, uint8_t* kinds,
                          uint32_t* cards) {
    STORM_t* s = STORM_new();
    STORM_add(s, values, n);
    const STORM_bitmap_cont_t& c = s->conts[0];
    for (uint32_t k = 0; k < c.n_bitmaps; ++k) {
        ids[k] = c.block_ids[k];
        kinds[k] = c.bitmaps[k].n_bitmap ? 1 : 0;
        cards[k] = c.bitmaps[k].n_bits_set;
    }
    const uint32_t nb = c.n_bitmaps;
    STORM_free(s);
    return nb;
}

/* Low-level reference kernels, exported unchanged for golden vectors. */
uint64_t ref_vector16(const uint16_t* a, const uint16_t* b, uint32_t na, uint32_t nb) {
    return STORM_intersect_vector16_cardinality(a, b, na, nb);
}
uint64_t ref_vector32(const uint32_t* a, const uint32_t* b, uint32_t na, uint32_t nb, uint32_t* out) {
    return STORM_intersect_vector32_unsafe(a, b, na, nb, out);
}
uint64_t ref_bitmaps_scalar_list(const uint64_t* b1, const uint64_t* b2, const uint32_t* l1,
                                 const uint32_t* l2, uint32_t n1, uint32_t n2) {
    return STORM_intersect_bitmaps_scalar_list(b1, b2, l1, l2, n1, n2);
}
uint64_t ref_wrapper_diag(uint32_t n, const uint64_t* vals, uint32_t n_ints, uint32_t block) {
    const STORM_compute_func f = STORM_get_intersect_count_func(n_ints);
    return block ? STORM_wrapper_diag_blocked(n, vals, n_ints, f, block)
                 : STORM_wrapper_diag(n, vals, n_ints, f);
}

/* ---- kernel layer (kernels/) ------------------------------------------ */
static void build_rows(std::vector<storm::Row>& rows, const uint32_t* values, const uint64_t* offsets,
                       uint64_t n, uint32_t universe) {
    rows.resize(n);
    for (uint64_t r = 0; r < n; ++r)
        storm::build_row(rows[r], values + offsets[r], offsets[r + 1] - offsets[r], universe);
}

/* storm::allpairs_sum (storm_allpairs.cpp:486) with the default model.
 * stats[0..3] = sum, pairs, skipped, decisions. */
void ref_allpairs_sum(const uint32_t* values, const uint64_t* offsets, uint64_t n, uint32_t universe,
                      uint32_t policy, uint32_t tile, uint64_t* stats) {
    std::vector<storm::Row> rows;
    build_rows(rows, values, offsets, n, universe);
    storm::CostModel m;
    storm::default_model(m);
    const storm::AllPairsStats st = storm::allpairs_sum(rows, m, (storm::Policy)policy, tile);
    stats[0] = st.sum;
    stats[1] = st.pairs;
    stats[2] = st.skipped;
    stats[3] = st.decisions;
}

struct TileSink { uint32_t tile; uint64_t n; uint32_t* out; };
static void tile_sink(uint32_t i0, uint32_t j0, uint32_t nr, uint32_t nc, const uint32_t* counts,
                      void* vp) {
    TileSink* s = (TileSink*)vp;
    for (uint32_t a = 0; a < nr; ++a)
        for (uint32_t b = 0; b < nc; ++b) {
            const uint64_t i = i0 + a, j = j0 + b;
            if (j <= i) continue;
            s->out[i * s->n - (i * (i - 1)) / 2 + (j - i)] = counts[(size_t)a * s->tile + b];
        }
}

/* storm::allpairs_tiles (storm_allpairs.cpp:677) under Policy::AllBitmap
 * (identity row order, so tile coordinates are original rows), scattered into
 * the packed strict upper triangle.  Returns the stats sum. */
uint64_t ref_allpairs_tiles(const uint32_t* values, const uint64_t* offsets, uint64_t n,
                            uint32_t universe, uint32_t tile, uint32_t* out) {
    std::vector<storm::Row> rows;
    build_rows(rows, values, offsets, n, universe);
    storm::CostModel m;
    storm::default_model(m);
    TileSink s{tile, n, out};
    const storm::AllPairsStats st =
        storm::allpairs_tiles(rows, m, storm::Policy::AllBitmap, tile_sink, &s, tile);
    return st.sum;
}

/* kernels/oracle.cpp:28 on one pair. */
uint64_t ref_oracle_intersect(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb,
                              uint32_t universe) {
    storm::Row ra, rb;
    storm::build_row(ra, a, na, universe);
    storm::build_row(rb, b, nb, universe);
    return storm::oracle_intersect(ra, rb);
}

/* Representations built by storm::build_row (storm_repr.cpp:102-207).
 * Returns counts in sizes[0..5] = runs, ewah words, rank words, occ words,
 * complement list length, complement runs; meta[0..7] as RowMeta. */
void ref_build_row(const uint32_t* v, uint64_t n, uint32_t universe, uint32_t* run_start,
                   uint32_t* run_end, uint64_t* ewah, uint64_t* rank, uint64_t* occ,
                   uint32_t* comp, uint64_t* sizes, uint32_t* meta) {
    storm::Row r;
    storm::build_row(r, v, n, universe);
    sizes[0] = r.run_start.size();
    sizes[1] = r.ewah.size();
    sizes[2] = r.rank.size();
    sizes[3] = r.occ.size();
    sizes[4] = r.comp_list.size();
    sizes[5] = r.comp_start.size();
    if (run_start) std::copy(r.run_start.begin(), r.run_start.end(), run_start);
    if (run_end) std::copy(r.run_end.begin(), r.run_end.end(), run_end);
    if (ewah) std::copy(r.ewah.begin(), r.ewah.end(), ewah);
    if (rank) std::copy(r.rank.begin(), r.rank.end(), rank);
    if (occ) std::copy(r.occ.begin(), r.occ.end(), occ);
    if (comp) std::copy(r.comp_list.begin(), r.comp_list.end(), comp);
    meta[0] = r.meta.cardinality;
    meta[1] = r.meta.n_runs;
    meta[2] = r.meta.n_words;
    meta[3] = r.meta.n_nonzero_w;
    meta[4] = r.meta.first_set;
    meta[5] = r.meta.last_set;
    meta[6] = r.meta.has_rank;
    meta[7] = r.meta.has_occ;
}

/* storm::select_pairing with the default model (storm_cost.cpp:422) on two
 * RowMeta records given as 8-word arrays; also returns predict() of every
 * pairing into pred[0..10]. */
uint32_t ref_select_pairing(const uint32_t* ma, const uint32_t* mb, double* pred) {
    auto mk = [](const uint32_t* m) {
        storm::RowMeta r;
        r.cardinality = m[0]; r.n_runs = m[1]; r.n_words = m[2]; r.n_nonzero_w = m[3];
        r.first_set = m[4]; r.last_set = m[5]; r.has_rank = m[6] != 0; r.has_occ = m[7] != 0;
        return r;
    };
    storm::CostModel m;
    storm::default_model(m);
    const storm::RowMeta a = mk(ma), b = mk(mb);
    if (pred)
        for (int p = 0; p <= (int)storm::Pairing::Empty; ++p)
            pred[p] = storm::predict(m, (storm::Pairing)p, a, b);
    return (uint32_t)storm::select_pairing(m, a, b);
}

/* Every variant of every cell on one ordered pair, for kernel-level golden
 * vectors: results[] in registry order bb, bs, br, bw, ss, sr, sw, rr, rw, ww, cb.
 * Returns the number written. */
uint32_t ref_all_cells(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb,
                       uint32_t universe, uint64_t* results) {
    storm::Row ra, rb;
    storm::build_row(ra, a, na, universe);
    storm::build_row(rb, b, nb, universe);
    uint32_t k = 0;
    auto bb = storm::cell_bb(); for (size_t i = 0; i < bb.n; ++i) results[k++] = bb.v[i].fn(ra.B(), rb.B());
    auto bs = storm::cell_bs(); for (size_t i = 0; i < bs.n; ++i) results[k++] = bs.v[i].fn(ra.B(), rb.S());
    auto br = storm::cell_br(); for (size_t i = 0; i < br.n; ++i) results[k++] = br.v[i].fn(ra.B(), rb.R());
    auto bw = storm::cell_bw(); for (size_t i = 0; i < bw.n; ++i) results[k++] = bw.v[i].fn(ra.B(), rb.W());
    auto ss = storm::cell_ss(); for (size_t i = 0; i < ss.n; ++i) results[k++] = ss.v[i].fn(ra.S(), rb.S());
    auto sr = storm::cell_sr(); for (size_t i = 0; i < sr.n; ++i) results[k++] = sr.v[i].fn(ra.S(), rb.R());
    auto sw = storm::cell_sw(); for (size_t i = 0; i < sw.n; ++i) results[k++] = sw.v[i].fn(ra.S(), rb.W());
    auto rr = storm::cell_rr(); for (size_t i = 0; i < rr.n; ++i) results[k++] = rr.v[i].fn(ra.R(), rb.R());
    auto rw = storm::cell_rw(); for (size_t i = 0; i < rw.n; ++i) results[k++] = rw.v[i].fn(ra.R(), rb.W());
    auto ww = storm::cell_ww(); for (size_t i = 0; i < ww.n; ++i) results[k++] = ww.v[i].fn(ra.W(), rb.W());
    if (ra.C().valid) {
        auto cb = storm::cell_cb(); for (size_t i = 0; i < cb.n; ++i) results[k++] = cb.v[i].fn(ra.C(), rb.B());
    }
    return k;
}

} /* extern "C" */
