/*
 * storm_oracle.c -- CPU ORACLE for the all-pairs intersection path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg use it, and only as the checker.
 *
 * It restates, in plain C, what the StormBitmaps reference computes on this
 * path, each function citing the reference code it follows:
 *
 *   - per-pair |Xi & Xj| over packed bitmap rows: the contiguous container's
 *     dispatch (storm.cpp:1144-1156) and libalgebra's AND+popcount kernels
 *     (libalgebra.h:2996 scalar form).  All dispatch branches compute the same
 *     set-intersection cardinality, so one AND+popcount loop restates them.
 *   - per-pair |Xi & Xj| over sorted position lists: kernels/oracle.cpp:28-38
 *     (rebuild both sides from positions, count common bits) -- restated as a
 *     two-pointer merge over the sorted distinct lists.
 *   - the STORM_t chunk split (storm.cpp:737-803): chunk = value / 65536,
 *     list chunk when fewer than 4096 values, bitmap chunk otherwise; and
 *     STORM_t counted chunk by chunk as the reference counts it, which
 *     differs from the set intersection for rows with repeated or
 *     out-of-order list entries (oracle_storm_matrix).
 *   - representation builders of kernels/storm_repr.cpp: maximal runs
 *     (:118-128), EWAH-64 (:78-100, marker layout storm_repr.h:28-31),
 *     rank9 (:25-45), zone map (:47-59), complement (:139-154) and RowMeta
 *     (:186-206).
 *
 * The popcount here is a SWAR bit count (no compiler builtin), so a broken
 * intrinsic path in a build cannot also break the checker -- the same
 * independence rule as kernels/oracle.cpp:17-24.
 *
 * Parity pinning: tests/golden/ holds outputs of the reference itself,
 * compiled from its own sources (oracle/Makefile) and run on seeded inputs
 * (tests/golden/make_golden.py); tests/test_oracle.py checks this file
 * against every one of them.
 */
#include <stdint.h>
#include <stddef.h>
#include <string.h>
#include <stdlib.h>

static uint32_t oracle_popcount64(uint64_t x) {
    x = x - ((x >> 1) & 0x5555555555555555ull);
    x = (x & 0x3333333333333333ull) + ((x >> 2) & 0x3333333333333333ull);
    x = (x + (x >> 4)) & 0x0F0F0F0F0F0F0F0Full;
    return (uint32_t)((x * 0x0101010101010101ull) >> 56);
}

/* |A & B| over nw words (libalgebra.h:2996, storm.cpp:1155). */
uint64_t oracle_and_popcount(const uint64_t* a, const uint64_t* b, uint64_t nw) {
    uint64_t c = 0;
    for (uint64_t k = 0; k < nw; ++k) c += oracle_popcount64(a[k] & b[k]);
    return c;
}

/* Packed upper triangle (i <= j, diagonal included) of per-pair counts over
 * n packed bitmap rows of nw words, plus the reference's sum over i < j
 * (storm.cpp:1232-1240).  `out` may be NULL.  Rows [r0, r1) only, so a
 * caller can sample a bounded slice; rows outside contribute nothing. */
uint64_t oracle_contig_matrix(const uint64_t* words, uint64_t n, uint64_t nw,
                              uint64_t r0, uint64_t r1, uint32_t* out) {
    uint64_t sum = 0;
    for (uint64_t i = r0; i < r1 && i < n; ++i) {
        const uint64_t* a = words + i * nw;
        const uint64_t base = i * n - (i * (i - 1)) / 2 - i;
        for (uint64_t j = i; j < n; ++j) {
            const uint64_t c = oracle_and_popcount(a, words + j * nw, nw);
            if (out) out[base + j] = (uint32_t)c;
            if (j > i) sum += c;
        }
    }
    return sum;
}

/* |A & B| of two sorted, distinct position lists (kernels/oracle.cpp:28-38:
 * the set intersection of the two rows). */
uint64_t oracle_list_intersect(const uint32_t* a, uint64_t na,
                               const uint32_t* b, uint64_t nb) {
    uint64_t i = 0, j = 0, c = 0;
    while (i < na && j < nb) {
        if (a[i] < b[j]) ++i;
        else if (b[j] < a[i]) ++j;
        else { ++c; ++i; ++j; }
    }
    return c;
}

/* Per-pair counts over n rows given as sorted distinct lists in CSR form
 * (values[offsets[r] .. offsets[r+1])).  Same output convention as
 * oracle_contig_matrix.  This is the count every STORM_t and kernel-layer
 * all-pairs call must reproduce (storm.cpp:927-945; storm_allpairs.cpp:677-732). */
uint64_t oracle_sets_matrix(const uint32_t* values, const uint64_t* offsets, uint64_t n,
                            uint64_t r0, uint64_t r1, uint32_t* out) {
    uint64_t sum = 0;
    for (uint64_t i = r0; i < r1 && i < n; ++i) {
        const uint64_t base = i * n - (i * (i - 1)) / 2 - i;
        for (uint64_t j = i; j < n; ++j) {
            const uint64_t c = oracle_list_intersect(values + offsets[i], offsets[i + 1] - offsets[i],
                                                     values + offsets[j], offsets[j + 1] - offsets[j]);
            if (out) out[base + j] = (uint32_t)c;
            if (j > i) sum += c;
        }
    }
    return sum;
}

/* Rectangular form: sum over all (i in X, j in Y) (storm.cpp:1027-1046). */
uint64_t oracle_sets_square(const uint32_t* xv, const uint64_t* xo, uint64_t nx,
                            const uint32_t* yv, const uint64_t* yo, uint64_t ny) {
    uint64_t sum = 0;
    for (uint64_t i = 0; i < nx; ++i)
        for (uint64_t j = 0; j < ny; ++j)
            sum += oracle_list_intersect(xv + xo[i], xo[i + 1] - xo[i], yv + yo[j], yo[j + 1] - yo[j]);
    return sum;
}

/* ---- STORM_t counted chunk by chunk, as the reference counts it ----------
 * For rows handed to STORM_add as given (sorted, repeats allowed; values out
 * of order only inside one chunk), the count STORM_pairw_intersect_cardinality
 * and STORM_bitmap_cont_intersect_cardinality produce, which for rows with
 * repeated or out-of-order list entries is not the set intersection:
 *   - each row is cut into chunks as STORM_bitmap_cont_add does
 *     (storm.cpp:737-803): a run of consecutive values with one chunk id
 *     (value / 65536) is a u16 list (entries as given) when it has fewer
 *     than 4096 values, else a 1024-word bitmap;
 *   - the chunk ids of two rows are matched by the two-pointer loop of
 *     STORM_intersect_vector32_unsafe (storm.cpp:90-121);
 *   - each matched pair is counted by STORM_bitmap_intersect_cardinality_func
 *     (storm.cpp:652-690): list x list by the SSE4.2 build of
 *     STORM_intersect_vector16_cardinality (storm.cpp:15-88, restated in
 *     oracle_list16_blocked), bitmap x list one bit test per list entry,
 *     bitmap x bitmap AND + popcount over 1024 words. */

/* Entries of an 8-entry block before its first 0 (8 if none): the implicit
 * string length of the reference's _mm_cmpistrm compare. */
static uint32_t o_block_len(const uint16_t* b) {
    uint32_t n = 0;
    while (n < 8 && b[n] != 0) ++n;
    return n;
}

/* Entries i < la of a equal to some entry k < lb of b (the "equal any" mask
 * of the reference's _mm_cmpestrm / _mm_cmpistrm, popcounted). */
static uint32_t o_block_any(const uint16_t* a, uint32_t la, const uint16_t* b, uint32_t lb) {
    uint32_t c = 0;
    for (uint32_t i = 0; i < la; ++i) {
        uint32_t hit = 0;
        for (uint32_t k = 0; k < lb; ++k) hit |= a[i] == b[k];
        c += hit;
    }
    return c;
}

/* storm.cpp:15-88 (SSE4.2 build): blocks of 8 while both lists have a whole
 * block left -- full-length compares while either block starts with 0, then
 * compares ending each block at its first 0; the block with the smaller last
 * entry advances (both on a tie) -- then the scalar merge of the rest. */
uint64_t oracle_list16_blocked(const uint16_t* v1, const uint16_t* v2, uint32_t len1, uint32_t len2) {
    uint64_t count = 0;
    uint32_t ia = 0, ib = 0;
    const uint32_t sta = len1 / 8 * 8, stb = len2 / 8 * 8;
    if (ia < sta && ib < stb) {
        int done = 0;
        while (v1[ia] == 0 || v2[ib] == 0) {
            count += o_block_any(v1 + ia, 8, v2 + ib, 8);
            const uint16_t am = v1[ia + 7], bm = v2[ib + 7];
            if (am <= bm) { ia += 8; if (ia == sta) { done = 1; break; } }
            if (bm <= am) { ib += 8; if (ib == stb) { done = 1; break; } }
        }
        if (!done && ia < sta && ib < stb)
            for (;;) {
                count += o_block_any(v1 + ia, o_block_len(v1 + ia), v2 + ib, o_block_len(v2 + ib));
                const uint16_t am = v1[ia + 7], bm = v2[ib + 7];
                if (am <= bm) { ia += 8; if (ia == sta) break; }
                if (bm <= am) { ib += 8; if (ib == stb) break; }
            }
    }
    while (ia < len1 && ib < len2) {
        if (v1[ia] < v2[ib]) ++ia;
        else if (v2[ib] < v1[ia]) ++ib;
        else { ++count; ++ia; ++ib; }
    }
    return count;
}

typedef struct {
    uint32_t id, bitmap, len;   /* len: list entries (bitmap chunks: 0) */
    uint64_t off;               /* into the list pool (u16) or the bitmap pool (words) */
} o_chunk;

typedef struct {
    o_chunk* ch;
    uint64_t* row;              /* row r: chunks [row[r], row[r+1]) */
    uint16_t* lst;
    uint64_t* bm;
} o_rows;

static void o_rows_build(const uint32_t* values, const uint64_t* offsets, uint64_t n, o_rows* R) {
    uint64_t nch = 0, nl = 0, nb = 0;
    for (uint64_t r = 0; r < n; ++r)
        for (uint64_t s = offsets[r]; s < offsets[r + 1];) {
            const uint32_t id = values[s] / 65536u;
            uint64_t e = s;
            while (e < offsets[r + 1] && values[e] / 65536u == id) ++e;
            ++nch;
            if (e - s < 4096) nl += e - s; else ++nb;
            s = e;
        }
    R->ch = (o_chunk*)malloc(sizeof(o_chunk) * (nch ? nch : 1));
    R->row = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
    R->lst = (uint16_t*)malloc(sizeof(uint16_t) * (nl ? nl : 1));
    R->bm = (uint64_t*)calloc((nb ? nb : 1) * 1024, sizeof(uint64_t));
    uint64_t c = 0, l = 0, b = 0;
    for (uint64_t r = 0; r < n; ++r) {
        R->row[r] = c;
        for (uint64_t s = offsets[r]; s < offsets[r + 1];) {
            const uint32_t id = values[s] / 65536u;
            uint64_t e = s;
            while (e < offsets[r + 1] && values[e] / 65536u == id) ++e;
            o_chunk* k = &R->ch[c++];
            k->id = id;
            if (e - s < 4096) {
                k->bitmap = 0;
                k->len = (uint32_t)(e - s);
                k->off = l;
                for (uint64_t q = s; q < e; ++q) R->lst[l++] = (uint16_t)(values[q] - id * 65536u);
            } else {
                k->bitmap = 1;
                k->len = 0;
                k->off = b * 1024;
                for (uint64_t q = s; q < e; ++q) {
                    const uint32_t x = values[q] - id * 65536u;
                    R->bm[b * 1024 + (x >> 6)] |= 1ull << (x & 63);
                }
                ++b;
            }
            s = e;
        }
    }
    R->row[n] = c;
}

static void o_rows_free(o_rows* R) {
    free(R->ch);
    free(R->row);
    free(R->lst);
    free(R->bm);
}

static uint64_t o_chunk_pair(const o_rows* R, const o_chunk* a, const o_chunk* b) {
    if (!a->bitmap && !b->bitmap) return oracle_list16_blocked(R->lst + a->off, R->lst + b->off, a->len, b->len);
    if (a->bitmap && b->bitmap) return oracle_and_popcount(R->bm + a->off, R->bm + b->off, 1024);
    const o_chunk* bmc = a->bitmap ? a : b;
    const o_chunk* lc = a->bitmap ? b : a;
    uint64_t c = 0;
    for (uint32_t e = 0; e < lc->len; ++e) {
        const uint32_t x = R->lst[lc->off + e];
        c += (R->bm[bmc->off + (x >> 6)] >> (x & 63)) & 1u;
    }
    return c;
}

/* Two rows: STORM_intersect_vector32_unsafe's chunk-id loop (storm.cpp:90-121),
 * then the matched chunk pairs (storm.cpp:835-860). */
static uint64_t o_row_pair(const o_rows* R, uint64_t i, uint64_t j) {
    const o_chunk* a = R->ch + R->row[i];
    const o_chunk* b = R->ch + R->row[j];
    const uint64_t la = R->row[i + 1] - R->row[i], lb = R->row[j + 1] - R->row[j];
    if (la == 0 || lb == 0) return 0;
    uint64_t A = 0, B = 0, c = 0;
    for (;;) {
        while (a[A].id < b[B].id)
            if (++A == la) return c;
        while (a[A].id > b[B].id)
            if (++B == lb) return c;
        if (a[A].id == b[B].id) {
            c += o_chunk_pair(R, &a[A], &b[B]);
            if (++A == la || ++B == lb) return c;
        } else if (++A == la) {
            return c;
        }
    }
}

/* Per-pair counts (packed upper triangle incl. the diagonal, the same
 * convention as oracle_contig_matrix) and the sum over i < j. */
uint64_t oracle_storm_matrix(const uint32_t* values, const uint64_t* offsets, uint64_t n, uint32_t* out) {
    o_rows R;
    o_rows_build(values, offsets, n, &R);
    uint64_t sum = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t base = i * n - (i * (i - 1)) / 2 - i;
        for (uint64_t j = i; j < n; ++j) {
            const uint64_t c = o_row_pair(&R, i, j);
            if (out) out[base + j] = (uint32_t)c;
            if (j > i) sum += c;
        }
    }
    o_rows_free(&R);
    return sum;
}

/* ---- STORM_t chunk split (storm.cpp:737-803) ----------------------------
 * For one sorted row, writes per chunk: id, kind (0 = list, 1 = bitmap) and
 * value count.  Returns the number of chunks. */
uint64_t oracle_chunk_split(const uint32_t* v, uint64_t n, uint32_t* ids, uint8_t* kinds,
                            uint32_t* counts) {
    uint64_t k = 0, s = 0;
    while (s < n) {
        const uint32_t id = v[s] / 65536u;
        uint64_t e = s;
        while (e < n && v[e] / 65536u == id) ++e;
        ids[k] = id;
        counts[k] = (uint32_t)(e - s);
        kinds[k] = (e - s) < 4096 ? 0 : 1;
        ++k;
        s = e;
    }
    return k;
}

/* ---- representation builders (kernels/storm_repr.cpp) ------------------ */

/* Maximal runs [start, end) of a sorted distinct list (storm_repr.cpp:118-128). */
uint64_t oracle_runs(const uint32_t* v, uint64_t n, uint32_t* start, uint32_t* end) {
    uint64_t r = 0;
    for (uint64_t i = 0; i < n;) {
        uint64_t j = i;
        while (j + 1 < n && v[j + 1] == v[j] + 1) ++j;
        start[r] = v[i];
        end[r] = v[j] + 1;
        ++r;
        i = j + 1;
    }
    return r;
}

/* EWAH-64 encoding of a bitmap (storm_repr.cpp:78-100).  Marker: bit 0 fill
 * value, bits 1..31 fill length, bits 32..63 literal count
 * (storm_repr.h:28-31).  A maximal stretch of all-zero or all-one words (at
 * most 2^31-1) is a fill; the non-fill words after it are literals.  `out`
 * must hold 2*nw+1 words.  Returns the stream length. */
uint64_t oracle_ewah(const uint64_t* w, uint64_t nw, uint64_t* out) {
    uint64_t o = 0, i = 0;
    while (i < nw) {
        uint64_t fv = (w[i] == ~0ull) ? 1 : 0;
        uint64_t fl = 0;
        if (w[i] == 0 || fv) {
            const uint64_t pat = fv ? ~0ull : 0ull;
            while (i < nw && w[i] == pat && fl < 0x7FFFFFFFull) { ++i; ++fl; }
        } else {
            fv = 0;
        }
        const uint64_t l0 = i;
        while (i < nw && w[i] != 0 && w[i] != ~0ull) ++i;
        const uint64_t ll = i - l0;
        out[o++] = fv | (fl << 1) | (ll << 32);
        for (uint64_t k = 0; k < ll; ++k) out[o++] = w[l0 + k];
    }
    if (o == 0) out[o++] = 0;
    return o;
}

/* Decode EWAH-64 back to nw words (storm_repr.cpp:61-74). */
void oracle_ewah_decode(const uint64_t* buf, uint64_t n, uint64_t* out) {
    uint64_t i = 0, o = 0;
    while (i < n) {
        const uint64_t m = buf[i++];
        const uint64_t fl = (m >> 1) & 0x7FFFFFFFull, ll = m >> 32;
        const uint64_t fv = (m & 1) ? ~0ull : 0ull;
        for (uint64_t k = 0; k < fl; ++k) out[o++] = fv;
        for (uint64_t k = 0; k < ll; ++k) out[o++] = buf[i++];
    }
}

/* rank9 index, 2*(nblk+1) words (storm_repr.cpp:25-45; layout storm_repr.h:78-93). */
void oracle_rank9(const uint64_t* w, uint64_t nw, uint64_t* out) {
    const uint64_t nblk = (nw + 7) / 8;
    uint64_t acc = 0;
    for (uint64_t b = 0; b < nblk; ++b) {
        uint64_t rel = 0, sub = 0;
        out[2 * b] = acc;
        for (uint64_t k = 0; k < 8; ++k) {
            if (k >= 1) sub |= (rel & 0x1FFull) << (9 * (k - 1));
            if (b * 8 + k < nw) rel += oracle_popcount64(w[b * 8 + k]);
        }
        out[2 * b + 1] = sub;
        acc += rel;
    }
    out[2 * nblk] = acc;
    out[2 * nblk + 1] = 0;
}

/* Zone map: one bit per bin of `bin` words, set when the bin is non-zero
 * (storm_repr.cpp:47-59).  out holds ceil(ceil(nw/bin)/64) words. */
void oracle_occ(const uint64_t* w, uint64_t nw, uint64_t bin, uint64_t* out) {
    const uint64_t bins = (nw + bin - 1) / bin;
    memset(out, 0, ((bins + 63) / 64) * 8);
    for (uint64_t b = 0; b < bins; ++b) {
        uint64_t any = 0;
        for (uint64_t k = b * bin; k < (b + 1) * bin && k < nw; ++k) any |= w[k];
        if (any) out[b >> 6] |= 1ull << (b & 63);
    }
}

/* RowMeta of a sorted distinct list over `universe` bits
 * (storm_repr.cpp:186-206, storm_repr.h:213-231).  meta[0..7] =
 * cardinality, n_runs, n_words, n_nonzero_w, first_set, last_set, has_rank,
 * has_occ. */
void oracle_row_meta(const uint32_t* v, uint64_t n, uint32_t universe, uint32_t* meta) {
    const uint32_t nw = (universe + 63u) / 64u;
    uint32_t runs = 0, nnz = 0;
    int64_t last_word = -1;
    for (uint64_t i = 0; i < n; ++i) {
        if (i == 0 || v[i] != v[i - 1] + 1) ++runs;
        if ((int64_t)(v[i] >> 6) != last_word) { ++nnz; last_word = v[i] >> 6; }
    }
    meta[0] = (uint32_t)n;
    meta[1] = runs;
    meta[2] = nw;
    meta[3] = nnz;
    meta[4] = n ? v[0] : 0xFFFFFFFFu;
    meta[5] = n ? v[n - 1] : 0;
    meta[6] = (runs && n / runs >= 512) ? 1 : 0;
    meta[7] = ((uint64_t)n * 512 > (uint64_t)universe) ? 1 : 0;
}

/* Complement positions of a sorted distinct list (storm_repr.cpp:139-146). */
uint64_t oracle_complement(const uint32_t* v, uint64_t n, uint32_t universe, uint32_t* out) {
    uint64_t o = 0;
    uint32_t prev = 0;
    for (uint64_t i = 0; i < n; ++i) {
        for (uint32_t p = prev; p < v[i]; ++p) out[o++] = p;
        prev = v[i] + 1;
    }
    for (uint32_t p = prev; p < universe; ++p) out[o++] = p;
    return o;
}

/* One row's strip of the packed triangle: out[j - i] = |Xi & Xj| for
 * j in [i, n).  Same counts as oracle_contig_matrix, without the n^2 buffer. */
uint64_t oracle_contig_row(const uint64_t* words, uint64_t n, uint64_t nw, uint64_t i, uint32_t* out) {
    uint64_t sum = 0;
    for (uint64_t j = i; j < n; ++j) {
        const uint64_t c = oracle_and_popcount(words + i * nw, words + j * nw, nw);
        out[j - i] = (uint32_t)c;
        if (j > i) sum += c;
    }
    return sum;
}

/* Cardinality of each packed row (the diagonal of the all-pairs matrix). */
void oracle_row_popcounts(const uint64_t* words, uint64_t n, uint64_t nw, uint32_t* out) {
    for (uint64_t r = 0; r < n; ++r) {
        uint64_t c = 0;
        for (uint64_t k = 0; k < nw; ++k) c += oracle_popcount64(words[r * nw + k]);
        out[r] = (uint32_t)c;
    }
}

/* Strips of the per-pair matrix for up to 8 query rows against many rows,
 * without the n^2 buffer: |Q_k & R_j| = the number of values of R_j that Q_k
 * holds (the set intersection oracle_sets_matrix counts, by a membership
 * table instead of a merge).  o_strip_new builds the table: byte v has bit k
 * set when query k holds value v (values < universe).  o_strip_count fills
 * out[j * nq + k] for rows j of a CSR batch and may be called from several
 * threads at once on disjoint batches. */
typedef struct {
    uint8_t* mask;
    uint64_t universe;
    uint32_t nq;
} o_strip;

void* oracle_strip_new(const uint32_t* qvals, const uint64_t* qoffs, uint32_t nq, uint64_t universe) {
    if (nq == 0 || nq > 8) return NULL;
    o_strip* h = (o_strip*)malloc(sizeof(o_strip));
    if (!h) return NULL;
    h->mask = (uint8_t*)calloc(universe ? universe : 1, 1);
    if (!h->mask) {
        free(h);
        return NULL;
    }
    h->universe = universe;
    h->nq = nq;
    for (uint32_t k = 0; k < nq; ++k)
        for (uint64_t e = qoffs[k]; e < qoffs[k + 1]; ++e)
            if (qvals[e] < universe) h->mask[qvals[e]] |= (uint8_t)(1u << k);
    return h;
}

void oracle_strip_count(const void* hp, const uint32_t* vals, const uint64_t* offs, uint64_t n, uint32_t* out) {
    const o_strip* h = (const o_strip*)hp;
    for (uint64_t j = 0; j < n; ++j) {
        uint32_t c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (uint64_t e = offs[j]; e < offs[j + 1]; ++e) {
            const uint32_t v = vals[e];
            if (v >= h->universe) continue;
            const uint32_t m = h->mask[v];
            for (uint32_t k = 0; k < h->nq; ++k) c[k] += (m >> k) & 1u;
        }
        for (uint32_t k = 0; k < h->nq; ++k) out[j * h->nq + k] = c[k];
    }
}

void oracle_strip_free(void* hp) {
    o_strip* h = (o_strip*)hp;
    if (!h) return;
    free(h->mask);
    free(h);
}

/* The same strips for rows given as packed bitmaps (nw words each):
 * out[j * nq + k] = |Q_k & R_j| by AND + popcount (oracle_and_popcount). */
void oracle_contig_strip(const uint64_t* q, uint32_t nq, const uint64_t* words, uint64_t n, uint64_t nw,
                         uint32_t* out) {
    for (uint64_t j = 0; j < n; ++j)
        for (uint32_t k = 0; k < nq; ++k)
            out[j * nq + k] = (uint32_t)oracle_and_popcount(q + (uint64_t)k * nw, words + j * nw, nw);
}
