// rows_cells.cuh -- the pairing matrix (kernels/storm_cells.h) as
// warp-cooperative device cells.  Each cell returns this lane's share of
// |A & B|; the caller sums the warp.  Every lane of the warp calls the cell
// with the same arguments.  Orientation follows the reference's signatures:
// the first argument supplies the first representation of the cell's name
// (B x S takes (bitmap row, list row)).
//
//   B x B  dense AND+POPC over nw words (cell_bb.cpp:402 `dense`), or, when
//          both rows carry a zone map, only the 8-word bins live on both
//          sides (cell_bb.cpp:466-550 `occ` / `occ_sel`).
//   B x S  one bit test per list element (cell_bs.cpp:62 `ilp8`).
//   B x R  per run, rank difference when the bitmap has rank9
//          (cell_br.cpp:114-199), else a masked word popcount.
//   B x W  per EWAH marker: all-one fills count the bitmap's words, literals
//          AND with them (cell_wah.cpp:103-288).
//   S x S  each element of the shorter list binary-searches the longer
//          (cell_sparse.cpp:40-230, gallop family).
//   S x R  each element binary-searches the runs (cell_sparse.cpp:284-377).
//   S x W  each element finds its word's marker by binary search.
//   R x R  each run of the shorter side binary-searches the first overlapping
//          run and sums overlaps (cell_sparse.cpp:438-558).
//   R x W  per run, EWAH words covering it (cell_wah.cpp:483-573).
//   W x W  per marker of A: B's bits under A's one-fills plus A's literals
//          AND B's words (cell_wah.cpp:294-372).
//   C x B  |A & B| = |B| - |A' & B| with A' the complement list
//          (cell_comp.cpp:35-74).
#pragma once
#include "rows_engine.cuh"

namespace sb200 {

__device__ __forceinline__ uint32_t popc64d(uint64_t x) { return (uint32_t)__popcll(x); }

// First index in [0, n) with a[i] > x.
template <class T>
__device__ __forceinline__ uint32_t upper_bound_d(const T* a, uint32_t n, T x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}
template <class T>
__device__ __forceinline__ uint32_t lower_bound_d(const T* a, uint32_t n, T x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Set bits of bitmap words in [w0, w1).
__device__ __forceinline__ uint32_t bm_count_words(const uint64_t* bm, uint32_t w0, uint32_t w1) {
    uint32_t c = 0;
    for (uint32_t w = w0; w < w1; ++w) c += popc64d(bm[w]);
    return c;
}

// Set bits of a bitmap in [a, b) (bit positions), a < b.
__device__ __forceinline__ uint32_t bm_count_range(const uint64_t* bm, uint32_t a, uint32_t b) {
    const uint32_t wa = a >> 6, wb = (b - 1) >> 6;
    const uint64_t ma = ~0ull << (a & 63);
    const uint64_t mb = ((b & 63) == 0) ? ~0ull : ((1ull << (b & 63)) - 1);
    if (wa == wb) return popc64d(bm[wa] & ma & mb);
    uint32_t c = popc64d(bm[wa] & ma) + popc64d(bm[wb] & mb);
    for (uint32_t w = wa + 1; w < wb; ++w) c += popc64d(bm[w]);
    return c;
}

// rank9: set bits strictly below x (storm_repr.h:129-136).
__device__ __forceinline__ uint64_t rank_at_d(const uint64_t* bm, const uint64_t* rk, uint32_t nw, uint32_t x) {
    const uint32_t wi = x >> 6;
    if (wi >= nw) return rk[2 * ((nw + 7) / 8)];
    const uint32_t blk = wi >> 3, k = wi & 7;
    uint64_t r = rk[2 * blk];
    if (k) r += (rk[2 * blk + 1] >> (9 * (k - 1))) & 0x1FF;
    return r + popc64d(bm[wi] & ((1ull << (x & 63)) - 1));
}

// ---- EWAH helpers ----------------------------------------------------------
struct Ewah {
    const uint64_t* buf;   // stream
    const uint2* mk;       // marker table (stream pos, first word)
    uint32_t nm;           // markers
};

__device__ __forceinline__ Ewah ewah_of(const RowsView& v, uint32_t r) {
    Ewah e;
    e.buf = v.w_buf + v.w_off[r];
    e.mk = v.m_tab + v.m_off[r];
    e.nm = (uint32_t)(v.m_off[r + 1] - v.m_off[r]);
    return e;
}

// Index of the marker whose segment holds decoded word `w`.
__device__ __forceinline__ uint32_t ewah_find(const Ewah& e, uint32_t w) {
    uint32_t lo = 0, hi = e.nm;   // last marker with first word <= w
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (e.mk[mid].y <= w) lo = mid; else hi = mid;
    }
    return lo;
}

// Decoded word w of the stream, given the marker m that covers it.
__device__ __forceinline__ uint64_t ewah_word_in(const Ewah& e, uint32_t m, uint32_t w) {
    const uint64_t mw = e.buf[e.mk[m].x];
    const uint32_t fl = (uint32_t)((mw >> 1) & 0x7FFFFFFFull), ll = (uint32_t)(mw >> 32);
    const uint32_t off = w - e.mk[m].y;
    if (off < fl) return (mw & 1) ? ~0ull : 0ull;
    if (off - fl < ll) return e.buf[e.mk[m].x + 1 + (off - fl)];
    return 0ull;
}

// Walks decoded words of a stream from word w0 upwards.
struct EwahCursor {
    const Ewah* e;
    uint32_t m, w;
    __device__ __forceinline__ void seek(const Ewah& s, uint32_t w0) {
        e = &s;
        m = ewah_find(s, w0);
        w = w0;
    }
    __device__ __forceinline__ uint64_t next() {
        while (m + 1 < e->nm && e->mk[m + 1].y <= w) ++m;
        return ewah_word_in(*e, m, w++);
    }
};

// Set bits of the stream's decoded words in [w0, w1).
__device__ __forceinline__ uint32_t ewah_count_words(const Ewah& e, uint32_t w0, uint32_t w1) {
    if (w0 >= w1) return 0;
    uint32_t m = ewah_find(e, w0), c = 0, w = w0;
    while (w < w1 && m < e.nm) {
        const uint64_t mw = e.buf[e.mk[m].x];
        const uint32_t fl = (uint32_t)((mw >> 1) & 0x7FFFFFFFull), ll = (uint32_t)(mw >> 32);
        const uint32_t s0 = e.mk[m].y, fend = s0 + fl, lend = fend + ll;
        if (w < fend) {
            const uint32_t e1 = fend < w1 ? fend : w1;
            if (mw & 1) c += 64u * (e1 - w);
            w = e1;
        }
        while (w < lend && w < w1) {
            c += popc64d(e.buf[e.mk[m].x + 1 + (w - fend)]);
            ++w;
        }
        ++m;
    }
    return c;
}

// ---- cells -----------------------------------------------------------------
__device__ __forceinline__ uint32_t cell_bb(const RowsView& v, uint32_t a, uint32_t b, int lane, bool zone_map) {
    const uint64_t* wa = v.bm + v.b_off[a];
    const uint64_t* wb = v.bm + v.b_off[b];
    uint32_t c = 0;
    if (zone_map && v.oc_off[a] != NONE && v.oc_off[b] != NONE) {
        const uint64_t* oa = v.oc + v.oc_off[a];
        const uint64_t* ob = v.oc + v.oc_off[b];
        for (uint32_t k = 0; k < v.n_occ; ++k) {
            uint64_t live = oa[k] & ob[k];
            // bins of this occ word, spread over the warp
            while (live) {
                const uint32_t bit = __ffsll((long long)live) - 1;
                live &= live - 1;
                const uint32_t w = (k * 64 + bit) * 8 + (lane & 7);
                if ((lane >> 3) == 0 && w < v.nw) c += popc64d(wa[w] & wb[w]);
            }
        }
        return c;
    }
    for (uint32_t w = lane; w < v.nw; w += 32) c += popc64d(wa[w] & wb[w]);
    return c;
}

__device__ __forceinline__ uint32_t cell_bs(const RowsView& v, uint32_t bmrow, uint32_t lrow, int lane) {
    const uint64_t* w = v.bm + v.b_off[bmrow];
    const uint32_t* l = v.s_val + v.s_off[lrow];
    const uint32_t n = (uint32_t)(v.s_off[lrow + 1] - v.s_off[lrow]);
    uint32_t c = 0;
    for (uint32_t e = lane; e < n; e += 32) {
        const uint32_t x = l[e];
        c += (uint32_t)(w[x >> 6] >> (x & 63)) & 1u;
    }
    return c;
}

__device__ __forceinline__ uint32_t cell_br(const RowsView& v, uint32_t bmrow, uint32_t rrow, int lane) {
    const uint64_t* w = v.bm + v.b_off[bmrow];
    const bool rank = v.rk_off[bmrow] != NONE;
    const uint64_t* rk = rank ? v.rk + v.rk_off[bmrow] : nullptr;
    const uint64_t r0 = v.r_off[rrow];
    const uint32_t n = (uint32_t)(v.r_off[rrow + 1] - r0);
    uint32_t c = 0;
    for (uint32_t e = lane; e < n; e += 32) {
        const uint32_t a = v.r_start[r0 + e], b = v.r_end[r0 + e];
        // hybrid: rank for runs of at least 4 words (cell_br.cpp:187-199)
        if (rank && (b - a) >= 256) c += (uint32_t)(rank_at_d(w, rk, v.nw, b) - rank_at_d(w, rk, v.nw, a));
        else c += bm_count_range(w, a, b);
    }
    return c;
}

__device__ __forceinline__ uint32_t cell_bw(const RowsView& v, uint32_t bmrow, uint32_t wrow, int lane) {
    const uint64_t* w = v.bm + v.b_off[bmrow];
    const Ewah e = ewah_of(v, wrow);
    uint32_t c = 0;
    for (uint32_t m = lane; m < e.nm; m += 32) {
        const uint64_t mw = e.buf[e.mk[m].x];
        const uint32_t fl = (uint32_t)((mw >> 1) & 0x7FFFFFFFull), ll = (uint32_t)(mw >> 32);
        const uint32_t s0 = e.mk[m].y;
        if (mw & 1) c += bm_count_words(w, s0, s0 + fl);
        for (uint32_t k = 0; k < ll; ++k) c += popc64d(w[s0 + fl + k] & e.buf[e.mk[m].x + 1 + k]);
    }
    return c;
}

__device__ __forceinline__ uint32_t cell_ss(const RowsView& v, uint32_t a, uint32_t b, int lane) {
    const uint32_t na = (uint32_t)(v.s_off[a + 1] - v.s_off[a]), nb = (uint32_t)(v.s_off[b + 1] - v.s_off[b]);
    const bool a_short = na <= nb;
    const uint32_t* s = v.s_val + v.s_off[a_short ? a : b];
    const uint32_t* l = v.s_val + v.s_off[a_short ? b : a];
    const uint32_t ns = a_short ? na : nb, nl = a_short ? nb : na;
    uint32_t c = 0;
    for (uint32_t e = lane; e < ns; e += 32) {
        const uint32_t x = s[e];
        const uint32_t p = lower_bound_d<uint32_t>(l, nl, x);
        c += (p < nl && l[p] == x) ? 1u : 0u;
    }
    return c;
}

__device__ __forceinline__ uint32_t cell_sr(const RowsView& v, uint32_t lrow, uint32_t rrow, int lane) {
    const uint32_t* l = v.s_val + v.s_off[lrow];
    const uint32_t n = (uint32_t)(v.s_off[lrow + 1] - v.s_off[lrow]);
    const uint64_t r0 = v.r_off[rrow];
    const uint32_t nr = (uint32_t)(v.r_off[rrow + 1] - r0);
    const uint32_t* st = v.r_start + r0;
    const uint32_t* en = v.r_end + r0;
    uint32_t c = 0;
    for (uint32_t e = lane; e < n; e += 32) {
        const uint32_t x = l[e];
        const uint32_t p = upper_bound_d<uint32_t>(st, nr, x);   // runs starting at or before x
        c += (p > 0 && x < en[p - 1]) ? 1u : 0u;
    }
    return c;
}

__device__ __forceinline__ uint32_t cell_sw(const RowsView& v, uint32_t lrow, uint32_t wrow, int lane) {
    const uint32_t* l = v.s_val + v.s_off[lrow];
    const uint32_t n = (uint32_t)(v.s_off[lrow + 1] - v.s_off[lrow]);
    const Ewah e = ewah_of(v, wrow);
    uint32_t c = 0;
    for (uint32_t i = lane; i < n; i += 32) {
        const uint32_t x = l[i];
        const uint32_t m = ewah_find(e, x >> 6);
        c += (uint32_t)(ewah_word_in(e, m, x >> 6) >> (x & 63)) & 1u;
    }
    return c;
}

__device__ __forceinline__ uint32_t cell_rr(const RowsView& v, uint32_t a, uint32_t b, int lane) {
    const uint32_t na = (uint32_t)(v.r_off[a + 1] - v.r_off[a]), nb = (uint32_t)(v.r_off[b + 1] - v.r_off[b]);
    const bool a_short = na <= nb;
    const uint64_t s0 = v.r_off[a_short ? a : b], l0 = v.r_off[a_short ? b : a];
    const uint32_t ns = a_short ? na : nb, nl = a_short ? nb : na;
    const uint32_t* le = v.r_end + l0;
    uint32_t c = 0;
    for (uint32_t e = lane; e < ns; e += 32) {
        const uint32_t sa = v.r_start[s0 + e], sb = v.r_end[s0 + e];
        for (uint32_t q = upper_bound_d<uint32_t>(le, nl, sa); q < nl; ++q) {   // first run ending after sa
            const uint32_t ta = v.r_start[l0 + q], tb = le[q];
            if (ta >= sb) break;
            const uint32_t lo = sa > ta ? sa : ta, hi = sb < tb ? sb : tb;
            c += hi - lo;
        }
    }
    return c;
}

__device__ __forceinline__ uint32_t cell_rw(const RowsView& v, uint32_t rrow, uint32_t wrow, int lane) {
    const uint64_t r0 = v.r_off[rrow];
    const uint32_t nr = (uint32_t)(v.r_off[rrow + 1] - r0);
    const Ewah e = ewah_of(v, wrow);
    uint32_t c = 0;
    for (uint32_t i = lane; i < nr; i += 32) {
        const uint32_t a = v.r_start[r0 + i], b = v.r_end[r0 + i];
        const uint32_t wa = a >> 6, wb = (b - 1) >> 6;
        EwahCursor cur;
        cur.seek(e, wa);
        for (uint32_t w = wa; w <= wb; ++w) {
            uint64_t x = cur.next();
            if (w == wa) x &= ~0ull << (a & 63);
            if (w == wb && (b & 63)) x &= (1ull << (b & 63)) - 1;
            c += popc64d(x);
        }
    }
    return c;
}

__device__ __forceinline__ uint32_t cell_ww(const RowsView& v, uint32_t a, uint32_t b, int lane) {
    const Ewah ea = ewah_of(v, a), eb = ewah_of(v, b);
    uint32_t c = 0;
    for (uint32_t m = lane; m < ea.nm; m += 32) {
        const uint64_t mw = ea.buf[ea.mk[m].x];
        const uint32_t fl = (uint32_t)((mw >> 1) & 0x7FFFFFFFull), ll = (uint32_t)(mw >> 32);
        const uint32_t s0 = ea.mk[m].y;
        if (mw & 1) c += ewah_count_words(eb, s0, s0 + fl);
        if (ll) {
            EwahCursor cur;
            cur.seek(eb, s0 + fl);
            for (uint32_t k = 0; k < ll; ++k) c += popc64d(ea.buf[ea.mk[m].x + 1 + k] & cur.next());
        }
    }
    return c;
}

// C x B: `crow` supplies its complement list, `bmrow` its bitmap.  The
// returned lane share sums to |crow & bmrow| over the warp.
__device__ __forceinline__ uint32_t cell_cb(const RowsView& v, uint32_t crow, uint32_t bmrow, int lane) {
    const uint64_t* w = v.bm + v.b_off[bmrow];
    const uint32_t* l = v.c_val + v.c_off[crow];
    const uint32_t n = (uint32_t)(v.c_off[crow + 1] - v.c_off[crow]);
    uint32_t miss = 0;
    for (uint32_t e = lane; e < n; e += 32) {
        const uint32_t x = l[e];
        miss += (uint32_t)(w[x >> 6] >> (x & 63)) & 1u;
    }
    return (lane == 0 ? v.meta[bmrow].card : 0u) - miss;   // wraps per lane; the warp sum is exact
}

// Run pairing p on the ordered pair (d, s) with the driver's orientation
// rules (storm_allpairs.cpp:192-251): d is the denser row; B x R and B x W
// hand the bitmap to the row with more runs when the other has at least 16x
// fewer (the run-count orientation).
__device__ __forceinline__ uint32_t run_cell(const RowsView& v, int p, uint32_t d, uint32_t s, int lane,
                                             bool zone_map) {
    switch (p) {
        case P_BB: return cell_bb(v, d, s, lane, zone_map);
        case P_BS: return cell_bs(v, d, s, lane);
        case P_BR: {
            const bool sw = (double)v.meta[d].runs * BR_ORIENT_MARGIN <= (double)v.meta[s].runs;
            return sw ? cell_br(v, s, d, lane) : cell_br(v, d, s, lane);
        }
        case P_BW: {
            const bool sw = (double)v.meta[d].runs * BR_ORIENT_MARGIN <= (double)v.meta[s].runs;
            return sw ? cell_bw(v, s, d, lane) : cell_bw(v, d, s, lane);
        }
        case P_SS: return cell_ss(v, d, s, lane);
        case P_SR: return cell_sr(v, s, d, lane);
        case P_SW: return cell_sw(v, s, d, lane);
        case P_RR: return cell_rr(v, d, s, lane);
        case P_RW: return cell_rw(v, s, d, lane);
        case P_WW: return cell_ww(v, d, s, lane);
        case P_CB: return cell_cb(v, d, s, lane);   // the denser row's complement, the other's bitmap
        default: return 0;
    }
}

}  // namespace sb200
