// rows_pack.cu -- build the reference's row representations (storm_repr.cpp)
// from sorted positions and move them to HBM.
//
// Same outputs as storm::build_row, computed without materialising a bitmap
// for rows that do not get one: the EWAH stream is produced from the row's
// non-zero words, reproducing build_ewah's segmentation exactly (a maximal
// run of all-zero or all-one words, capped at 2^31-1, then the literal words
// up to the next fill; storm_repr.cpp:78-100).
#include <algorithm>
#include <cstring>

#include "rows_engine.cuh"

namespace sb200 {

static inline uint32_t popc64(uint64_t x) { return (uint32_t)__builtin_popcountll(x); }

namespace {

// Non-zero words of a sorted position list: (index, value), ascending.
void nonzero_words(const uint32_t* v, uint64_t n, std::vector<uint32_t>& idx, std::vector<uint64_t>& val) {
    idx.clear();
    val.clear();
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t w = v[i] >> 6;
        if (idx.empty() || idx.back() != w) {
            idx.push_back(w);
            val.push_back(0);
        }
        val.back() |= 1ull << (v[i] & 63);
    }
}

// EWAH-64 of a row given its non-zero words (storm_repr.cpp:78-100 semantics).
void ewah_sparse(const std::vector<uint32_t>& idx, const std::vector<uint64_t>& val, uint32_t nw,
                 std::vector<uint64_t>& out, std::vector<uint2>& markers) {
    const uint64_t FULL = ~0ull, CAP = 0x7FFFFFFFull;
    size_t k = 0;   // next non-zero word
    uint32_t i = 0; // current word
    auto word_at = [&](uint32_t w) -> uint64_t {  // only valid for w >= idx[k-?]; advance k lazily
        while (k < idx.size() && idx[k] < w) ++k;
        return (k < idx.size() && idx[k] == w) ? val[k] : 0ull;
    };
    const size_t start = out.size();
    while (i < nw) {
        const uint64_t w0 = word_at(i);
        uint64_t fv = (w0 == FULL) ? 1 : 0, fl = 0;
        const uint32_t first_word = i;
        if (w0 == 0 || fv) {
            if (fv) {
                while (i < nw && word_at(i) == FULL && fl < CAP) { ++i; ++fl; }
            } else {
                // zero fill up to the next non-zero word
                const uint32_t next = (k < idx.size()) ? idx[k] : nw;   // word_at advanced k to >= i
                uint64_t len = (uint64_t)std::min(next, nw) - i;
                if (len > CAP) len = CAP;
                i += (uint32_t)len;
                fl = len;
            }
        } else {
            fv = 0;
        }
        const size_t marker_pos = out.size();
        out.push_back(0);
        uint64_t ll = 0;
        while (i < nw) {
            const uint64_t w = word_at(i);
            if (w == 0 || w == FULL) break;
            out.push_back(w);
            ++ll;
            ++i;
        }
        out[marker_pos] = fv | (fl << 1) | (ll << 32);
        markers.push_back(make_uint2((uint32_t)(marker_pos - start), first_word));
    }
    if (out.size() == start) {
        out.push_back(0);
        markers.push_back(make_uint2(0, 0));
    }
}

}  // namespace

void pack_rows(const std::vector<uint32_t>& vals, const std::vector<uint64_t>& offs, uint32_t universe,
               const std::vector<uint8_t>& bm_rows, RowsPack& p) {
    const uint64_t n = offs.size() - 1;
    const uint32_t nw = (uint32_t)(((uint64_t)universe + 63) / 64);
    const uint32_t nw_pad = (nw + 1) & ~1u;
    const uint32_t nblk = (nw + 7) / 8;
    const uint32_t n_occ = (nblk + 63) / 64;
    p = RowsPack();
    p.meta.resize(n);
    p.b_off.assign(n, NONE);
    p.rk_off.assign(n, NONE);
    p.oc_off.assign(n, NONE);
    p.s_val.assign(vals.begin(), vals.end());
    p.s_off.assign(offs.begin(), offs.end());
    std::vector<uint32_t> idx;
    std::vector<uint64_t> wv;
    for (uint64_t r = 0; r < n; ++r) {
        const uint32_t* v = vals.data() + offs[r];
        const uint64_t len = offs[r + 1] - offs[r];
        // R: maximal runs (storm_repr.cpp:118-128)
        for (uint64_t i = 0; i < len;) {
            uint64_t j = i;
            while (j + 1 < len && v[j + 1] == v[j] + 1) ++j;
            p.r_start.push_back(v[i]);
            p.r_end.push_back(v[j] + 1);
            i = j + 1;
        }
        const uint64_t runs = p.r_start.size() - p.r_off.back();
        p.r_off.push_back(p.r_start.size());
        // W
        nonzero_words(v, len, idx, wv);
        const size_t w0 = p.w_buf.size();
        ewah_sparse(idx, wv, nw, p.w_buf, p.m_tab);
        (void)w0;
        p.w_off.push_back(p.w_buf.size());
        p.m_off.push_back(p.m_tab.size());
        // B (+ rank, zone map) for rows that get a bitmap
        const bool has_bm = bm_rows.empty() ? true : bm_rows[r] != 0;
        const uint64_t mean_rl = runs ? len / runs : 0;
        const bool want_rank = has_bm && mean_rl >= 512;
        const bool want_occ = has_bm && len * 512 > (uint64_t)universe;
        if (has_bm) {
            const uint64_t off = p.bm.size();
            p.b_off[r] = off;
            p.bm.resize(off + nw_pad, 0);
            for (size_t k = 0; k < idx.size(); ++k) p.bm[off + idx[k]] = wv[k];
            if (want_rank) {   // storm_repr.cpp:25-45
                const uint64_t ro = p.rk.size();
                p.rk_off[r] = ro;
                p.rk.resize(ro + 2 * (uint64_t)(nblk + 1), 0);
                uint64_t acc = 0;
                for (uint32_t b = 0; b < nblk; ++b) {
                    uint64_t rel = 0, sub = 0;
                    p.rk[ro + 2 * b] = acc;
                    for (uint32_t q = 0; q < 8; ++q) {
                        if (q >= 1) sub |= (rel & 0x1FFull) << (9 * (q - 1));
                        if (b * 8 + q < nw) rel += popc64(p.bm[off + b * 8 + q]);
                    }
                    p.rk[ro + 2 * b + 1] = sub;
                    acc += rel;
                }
                p.rk[ro + 2 * nblk] = acc;
            }
            if (want_occ) {    // storm_repr.cpp:47-59, 8-word bins
                const uint64_t oo = p.oc.size();
                p.oc_off[r] = oo;
                p.oc.resize(oo + n_occ, 0);
                for (size_t k = 0; k < idx.size(); ++k) {
                    const uint32_t bin = idx[k] / 8;
                    p.oc[oo + (bin >> 6)] |= 1ull << (bin & 63);
                }
            }
        }
        // C: complement when density > 1/2 (storm_repr.cpp:139-154)
        // (an empty complement -- a full row -- is not a usable form, storm_repr.h:185-192)
        const bool has_comp = has_bm && len * 2 > (uint64_t)universe && len < (uint64_t)universe;
        if (has_comp) {
            uint32_t prev = 0;
            for (uint64_t i = 0; i < len; ++i) {
                for (uint32_t q = prev; q < v[i]; ++q) p.c_val.push_back(q);
                prev = v[i] + 1;
            }
            for (uint32_t q = prev; q < universe; ++q) p.c_val.push_back(q);
        }
        p.c_off.push_back(p.c_val.size());
        RowMetaD& m = p.meta[r];
        m.card = (uint32_t)len;
        m.runs = (uint32_t)runs;
        m.nw = nw;
        m.nnz = (uint32_t)idx.size();
        m.first = len ? v[0] : 0xFFFFFFFFu;
        m.last = len ? v[len - 1] : 0;
        m.has_rank = want_rank;
        m.has_occ = want_occ;
        m.has_bm = has_bm;
        m.has_comp = has_comp;
    }
}

void upload_rows(const RowsPack& p, uint32_t universe, RowsDev& d, cudaStream_t st) {
    d.meta.put(p.meta, st);
    d.s_off.put(p.s_off, st);
    d.s_val.put(p.s_val, st);
    d.r_off.put(p.r_off, st);
    d.r_start.put(p.r_start, st);
    d.r_end.put(p.r_end, st);
    d.w_off.put(p.w_off, st);
    d.w_buf.put(p.w_buf, st);
    d.m_off.put(p.m_off, st);
    d.m_tab.put(p.m_tab, st);
    d.b_off.put(p.b_off, st);
    d.bm.put(p.bm, st);
    d.rk_off.put(p.rk_off, st);
    d.rk.put(p.rk, st);
    d.oc_off.put(p.oc_off, st);
    d.oc.put(p.oc, st);
    d.c_off.put(p.c_off, st);
    d.c_val.put(p.c_val, st);
    SB_CUDA(cudaStreamSynchronize(st));
    RowsView& v = d.view;
    v.n = (uint32_t)p.meta.size();
    v.universe = universe;
    v.nw = (uint32_t)(((uint64_t)universe + 63) / 64);
    v.n_occ = ((v.nw + 7) / 8 + 63) / 64;
    v.meta = d.meta.buf.p;
    v.s_off = d.s_off.buf.p;
    v.s_val = d.s_val.buf.p;
    v.r_off = d.r_off.buf.p;
    v.r_start = d.r_start.buf.p;
    v.r_end = d.r_end.buf.p;
    v.w_off = d.w_off.buf.p;
    v.w_buf = d.w_buf.buf.p;
    v.m_off = d.m_off.buf.p;
    v.m_tab = d.m_tab.buf.p;
    v.b_off = d.b_off.buf.p;
    v.bm = d.bm.buf.p;
    v.rk_off = d.rk_off.buf.p;
    v.rk = d.rk.buf.p;
    v.oc_off = d.oc_off.buf.p;
    v.oc = d.oc.buf.p;
    v.c_off = d.c_off.buf.p;
    v.c_val = d.c_val.buf.p;
}

}  // namespace sb200
