// rows_pack.cu -- build the reference's row representations (storm::build_row,
// storm_repr.cpp:25-207) on the device from the rows' sorted positions.
//
// The positions (S) and their CSR offsets are the only upload; everything
// else is derived in HBM by one thread block per row:
//   repr_count_kernel  per row: run count, non-zero words, EWAH markers and
//                      stream words (block reductions over the positions);
//   (host)             exclusive scans of those counts into the pool offsets,
//                      the representation gates of storm_repr.cpp:186-189;
//   repr_fill_kernel   per row, positions in tiles of PK_THREADS with block
//                      scans carried across tiles: R (maximal runs), B
//                      (each word built by the thread holding its first
//                      position), the zone map, the EWAH literals, marker
//                      slots and the marker table; then, after a barrier,
//                      the marker words, rank9 and the complement (C) from
//                      the row's own bitmap.
//
// EWAH-64 segmentation (storm_repr.cpp:78-100): a marker is a fill run (all
// zero or all one words) followed by the literal words up to the next fill.
// Over the row's non-zero words k (index w_k) a marker starts
//   * at every zero gap (words w_{k-1}+1 .. w_k - 1, or before the first /
//     after the last non-zero word, or the whole row when it is empty);
//   * at every full word whose predecessor is not an adjacent full word;
//   * at word 0 when it is a literal (a marker without fill).
// A word is full when 64 consecutive positions start at its first bit --
// a test on two positions of the sorted row. Marker q's literal count and
// fill length follow from the next marker (position p, first word f):
// ll = p_{q+1} - p_q - 1 and fl = f_{q+1} - f_q - ll, with (stream length,
// word count) after the last; so the fill pass writes only the marker table
// and the full-fill flag, and the marker words are assembled afterwards.
// Fill runs never reach the reference's 2^31 - 1 cap: a universe of at most
// 2^32 bits has 2^26 words.
#include <algorithm>
#include <cstring>

#include "rows_engine.cuh"

namespace sb200 {

namespace {

constexpr int PK_THREADS = 256;
constexpr int PK_WARPS = PK_THREADS / 32;

// What one position contributes: run start / end, and, when it is the first
// position of a word, the word's EWAH items.
struct PosInfo {
    uint32_t run_start, run_end;
    uint32_t word_start, full;
    uint32_t gap, gap_first, fullstart, lit0, trailing;
    uint32_t w;
};

__device__ __forceinline__ PosInfo classify(const uint32_t* __restrict__ v, uint64_t i, uint64_t len, uint32_t nw) {
    PosInfo p{};
    const uint32_t x = v[i];
    p.w = x >> 6;
    p.run_start = (i == 0) || v[i - 1] + 1 != x;
    p.run_end = (i + 1 == len) || v[i + 1] != x + 1;
    const uint32_t pw = i ? v[i - 1] >> 6 : 0;
    p.word_start = (i == 0) || pw != p.w;
    if (p.word_start) {
        p.full = (x & 63u) == 0 && i + 63 < len && v[i + 63] == x + 63;
        // previous non-zero word full: its last position is bit 63 and the
        // position 63 places earlier is its bit 0
        const bool pfull = i > 0 && (v[i - 1] & 63u) == 63 && i >= 64 && v[i - 64] == v[i - 1] - 63;
        if (i == 0) {
            p.gap = p.w > 0;
            p.gap_first = 0;
        } else {
            p.gap = p.w > pw + 1;
            p.gap_first = pw + 1;
        }
        p.fullstart = p.full && (i == 0 || p.gap || !pfull);
        p.lit0 = (i == 0) && p.w == 0 && !p.full;
    }
    p.trailing = (i + 1 == len) && p.w + 1 < nw;
    return p;
}

__device__ __forceinline__ uint32_t markers_of(const PosInfo& p) {
    return p.word_start ? p.gap + p.fullstart + p.lit0 + p.trailing : p.trailing;
}

__device__ __forceinline__ uint32_t stream_of(const PosInfo& p) {
    return markers_of(p) + (p.word_start && !p.full ? 1u : 0u);
}

// Block-wide exclusive scan of four counters; `total` receives the block's
// sums. All threads of the block must call it.
__device__ __forceinline__ uint4 block_scan4(uint4 x, uint4& total, uint4* sm /* [PK_WARPS + 1] */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint4 inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t a = __shfl_up_sync(0xffffffffu, inc.x, o), b = __shfl_up_sync(0xffffffffu, inc.y, o);
        const uint32_t c = __shfl_up_sync(0xffffffffu, inc.z, o), d = __shfl_up_sync(0xffffffffu, inc.w, o);
        if (lane >= o) {
            inc.x += a;
            inc.y += b;
            inc.z += c;
            inc.w += d;
        }
    }
    if (lane == 31) sm[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint4 s = lane < PK_WARPS ? sm[lane] : make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int o = 1; o < PK_WARPS; o <<= 1) {
            const uint32_t a = __shfl_up_sync(0xffffffffu, s.x, o), b = __shfl_up_sync(0xffffffffu, s.y, o);
            const uint32_t c = __shfl_up_sync(0xffffffffu, s.z, o), d = __shfl_up_sync(0xffffffffu, s.w, o);
            if (lane >= o) {
                s.x += a;
                s.y += b;
                s.z += c;
                s.w += d;
            }
        }
        if (lane < PK_WARPS) sm[lane] = s;   // inclusive per warp
    }
    __syncthreads();
    const uint4 base = wid ? sm[wid - 1] : make_uint4(0, 0, 0, 0);
    total = sm[PK_WARPS - 1];
    __syncthreads();   // sm is reused by the next call
    return make_uint4(base.x + inc.x - x.x, base.y + inc.y - x.y, base.z + inc.z - x.z, base.w + inc.w - x.w);
}

// Per row: x = runs, y = non-zero words, z = EWAH markers, w = EWAH words.
__global__ void __launch_bounds__(PK_THREADS) repr_count_kernel(const uint32_t* __restrict__ vals,
                                                                const uint64_t* __restrict__ offs, uint32_t nw,
                                                                uint4* __restrict__ counts) {
    __shared__ uint4 sm[PK_WARPS + 1];
    const uint64_t r = blockIdx.x;
    const uint64_t o = offs[r], len = offs[r + 1] - o;
    const uint32_t* v = vals + o;
    uint4 acc = make_uint4(0, 0, 0, 0);
    for (uint64_t i = threadIdx.x; i < len; i += PK_THREADS) {
        const PosInfo p = classify(v, i, len, nw);
        acc.x += p.run_start;
        acc.y += p.word_start;
        acc.z += markers_of(p);
        acc.w += stream_of(p);
    }
    uint4 tot;
    block_scan4(acc, tot, sm);
    if (threadIdx.x == 0) {
        if (len == 0) tot = make_uint4(0, 0, 1, 1);   // one zero fill over the row (or an empty marker)
        counts[r] = tot;
    }
}

struct FillArgs {
    const uint32_t* vals;
    const uint64_t* offs;
    const RowMetaD* meta;
    uint32_t universe, nw, nblk;
    const uint64_t *r_off, *w_off, *m_off, *b_off, *rk_off, *oc_off, *c_off;
    uint32_t *r_start, *r_end, *c_val;
    uint64_t *w_buf, *bm, *rk, *oc;
    uint2* m_tab;
};

__global__ void __launch_bounds__(PK_THREADS) repr_fill_kernel(FillArgs a) {
    __shared__ uint4 sm[PK_WARPS + 1];
    const uint64_t r = blockIdx.x;
    const uint64_t o = a.offs[r], len = a.offs[r + 1] - o;
    const uint32_t* v = a.vals + o;
    const RowMetaD m = a.meta[r];
    uint32_t* rs = a.r_start + a.r_off[r];
    uint32_t* re = a.r_end + a.r_off[r];
    uint64_t* ew = a.w_buf + a.w_off[r];
    uint2* mt = a.m_tab + a.m_off[r];
    const uint32_t n_mark = (uint32_t)(a.m_off[r + 1] - a.m_off[r]);
    const uint32_t n_stream = (uint32_t)(a.w_off[r + 1] - a.w_off[r]);
    uint64_t* bm = m.has_bm ? a.bm + a.b_off[r] : nullptr;
    uint64_t* oc = m.has_occ ? a.oc + a.oc_off[r] : nullptr;

    // ---- phase 1: runs, words, marker table, literals
    if (len == 0 && threadIdx.x == 0) {
        mt[0] = make_uint2(0, 0);
        ew[0] = 0;
    }
    uint4 carry = make_uint4(0, 0, 0, 0);   // runs, markers, stream words
    for (uint64_t base = 0; base < len; base += PK_THREADS) {
        const uint64_t i = base + threadIdx.x;
        PosInfo p{};
        uint64_t word = 0;
        if (i < len) {
            p = classify(v, i, len, a.nw);
            if (p.word_start)
                for (uint64_t j = i; j < len && (v[j] >> 6) == p.w; ++j) word |= 1ull << (v[j] & 63u);
        }
        const uint4 mine = i < len ? make_uint4(p.run_start, markers_of(p), stream_of(p), 0) : make_uint4(0, 0, 0, 0);
        uint4 tot;
        const uint4 ex = block_scan4(mine, tot, sm);
        if (i < len) {
            const uint32_t run = carry.x + ex.x + p.run_start - 1;   // index of the run holding i
            if (p.run_start) rs[run] = v[i];
            if (p.run_end) re[run] = v[i] + 1;
            uint32_t q = carry.y + ex.y, s = carry.z + ex.z;
            if (p.word_start) {
                if (p.gap) {
                    mt[q++] = make_uint2(s, p.gap_first);
                    ew[s++] = 0;
                }
                if (p.fullstart || p.lit0) {
                    mt[q++] = make_uint2(s, p.w);
                    ew[s++] = p.fullstart ? 1ull : 0ull;   // the fill value bit; lengths below
                }
                if (!p.full) ew[s++] = word;
                if (bm) bm[p.w] = word;
                if (oc && (i == 0 || (v[i - 1] >> 9) != (p.w >> 3)))
                    atomicOr((unsigned long long*)&oc[(p.w >> 3) >> 6], 1ull << ((p.w >> 3) & 63u));
            }
            if (p.trailing) {
                mt[q++] = make_uint2(s, p.w + 1);
                ew[s++] = 0;
            }
        }
        carry.x += tot.x;
        carry.y += tot.y;
        carry.z += tot.z;
    }
    __syncthreads();   // the row's stream, table and bitmap are complete

    // ---- phase 2: marker words (fill length and literal count)
    for (uint32_t q = threadIdx.x; q < n_mark; q += PK_THREADS) {
        const uint2 cur = mt[q];
        const uint2 nxt = q + 1 < n_mark ? mt[q + 1] : make_uint2(n_stream, a.nw);
        const uint64_t ll = nxt.x - cur.x - 1;
        const uint64_t fl = (uint64_t)nxt.y - cur.y - ll;
        ew[cur.x] = (ew[cur.x] & 1ull) | (fl << 1) | (ll << 32);
    }

    // ---- phase 3: rank9 (storm_repr.cpp:25-45) from the row's bitmap
    if (m.has_rank) {
        uint64_t* rk = a.rk + a.rk_off[r];
        uint64_t acc = 0;
        for (uint32_t b0 = 0; b0 < a.nblk; b0 += PK_THREADS) {
            const uint32_t b = b0 + threadIdx.x;
            uint32_t rel = 0;
            uint64_t sub = 0;
            if (b < a.nblk)
                for (uint32_t q = 0; q < 8; ++q) {
                    if (q >= 1) sub |= (uint64_t)(rel & 0x1FFu) << (9 * (q - 1));
                    if (b * 8 + q < a.nw) rel += __popcll(bm[b * 8 + q]);
                }
            uint4 tot;
            const uint4 ex = block_scan4(make_uint4(rel, 0, 0, 0), tot, sm);
            if (b < a.nblk) {
                rk[2 * b] = acc + ex.x;
                rk[2 * b + 1] = sub;
            }
            acc += tot.x;
        }
        if (threadIdx.x == 0) {
            rk[2 * a.nblk] = acc;
            rk[2 * a.nblk + 1] = 0;
        }
    }

    // ---- phase 4: complement positions (storm_repr.cpp:139-154): the zero
    // bits of the bitmap below the universe, in order
    if (m.has_comp) {
        uint32_t* cv = a.c_val + a.c_off[r];
        uint32_t acc = 0;
        for (uint32_t k0 = 0; k0 < a.nw; k0 += PK_THREADS) {
            const uint32_t k = k0 + threadIdx.x;
            uint64_t z = 0;
            if (k < a.nw) {
                z = ~bm[k];
                const uint64_t hi = (uint64_t)k * 64 + 64;
                if (hi > a.universe) z &= (1ull << (a.universe - (uint64_t)k * 64)) - 1;
            }
            uint4 tot;
            const uint4 ex = block_scan4(make_uint4((uint32_t)__popcll(z), 0, 0, 0), tot, sm);
            uint32_t at = acc + ex.x;
            while (z) {
                const int b = __ffsll((long long)z) - 1;
                cv[at++] = k * 64 + (uint32_t)b;
                z &= z - 1;
            }
            acc += tot.x;
        }
    }
}

template <class T>
void put(DevBuf<T>& d, const T* h, size_t n, cudaStream_t st) {
    d.reserve(n ? n : 1);
    if (n) SB_CUDA(cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
}

template <class T>
void zeroed(DevBuf<T>& d, size_t n, cudaStream_t st) {
    d.reserve(n ? n : 1);
    SB_CUDA(cudaMemsetAsync(d.p, 0, (n ? n : 1) * sizeof(T), st));
}

}  // namespace

void build_rows(const std::vector<uint32_t>& vals, const std::vector<uint64_t>& offs, uint32_t universe,
                const std::vector<uint8_t>& bm_rows, RowsDev& d, cudaStream_t st) {
    const uint64_t n = offs.size() - 1;
    const uint32_t nw = (uint32_t)(((uint64_t)universe + 63) / 64);
    const uint32_t nw_pad = (nw + 1) & ~1u;
    const uint32_t nblk = (nw + 7) / 8;
    const uint32_t n_occ = (nblk + 63) / 64;
    put(d.s_val, vals.data(), vals.size(), st);
    put(d.s_off, offs.data(), offs.size(), st);
    std::vector<uint4> cnt(n);
    if (n) {
        d.counts.reserve(n);
        repr_count_kernel<<<(unsigned)n, PK_THREADS, 0, st>>>(d.s_val.p, d.s_off.p, nw, d.counts.p);
        SB_CUDA(cudaGetLastError());
        SB_CUDA(cudaMemcpyAsync(cnt.data(), d.counts.p, n * sizeof(uint4), cudaMemcpyDeviceToHost, st));
    }
    SB_CUDA(cudaStreamSynchronize(st));

    // Pool offsets and the representation gates (storm_repr.cpp:186-189).
    std::vector<uint64_t> r_off(n + 1), w_off(n + 1), m_off(n + 1), c_off(n + 1);
    std::vector<uint64_t> b_off(n, NONE), rk_off(n, NONE), oc_off(n, NONE);
    d.h_meta.assign(n, RowMetaD{});
    uint64_t nb = 0, nrk = 0, noc = 0;
    r_off[0] = w_off[0] = m_off[0] = c_off[0] = 0;
    for (uint64_t r = 0; r < n; ++r) {
        const uint64_t len = offs[r + 1] - offs[r];
        const uint32_t runs = cnt[r].x;
        const bool has_bm = bm_rows.empty() ? true : bm_rows[r] != 0;
        const uint64_t mean_rl = runs ? len / runs : 0;
        const bool want_rank = has_bm && mean_rl >= 512;
        const bool want_occ = has_bm && len * 512 > (uint64_t)universe;
        // an empty complement (a full row) is not a usable form (storm_repr.h:185-192)
        const bool has_comp = has_bm && len * 2 > (uint64_t)universe && len < (uint64_t)universe;
        RowMetaD& m = d.h_meta[r];
        m.card = (uint32_t)len;
        m.runs = runs;
        m.nw = nw;
        m.nnz = cnt[r].y;
        m.first = len ? vals[offs[r]] : 0xFFFFFFFFu;
        m.last = len ? vals[offs[r + 1] - 1] : 0;
        m.has_rank = want_rank;
        m.has_occ = want_occ;
        m.has_bm = has_bm;
        m.has_comp = has_comp;
        r_off[r + 1] = r_off[r] + runs;
        m_off[r + 1] = m_off[r] + cnt[r].z;
        w_off[r + 1] = w_off[r] + cnt[r].w;
        c_off[r + 1] = c_off[r] + (has_comp ? universe - len : 0);
        if (has_bm) {
            b_off[r] = nb;
            nb += nw_pad;
        }
        if (want_rank) {
            rk_off[r] = nrk;
            nrk += 2 * (uint64_t)(nblk + 1);
        }
        if (want_occ) {
            oc_off[r] = noc;
            noc += n_occ;
        }
    }
    put(d.meta, d.h_meta.data(), n, st);
    put(d.r_off, r_off.data(), n + 1, st);
    put(d.w_off, w_off.data(), n + 1, st);
    put(d.m_off, m_off.data(), n + 1, st);
    put(d.c_off, c_off.data(), n + 1, st);
    put(d.b_off, b_off.data(), n, st);
    put(d.rk_off, rk_off.data(), n, st);
    put(d.oc_off, oc_off.data(), n, st);
    d.r_start.reserve(std::max<uint64_t>(1, r_off[n]));
    d.r_end.reserve(std::max<uint64_t>(1, r_off[n]));
    d.w_buf.reserve(std::max<uint64_t>(1, w_off[n]));
    d.m_tab.reserve(std::max<uint64_t>(1, m_off[n]));
    d.c_val.reserve(std::max<uint64_t>(1, c_off[n]));
    d.rk.reserve(std::max<uint64_t>(1, nrk));
    zeroed(d.bm, nb, st);    // words without a position stay zero
    zeroed(d.oc, noc, st);   // zone-map bits are OR-ed in
    if (n) {
        FillArgs a;
        a.vals = d.s_val.p;
        a.offs = d.s_off.p;
        a.meta = d.meta.p;
        a.universe = universe;
        a.nw = nw;
        a.nblk = nblk;
        a.r_off = d.r_off.p;
        a.w_off = d.w_off.p;
        a.m_off = d.m_off.p;
        a.b_off = d.b_off.p;
        a.rk_off = d.rk_off.p;
        a.oc_off = d.oc_off.p;
        a.c_off = d.c_off.p;
        a.r_start = d.r_start.p;
        a.r_end = d.r_end.p;
        a.c_val = d.c_val.p;
        a.w_buf = d.w_buf.p;
        a.bm = d.bm.p;
        a.rk = d.rk.p;
        a.oc = d.oc.p;
        a.m_tab = d.m_tab.p;
        repr_fill_kernel<<<(unsigned)n, PK_THREADS, 0, st>>>(a);
        SB_CUDA(cudaGetLastError());
    }
    SB_CUDA(cudaStreamSynchronize(st));
    RowsView& v = d.view;
    v.n = (uint32_t)n;
    v.universe = universe;
    v.nw = nw;
    v.n_occ = n_occ;
    v.meta = d.meta.p;
    v.s_off = d.s_off.p;
    v.s_val = d.s_val.p;
    v.r_off = d.r_off.p;
    v.r_start = d.r_start.p;
    v.r_end = d.r_end.p;
    v.w_off = d.w_off.p;
    v.w_buf = d.w_buf.p;
    v.m_off = d.m_off.p;
    v.m_tab = d.m_tab.p;
    v.b_off = d.b_off.p;
    v.bm = d.bm.p;
    v.rk_off = d.rk_off.p;
    v.rk = d.rk.p;
    v.oc_off = d.oc_off.p;
    v.oc = d.oc.p;
    v.c_off = d.c_off.p;
    v.c_val = d.c_val.p;
}

}  // namespace sb200
