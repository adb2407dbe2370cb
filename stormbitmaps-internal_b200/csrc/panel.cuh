// panel.cuh -- sparse rows against a transposed dense panel: the bit-slice
// engine of the STORM_t all-pairs planner.
//
// The tensor cores pay for a pair in proportion to the universe, whatever
// the rows hold; a pair of a sparse row x and a dense row p costs only
// |x| bits of p.  For a block of up to 2048 panel rows the engine stores the
// panel TRANSPOSED: DT[v] = 2048 bits, bit r set when panel row r holds
// value v (32 u64 words per value, U x 256 bytes in HBM).  A query row x is
// then one warp: lane w owns panel rows 64w .. 64w + 63, and for every value
// v of x it loads DT[v][w] (one coalesced 256-byte line per value for the
// warp) and adds its 64 bits into 64 per-row counters held bit-sliced:
// carry-save adders fold eight words into ones/twos/fours and a carry of
// weight 8, which ripples into NP vertical counter planes.  After the row,
// each lane turns its planes into 64 counts, the warp stages the 2048 counts
// in shared memory and writes them into the packed triangle.  Work per pair
// is |x| / 64 word additions and |x| / 8 bytes of panel traffic, against
// the universe's bits on the tensor cores.
//
// A query row is one work item, or -- when it holds many values -- several:
// items cover ranges of the row's chunks, so that no warp walks millions of
// values alone while the others wait (each value costs one dependent
// round trip to HBM per 16 values in flight).  The items of a split row
// write their counts into scratch slots, and panel_reduce_kernel adds the
// slots of each split row into the triangle.
//
// Bound: HBM (the DT lines: 256 bytes per value of a query row per block).
#pragma once
#include "chunk_engine.cuh"

namespace sb200 {

constexpr uint32_t PANEL_ROWS = 2048;                  // panel rows per block
constexpr uint32_t PANEL_WORDS = PANEL_ROWS / 64;      // DT words per value
constexpr uint32_t PANEL_T_WORDS = 4;                  // row words per transpose CTA (256 values)
constexpr uint32_t PANEL_Q_WARPS = 4;                  // warps per query CTA (33 KiB of shared memory)
constexpr uint32_t PANEL_NO_VALUE = 0xFFFFFFFFu;
constexpr uint64_t PANEL_MAX_UNIVERSE = 1ull << 26;    // 16 GiB of transposed block
constexpr uint64_t PANEL_MIN_SEG = 8192;               // values per work item of a split row, at least
constexpr uint32_t PANEL_MAX_SLOTS = 8192;             // scratch slots of split rows (64 MiB)

// X: PANEL_ROWS expanded rows of W words (rows past the block's end are
// zero).  DT[v * PANEL_WORDS + w] bit r = bit v of row 64 w + r.  CTA: 32
// warps, warp w transposes rows 64w .. 64w + 63 for PANEL_T_WORDS words: each
// 32 x 32 bit block (32 rows' 32-bit half-word, one per lane) is transposed
// in registers by five butterfly stages (shfl_xor over lanes 16, 8, 4, 2, 1),
// after which lane l holds bit l of that half-word across the 32 rows.  The
// CTA stages the 256 x 32 result (PANEL_T_SMEM bytes of dynamic shared
// memory, each value's 32 words rotated by the value so that a warp's 32
// stores hit distinct banks) and writes it out in order.
constexpr uint32_t PANEL_T_SMEM = 64 * PANEL_T_WORDS * PANEL_WORDS * 8;    // 64 KiB

// 32 x 32 bit transpose across a warp: on entry lane r holds row r (bit c =
// column c); on return lane c holds column c (bit r = row r).
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, uint32_t lane) {
#pragma unroll
    for (uint32_t j = 16; j > 0; j >>= 1) {
        // the lanes with bit j clear trade their high j-bit groups for the
        // low groups of lane ^ j
        const uint32_t m = j == 16 ? 0x0000FFFFu : j == 8 ? 0x00FF00FFu : j == 4 ? 0x0F0F0F0Fu
                         : j == 2 ? 0x33333333u : 0x55555555u;
        const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
        x = (lane & j) ? (x & ~m) | ((y >> j) & m) : (x & m) | ((y << j) & ~m);
    }
    return x;
}

__global__ void __launch_bounds__(1024)
panel_transpose_kernel(const uint64_t* __restrict__ X, uint64_t W, uint64_t* __restrict__ DT) {
    extern __shared__ unsigned long long stage[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t k0 = (uint64_t)blockIdx.x * PANEL_T_WORDS;
    const uint64_t* ra = X + (uint64_t)(64 * warp + lane) * W + k0;
    const uint64_t* rb = X + (uint64_t)(64 * warp + 32 + lane) * W + k0;
    uint64_t xa[PANEL_T_WORDS], xb[PANEL_T_WORDS];
#pragma unroll
    for (uint32_t q = 0; q < PANEL_T_WORDS; ++q) {
        xa[q] = __ldg(ra + q);
        xb[q] = __ldg(rb + q);
    }
#pragma unroll
    for (uint32_t q = 0; q < PANEL_T_WORDS; ++q) {
#pragma unroll
        for (uint32_t h = 0; h < 2; ++h) {
            const uint32_t lo = warp_transpose32((uint32_t)(xa[q] >> (32 * h)), lane);
            const uint32_t hi = warp_transpose32((uint32_t)(xb[q] >> (32 * h)), lane);
            const uint32_t v = 64 * q + 32 * h + lane;     // value within the CTA's 256
            stage[v * PANEL_WORDS + ((warp + v) & (PANEL_WORDS - 1))] = ((uint64_t)hi << 32) | lo;
        }
    }
    __syncthreads();
    uint64_t* dst = DT + k0 * 64 * PANEL_WORDS;
    for (uint32_t t = threadIdx.x; t < 64 * PANEL_T_WORDS * PANEL_WORDS; t += blockDim.x) {
        const uint32_t v = t / PANEL_WORDS, w = t % PANEL_WORDS;
        dst[t] = stage[v * PANEL_WORDS + ((w + v) & (PANEL_WORDS - 1))];
    }
}

__device__ __forceinline__ void panel_csa(uint64_t& h, uint64_t& l, uint64_t a, uint64_t b, uint64_t c) {
    const uint64_t u = a ^ b;
    h = (a & b) | (u & c);
    l = u ^ c;
}

// Adds eight words into the bit-sliced counters: count = s1 + 2 s2 + 4 s4 +
// sum_k 2^(k+3) planes[k], per bit position.
template <int NP>
__device__ __forceinline__ void panel_add8(const uint64_t* w, uint64_t& s1, uint64_t& s2, uint64_t& s4,
                                           uint64_t (&planes)[NP]) {
    uint64_t t2a, t2b, t2c, t2d, t4a, t4b, t8;
    panel_csa(t2a, s1, s1, w[0], w[1]);
    panel_csa(t2b, s1, s1, w[2], w[3]);
    panel_csa(t4a, s2, s2, t2a, t2b);
    panel_csa(t2c, s1, s1, w[4], w[5]);
    panel_csa(t2d, s1, s1, w[6], w[7]);
    panel_csa(t4b, s2, s2, t2c, t2d);
    panel_csa(t8, s4, s4, t4a, t4b);
    uint64_t c = t8;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        const uint64_t nc = planes[k] & c;
        planes[k] ^= c;
        c = nc;
    }
}

// 32 values (one per lane, PANEL_NO_VALUE = none) into the counters.
template <int NP>
__device__ __forceinline__ void panel_batch(uint32_t myv, const uint64_t* __restrict__ DT, uint32_t lane,
                                            uint64_t& s1, uint64_t& s2, uint64_t& s4, uint64_t (&planes)[NP]) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        uint64_t w[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            const uint32_t v = __shfl_sync(0xffffffffu, myv, 16 * h + t);
            w[t] = v != PANEL_NO_VALUE ? __ldg(DT + (uint64_t)v * PANEL_WORDS + lane) : 0ull;
        }
        panel_add8<NP>(w, s1, s2, s4, planes);
        panel_add8<NP>(w + 8, s1, s2, s4, planes);
    }
}

// One warp per (work item, block): items[k] (heaviest first), taken from a
// shared counter; the block holds the panel rows at walk positions
// [pw0, pw0 + prows).  Pairs with a panel row at a walk position after the
// query row's are written: out[(i, j)] with i, j the rows' stored indices
// (perm) -- or, for an item of a split row, scratch[slot][t] for panel row t
// -- and the sum over them added into flags.
// Shared memory: per warp 64 staged values + 2048 counts.
template <int NP>
__global__ void __launch_bounds__(PANEL_Q_WARPS * 32)
panel_query_kernel(ChunkView v, const uint32_t* __restrict__ perm, const PanelItem* __restrict__ items, uint32_t n_items,
                   uint64_t pw0, uint32_t prows, const uint64_t* __restrict__ DT, uint64_t n,
                   uint32_t* __restrict__ out, uint32_t* __restrict__ scratch, DeviceFlags* __restrict__ flags,
                   unsigned long long* __restrict__ counter) {
    __shared__ uint32_t vbuf[PANEL_Q_WARPS][64];
    __shared__ uint32_t cnt[PANEL_Q_WARPS][PANEL_ROWS];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* vb = vbuf[warp];
    uint32_t* cs = cnt[warp];
    unsigned long long local = 0;
    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= n_items) break;
        const PanelItem it = items[item];
        const uint64_t xw = it.xw;
        if (xw + 1 >= pw0 + prows) continue;              // no panel row after it in this block
        const uint32_t sx = perm[xw];
        const uint64_t c0 = v.row_off[sx];
        uint64_t s1 = 0, s2 = 0, s4 = 0;
        uint64_t planes[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) planes[k] = 0;
        uint32_t fill = 0;                                // staged values (warp-uniform)
        auto push = [&](bool valid, uint32_t val) {
            const uint32_t m = __ballot_sync(0xffffffffu, valid);
            if (valid) vb[fill + __popc(m & ((1u << lane) - 1u))] = val;
            fill += __popc(m);
            __syncwarp();
            if (fill >= 32) {
                panel_batch<NP>(vb[lane], DT, lane, s1, s2, s4, planes);
                const uint32_t rest = fill - 32;
                const uint32_t carry = lane < rest ? vb[32 + lane] : 0u;
                __syncwarp();
                if (lane < rest) vb[lane] = carry;
                fill = rest;
                __syncwarp();
            }
        };
        for (uint64_t c = c0 + it.c_lo; c < c0 + it.c_hi; ++c) {
            const uint32_t k = v.ckl[c];
            const uint32_t base = v.cid[c] << 16;
            if (k & CK_BITMAP) {
                const uint64_t* wd = v.bm + v.coff[c];
                for (uint32_t q0 = 0; q0 < CHUNK_WORDS; q0 += 32) {
                    uint64_t w = wd[q0 + lane];
                    while (__any_sync(0xffffffffu, w != 0)) {
                        const bool has = w != 0;
                        const uint32_t val = has ? base | ((q0 + lane) << 6) | (uint32_t)(__ffsll((long long)w) - 1) : 0u;
                        w &= w - 1;
                        push(has, val);
                    }
                }
            } else {
                const uint16_t* l = v.lst + v.coff[c];
                const uint32_t e = k & CK_LEN;
                for (uint32_t e0 = 0; e0 < e; e0 += 32) {
                    const bool has = e0 + lane < e;
                    push(has, has ? base | l[e0 + lane] : 0u);
                }
            }
        }
        if (fill) panel_batch<NP>(lane < fill ? vb[lane] : PANEL_NO_VALUE, DT, lane, s1, s2, s4, planes);
        // 64 counts of this lane's panel rows 64 lane + r, staged so that
        // the write-out below reads consecutive rows (XOR swizzle by lane)
#pragma unroll 4
        for (uint32_t r = 0; r < 64; ++r) {
            uint32_t x = (uint32_t)((s1 >> r) & 1u) + 2u * (uint32_t)((s2 >> r) & 1u) + 4u * (uint32_t)((s4 >> r) & 1u);
#pragma unroll
            for (int k = 0; k < NP; ++k) x += (uint32_t)((planes[k] >> r) & 1u) << (k + 3);
            cs[64 * lane + (r ^ lane)] = x;
        }
        __syncwarp();
        uint32_t* slot = it.slot != PANEL_NO_VALUE && out ? scratch + (uint64_t)it.slot * PANEL_ROWS : nullptr;
        for (uint32_t t = lane; t < prows; t += 32) {
            const uint64_t pw = pw0 + t;
            if (pw <= xw) continue;
            const uint32_t x = cs[(t & ~63u) + ((t & 63u) ^ (t >> 6))];
            if (slot) {
                slot[t] = x;
            } else if (out) {
                const uint32_t sp = perm[pw];
                const uint64_t i = sx < sp ? sx : sp, j = sx < sp ? sp : sx;
                out[tri_index(n, i, j)] = x;
            }
            local += x;
        }
        __syncwarp();
    }
    local = warp_sum_u64(local);
    if (lane == 0 && local) atomicAdd(&flags->sum, local);
}

// The counts of every split row against the block: the sum of its items'
// slots, written into the triangle (the sum over pairs was added by the
// items).  CTA per split row, threads over the block's panel rows.
__global__ void __launch_bounds__(256)
panel_reduce_kernel(const uint32_t* __restrict__ perm, const PanelSplit* __restrict__ splits, uint32_t n_splits,
                    uint64_t pw0, uint32_t prows, const uint32_t* __restrict__ scratch, uint64_t n,
                    uint32_t* __restrict__ out) {
    for (uint32_t r = blockIdx.x; r < n_splits; r += gridDim.x) {
        const PanelSplit sp = splits[r];
        const uint64_t xw = sp.xw;
        if (xw + 1 >= pw0 + prows) continue;
        const uint32_t sx = perm[xw];
        for (uint32_t t = threadIdx.x; t < prows; t += blockDim.x) {
            const uint64_t pw = pw0 + t;
            if (pw <= xw) continue;
            uint32_t x = 0;
            for (uint32_t k = 0; k < sp.nslots; ++k) x += scratch[(uint64_t)(sp.slot0 + k) * PANEL_ROWS + t];
            const uint32_t sq = perm[pw];
            const uint64_t i = sx < sq ? sx : sq, j = sx < sq ? sq : sx;
            out[tri_index(n, i, j)] = x;
        }
    }
}

}  // namespace sb200
