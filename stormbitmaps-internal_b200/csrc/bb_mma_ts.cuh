// bb_mma_ts.cuh -- B x B on tcgen05 with the A operand in tensor memory.
//
// Same arithmetic as bb_mma.cuh (u8 x u8 -> s32, A bytes weighted 2^(k mod 8),
// B bytes 2^(7 - k mod 8), D = 128 |Xi & Xj|), different data movement: the
// 128 rows of the A panel are expanded by their own threads straight into
// TMEM with tcgen05.st (lane = row, four K bytes per 32-bit column), so only
// the 256 B rows pass through shared memory.  Measured on the SS form, the
// shared-memory pipe (expansion stores + the tensor core's operand reads)
// was the bottleneck; this removes a third of that traffic.
//
// Warp roles (416 threads): warps 0-3 expand A rows into TMEM, warps 4-11
// expand B rows into the swizzled smem ring, warp 12 owns TMEM and issues
// the MMAs; warps 0-7 drain the accumulator in the epilogue.  Stages are 256
// row bits: 64 TMEM columns of A + 64 KB of B, three in flight.  TMEM: 512
// columns = accumulator [0, 256) + A stages [256, 448).
#pragma once
#include "bb_mma.cuh"

namespace sb200 {

constexpr int TS_BM = 128;
constexpr int TS_BN = 256;
constexpr int TS_KBITS = 256;                              // row bits per stage
constexpr int TS_STAGES = 3;
constexpr int TS_A_THREADS = 128;
constexpr int TS_B_THREADS = 256;
constexpr int TS_PRODUCERS = TS_A_THREADS + TS_B_THREADS;
constexpr int TS_THREADS = TS_PRODUCERS + 32;
constexpr int TS_MMA_WARP = TS_PRODUCERS / 32;             // 12
constexpr uint32_t TS_B_ATOM_BYTES = TS_BN * 128;          // one 128-byte K atom of B
constexpr uint32_t TS_B_STAGE_BYTES = TS_B_ATOM_BYTES * (TS_KBITS / 128);
constexpr uint32_t TS_TMEM_COLS = 512;
constexpr uint32_t TS_A_COL0 = 256;
constexpr uint32_t TS_EPI_BYTES = 8 * 32 * 32 * 4;         // per epilogue warp: a 32 x 32 u32 block
constexpr uint32_t TS_SMEM_BYTES = TS_STAGES * TS_B_STAGE_BYTES + 1024 + 256 + TS_EPI_BYTES;
constexpr uint32_t TS_SMEM_BYTES_LEAN = TS_STAGES * TS_B_STAGE_BYTES + 1024 + 256;
// Rows up to this many bits take the coalesced epilogue (the epilogue is a
// larger share of a short tile); longer rows the lean launch.
constexpr uint64_t TS_COALESCE_MAX_BITS = 1u << 17;

struct TsCtl {
    uint64_t full[TS_STAGES];
    uint64_t empty[TS_STAGES];
    uint64_t acc_full, acc_empty, drain;
    uint32_t tmem_base;
    volatile uint32_t abort;
};

__device__ __forceinline__ bool ts_wait(uint32_t bar, uint32_t parity, TsCtl* ctl, DeviceFlags* flags,
                                        uint32_t site, bool drain = false, uint64_t limit_ns = WAIT_LIMIT_NS) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (!drain && ctl->abort) return false;
        if (globaltimer_ns() - t0 > limit_ns) {
            atomicCAS(&flags->error, 0u, site);
            ctl->abort = 1;
            return false;
        }
    }
}

// 64 packed bits -> 16 u32 of A-weighted bytes (byte k carries bit k at
// 2^(k mod 8), or 2^(k mod 4) with kW4).
template <bool kW4>
__device__ __forceinline__ void expand_a64(uint64_t v, uint32_t* o) {
    const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
#pragma unroll
    for (uint32_t b = 0; b < 8; ++b) {
        const uint32_t r = __byte_perm(b < 4 ? lo : hi, 0, (b & 3) * 0x1111u);
        o[2 * b] = r & 0x08040201u;
        o[2 * b + 1] = kW4 ? (r >> 4) & 0x08040201u : r & 0x80402010u;
    }
}

// Where count (i, j) of the local rows goes: the packed triangle of these
// rows, or -- through row_map -- the packed triangle of n_out rows that these
// rows are a subset of (local row r is row row_map[r] there).
// Row-mapped launches may hold padding rows, mapped to ~0: nothing of
// theirs is written.
template <bool kRowMap>
__device__ __forceinline__ bool ts_mapped(const uint32_t* row_map, uint64_t i, uint64_t j) {
    return !kRowMap || (row_map[i] != ~0u && row_map[j] != ~0u);
}

template <bool kRowMap>
__device__ __forceinline__ uint64_t ts_out_index(uint64_t n, uint64_t i, uint64_t j, const uint32_t* row_map,
                                                 uint64_t n_out) {
    if (!kRowMap) return tri_index(n, i, i) - i + j;
    const uint64_t a = row_map[i], b = row_map[j];
    return a < b ? tri_index(n_out, a, b) : tri_index(n_out, b, a);
}

// Work schedule, identical in the three roles of a CTA. k_splits >= 1:
// whole tiles (or k_splits even K slices of each) dealt round robin over the
// grid. k_splits == 0 (stream-K, data-parallel head): the first
// W = floor(tiles / G) x G tiles go whole, round robin (G = grid); CTA c then
// takes the contiguous range [W nk + S c / G, W nk + S (c + 1) / G) of the
// remaining tiles' flattened (tile, K stage) space, S = (tiles - W) x nk,
// cut at tile boundaries into segments. A segment that is not a whole tile
// adds its partial counts into the output, which must be zeroed for the
// tiles from W on; whole tiles store theirs.
struct TsSched {
    uint32_t nk, n_tiles, k_splits, it, whole = 0;
    uint64_t pos = 0, end = 0;
    __device__ __forceinline__ TsSched(uint32_t nk_, uint32_t n_tiles_, uint32_t k_splits_)
        : nk(nk_), n_tiles(n_tiles_), k_splits(k_splits_), it(blockIdx.x) {
        if (k_splits == 0) {
            whole = (n_tiles / gridDim.x) * gridDim.x;
            const uint64_t S = (uint64_t)(n_tiles - whole) * nk;
            pos = (uint64_t)whole * nk + S * blockIdx.x / gridDim.x;
            end = (uint64_t)whole * nk + S * (blockIdx.x + 1) / gridDim.x;
        }
    }
    __device__ __forceinline__ bool next(uint32_t& t, uint32_t& kb0, uint32_t& kb1, bool& partial) {
        if (k_splits == 0) {
            if (it < whole) {
                t = it;
                kb0 = 0;
                kb1 = nk;
                partial = false;
                it += gridDim.x;
                return true;
            }
            if (pos >= end) return false;
            t = (uint32_t)(pos / nk);
            kb0 = (uint32_t)(pos % nk);
            const uint64_t stop = (uint64_t)kb0 + (end - pos);
            kb1 = stop < nk ? (uint32_t)stop : nk;
            pos += kb1 - kb0;
            partial = kb0 != 0 || kb1 != nk;
            return true;
        }
        if (it >= n_tiles * k_splits) return false;
        t = it / k_splits;
        const uint32_t ks = it % k_splits;
        kb0 = (uint32_t)((uint64_t)nk * ks / k_splits);
        kb1 = (uint32_t)((uint64_t)nk * (ks + 1) / k_splits);
        partial = k_splits > 1;
        it += gridDim.x;
        return true;
    }
};

// Thresholded output (the opt-in contract of the reference's thresholded
// mode, bench/bench_threshold.cpp:129-132): pair i < j is reported when its
// count v > 0 and v / (|Xi| + |Xj| - v) >= t in double precision; reported
// pairs are appended (unordered) to pairs/cnts, found counts all of them
// (entries past cap are counted, not written).
struct TsThresh {
    const uint32_t* card;            // |Xi| per row
    double t;
    uint2* pairs;
    uint32_t* cnts;
    unsigned long long cap;
    unsigned long long* found;
};

template <bool kRowMap, bool kW4, bool kThresh = false>
__device__ __forceinline__ void ts_body(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay,
                                        const uint2* __restrict__ tiles, uint32_t n_tiles,
                                        uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags,
                                        const uint32_t* __restrict__ row_map, uint64_t n_out, uint32_t k_splits,
                                        TsThresh th = TsThresh{}) {
    extern __shared__ __align__(1024) unsigned char ts_smem[];
    const uint32_t raw_addr = smem_u32(ts_smem);
    const uint32_t pad = ((raw_addr + 1023u) & ~1023u) - raw_addr;
    uint8_t* ring = ts_smem + pad;
    const uint32_t ring_addr = raw_addr + pad;
    TsCtl* ctl = reinterpret_cast<TsCtl*>(ring + TS_STAGES * TS_B_STAGE_BYTES);
    uint32_t* epi = reinterpret_cast<uint32_t*>(ring + TS_STAGES * TS_B_STAGE_BYTES + 256);
    // The launch decides the epilogue: with TS_SMEM_BYTES of dynamic shared
    // memory the counts are staged through smem and stored coalesced; with
    // TS_SMEM_BYTES_LEAN (no staging buffer, more L1 left for the loads that
    // feed long rows) each lane stores its own row.
    uint32_t dyn_smem;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn_smem));
    const bool coalesced = !kThresh && dyn_smem >= TS_SMEM_BYTES;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t nk = w_pad / (TS_KBITS / 64);               // stages per tile (w_pad % 8 == 0)

    if (tid == 0) {
        for (int s = 0; s < TS_STAGES; ++s) {
            mbar_init(smem_u32(&ctl->full[s]), TS_PRODUCERS);
            mbar_init(smem_u32(&ctl->empty[s]), 1);
        }
        mbar_init(smem_u32(&ctl->acc_full), 1);
        mbar_init(smem_u32(&ctl->acc_empty), 256);
        mbar_init(smem_u32(&ctl->drain), 1);
        ctl->abort = 0;
        fence_barrier_init();
    }
    if (warp == TS_MMA_WARP) {
        tmem_alloc(smem_u32(&ctl->tmem_base), TS_TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = ctl->tmem_base;

    if (warp < TS_MMA_WARP) {
        const bool is_a = tid < TS_A_THREADS;
        const uint32_t prow = is_a ? (uint32_t)tid : (uint32_t)(tid - TS_A_THREADS);   // operand row
        uint32_t g = 0, tcount = 0;
        bool ok = true;
        TsSched sched(nk, n_tiles, k_splits);
        uint32_t t, kb0, kb1;
        bool partial;
        for (; ok && sched.next(t, kb0, kb1, partial); ++tcount) {
            const uint64_t i0 = (uint64_t)tiles[t].x * TS_BM;
            const uint64_t j0 = (uint64_t)tiles[t].y * TS_BN;
            const uint64_t* src = X + (is_a ? i0 + prow : j0 + prow) * lay.pitch;
            // loads run two stages ahead of the expansion
            Row32 v = ldg_row32(stage_ptr(src, kb0, lay.kstride)), nv{};
            if (kb0 + 1 < kb1) nv = ldg_row32(stage_ptr(src, kb0 + 1, lay.kstride));
            for (uint32_t kb = kb0; kb < kb1; ++kb, ++g) {
                const uint32_t s = g % TS_STAGES;
                const uint32_t round = g / TS_STAGES;
                Row32 nnv{};
                if (kb + 2 < kb1) nnv = ldg_row32(stage_ptr(src, kb + 2, lay.kstride));
                if (!ts_wait(smem_u32(&ctl->empty[s]), (round & 1) ^ 1, ctl, flags, ERR_PROD_EMPTY)) {
                    ok = false;
                    break;
                }
                const uint64_t (&w)[4] = v.w;
                if (is_a) {
                    // lanes 32*(warp%4).. ; columns A_COL0 + 64 s + [0, 64)
                    const uint32_t taddr = tmem_base + ((uint32_t)(warp & 3) * 32u << 16) + TS_A_COL0 + 64u * s;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        uint32_t r[32];
                        expand_a64<kW4>(w[2 * h], r);
                        expand_a64<kW4>(w[2 * h + 1], r + 16);
                        tmem_st_32x32b_x32(taddr + 32u * h, r);
                    }
                    tmem_st_wait();
                    tc_fence_before();
                } else {
                    uint8_t* b_stage = ring + s * TS_B_STAGE_BYTES;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        // word q covers K bytes [64q, 64q + 64): atom q/2, chunks 4(q%2)..
                        expand_store<true, kW4>(b_stage + (q >> 1) * TS_B_ATOM_BYTES, prow, (uint32_t)(q & 1),
                                                w[q]);
                    }
                    fence_proxy_async_smem();
                }
                mbar_arrive(smem_u32(&ctl->full[s]));
                v = nv;
                nv = nnv;
            }
            if (!ok) break;
            if (warp >= 8) continue;   // warps 8-11 do not take part in the epilogue
            if (!ts_wait(smem_u32(&ctl->acc_full), tcount & 1, ctl, flags, ERR_PROD_ACCFULL)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t lane_grp = (uint32_t)(warp & 3) * 32u;
            const uint32_t col0 = (uint32_t)(warp >> 2) * 128u;
            unsigned long long local = 0;
            if (coalesced) {
                // Each 32 x 32 block goes through this warp's smem buffer
                // (16-byte chunks XOR-swizzled by row) so that one store
                // instruction writes 32 consecutive counts of one row.
                uint32_t* buf = epi + warp * 1024;
#pragma unroll 1
                for (uint32_t c = 0; c < 4; ++c) {
                    uint32_t r[32];
                    tmem_ld_32x32b_x32(tmem_base + (lane_grp << 16) + col0 + 32u * c, r);
                    tmem_ld_wait();
#pragma unroll
                    for (uint32_t k = 0; k < 8; ++k)
                        *reinterpret_cast<uint4*>(buf + lane * 32 + ((k ^ (lane & 7)) << 2)) =
                            make_uint4(r[4 * k], r[4 * k + 1], r[4 * k + 2], r[4 * k + 3]);
                    __syncwarp();
                    const uint64_t j = j0 + col0 + 32u * c + lane;
#pragma unroll 4
                    for (uint32_t rr = 0; rr < 32; ++rr) {
                        const uint64_t i = i0 + lane_grp + rr;
                        const uint32_t cnt =
                            buf[rr * 32 + ((((uint32_t)lane >> 2) ^ (rr & 7)) << 2) + (lane & 3)] >> (kW4 ? 3 : 7);
                        if (i < n && j >= i && j < n && ts_mapped<kRowMap>(row_map, i, j)) {
                            if (out) {
                                uint32_t* dst = out + ts_out_index<kRowMap>(n, i, j, row_map, n_out);
                                if (partial) atomicAdd(dst, cnt);   // one K segment's share
                                else *dst = cnt;
                            }
                            if (j > i) local += cnt;
                        }
                    }
                    __syncwarp();
                }
            } else {
                // Lean form (no staging buffer): each lane writes its own row.
                const uint64_t i = i0 + lane_grp + lane;
                const bool row_ok = i < n;
                const uint64_t base = row_ok ? tri_index(n, i, i) - i : 0;
#pragma unroll 1
                for (uint32_t c = 0; c < 4; ++c) {
                    uint32_t r[32];
                    tmem_ld_32x32b_x32(tmem_base + (lane_grp << 16) + col0 + 32u * c, r);
                    tmem_ld_wait();
                    if constexpr (kThresh) {
                        // whole tiles only (no partial segments); every lane
                        // stays in the loop for the warp-aggregated appends
                        const uint64_t jb = j0 + col0 + 32u * c;
                        const double ci = row_ok ? (double)th.card[i] : 0.0;
#pragma unroll
                        for (int e = 0; e < 32; ++e) {
                            const uint64_t j = jb + e;
                            const uint32_t cnt = r[e] >> (kW4 ? 3 : 7);
                            bool pass = false;
                            if (row_ok && j > i && j < n) {
                                local += cnt;
                                if (cnt) {
                                    const double u = ci + (double)th.card[j] - (double)cnt;
                                    pass = u > 0.0 && (double)cnt / u >= th.t;
                                }
                            }
                            const uint32_t m = __ballot_sync(0xffffffffu, pass);
                            if (m) {
                                const int leader = __ffs(m) - 1;
                                unsigned long long b0 = 0;
                                if (lane == leader) b0 = atomicAdd(th.found, (unsigned long long)__popc(m));
                                b0 = __shfl_sync(0xffffffffu, b0, leader);
                                if (pass) {
                                    const unsigned long long k = b0 + __popc(m & ((1u << lane) - 1u));
                                    if (k < th.cap) {
                                        th.pairs[k] = make_uint2((uint32_t)i, (uint32_t)j);
                                        th.cnts[k] = cnt;
                                    }
                                }
                            }
                        }
                    } else if (row_ok) {
                        const uint64_t jb = j0 + col0 + 32u * c;
#pragma unroll
                        for (int e = 0; e < 32; ++e) {
                            const uint64_t j = jb + e;
                            const uint32_t cnt = r[e] >> (kW4 ? 3 : 7);
                            if (j >= i && j < n && ts_mapped<kRowMap>(row_map, i, j)) {
                                if (out) {
                                    uint32_t* dst = out + (kRowMap ? ts_out_index<true>(n, i, j, row_map, n_out)
                                                                   : base + j);
                                    if (partial) atomicAdd(dst, cnt);
                                    else *dst = cnt;
                                }
                                if (j > i) local += cnt;
                            }
                        }
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(smem_u32(&ctl->acc_empty));
            local = warp_sum_u64(local);
            if (lane == 0 && local) atomicAdd(&flags->sum, local);
        }
    } else if (lane == 0) {
        const uint32_t idesc = umma_idesc_u8_s32(TS_BM, TS_BN);
        uint32_t g = 0, tcount = 0;
        bool issued = false;
        TsSched sched(nk, n_tiles, k_splits);
        uint32_t t, kb0, kb1;
        bool partial;
        for (; sched.next(t, kb0, kb1, partial); ++tcount) {
            if (!ts_wait(smem_u32(&ctl->acc_empty), (tcount & 1) ^ 1, ctl, flags, ERR_MMA_ACCEMPTY)) break;
            tc_fence_after();
            bool ok = true;
            for (uint32_t kb = kb0; kb < kb1; ++kb, ++g) {
                const uint32_t s = g % TS_STAGES;
                if (!ts_wait(smem_u32(&ctl->full[s]), (g / TS_STAGES) & 1, ctl, flags, ERR_MMA_FULL)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t b_addr = ring_addr + s * TS_B_STAGE_BYTES;
                const uint32_t a_col = tmem_base + TS_A_COL0 + 64u * s;
#pragma unroll
                for (uint32_t kk = 0; kk < TS_KBITS / 32; ++kk) {
                    const uint32_t boff = (kk >> 2) * TS_B_ATOM_BYTES + (kk & 3) * 32u;
                    mma_u8_ts(tmem_base, a_col + 8u * kk, umma_desc_sw128(b_addr + boff, 1024), idesc,
                              (kb != kb0 || kk != 0) ? 1u : 0u);
                }
                issued = true;
                tc_commit(smem_u32(&ctl->empty[s]));
            }
            if (!ok) break;
            tc_commit(smem_u32(&ctl->acc_full));
        }
        if (issued) {
            tc_commit(smem_u32(&ctl->drain));
            ts_wait(smem_u32(&ctl->drain), 0, ctl, flags, ERR_MMA_DRAIN, true);
        }
    }
    if (warp == TS_MMA_WARP) __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == TS_MMA_WARP) {
        tc_fence_after();
        tmem_dealloc(tmem_base, TS_TMEM_COLS);
    }
}

// k_splits: the work schedule (TsSched). 1 = whole tiles round robin;
// > 1 = that many K slices per tile; 0 = stream-K. For any value but 1 the
// partial counts are added into out with atomics (out zeroed beforehand).
__global__ void __launch_bounds__(TS_THREADS, 1)
bb_mma_ts_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* __restrict__ tiles,
                 uint32_t n_tiles, uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags, uint32_t k_splits) {
    ts_body<false, false>(X, n, w_pad, lay, tiles, n_tiles, out, flags, nullptr, 0, k_splits);
}

// Rows of 2^23 .. 2^27 bits: the 4-byte weight cycle keeps D = 8 x count < 2^31.
__global__ void __launch_bounds__(TS_THREADS, 1)
bb_mma_ts_long_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* __restrict__ tiles,
                      uint32_t n_tiles, uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags,
                      uint32_t k_splits) {
    ts_body<false, true>(X, n, w_pad, lay, tiles, n_tiles, out, flags, nullptr, 0, k_splits);
}

// Same kernel over a gathered subset of rows, writing into the triangle of
// the full row set through row_map (the kernel layer's dense block).
__global__ void __launch_bounds__(TS_THREADS, 1)
bb_mma_ts_rows_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* __restrict__ tiles,
                      uint32_t n_tiles, uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags,
                      const uint32_t* __restrict__ row_map, uint64_t n_out, uint32_t k_splits) {
    ts_body<true, false>(X, n, w_pad, lay, tiles, n_tiles, out, flags, row_map, n_out, k_splits);
}

__global__ void __launch_bounds__(TS_THREADS, 1)
bb_mma_ts_rows_long_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay,
                           const uint2* __restrict__ tiles, uint32_t n_tiles, uint32_t* __restrict__ out,
                           DeviceFlags* __restrict__ flags, const uint32_t* __restrict__ row_map, uint64_t n_out,
                           uint32_t k_splits) {
    ts_body<true, true>(X, n, w_pad, lay, tiles, n_tiles, out, flags, row_map, n_out, k_splits);
}

// Thresholded form over contiguous rows (whole tiles round robin).
__global__ void __launch_bounds__(TS_THREADS, 1)
bb_mma_ts_thresh_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* __restrict__ tiles,
                        uint32_t n_tiles, DeviceFlags* __restrict__ flags, TsThresh th) {
    ts_body<false, false, true>(X, n, w_pad, lay, tiles, n_tiles, nullptr, flags, nullptr, 0, 1u, th);
}

__global__ void __launch_bounds__(TS_THREADS, 1)
bb_mma_ts_thresh_long_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay,
                             const uint2* __restrict__ tiles, uint32_t n_tiles, DeviceFlags* __restrict__ flags,
                             TsThresh th) {
    ts_body<false, true, true>(X, n, w_pad, lay, tiles, n_tiles, nullptr, flags, nullptr, 0, 1u, th);
}

}  // namespace sb200
