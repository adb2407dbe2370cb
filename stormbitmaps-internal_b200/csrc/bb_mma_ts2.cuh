// bb_mma_ts2.cuh -- the tcgen05 B x B kernel of bb_mma_ts.cuh with a
// double-buffered accumulator, for short rows.
//
// Same arithmetic (u8 x u8 -> s32, A bytes weighted 2^(k mod 8) or 2^(k mod 4),
// B bytes bit-reversed), same operand movement (A expanded into TMEM by its
// own threads, B expanded into a 128-byte-swizzled smem ring), but the tile
// is 128 x 192 pairs so that TMEM holds two accumulators: [0, 192) and
// [256, 448), with the two A stages at [192, 256) and [448, 512). Dedicated
// epilogue warps drain one accumulator while the MMAs fill the other, so a
// tile boundary no longer stalls the tensor pipe -- the cost that dominates
// when a tile has few K stages (rows of tens of thousands of bits).
//
// Warp roles (480 threads): warps 0-3 expand A rows into TMEM, warps 4-9
// expand B rows into the ring, warp 10 owns TMEM and issues the MMAs, warps
// 11-14 drain the accumulators (warp w reads TMEM lanes 32 (w % 4) ..).
// Two stages of 256 row bits in flight. Whole tiles or stream-K (TsSched).
#pragma once
#include "bb_mma_ts.cuh"

namespace sb200 {

constexpr int T2_BM = 128;
constexpr int T2_BN = 192;
constexpr int T2_STAGES = 2;
constexpr int T2_A_THREADS = 128;
constexpr int T2_B_THREADS = 192;
constexpr int T2_PRODUCERS = T2_A_THREADS + T2_B_THREADS;   // 320
constexpr int T2_MMA_WARP = T2_PRODUCERS / 32;              // 10
constexpr int T2_EPI_WARP0 = T2_MMA_WARP + 1;               // 11 .. 14
constexpr int T2_THREADS = (T2_EPI_WARP0 + 4) * 32;         // 480
constexpr uint32_t T2_B_ATOM_BYTES = T2_BN * 128;
constexpr uint32_t T2_B_STAGE_BYTES = T2_B_ATOM_BYTES * (TS_KBITS / 128);
constexpr uint32_t T2_EPI_BYTES = 4 * 32 * 32 * 4;
constexpr uint32_t T2_SMEM_BYTES = T2_STAGES * T2_B_STAGE_BYTES + 1024 + 256 + T2_EPI_BYTES;

struct T2Ctl {
    uint64_t full[T2_STAGES];
    uint64_t empty[T2_STAGES];
    uint64_t acc_full[2], acc_empty[2], drain;
    uint32_t tmem_base;
    volatile uint32_t abort;
};

__device__ __forceinline__ uint32_t t2_acc_col(uint32_t b) { return b ? 256u : 0u; }
__device__ __forceinline__ uint32_t t2_a_col(uint32_t s) { return s ? 448u : 192u; }

__device__ __forceinline__ bool t2_wait(uint32_t bar, uint32_t parity, T2Ctl* ctl, DeviceFlags* flags,
                                        uint32_t site, bool drain = false) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (!drain && ctl->abort) return false;
        if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
            atomicCAS(&flags->error, 0u, site);
            ctl->abort = 1;
            return false;
        }
    }
}

// tiles[t] = (bi, bj): rows [128 bi, +128) x rows [192 bj, +192). Rows at or
// past n read as zero (no padding needed beyond the rows' own buffer).
template <bool kW4>
__device__ __forceinline__ void ts2_body(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay,
                                         const uint2* __restrict__ tiles, uint32_t n_tiles,
                                         uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags,
                                         uint32_t k_splits) {
    extern __shared__ __align__(1024) unsigned char t2_smem[];
    const uint32_t raw_addr = smem_u32(t2_smem);
    const uint32_t pad = ((raw_addr + 1023u) & ~1023u) - raw_addr;
    uint8_t* ring = t2_smem + pad;
    const uint32_t ring_addr = raw_addr + pad;
    T2Ctl* ctl = reinterpret_cast<T2Ctl*>(ring + T2_STAGES * T2_B_STAGE_BYTES);
    uint32_t* epi = reinterpret_cast<uint32_t*>(ring + T2_STAGES * T2_B_STAGE_BYTES + 256);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t nk = w_pad / (TS_KBITS / 64);

    if (tid == 0) {
        for (int s = 0; s < T2_STAGES; ++s) {
            mbar_init(smem_u32(&ctl->full[s]), T2_PRODUCERS);
            mbar_init(smem_u32(&ctl->empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&ctl->acc_full[b]), 1);
            mbar_init(smem_u32(&ctl->acc_empty[b]), 128);
        }
        mbar_init(smem_u32(&ctl->drain), 1);
        ctl->abort = 0;
        fence_barrier_init();
    }
    if (warp == T2_MMA_WARP) {
        tmem_alloc(smem_u32(&ctl->tmem_base), TS_TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = ctl->tmem_base;

    if (warp < T2_MMA_WARP) {
        // ---- producers
        const bool is_a = tid < T2_A_THREADS;
        const uint32_t prow = is_a ? (uint32_t)tid : (uint32_t)(tid - T2_A_THREADS);
        uint32_t g = 0;
        bool ok = true;
        TsSched sched(nk, n_tiles, k_splits);
        uint32_t t, kb0, kb1;
        bool partial;
        while (ok && sched.next(t, kb0, kb1, partial)) {
            const uint64_t row = is_a ? (uint64_t)tiles[t].x * T2_BM + prow : (uint64_t)tiles[t].y * T2_BN + prow;
            const bool live = row < n;
            const uint64_t* src = X + (live ? row : 0) * lay.pitch;
            // loads run two stages ahead of the expansion
            Row32 v{}, nv{};
            if (live) v = ldg_row32(stage_ptr(src, kb0, lay.kstride));
            if (live && kb0 + 1 < kb1) nv = ldg_row32(stage_ptr(src, kb0 + 1, lay.kstride));
            for (uint32_t kb = kb0; kb < kb1; ++kb, ++g) {
                const uint32_t s = g % T2_STAGES;
                const uint32_t round = g / T2_STAGES;
                Row32 nnv{};
                if (live && kb + 2 < kb1) nnv = ldg_row32(stage_ptr(src, kb + 2, lay.kstride));
                if (!t2_wait(smem_u32(&ctl->empty[s]), (round & 1) ^ 1, ctl, flags, ERR_PROD_EMPTY)) {
                    ok = false;
                    break;
                }
                const uint64_t (&w)[4] = v.w;
                if (is_a) {
                    const uint32_t taddr = tmem_base + ((uint32_t)(warp & 3) * 32u << 16) + t2_a_col(s);
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
                    uint8_t* b_stage = ring + s * T2_B_STAGE_BYTES;
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        expand_store<true, kW4>(b_stage + (q >> 1) * T2_B_ATOM_BYTES, prow, (uint32_t)(q & 1),
                                                w[q]);
                    fence_proxy_async_smem();
                }
                mbar_arrive(smem_u32(&ctl->full[s]));
                v = nv;
                nv = nnv;
            }
        }
    } else if (warp == T2_MMA_WARP) {
        // ---- MMA issuer: accumulator b = item % 2
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_u8_s32(T2_BM, T2_BN);
            uint32_t g = 0, tc = 0;
            bool issued = false;
            TsSched sched(nk, n_tiles, k_splits);
            uint32_t t, kb0, kb1;
            bool partial;
            for (; sched.next(t, kb0, kb1, partial); ++tc) {
                const uint32_t b = tc & 1, use = tc >> 1;
                if (!t2_wait(smem_u32(&ctl->acc_empty[b]), (use & 1) ^ 1, ctl, flags, ERR_MMA_ACCEMPTY)) break;
                tc_fence_after();
                bool ok = true;
                for (uint32_t kb = kb0; kb < kb1; ++kb, ++g) {
                    const uint32_t s = g % T2_STAGES;
                    if (!t2_wait(smem_u32(&ctl->full[s]), (g / T2_STAGES) & 1, ctl, flags, ERR_MMA_FULL)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t b_addr = ring_addr + s * T2_B_STAGE_BYTES;
                    const uint32_t a_col = tmem_base + t2_a_col(s);
#pragma unroll
                    for (uint32_t kk = 0; kk < TS_KBITS / 32; ++kk) {
                        const uint32_t boff = (kk >> 2) * T2_B_ATOM_BYTES + (kk & 3) * 32u;
                        mma_u8_ts(tmem_base + t2_acc_col(b), a_col + 8u * kk, umma_desc_sw128(b_addr + boff, 1024),
                                  idesc, (kb != kb0 || kk != 0) ? 1u : 0u);
                    }
                    issued = true;
                    tc_commit(smem_u32(&ctl->empty[s]));
                }
                if (!ok) break;
                tc_commit(smem_u32(&ctl->acc_full[b]));
            }
            if (issued) {
                tc_commit(smem_u32(&ctl->drain));
                t2_wait(smem_u32(&ctl->drain), 0, ctl, flags, ERR_MMA_DRAIN, true);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: this warp drains TMEM lanes 32 (warp % 4) .., all 192 columns
        const uint32_t lane_grp = (uint32_t)(warp & 3) * 32u;
        uint32_t* buf = epi + (warp - T2_EPI_WARP0) * 1024;
        uint32_t tc = 0;
        TsSched sched(nk, n_tiles, k_splits);
        uint32_t t, kb0, kb1;
        bool partial;
        for (; sched.next(t, kb0, kb1, partial); ++tc) {
            const uint32_t b = tc & 1, use = tc >> 1;
            if (!t2_wait(smem_u32(&ctl->acc_full[b]), use & 1, ctl, flags, ERR_PROD_ACCFULL)) break;
            tc_fence_after();
            const uint64_t i0 = (uint64_t)tiles[t].x * T2_BM, j0 = (uint64_t)tiles[t].y * T2_BN;
            unsigned long long local = 0;
#pragma unroll 1
            for (uint32_t c = 0; c < T2_BN / 32; ++c) {
                uint32_t r[32];
                tmem_ld_32x32b_x32(tmem_base + (lane_grp << 16) + t2_acc_col(b) + 32u * c, r);
                tmem_ld_wait();
#pragma unroll
                for (uint32_t k = 0; k < 8; ++k)
                    *reinterpret_cast<uint4*>(buf + lane * 32 + ((k ^ (lane & 7)) << 2)) =
                        make_uint4(r[4 * k], r[4 * k + 1], r[4 * k + 2], r[4 * k + 3]);
                __syncwarp();
                const uint64_t j = j0 + 32u * c + lane;
#pragma unroll 4
                for (uint32_t rr = 0; rr < 32; ++rr) {
                    const uint64_t i = i0 + lane_grp + rr;
                    const uint32_t cnt =
                        buf[rr * 32 + ((((uint32_t)lane >> 2) ^ (rr & 7)) << 2) + (lane & 3)] >> (kW4 ? 3 : 7);
                    if (i < n && j >= i && j < n) {
                        if (out) {
                            uint32_t* dst = out + tri_index(n, i, i) - i + j;
                            if (partial) atomicAdd(dst, cnt);
                            else *dst = cnt;
                        }
                        if (j > i) local += cnt;
                    }
                }
                __syncwarp();
            }
            tc_fence_before();
            mbar_arrive(smem_u32(&ctl->acc_empty[b]));
            local = warp_sum_u64(local);
            if (lane == 0 && local) atomicAdd(&flags->sum, local);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == T2_MMA_WARP) {
        tc_fence_after();
        tmem_dealloc(tmem_base, TS_TMEM_COLS);
    }
}

__global__ void __launch_bounds__(T2_THREADS, 1)
bb_mma_ts2_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* __restrict__ tiles,
                  uint32_t n_tiles, uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags, uint32_t k_splits) {
    ts2_body<false>(X, n, w_pad, lay, tiles, n_tiles, out, flags, k_splits);
}

__global__ void __launch_bounds__(T2_THREADS, 1)
bb_mma_ts2_long_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* __restrict__ tiles,
                       uint32_t n_tiles, uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags,
                       uint32_t k_splits) {
    ts2_body<true>(X, n, w_pad, lay, tiles, n_tiles, out, flags, k_splits);
}

}  // namespace sb200
