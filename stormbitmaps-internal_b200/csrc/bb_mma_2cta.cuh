// bb_mma_2cta.cuh -- the tcgen05 B x B kernel on CTA pairs (cta_group::2).
//
// Same arithmetic as bb_mma_ts.cuh (u8 x u8 -> s32, A bytes weighted
// 2^(k mod 8) or 2^(k mod 4), B bytes bit-reversed, D = 128 |Xi & Xj| or
// 8 |Xi & Xj|), on a different machine shape.  The single-CTA kernels are fed
// through shared memory: per 256-bit stage a CTA writes 64 KiB of expanded B
// and its MMAs read the same 64 KiB back while they compute 128 x 256 x 256
// MACs -- shared memory and the tensor pipe both at their limit.  Here two
// CTAs of a cluster share one MMA of M = 256 (each CTA's 128 A rows in its
// own tensor memory) against N = 256 B rows, of which each CTA expands and
// holds only its 128: the hardware reads each half once for both SMs, so the
// shared-memory bytes per MAC halve and the tensor pipe sets the pace.
//
// Per CTA (288 threads): warps 0-3 expand its A rows into TMEM
// (tcgen05.st), warps 4-7 expand its half of the B rows into a 4-stage
// 128-byte-swizzled ring, warp 8 owns TMEM; in the even CTA of the pair
// (the leader) warp 8's elected lane issues tcgen05.mma.cta_group::2 and
// tcgen05.commit with .multicast::cluster, so that stage releases and
// accumulator-ready signals reach both CTAs' barriers.  Producers and the
// epilogue of both CTAs arrive on the leader's barriers (mapa +
// mbarrier.arrive.release.cluster, one arrival per warp).  Warps 0-7 drain
// the CTA's 128 x 256 accumulator.  TMEM (both CTAs, allocated as a pair):
// accumulator [0, 256) + A stages 4 x 64.  Every wait is bounded (2 s); on
// expiry the site is recorded and the roles stop; both CTAs meet at a cluster
// barrier before tensor memory is freed, so neither leaves while the other
// can still signal it.
//
// tiles[t] = (bi, bj), bi <= bj: A rows [256 bi, +256) x B rows [256 bj,
// +256); the pair's CTA r takes A rows 256 bi + 128 r .. and B rows
// 256 bj + 128 r ..; accumulator column c is B row 256 bj + c.  Whole tiles
// dealt round robin over the clusters.  No TMA anywhere: operands are
// expanded by threads from global loads.
#pragma once
#include "bb_mma_ts.cuh"

namespace sb200 {

constexpr int C2_BM = 256;                                 // A rows per tile (128 per CTA)
constexpr int C2_BN = 256;                                 // B rows per tile (128 per CTA)
constexpr int C2_STAGES = 4;
constexpr int C2_A_THREADS = 128;
constexpr int C2_B_THREADS = 128;
constexpr int C2_PRODUCERS = C2_A_THREADS + C2_B_THREADS;  // 256
constexpr int C2_MMA_WARP = C2_PRODUCERS / 32;             // 8
constexpr int C2_THREADS = C2_PRODUCERS + 32;              // 288
constexpr uint32_t C2_B_ATOM_BYTES = 128 * 128;            // 128 rows x one 128-byte K atom
constexpr uint32_t C2_B_STAGE_BYTES = C2_B_ATOM_BYTES * (TS_KBITS / 128);   // 32 KiB
constexpr uint32_t C2_TMEM_COLS = 512;
constexpr uint32_t C2_A_COL0 = 256;
constexpr uint32_t C2_EPI_BYTES = 8 * 32 * 32 * 4;         // per epilogue warp: a 32 x 32 u32 block
constexpr uint32_t C2_SMEM_BYTES = C2_STAGES * C2_B_STAGE_BYTES + 1024 + 256 + C2_EPI_BYTES;
constexpr uint32_t C2_WARPS_PER_SIDE = 8;                  // arrivals per CTA on full / acc_empty

enum : uint32_t {
    ERR_C2_PROD_EMPTY = 0x401, ERR_C2_PROD_ACCFULL = 0x402,
    ERR_C2_MMA_ACCEMPTY = 0x403, ERR_C2_MMA_FULL = 0x404, ERR_C2_DRAIN = 0x405,
};

struct C2Ctl {
    uint64_t full[C2_STAGES];       // leader: both CTAs' producer warps
    uint64_t empty[C2_STAGES];      // both: the leader's commit
    uint64_t acc_full, acc_empty, drain;
    uint32_t tmem_base;
    volatile uint32_t abort;
};

__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// The shared::cluster address of the same shared-memory offset in CTA `rank`.
__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_cluster(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc_pair(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish_pair() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Arrive on `bar` (the same offset) in every CTA of cta_mask once the pair's
// tcgen05 operations issued so far by this thread have completed.
__device__ __forceinline__ void tc_commit_pair(uint32_t bar, uint16_t cta_mask) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            bar),
        "h"(cta_mask)
        : "memory");
}

// D[tmem] (+)= A[tmem] * B[smem]^T over the CTA pair: M = 256 (128 lanes of
// A and D in each CTA's TMEM), B's N rows split over the two CTAs' smem.
__device__ __forceinline__ void mma_u8_pair(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

template <bool kCluster>
__device__ __forceinline__ bool c2_wait(uint32_t bar, uint32_t parity, C2Ctl* ctl, DeviceFlags* flags, uint32_t site,
                                        bool drain = false) {
    auto poll = [&]() { return kCluster ? mbar_try_wait_cluster(bar, parity) : mbar_try_wait(bar, parity); };
    if (poll()) return true;
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        if (poll()) return true;
        if (!drain && ctl->abort) return false;
        if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
            atomicCAS(&flags->error, 0u, site);
            ctl->abort = 1;
            return false;
        }
    }
}

template <bool kW4>
__device__ __forceinline__ void c2_body(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay,
                                        const uint2* __restrict__ tiles, uint32_t n_tiles,
                                        uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags) {
    extern __shared__ __align__(1024) unsigned char c2_smem[];
    const uint32_t raw_addr = smem_u32(c2_smem);
    const uint32_t pad = ((raw_addr + 1023u) & ~1023u) - raw_addr;   // the same in both CTAs
    uint8_t* ring = c2_smem + pad;
    const uint32_t ring_addr = raw_addr + pad;
    C2Ctl* ctl = reinterpret_cast<C2Ctl*>(ring + C2_STAGES * C2_B_STAGE_BYTES);
    uint32_t* epi = reinterpret_cast<uint32_t*>(ring + C2_STAGES * C2_B_STAGE_BYTES + 256);
    uint32_t dyn_smem;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn_smem));
    const bool coalesced = dyn_smem >= C2_SMEM_BYTES;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = cluster_ctarank();
    const bool leader = rank == 0;
    const uint32_t cid = blockIdx.x >> 1, n_clusters = gridDim.x >> 1;
    const uint32_t nk = w_pad / (TS_KBITS / 64);              // stages per tile (w_pad % 8 == 0)

    if (tid == 0) {
        for (int s = 0; s < C2_STAGES; ++s) {
            mbar_init(smem_u32(&ctl->full[s]), 2 * C2_WARPS_PER_SIDE);
            mbar_init(smem_u32(&ctl->empty[s]), 1);
        }
        mbar_init(smem_u32(&ctl->acc_full), 1);
        mbar_init(smem_u32(&ctl->acc_empty), 2 * C2_WARPS_PER_SIDE);
        mbar_init(smem_u32(&ctl->drain), 1);
        ctl->abort = 0;
        fence_barrier_init();
    }
    if (warp == C2_MMA_WARP) {
        tmem_alloc_pair(smem_u32(&ctl->tmem_base), C2_TMEM_COLS);
        tmem_relinquish_pair();
    }
    tc_fence_before();
    cluster_sync_all();            // barriers initialised in both CTAs before any remote arrival
    tc_fence_after();
    const uint32_t tmem_base = ctl->tmem_base;
    const uint32_t lead_full0 = mapa_shared(smem_u32(&ctl->full[0]), 0);
    const uint32_t lead_acc_empty = mapa_shared(smem_u32(&ctl->acc_empty), 0);
    const bool has_work = cid < n_tiles;

    if (warp < C2_MMA_WARP) {
        const bool is_a = tid < C2_A_THREADS;
        const uint32_t prow = is_a ? (uint32_t)tid : (uint32_t)(tid - C2_A_THREADS);   // row within the CTA's half
        uint32_t g = 0, tcount = 0;
        bool ok = true;
        for (uint32_t t = cid; ok && t < n_tiles; t += n_clusters, ++tcount) {
            const uint64_t i0 = (uint64_t)tiles[t].x * C2_BM + 128u * rank;
            const uint64_t j0 = (uint64_t)tiles[t].y * C2_BN;
            const uint64_t* src = X + (is_a ? i0 + prow : j0 + 128u * rank + prow) * lay.pitch;
            // loads run two stages ahead of the expansion
            Row32 v = ldg_row32(src), nv{};
            if (1 < nk) nv = ldg_row32(stage_ptr(src, 1, lay.kstride));
            for (uint32_t kb = 0; kb < nk; ++kb, ++g) {
                const uint32_t s = g % C2_STAGES;
                const uint32_t round = g / C2_STAGES;
                Row32 nnv{};
                if (kb + 2 < nk) nnv = ldg_row32(stage_ptr(src, kb + 2, lay.kstride));
                if (!c2_wait<true>(smem_u32(&ctl->empty[s]), (round & 1) ^ 1, ctl, flags, ERR_C2_PROD_EMPTY)) {
                    ok = false;
                    break;
                }
                const uint64_t (&w)[4] = v.w;
                if (is_a) {
                    const uint32_t taddr = tmem_base + ((uint32_t)(warp & 3) * 32u << 16) + C2_A_COL0 + 64u * s;
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
                    uint8_t* b_stage = ring + s * C2_B_STAGE_BYTES;
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        expand_store<true, kW4>(b_stage + (q >> 1) * C2_B_ATOM_BYTES, prow, (uint32_t)(q & 1), w[q]);
                    fence_proxy_async_smem();
                }
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(lead_full0 + 8u * s);
                v = nv;
                nv = nnv;
            }
            if (!ok) break;
            // ---- epilogue: this CTA's 128 x 256 accumulator
            if (!c2_wait<true>(smem_u32(&ctl->acc_full), tcount & 1, ctl, flags, ERR_C2_PROD_ACCFULL)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t lane_grp = (uint32_t)(warp & 3) * 32u;
            const uint32_t col0 = (uint32_t)(warp >> 2) * 128u;
            unsigned long long local = 0;
            if (coalesced) {
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
                        if (i < n && j >= i && j < n) {
                            if (out) out[tri_index(n, i, i) - i + j] = cnt;
                            if (j > i) local += cnt;
                        }
                    }
                    __syncwarp();
                }
            } else {
                const uint64_t i = i0 + lane_grp + lane;
                const bool row_ok = i < n;
                const uint64_t base = row_ok ? tri_index(n, i, i) - i : 0;
#pragma unroll 1
                for (uint32_t c = 0; c < 4; ++c) {
                    uint32_t r[32];
                    tmem_ld_32x32b_x32(tmem_base + (lane_grp << 16) + col0 + 32u * c, r);
                    tmem_ld_wait();
                    if (row_ok) {
                        const uint64_t jb = j0 + col0 + 32u * c;
#pragma unroll
                        for (int e = 0; e < 32; ++e) {
                            const uint64_t j = jb + e;
                            const uint32_t cnt = r[e] >> (kW4 ? 3 : 7);
                            if (j >= i && j < n) {
                                if (out) out[base + j] = cnt;
                                if (j > i) local += cnt;
                            }
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(lead_acc_empty);
            local = warp_sum_u64(local);
            if (lane == 0 && local) atomicAdd(&flags->sum, local);
        }
    } else if (leader && lane == 0) {
        const uint32_t idesc = umma_idesc_u8_s32(C2_BM, C2_BN);
        uint32_t g = 0, tcount = 0;
        bool issued = false;
        for (uint32_t t = cid; t < n_tiles; t += n_clusters, ++tcount) {
            if (!c2_wait<true>(smem_u32(&ctl->acc_empty), (tcount & 1) ^ 1, ctl, flags, ERR_C2_MMA_ACCEMPTY)) break;
            tc_fence_after();
            bool ok = true;
            for (uint32_t kb = 0; kb < nk; ++kb, ++g) {
                const uint32_t s = g % C2_STAGES;
                if (!c2_wait<true>(smem_u32(&ctl->full[s]), (g / C2_STAGES) & 1, ctl, flags, ERR_C2_MMA_FULL)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t b_addr = ring_addr + s * C2_B_STAGE_BYTES;
                const uint32_t a_col = tmem_base + C2_A_COL0 + 64u * s;
#pragma unroll
                for (uint32_t kk = 0; kk < TS_KBITS / 32; ++kk) {
                    const uint32_t boff = (kk >> 2) * C2_B_ATOM_BYTES + (kk & 3) * 32u;
                    mma_u8_pair(tmem_base, a_col + 8u * kk, umma_desc_sw128(b_addr + boff, 1024), idesc,
                                (kb != 0 || kk != 0) ? 1u : 0u);
                }
                issued = true;
                tc_commit_pair(smem_u32(&ctl->empty[s]), 0x3);
            }
            if (!ok) break;
            tc_commit_pair(smem_u32(&ctl->acc_full), 0x3);
        }
        if (issued) tc_commit_pair(smem_u32(&ctl->drain), 0x3);
    }
    // Both CTAs: the pair's MMAs must have completed before tensor memory is
    // freed (the leader's last commit reaches both drain barriers).
    if (warp == C2_MMA_WARP && lane == 0 && has_work)
        c2_wait<true>(smem_u32(&ctl->drain), 0, ctl, flags, ERR_C2_DRAIN, true);
    if (warp == C2_MMA_WARP) __syncwarp();
    tc_fence_before();
    __syncthreads();
    cluster_sync_all();            // neither CTA leaves while the other can still signal it
    if (warp == C2_MMA_WARP) {
        tc_fence_after();
        tmem_dealloc_pair(tmem_base, C2_TMEM_COLS);
    }
}

__global__ void __launch_bounds__(C2_THREADS, 1)
bb_mma_2cta_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* __restrict__ tiles,
                   uint32_t n_tiles, uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags) {
    c2_body<false>(X, n, w_pad, lay, tiles, n_tiles, out, flags);
}

__global__ void __launch_bounds__(C2_THREADS, 1)
bb_mma_2cta_long_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* __restrict__ tiles,
                        uint32_t n_tiles, uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags) {
    c2_body<true>(X, n, w_pad, lay, tiles, n_tiles, out, flags);
}

}  // namespace sb200
