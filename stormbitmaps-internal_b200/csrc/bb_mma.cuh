// bb_mma.cuh -- B x B cell on the 5th-generation tensor cores (tcgen05).
//
// Same contract as bb_popc.cuh (the reference's dense cell, storm.cpp:1155 /
// libalgebra.h:2884): per-pair |Xi & Xj| over packed rows, packed upper
// triangle out, sum over i < j.  Here the pair counts are an integer matrix
// product computed exactly on the tensor cores:
//
//   * A 128 x 256 tile of pairs is one tcgen05.mma (kind::i8, M=128, N=256,
//     K=32) chain accumulating in TMEM (256 of the 512 columns, s32).
//   * Packed bits are expanded to u8 in shared memory, in the K-major
//     128-byte-swizzle layout the MMA reads.  Expansion is one PRMT (replicate
//     a byte) and one AND per 4 output bytes: A bytes carry their bit at
//     weight 2^(k mod 8), B bytes at weight 2^(7 - k mod 8) (bit-reversed
//     word), so every product is 0 or exactly 128 and D = 128 * |Xi & Xj|.
//     The u8 x u8 -> s32 accumulation is exact; counts must stay below 2^24
//     (D < 2^31), so rows longer than 2^23 bits use the POPC kernel.
//   * Warp roles: warps 0-7 load packed words (16 B per row per stage) and
//     expand them, then drain the accumulator (tcgen05.ld) for the epilogue;
//     warp 8 owns TMEM and one elected lane issues the MMAs.  A 4-stage
//     shared-memory ring (48 KB per stage: 128 + 256 rows x 128 K-bytes) is
//     handed over with mbarriers; tcgen05.commit releases a stage when the
//     MMAs reading it complete.
//   * Every wait is bounded (WAIT_LIMIT_NS); on expiry the kernel records
//     the site in flags->error, drains its own MMAs (bounded), frees TMEM and
//     returns -- it never spins forever.
//
// Roofline: tensor-bound.  Algorithmic work per pair = row bits (u8 MACs).
#pragma once
#include "common.cuh"
#include "tc_ptx.cuh"

namespace sb200 {

constexpr int MMA_BM = 128;
constexpr int MMA_BN = 256;
constexpr int MMA_KB = 128;                              // K bytes (= row bits) per stage
constexpr int MMA_STAGES = 4;
constexpr int MMA_PRODUCERS = 256;
constexpr int MMA_THREADS = MMA_PRODUCERS + 32;
constexpr uint32_t MMA_A_BYTES = MMA_BM * MMA_KB;        // 16 KB
constexpr uint32_t MMA_B_BYTES = MMA_BN * MMA_KB;        // 32 KB
constexpr uint32_t MMA_STAGE_BYTES = MMA_A_BYTES + MMA_B_BYTES;
constexpr uint32_t MMA_TMEM_COLS = 256;
constexpr uint32_t MMA_SMEM_BYTES = MMA_STAGES * MMA_STAGE_BYTES + 1024 /*align slack*/ + 256;
constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;        // 2 s per wait
constexpr uint32_t MMA_MAX_BITS = 1u << 23;        // 8-byte weight cycle (D = 128 x count)
constexpr uint32_t MMA_MAX_BITS_W4 = 1u << 27;     // 4-byte weight cycle (D = 8 x count)

// Error sites (flags->error = site).
enum : uint32_t {
    ERR_PROD_EMPTY = 0x101, ERR_PROD_ACCFULL = 0x102,
    ERR_MMA_ACCEMPTY = 0x201, ERR_MMA_FULL = 0x202, ERR_MMA_DRAIN = 0x203,
};

struct MmaCtl {
    uint64_t full[MMA_STAGES];
    uint64_t empty[MMA_STAGES];
    uint64_t acc_full, acc_empty, drain;
    uint32_t tmem_base;
    volatile uint32_t abort;
};

// Bounded mbarrier wait.  Gives up when another role has aborted (unless
// `drain`, which must outlive an abort) or after WAIT_LIMIT_NS.
__device__ __forceinline__ bool mma_wait(uint32_t bar, uint32_t parity, MmaCtl* ctl,
                                         DeviceFlags* flags, uint32_t site, bool drain = false) {
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

// Expand 64 packed bits (one task) into 4 swizzled 16-byte chunks.
// kW4: weights cycle over 4 bytes instead of 8 (A 2^(k mod 4), B 2^(3 - k mod 4),
// every product 0 or 8), exact for rows up to 2^27 bits instead of 2^23.
template <bool kIsB, bool kW4 = false>
__device__ __forceinline__ void expand_store(uint8_t* op_base, uint32_t r, uint32_t half, uint64_t v) {
    uint8_t* row = op_base + (r >> 3) * 1024u + (r & 7u) * 128u;
    const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
    const uint32_t rl = __brev(lo), rh = __brev(hi);
#pragma unroll
    for (uint32_t q = 0; q < 4; ++q) {
        uint4 o;
        const uint32_t b0 = 2 * q, b1 = 2 * q + 1;   // input byte indices 0..7 of v
        if (!kIsB) {
            const uint32_t src0 = b0 < 4 ? lo : hi, src1 = b1 < 4 ? lo : hi;
            const uint32_t r0 = __byte_perm(src0, 0, (b0 & 3) * 0x1111u);
            const uint32_t r1 = __byte_perm(src1, 0, (b1 & 3) * 0x1111u);
            o.x = r0 & 0x08040201u;
            o.y = kW4 ? (r0 >> 4) & 0x08040201u : r0 & 0x80402010u;
            o.z = r1 & 0x08040201u;
            o.w = kW4 ? (r1 >> 4) & 0x08040201u : r1 & 0x80402010u;
        } else {
            // Byte b of a 32-bit word, bit-reversed, is byte (3 - b) of __brev(word).
            const uint32_t src0 = b0 < 4 ? rl : rh, src1 = b1 < 4 ? rl : rh;
            const uint32_t r0 = __byte_perm(src0, 0, (3u - (b0 & 3)) * 0x1111u);
            const uint32_t r1 = __byte_perm(src1, 0, (3u - (b1 & 3)) * 0x1111u);
            o.x = kW4 ? (r0 >> 4) & 0x01020408u : r0 & 0x10204080u;
            o.y = r0 & 0x01020408u;
            o.z = kW4 ? (r1 >> 4) & 0x01020408u : r1 & 0x10204080u;
            o.w = r1 & 0x01020408u;
        }
        const uint32_t chunk = half * 4 + q;
        *reinterpret_cast<uint4*>(row + ((chunk ^ (r & 7u)) << 4)) = o;
    }
}

// tiles[t] = (bi, bj): rows [128 bi, +128) x rows [256 bj, +256).
__global__ void __launch_bounds__(MMA_THREADS, 1)
bb_mma_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, uint64_t pitch,
              const uint2* __restrict__ tiles, uint32_t n_tiles,
              uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags) {
    extern __shared__ __align__(1024) unsigned char mma_smem[];
    const uint32_t raw_addr = smem_u32(mma_smem);
    const uint32_t pad = ((raw_addr + 1023u) & ~1023u) - raw_addr;
    uint8_t* ring = mma_smem + pad;                           // 1024-aligned stages
    const uint32_t ring_addr = raw_addr + pad;
    MmaCtl* ctl = reinterpret_cast<MmaCtl*>(ring + MMA_STAGES * MMA_STAGE_BYTES);

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t nk = w_pad / 2;                            // 128-bit stages per row

    if (tid == 0) {
        for (int s = 0; s < MMA_STAGES; ++s) {
            mbar_init(smem_u32(&ctl->full[s]), MMA_PRODUCERS);
            mbar_init(smem_u32(&ctl->empty[s]), 1);
        }
        mbar_init(smem_u32(&ctl->acc_full), 1);
        mbar_init(smem_u32(&ctl->acc_empty), MMA_PRODUCERS);
        mbar_init(smem_u32(&ctl->drain), 1);
        ctl->abort = 0;
        fence_barrier_init();
    }
    if (warp == 8) {
        tmem_alloc(smem_u32(&ctl->tmem_base), MMA_TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = ctl->tmem_base;

    if (warp < 8) {
        // ------------------------------------------------ producers + epilogue
        uint32_t g = 0, tcount = 0;
        bool ok = true;
        for (uint32_t t = blockIdx.x; t < n_tiles && ok; t += gridDim.x, ++tcount) {
            const uint64_t i0 = (uint64_t)tiles[t].x * MMA_BM;
            const uint64_t j0 = (uint64_t)tiles[t].y * MMA_BN;
            // Three tasks per thread: task = (operand row, 64-bit half).
            const uint64_t* src[3];
            uint32_t trow[3], thalf[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const uint32_t task = tid + q * MMA_PRODUCERS;
                trow[q] = task >> 1;
                thalf[q] = task & 1;
                const uint64_t grow = trow[q] < MMA_BM ? i0 + trow[q] : j0 + (trow[q] - MMA_BM);
                src[q] = X + grow * pitch + thalf[q];
            }
            uint64_t v[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) v[q] = __ldg(src[q]);
            for (uint32_t kb = 0; kb < nk; ++kb, ++g) {
                const uint32_t s = g % MMA_STAGES;
                const uint32_t round = g / MMA_STAGES;
                uint64_t nv[3] = {0, 0, 0};
                if (kb + 1 < nk) {
#pragma unroll
                    for (int q = 0; q < 3; ++q) nv[q] = __ldg(src[q] + 2 * (kb + 1));
                }
                if (!mma_wait(smem_u32(&ctl->empty[s]), (round & 1) ^ 1, ctl, flags, ERR_PROD_EMPTY)) {
                    ok = false;
                    break;
                }
                uint8_t* a_op = ring + s * MMA_STAGE_BYTES;
                uint8_t* b_op = a_op + MMA_A_BYTES;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    if (trow[q] < MMA_BM) expand_store<false>(a_op, trow[q], thalf[q], v[q]);
                    else expand_store<true>(b_op, trow[q] - MMA_BM, thalf[q], v[q]);
                }
                fence_proxy_async_smem();
                mbar_arrive(smem_u32(&ctl->full[s]));
#pragma unroll
                for (int q = 0; q < 3; ++q) v[q] = nv[q];
            }
            if (!ok) break;
            // Epilogue: this warp reads TMEM lanes 32*(warp%4).. and 128 columns.
            if (!mma_wait(smem_u32(&ctl->acc_full), tcount & 1, ctl, flags, ERR_PROD_ACCFULL)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t lane_grp = (uint32_t)(warp & 3) * 32u;
            const uint32_t col0 = (uint32_t)(warp >> 2) * 128u;
            const uint64_t i = i0 + lane_grp + lane;
            const bool row_ok = i < n;
            const uint64_t base = row_ok ? tri_index(n, i, i) - i : 0;
            unsigned long long local = 0;
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
                        const uint32_t cnt = r[e] >> 7;
                        if (j >= i && j < n) {
                            if (out) out[base + j] = cnt;
                            if (j > i) local += cnt;
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
        // ------------------------------------------------ MMA issuer
        const uint32_t idesc = umma_idesc_u8_s32(MMA_BM, MMA_BN);
        uint32_t g = 0, tcount = 0;
        bool issued = false;
        for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x, ++tcount) {
            if (!mma_wait(smem_u32(&ctl->acc_empty), (tcount & 1) ^ 1, ctl, flags, ERR_MMA_ACCEMPTY)) break;
            tc_fence_after();
            bool ok = true;
            for (uint32_t kb = 0; kb < nk; ++kb, ++g) {
                const uint32_t s = g % MMA_STAGES;
                if (!mma_wait(smem_u32(&ctl->full[s]), (g / MMA_STAGES) & 1, ctl, flags, ERR_MMA_FULL)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t a_addr = ring_addr + s * MMA_STAGE_BYTES;
                const uint32_t b_addr = a_addr + MMA_A_BYTES;
#pragma unroll
                for (uint32_t kk = 0; kk < MMA_KB / 32; ++kk) {
                    mma_u8(tmem_base, umma_desc_sw128(a_addr + 32u * kk, 1024),
                           umma_desc_sw128(b_addr + 32u * kk, 1024), idesc, (kb | kk) != 0);
                }
                issued = true;
                tc_commit(smem_u32(&ctl->empty[s]));
            }
            if (!ok) break;
            tc_commit(smem_u32(&ctl->acc_full));
        }
        if (issued) {
            // Drain: every MMA this thread issued must finish before TMEM is freed.
            tc_commit(smem_u32(&ctl->drain));
            mma_wait(smem_u32(&ctl->drain), 0, ctl, flags, ERR_MMA_DRAIN, true);
        }
    }
    if (warp == 8) __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp == 8) {
        tc_fence_after();
        tmem_dealloc(tmem_base, MMA_TMEM_COLS);
    }
}

}  // namespace sb200
