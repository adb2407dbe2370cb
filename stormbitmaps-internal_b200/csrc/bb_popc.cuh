// bb_popc.cuh -- B x B cell on CUDA cores: tiled X X^T with AND + POPC.
//
// Replaces the reference's per-pair AND+popcount loop over packed words
// (storm.cpp:1155 -> libalgebra.h:2884/2168/2996 via
// STORM_get_intersect_count_func) with one persistent kernel over the whole
// upper triangle of row tiles.
//
// Layout: X is row-major [n_pad][w_pad] u64 in HBM (w_pad a multiple of
// POPC_BK).  A CTA owns a 128 x 128 tile of pairs (rows i0.., rows j0..) and
// walks K in chunks of POPC_BK words, staging both row panels k-major in
// shared memory (double buffered) so each thread reads its 8 + 8 words per k
// conflict-free.  Each of the 256 threads accumulates an 8 x 8 block of
// counts: rows ty + 16a, columns tx + 16b, so 16 neighbouring threads write
// 16 consecutive j of one row at the end (64-byte runs of the packed output).
//
// Roofline: the POPC pipe (16 x 32-bit POPC per SM per clock on sm_100) is
// the bound: 512 bit-ANDs per SM per clock.  Algorithmic work per pair is
// w words; bytes per launch are tiny next to it (compute bound).
#pragma once
#include "common.cuh"

namespace sb200 {

constexpr int POPC_BM = 128;
constexpr int POPC_BN = 128;
constexpr int POPC_BK = 8;             // words per stage
constexpr int POPC_THREADS = 256;
constexpr int POPC_PAD = 1;            // +1 word per k row of the panel: fewer bank conflicts

struct PopcSmem {
    uint64_t a[2][POPC_BK][POPC_BM + POPC_PAD];
    uint64_t b[2][POPC_BK][POPC_BN + POPC_PAD];
};

// Stage one K chunk of a 128-row panel into smem, k-major.
__device__ __forceinline__ void popc_stage(uint64_t (*dst)[POPC_BM + POPC_PAD],
                                           const uint64_t* __restrict__ X, uint64_t row0,
                                           uint64_t pitch, uint32_t k0, int tid) {
    // 128 rows x 8 words = 512 uint4 (2 words each); 2 per thread.
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int idx = tid + q * POPC_THREADS;
        const int r = idx >> 2, part = idx & 3;
        const uint4 v = *reinterpret_cast<const uint4*>(X + (row0 + r) * pitch + k0 + 2 * part);
        dst[2 * part][r] = ((uint64_t)v.y << 32) | v.x;
        dst[2 * part + 1][r] = ((uint64_t)v.w << 32) | v.z;
    }
}

// tiles[t] = (bi, bj) in units of 128 rows, bi <= bj, covering the triangle.
__global__ void __launch_bounds__(POPC_THREADS, 1)
bb_popc_kernel(const uint64_t* __restrict__ X, uint32_t n, uint32_t w_pad, uint64_t pitch,
               const uint2* __restrict__ tiles, uint32_t n_tiles,
               uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags) {
    extern __shared__ __align__(16) unsigned char popc_smem[];
    PopcSmem& sm = *reinterpret_cast<PopcSmem*>(popc_smem);
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const uint32_t nk = w_pad / POPC_BK;

    for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const uint64_t i0 = (uint64_t)tiles[t].x * POPC_BM;
        const uint64_t j0 = (uint64_t)tiles[t].y * POPC_BN;
        uint32_t acc[8][8];
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) acc[a][b] = 0;

        __syncthreads();   // previous tile's readers are done with both buffers
        popc_stage(sm.a[0], X, i0, pitch, 0, tid);
        popc_stage(sm.b[0], X, j0, pitch, 0, tid);
        __syncthreads();

        for (uint32_t kb = 0; kb < nk; ++kb) {
            const int cur = kb & 1;
            if (kb + 1 < nk) {
                popc_stage(sm.a[cur ^ 1], X, i0, pitch, (kb + 1) * POPC_BK, tid);
                popc_stage(sm.b[cur ^ 1], X, j0, pitch, (kb + 1) * POPC_BK, tid);
            }
#pragma unroll
            for (int k = 0; k < POPC_BK; ++k) {
                uint64_t av[8], bv[8];
#pragma unroll
                for (int a = 0; a < 8; ++a) av[a] = sm.a[cur][k][ty + 16 * a];
#pragma unroll
                for (int b = 0; b < 8; ++b) bv[b] = sm.b[cur][k][tx + 16 * b];
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int b = 0; b < 8; ++b) acc[a][b] += __popcll(av[a] & bv[b]);
            }
            __syncthreads();
        }

        // Epilogue: packed upper triangle (i <= j) plus the i < j sum.
        unsigned long long local = 0;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const uint64_t i = i0 + ty + 16 * a;
            if (i >= n) continue;
            const uint64_t base = tri_index(n, i, i) - i;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const uint64_t j = j0 + tx + 16 * b;
                if (j < i || j >= n) continue;
                if (out) out[base + j] = acc[a][b];
                if (j > i) local += acc[a][b];
            }
        }
        local = warp_sum_u64(local);
        if ((tid & 31) == 0 && local) atomicAdd(&flags->sum, local);
    }
}

}  // namespace sb200
