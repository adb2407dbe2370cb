// lowlevel.cu -- the reference's single-pair kernels and example wrappers
// (storm.h:56-148, storm.cpp:15-393), computed on the GPU.
//
// These calls take host pointers and answer one pair (or one small all-pairs
// sum), so each one is a copy in, one launch and a copy out; they exist so a
// program written against storm.h links and gets identical numbers.  The
// STORM_compute_func / STORM_compute_lfunc arguments select CPU SIMD kernels
// in the reference and are ignored here.
#include "oneshot.cuh"
#include <algorithm>
#include <vector>

#include "chunk_engine.cuh"
#include "dense.cuh"

namespace sb200 {

// Bit tests of list positions against a bitmap, summed (storm.cpp:128-141).
__global__ void probe_kernel(const uint64_t* __restrict__ bm, const uint32_t* __restrict__ list, uint32_t n,
                             DeviceFlags* flags) {
    uint32_t c = 0;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const uint32_t x = list[e];
        c += (uint32_t)(bm[x >> 6] >> (x & 63)) & 1u;
    }
    c = warp_sum_u32(c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&flags->sum, (unsigned long long)c);
}

// For every a[i]: the index in b of its two-pointer partner, or -1
// (storm.cpp:90-121: the k-th copy of a value pairs with the k-th copy).
__global__ void match32_kernel(const uint32_t* __restrict__ a, uint32_t na, const uint32_t* __restrict__ b,
                               uint32_t nb, int64_t* __restrict__ match) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x) {
        const uint32_t x = a[i];
        uint32_t lo = 0, hi = i;
        while (lo < hi) {
            const uint32_t m = (lo + hi) >> 1;
            if (a[m] < x) lo = m + 1; else hi = m;
        }
        const uint32_t r = i - lo;
        lo = 0;
        hi = nb;
        while (lo < hi) {
            const uint32_t m = (lo + hi) >> 1;
            if (b[m] < x) lo = m + 1; else hi = m;
        }
        const uint32_t q = lo + r;
        match[i] = (q < nb && b[q] == x) ? (int64_t)q : -1;
    }
}

// Sum of the packed-triangle counts over i < n1 <= j < n1 + n2.
__global__ void rect_sum_kernel(const uint32_t* __restrict__ tri, uint64_t n, uint64_t n1, uint64_t n2,
                                DeviceFlags* flags) {
    unsigned long long s = 0;
    const uint64_t total = n1 * n2;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total;
         p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = p / n2, j = n1 + p % n2;
        s += tri[tri_index(n, i, j)];
    }
    s = warp_sum_u64(s);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(&flags->sum, s);
}

// Upload n rows of n_ints words into a padded dense layout.
static void upload_dense(DevBuf<uint64_t>& d, const uint64_t* rows, uint64_t n, uint32_t n_ints, uint32_t& w_pad,
                         cudaStream_t st) {
    w_pad = (uint32_t)round_up(n_ints ? n_ints : 1, 8);
    const uint64_t n_pad = round_up(n ? n : 1, 256), pitch = dense_pitch(w_pad);
    d.reserve(n_pad * pitch);
    SB_CUDA(cudaMemsetAsync(d.p, 0, n_pad * pitch * sizeof(uint64_t), st));
    if (n && n_ints)
        SB_CUDA(cudaMemcpy2DAsync(d.p, pitch * sizeof(uint64_t), rows, n_ints * sizeof(uint64_t),
                                  n_ints * sizeof(uint64_t), n, cudaMemcpyHostToDevice, st));
}

static uint64_t dense_diag_sum(const uint64_t* vals, uint32_t n, uint32_t n_ints) {
    if (n < 2 || vals == NULL) return 0;
    OneShot& s = one_shot();
    uint32_t w_pad = 0;
    upload_dense(s.w64, vals, n, n_ints, w_pad, s.st);
    return s.dense.run(s.w64.p, n, w_pad, (uint64_t)n_ints * 64, nullptr, STORM_B200_KERNEL_AUTO, s.st);
}

}  // namespace sb200

using namespace sb200;

extern "C" {

uint64_t STORM_intersect_vector16_cardinality(const uint16_t* STORM_RESTRICT v1, const uint16_t* STORM_RESTRICT v2,
                                              const uint32_t len1, const uint32_t len2) {
    if (len1 == 0 || len2 == 0 || v1 == NULL || v2 == NULL) return 0;
    uint64_t r = 0;
    guard([&]() -> int {
        if (len1 > CK_LEN || len2 > CK_LEN) return STORM_B200_ELIMIT;
        STORM_bitmap_t a, b;
        STORM_bitmap_init(&a);
        STORM_bitmap_init(&b);
        a.scalar = const_cast<uint16_t*>(v1);
        a.n_scalar = len1;
        b.scalar = const_cast<uint16_t*>(v2);
        b.n_scalar = len2;
        OneShot& s = one_shot();
        s.pack.add_chunk(0, a);
        s.pack.end_row();
        s.pack.add_chunk(0, b);
        s.pack.end_row();
        r = s.rect(1, 1);
        return 0;
    });
    return r;
}

uint64_t STORM_intersect_vector32_unsafe(const uint32_t* STORM_RESTRICT v1, const uint32_t* STORM_RESTRICT v2,
                                         const uint32_t len1, const uint32_t len2, uint32_t* STORM_RESTRICT out) {
    if (out == NULL || v1 == NULL || v2 == NULL) return 0;
    if (len1 == 0 || len2 == 0) return 0;
    uint64_t r = 0;
    guard([&]() -> int {
        OneShot& s = one_shot();
        s.u32a.reserve(len1);
        s.u32b.reserve(len2);
        s.i64.reserve(len1);
        SB_CUDA(cudaMemcpyAsync(s.u32a.p, v1, len1 * sizeof(uint32_t), cudaMemcpyHostToDevice, s.st));
        SB_CUDA(cudaMemcpyAsync(s.u32b.p, v2, len2 * sizeof(uint32_t), cudaMemcpyHostToDevice, s.st));
        const uint32_t grid = std::min<uint32_t>((len1 + 255) / 256, 1024);
        match32_kernel<<<grid, 256, 0, s.st>>>(s.u32a.p, len1, s.u32b.p, len2, s.i64.p);
        SB_CUDA(cudaGetLastError());
        std::vector<int64_t> m(len1);
        SB_CUDA(cudaMemcpyAsync(m.data(), s.i64.p, len1 * sizeof(int64_t), cudaMemcpyDeviceToHost, s.st));
        SB_CUDA(cudaStreamSynchronize(s.st));
        // Emit the matched index pairs in the reference's order (ascending A).
        uint64_t k = 0;
        for (uint32_t i = 0; i < len1; ++i)
            if (m[i] >= 0) {
                out[k++] = i;
                out[k++] = (uint32_t)m[i];
            }
        r = k;
        return 0;
    });
    return r;
}

uint64_t STORM_intersect_bitmaps_scalar_list(const uint64_t* STORM_RESTRICT b1, const uint64_t* STORM_RESTRICT b2,
                                             const uint32_t* l1, const uint32_t* l2, const uint32_t n1,
                                             const uint32_t n2) {
    // storm.cpp:143-151: walk the shorter list against the other bitmap.
    const uint64_t* bm = (n1 < n2) ? b2 : b1;
    const uint32_t* list = (n1 < n2) ? l1 : l2;
    const uint32_t n = (n1 < n2) ? n1 : n2;
    if (n == 0 || bm == NULL || list == NULL) return 0;
    uint64_t r = 0;
    guard([&]() -> int {
        uint32_t mx = 0;
        for (uint32_t i = 0; i < n; ++i) mx = std::max(mx, list[i]);
        const uint64_t words = (uint64_t)(mx >> 6) + 1;   // the bitmap words the probes reach
        OneShot& s = one_shot();
        s.w64.reserve(words);
        s.u32a.reserve(n);
        s.flags.reserve(1);
        SB_CUDA(cudaMemcpyAsync(s.w64.p, bm, words * sizeof(uint64_t), cudaMemcpyHostToDevice, s.st));
        SB_CUDA(cudaMemcpyAsync(s.u32a.p, list, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s.st));
        SB_CUDA(cudaMemsetAsync(s.flags.p, 0, sizeof(DeviceFlags), s.st));
        probe_kernel<<<std::min<uint32_t>((n + 255) / 256, 512), 256, 0, s.st>>>(s.w64.p, s.u32a.p, n, s.flags.p);
        SB_CUDA(cudaGetLastError());
        r = s.read_sum(s.flags.p);
        return 0;
    });
    return r;
}

uint64_t STORM_wrapper_diag(const uint32_t n_vectors, const uint64_t* vals, const uint32_t n_ints,
                            const STORM_compute_func f) {
    (void)f;
    uint64_t r = 0;
    guard([&]() -> int {
        r = dense_diag_sum(vals, n_vectors, n_ints);
        return 0;
    });
    return r;
}

uint64_t STORM_wrapper_diag_blocked(const uint32_t n_vectors, const uint64_t* vals, const uint32_t n_ints,
                                    const STORM_compute_func f, uint32_t block_size) {
    (void)block_size;
    return STORM_wrapper_diag(n_vectors, vals, n_ints, f);
}

// The bitmaps are the data; the per-vector lists are a CPU shortcut to the
// same counts (storm.cpp:212-243), so the sum is taken over the bitmaps.
uint64_t STORM_wrapper_diag_list(const uint32_t n_vectors, const uint64_t* STORM_RESTRICT vals, const uint32_t n_ints,
                                 const uint32_t* STORM_RESTRICT n_alts, const uint32_t* STORM_RESTRICT alt_positions,
                                 const uint32_t* STORM_RESTRICT alt_offsets, const STORM_compute_func f,
                                 const STORM_compute_lfunc fl, const uint32_t cutoff) {
    (void)n_alts; (void)alt_positions; (void)alt_offsets; (void)fl; (void)cutoff;
    return STORM_wrapper_diag(n_vectors, vals, n_ints, f);
}

uint64_t STORM_wrapper_diag_list_blocked(const uint32_t n_vectors, const uint64_t* STORM_RESTRICT vals,
                                         const uint32_t n_ints, const uint32_t* STORM_RESTRICT n_alts,
                                         const uint32_t* STORM_RESTRICT alt_positions,
                                         const uint32_t* STORM_RESTRICT alt_offsets, const STORM_compute_func f,
                                         const STORM_compute_lfunc fl, const uint32_t cutoff, uint32_t block_size) {
    (void)block_size;
    return STORM_wrapper_diag_list(n_vectors, vals, n_ints, n_alts, alt_positions, alt_offsets, f, fl, cutoff);
}

// All pairs (i in vals1, j in vals2).  The reference loop never resets its
// second offset (storm.cpp:178-182) and so reads past vals2 for i > 0; this
// computes the documented rectangle.
uint64_t STORM_wrapper_square(const uint32_t n1, const uint64_t* STORM_RESTRICT vals1, const uint32_t n2,
                              const uint64_t* STORM_RESTRICT vals2, const uint32_t n_ints,
                              const STORM_compute_func f) {
    (void)f;
    if (n1 == 0 || n2 == 0 || vals1 == NULL || vals2 == NULL) return 0;
    uint64_t r = 0;
    guard([&]() -> int {
        OneShot& s = one_shot();
        const uint64_t n = (uint64_t)n1 + n2;
        std::vector<uint64_t> both(n * n_ints);
        std::copy(vals1, vals1 + (uint64_t)n1 * n_ints, both.begin());
        std::copy(vals2, vals2 + (uint64_t)n2 * n_ints, both.begin() + (uint64_t)n1 * n_ints);
        uint32_t w_pad = 0;
        upload_dense(s.w64, both.data(), n, n_ints, w_pad, s.st);
        s.tri.reserve(tri_size(n));
        s.dense.run(s.w64.p, n, w_pad, (uint64_t)n_ints * 64, s.tri.p, STORM_B200_KERNEL_AUTO, s.st);
        s.flags.reserve(1);
        SB_CUDA(cudaMemsetAsync(s.flags.p, 0, sizeof(DeviceFlags), s.st));
        const uint64_t total = (uint64_t)n1 * n2;
        const uint32_t grid = (uint32_t)std::min<uint64_t>((total + 255) / 256, 4096);
        rect_sum_kernel<<<grid, 256, 0, s.st>>>(s.tri.p, n, n1, n2, s.flags.p);
        SB_CUDA(cudaGetLastError());
        r = s.read_sum(s.flags.p);
        return 0;
    });
    return r;
}

}  // extern "C"
