// dense.cuh -- host side of the bitmap x bitmap all-pairs engine shared by
// STORM_contiguous_t, the STORM_wrapper_* calls and the dense tiles of the
// chunked engine.
#pragma once
#include <vector>
#include "common.cuh"

namespace sb200 {

// Device rows: X is [n_pad][w_pad] u64, zero padded, n_pad % 256 == 0 and
// w_pad % 8 == 0.
struct DenseEngine {
    DevBuf<uint2> d_tiles;
    uint64_t tiles_n = ~0ull;
    int tiles_kind = -1;
    uint32_t n_tiles = 0;
    DevBuf<DeviceFlags> d_flags;
    LaunchLog log;

    ~DenseEngine() { log.destroy(); }

    // Returns the sum over i < j; writes the packed upper triangle to d_out
    // when non-null.  `row_bits` is the logical row length (decides whether
    // the exact tensor-core kernel applies).  Synchronous.
    uint64_t run(const uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits, uint32_t* d_out,
                 int kernel_pref, cudaStream_t st);
};

inline uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

}  // namespace sb200
