// dense.cuh -- host side of the bitmap x bitmap all-pairs engine shared by
// STORM_contiguous_t, the STORM_wrapper_* calls and the dense tiles of the
// chunked engine.
#pragma once
#include <utility>
#include <vector>
#include "common.cuh"

namespace sb200 {

// Row pitch (words) of the dense engine's device rows of w_pad words: a
// pitch that is a multiple of 4 KiB gets 64 bytes more.  With a power-of-two
// pitch the same K stage of the 384 rows a tile reads falls on the same
// memory partitions, and their loads queue there; measured on B200 with the
// tensor-core kernel (ms, same rows): 65536 x 2^18 bits 368.6 -> 353.8,
// 16384 x 2^18 23.7 -> 21.6, 4096 x 2^16 0.484 -> 0.468, 4096 x 2^23 48.2
// -> 46.4.  (256 bytes more was slower than none at 2^18: 395.1.)
inline uint64_t dense_pitch(uint32_t w_pad) { return w_pad % 512 == 0 ? (uint64_t)w_pad + 8 : (uint64_t)w_pad; }

// Device rows: X is [n_pad][dense_pitch(w_pad)] u64, of which each row's
// first w_pad words are read (zero past the row's bits), n_pad % 256 == 0
// and w_pad % 8 == 0.
struct DenseEngine {
    int schedule = STORM_B200_SCHED_AUTO;   // tensor-core work schedule
    DevBuf<uint2> d_tiles;
    uint64_t tiles_n = ~0ull;
    int tiles_kind = -1;
    uint32_t n_tiles = 0;
    DevBuf<DeviceFlags> d_flags;
    LaunchLog log;

    ~DenseEngine() {
        log.destroy();
        for (cudaEvent_t e : panel_ev) cudaEventDestroy(e);
        for (cudaEvent_t e : h2d_ev) cudaEventDestroy(e);
    }

    // Returns the sum over i < j; writes the packed upper triangle to d_out
    // when non-null.  `row_bits` is the logical row length (decides whether
    // the exact tensor-core kernel applies).  Synchronous.
    uint64_t run(const uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits, uint32_t* d_out,
                 int kernel_pref, cudaStream_t st);

    // Same result, with the packed triangle also copied to host_out: the
    // tiles run in panels from the bottom of the triangle up, and the rows
    // each panel completes are copied on copy_st while the next computes.
    uint64_t run_to_host(const uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits, uint32_t* d_out,
                         uint32_t* host_out, int kernel_pref, cudaStream_t st, cudaStream_t copy_st);

    // run_to_host with the rows also coming from the host: host_rows (n x
    // host_wpr words, host memory) are copied into dX ([n_pad][pitch],
    // zero padded here) on h2d_st, last rows first, and each panel waits
    // only for the rows its tiles read, so the upload, the tiles and the
    // copy back overlap.
    uint64_t run_host_to_host(uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits,
                              const uint64_t* host_rows, uint32_t host_wpr, uint32_t* d_out, uint32_t* host_out,
                              int kernel_pref, cudaStream_t st, cudaStream_t copy_st, cudaStream_t h2d_st);

    // Thresholded form: the pairs i < j with count v > 0 and
    // v / (|Xi| + |Xj| - v) >= t, appended to d_pairs / d_cnts (up to cap,
    // unordered); returns how many pairs passed. The tensor-core kernel
    // filters in its epilogue (no triangle is written); other kernels write
    // the triangle into scratch and compact it. Synchronous.
    uint64_t run_threshold(const uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits, int kernel_pref,
                           double t, uint2* d_pairs, uint32_t* d_cnts, uint64_t cap, uint64_t* sum,
                           cudaStream_t st);
    DevBuf<uint32_t> d_card, d_scratch_tri;
    DevBuf<unsigned long long> d_found;

   private:
    int prepare(uint64_t n, uint64_t row_bits, int kernel_pref, cudaStream_t st);
    void launch(int kind, const uint64_t* dX, uint32_t n, uint32_t w_pad, uint32_t t0, uint32_t count,
                uint32_t* d_out, cudaStream_t st);
    void zero_stream_k_rows(uint32_t* d_out, uint32_t n, uint32_t grid, cudaStream_t st);
    uint64_t panels_to_host(const uint64_t* dX, uint64_t n, uint32_t w_pad, int kind, uint32_t* d_out,
                            uint32_t* host_out, cudaStream_t st, cudaStream_t copy_st, uint64_t chunk_rows);
    std::vector<uint2> h_tiles;
    std::vector<cudaEvent_t> panel_ev, h2d_ev;
};

inline uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

// Tiles (bi, bj) of 128 x 256 pairs covering the triangle of n rows.
void build_mma_tiles(std::vector<uint2>& t, uint64_t n);
// The tile list of a bitmap x bitmap kernel (STORM_B200_KERNEL_*): 128 x 256
// (tcgen05), 128 x 192 (double-buffered tcgen05) or 128 x 128 (POPC) tiles
// covering every pair i <= j < n once, ordered by A block.
void build_tiles(std::vector<uint2>& t, uint64_t n, int kind);
// Rows per A block / per B block of a kernel's tiles.
uint64_t tile_rows_a(int kind);
uint64_t tile_rows_b(int kind);
// Panels of the host-output forms over a tile list of n_tiles, in processing
// order (the end of the list first), each a whole number of waves but the
// last.
std::vector<std::pair<uint32_t, uint32_t>> host_panels(uint32_t n_tiles, uint32_t wave);
// Longest row the tensor-core kernels count exactly (4-byte weight cycle).
constexpr uint64_t TC_MAX_ROW_BITS = 1ull << 27;
// ... and the shared-memory form (8-byte weight cycle only).
constexpr uint64_t TC_SS_MAX_ROW_BITS = 1ull << 23;

// Tensor-core kernel over n gathered rows X (>= roundup(n, 256) rows of
// w_pad words in layout `lay`); count (i, j) lands at the packed index of
// (row_map[i], row_map[j]) in a
// triangle of n_out rows; the sum over i < j accumulates into flags->sum.
// With few tiles the K range is split and partial counts are added into
// out: out_zeroed says the caller has zeroed the triangle already, else it
// is zeroed here when a split is taken.  Asynchronous on st.
void launch_ts_rows(const uint64_t* X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* tiles, uint32_t n_tiles,
                    uint32_t* out, DeviceFlags* flags, const uint32_t* row_map, uint64_t n_out, cudaStream_t st,
                    bool out_zeroed = false);

// Thresholded pairs from a packed triangle of n rows already on the device
// (row cardinalities from its diagonal): appends the pairs i < j with
// v > 0 and v / (d_i + d_j - v) >= t to d_pairs / d_cnts (up to cap) and
// returns how many passed. card must hold n entries, found one. Synchronous.
uint64_t threshold_from_triangle(const uint32_t* d_tri, uint64_t n, double t, uint32_t* card,
                                 unsigned long long* found, uint2* d_pairs, uint32_t* d_cnts, uint64_t cap,
                                 cudaStream_t st);

// Host side of the thresholded C-ABI calls: copies min(found, cap) hits to
// the caller's arrays sorted by (i, j); returns 0, or STORM_B200_ESIZE when
// more pairs passed than cap (the arrays then hold cap of them).
int threshold_to_host(const uint2* d_pairs, const uint32_t* d_cnts, uint64_t found, uint64_t cap, uint32_t* out_i,
                      uint32_t* out_j, uint32_t* out_count, cudaStream_t st);

}  // namespace sb200
