// dense.cu -- launchers for the B x B kernels (POPC and tcgen05).
#include "dense.cuh"
#include "bb_popc.cuh"
#include "bb_mma.cuh"
#include "bb_mma_ts.cuh"
#include "bb_mma_ts2.cuh"
#include "bb_mma_2cta.cuh"

#include <algorithm>
#include <mutex>

namespace sb200 {

// Work schedule of the tensor-core kernel (TsSched in bb_mma_ts.cuh): whole
// tiles round robin when the last wave is nearly full (>= 98.5 %) or a tile
// has fewer than 128 K stages (32768 bits: shorter tiles lose more to the
// extra segment boundaries and partial-tile atomics than they gain); else
// stream-K over the (tile, K stage) space, at least 32 stages per CTA.
// Measured on B200: 272 tiles (1.8 waves) of 2^18-bit rows run 8 % faster
// under stream-K, 136 tiles 1.9x, 1088 tiles (92 % fill) 7 %, 4160 tiles
// (97 % fill) 3 %; 2176 tiles (98 % fill) of 2^16-bit rows 3 % slower, and
// 80-stage tiles (20000-bit rows) 7 % slower. Those figures are for stream-K
// over every tile; the kernels now run the first floor(tiles / grid) waves
// as whole tiles and stream-K only the rest (TsSched), which measured faster
// still on B200 (double-buffered kernel: 50000 x 20000 bits 7 %, 16384 x
// 262144 5 %, 4096 x 65536 1 %) with counts unchanged. Returns the kernel's
// k_splits argument (1 or 0) and sets the grid.
static uint32_t ts_schedule(uint32_t n_tiles, int sms, uint32_t w_pad, uint32_t& grid,
                            int pref = STORM_B200_SCHED_AUTO) {
    const uint64_t nk = w_pad / (TS_KBITS / 64);
    const uint64_t waves = ((uint64_t)n_tiles + sms - 1) / sms;
    const double fill = waves ? (double)n_tiles / (double)(waves * (uint64_t)sms) : 1.0;
    const bool tiles = pref == STORM_B200_SCHED_TILES ||
                       (pref == STORM_B200_SCHED_AUTO && (fill >= 0.985 || nk < 128));
    if (tiles) {
        grid = n_tiles < (uint32_t)sms ? n_tiles : (uint32_t)sms;
        return 1;
    }
    grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sms, (uint64_t)n_tiles * nk / 32));
    return 0;
}

constexpr uint64_t DB_AUTO_MAX_BITS = 1ull << 17;

// Rows per A block and per B block of a kernel's tiles.
uint64_t tile_rows_a(int kind) {
    return kind == STORM_B200_KERNEL_POPC ? POPC_BM : kind == STORM_B200_KERNEL_MMA_2CTA ? C2_BM : MMA_BM;
}
uint64_t tile_rows_b(int kind) {
    return kind == STORM_B200_KERNEL_POPC     ? POPC_BM
           : kind == STORM_B200_KERNEL_MMA_DB ? T2_BN
           : kind == STORM_B200_KERNEL_MMA_2CTA ? C2_BN
                                                : MMA_BN;
}

void build_tiles(std::vector<uint2>& t, uint64_t n, int kind) {
    t.clear();
    // tile indices and counts are 32-bit (the kernels' work lists); bound the
    // count by the full block grid before building anything
    const uint64_t bm = tile_rows_a(kind), bn = tile_rows_b(kind);
    if (((n + bm - 1) / bm) * ((n + bn - 1) / bn) > 0xFFFFFFFFull)
        fail(STORM_B200_ELIMIT, "more than 2^32 tiles: split the rows into several containers");
    if (kind == STORM_B200_KERNEL_MMA_2CTA) {
        const uint64_t nb = (n + C2_BM - 1) / C2_BM;
        for (uint64_t bi = 0; bi < nb; ++bi)
            for (uint64_t bj = bi; bj < nb; ++bj) t.push_back(make_uint2((uint32_t)bi, (uint32_t)bj));
    } else if (kind == STORM_B200_KERNEL_MMA || kind == STORM_B200_KERNEL_MMA_SS) {
        const uint64_t nbi = (n + MMA_BM - 1) / MMA_BM, nbj = (n + MMA_BN - 1) / MMA_BN;
        // Tile (bi, bj) holds a pair with i <= j iff 128 bi <= 256 bj + 255,
        // i.e. bj >= floor(bi / 2).
        for (uint64_t bi = 0; bi < nbi; ++bi)
            for (uint64_t bj = bi / 2; bj < nbj; ++bj) t.push_back(make_uint2((uint32_t)bi, (uint32_t)bj));
    } else if (kind == STORM_B200_KERNEL_MMA_DB) {
        const uint64_t nbi = (n + T2_BM - 1) / T2_BM, nbj = (n + T2_BN - 1) / T2_BN;
        // 128 bi <= 192 bj + 191  <=>  bj >= floor(128 bi / 192)
        for (uint64_t bi = 0; bi < nbi; ++bi)
            for (uint64_t bj = (128 * bi) / 192; bj < nbj; ++bj) t.push_back(make_uint2((uint32_t)bi, (uint32_t)bj));
    } else {
        const uint64_t nb = (n + POPC_BM - 1) / POPC_BM;
        for (uint64_t bi = 0; bi < nb; ++bi)
            for (uint64_t bj = bi; bj < nb; ++bj) t.push_back(make_uint2((uint32_t)bi, (uint32_t)bj));
    }
}

int DenseEngine::prepare(uint64_t n, uint64_t row_bits, int kernel_pref, cudaStream_t st) {
    if (n > 0xFFFFFFFFull) fail(STORM_B200_ELIMIT, "more than 2^32 rows");
    int kind = kernel_pref;
    // Automatic choice: rows of at most 2^17 bits (tiles of at most 512 K
    // stages) take the double-buffered tensor-core kernel, whose drain of one
    // tile overlaps the next tile's MMAs (measured on B200: 19 % faster at
    // 20000-bit rows, 3 % at 65536, even at 2^18); longer rows up to 2^27
    // bits the 128 x 256 kernel; past that the CUDA-core POPC kernel.
    if (kind == STORM_B200_KERNEL_AUTO)
        kind = row_bits <= DB_AUTO_MAX_BITS    ? STORM_B200_KERNEL_MMA_DB
               : row_bits <= MMA_MAX_BITS_W4 ? STORM_B200_KERNEL_MMA
                                             : STORM_B200_KERNEL_POPC;
    if ((kind == STORM_B200_KERNEL_MMA || kind == STORM_B200_KERNEL_MMA_DB || kind == STORM_B200_KERNEL_MMA_2CTA) &&
        row_bits > MMA_MAX_BITS_W4)
        fail(STORM_B200_ELIMIT, "tensor-core kernel is exact only for rows of at most 2^27 bits");
    if (kind == STORM_B200_KERNEL_MMA_SS && row_bits > MMA_MAX_BITS)
        fail(STORM_B200_ELIMIT, "shared-memory tensor-core kernel is exact only for rows of at most 2^23 bits");
    if (tiles_n != n || tiles_kind != kind) {
        build_tiles(h_tiles, n, kind);
        d_tiles.reserve(h_tiles.size());
        SB_CUDA(cudaMemcpyAsync(d_tiles.p, h_tiles.data(), h_tiles.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                                st));
        n_tiles = (uint32_t)h_tiles.size();
        tiles_n = n;
        tiles_kind = kind;
    }
    d_flags.reserve(1);
    SB_CUDA(cudaMemsetAsync(d_flags.p, 0, sizeof(DeviceFlags), st));
    log.ensure();
    return kind;
}

// Stream-K over the whole cached list (TsSched, k_splits 0): tiles from
// W = floor(tiles / grid) x grid on add into the output, and every one of them
// has its A block at or past tile W's (the list is ordered by A block), so
// zeroing the triangle from that block's first row on covers them.
static_assert(T2_BM == MMA_BM, "both tensor-core tilings use 128-row A blocks");

void DenseEngine::zero_stream_k_rows(uint32_t* d_out, uint32_t n, uint32_t grid, cudaStream_t st) {
    const uint32_t whole = (n_tiles / grid) * grid;
    if (whole >= n_tiles) return;
    const uint64_t r0 = (uint64_t)h_tiles[whole].x * MMA_BM;   // 128-row A blocks in both tensor-core tilings
    const uint64_t e0 = r0 * n - (r0 * (r0 - 1)) / 2;          // tri_index(n, r0, r0)
    SB_CUDA(cudaMemsetAsync(d_out + e0, 0, (tri_size(n) - e0) * sizeof(uint32_t), st));
}

// Tiles [t0, t0 + count) of the cached list.
void DenseEngine::launch(int kind, const uint64_t* dX, uint32_t n, uint32_t w_pad, uint32_t t0, uint32_t count,
                         uint32_t* d_out, cudaStream_t st) {
    const int sms = require_device();
    if (count == 0) return;
    const RowLayout lay = row_major(dense_pitch(w_pad));
    if (kind == STORM_B200_KERNEL_MMA) {
        static std::atomic<uint64_t> done_a{0}, done_b{0};
        smem_attr_once(bb_mma_ts_kernel, (int)TS_SMEM_BYTES, done_a);
        smem_attr_once(bb_mma_ts_long_kernel, (int)TS_SMEM_BYTES, done_b);
        // stream-K only for a launch over the whole tile list, whose output
        // triangle can be zeroed first for the partial-count atomics
        uint32_t grid = count < (uint32_t)sms ? count : (uint32_t)sms;
        const uint32_t ks = (t0 == 0 && count == n_tiles) ? ts_schedule(count, sms, w_pad, grid, schedule) : 1;
        if (ks != 1 && d_out) zero_stream_k_rows(d_out, n, grid, st);
        const uint32_t smem = (uint64_t)w_pad * 64 <= TS_COALESCE_MAX_BITS ? TS_SMEM_BYTES : TS_SMEM_BYTES_LEAN;
        if ((uint64_t)w_pad * 64 <= MMA_MAX_BITS)
            bb_mma_ts_kernel<<<grid, TS_THREADS, smem, st>>>(dX, n, w_pad, lay, d_tiles.p + t0, count, d_out, d_flags.p,
                                                             ks);
        else
            bb_mma_ts_long_kernel<<<grid, TS_THREADS, smem, st>>>(dX, n, w_pad, lay, d_tiles.p + t0, count, d_out,
                                                                  d_flags.p, ks);
    } else if (kind == STORM_B200_KERNEL_MMA_DB) {
        static std::atomic<uint64_t> done_a{0}, done_b{0};
        smem_attr_once(bb_mma_ts2_kernel, (int)T2_SMEM_BYTES, done_a);
        smem_attr_once(bb_mma_ts2_long_kernel, (int)T2_SMEM_BYTES, done_b);
        uint32_t grid = count < (uint32_t)sms ? count : (uint32_t)sms;
        const uint32_t ks = (t0 == 0 && count == n_tiles) ? ts_schedule(count, sms, w_pad, grid, schedule) : 1;
        if (ks != 1 && d_out) zero_stream_k_rows(d_out, n, grid, st);
        if ((uint64_t)w_pad * 64 <= MMA_MAX_BITS)
            bb_mma_ts2_kernel<<<grid, T2_THREADS, T2_SMEM_BYTES, st>>>(dX, n, w_pad, lay, d_tiles.p + t0, count, d_out,
                                                                      d_flags.p, ks);
        else
            bb_mma_ts2_long_kernel<<<grid, T2_THREADS, T2_SMEM_BYTES, st>>>(dX, n, w_pad, lay, d_tiles.p + t0, count,
                                                                           d_out, d_flags.p, ks);
    } else if (kind == STORM_B200_KERNEL_MMA_2CTA) {
        // CTA pairs (clusters of 2), one per two SMs, whole tiles round robin
        static std::atomic<uint64_t> done_a{0}, done_b{0};
        smem_attr_once(bb_mma_2cta_kernel, (int)C2_SMEM_BYTES, done_a);
        smem_attr_once(bb_mma_2cta_long_kernel, (int)C2_SMEM_BYTES, done_b);
        const uint32_t pairs = std::max<uint32_t>(1u, std::min<uint32_t>(count, (uint32_t)sms / 2));
        const uint32_t smem = (uint64_t)w_pad * 64 <= TS_COALESCE_MAX_BITS ? C2_SMEM_BYTES
                                                                          : C2_SMEM_BYTES - C2_EPI_BYTES;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * pairs, 1, 1);
        cfg.blockDim = dim3(C2_THREADS, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const uint2* tl = d_tiles.p + t0;
        if ((uint64_t)w_pad * 64 <= MMA_MAX_BITS)
            SB_CUDA(cudaLaunchKernelEx(&cfg, bb_mma_2cta_kernel, dX, n, w_pad, lay, tl, count, d_out, d_flags.p));
        else
            SB_CUDA(cudaLaunchKernelEx(&cfg, bb_mma_2cta_long_kernel, dX, n, w_pad, lay, tl, count, d_out, d_flags.p));
    } else if (kind == STORM_B200_KERNEL_MMA_SS) {
        static std::atomic<uint64_t> done{0};
        smem_attr_once(bb_mma_kernel, (int)MMA_SMEM_BYTES, done);
        const uint32_t grid = count < (uint32_t)sms ? count : (uint32_t)sms;
        bb_mma_kernel<<<grid, MMA_THREADS, MMA_SMEM_BYTES, st>>>(dX, n, w_pad, lay.pitch, d_tiles.p + t0, count, d_out,
                                                                  d_flags.p);
    } else {
        const size_t smem = sizeof(PopcSmem);
        static std::atomic<uint64_t> done{0};
        smem_attr_once(bb_popc_kernel, (int)smem, done);
        const uint32_t cap = (uint32_t)sms * 2;
        const uint32_t grid = count < cap ? count : cap;
        bb_popc_kernel<<<grid, POPC_THREADS, smem, st>>>(dX, n, w_pad, lay.pitch, d_tiles.p + t0, count, d_out, d_flags.p);
    }
    SB_CUDA(cudaGetLastError());
}

uint64_t DenseEngine::run(const uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits,
                          uint32_t* d_out, int kernel_pref, cudaStream_t st) {
    if (n == 0) {
        log.launches = 0;
        log.last_ms = 0.f;
        return 0;
    }
    const int kind = prepare(n, row_bits, kernel_pref, st);
    SB_CUDA(cudaEventRecord(log.ev0, st));
    launch(kind, dX, (uint32_t)n, w_pad, 0, n_tiles, d_out, st);
    SB_CUDA(cudaEventRecord(log.ev1, st));
    DeviceFlags f;
    SB_CUDA(cudaMemcpyAsync(&f, d_flags.p, sizeof(f), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    SB_CUDA(cudaEventElapsedTime(&log.last_ms, log.ev0, log.ev1));
    log.launches = 1;
    log.kernel = kind;
    if (f.error) fail(STORM_B200_ETIMEOUT, "bitmap x bitmap kernel: bounded wait expired");
    return f.sum;
}

// Panels of the host-output forms, in processing order (the bottom of the
// triangle first): [t0, t1) ranges of the tile list. Sizes are whole waves of
// the launch's grid (no SM idles at a launch's end), growing from one wave at
// both ends -- the first panel reads only the last rows, the last panel's
// rows are the only copy still running when the tiles end -- to about 1/24
// of the tiles. Small lists run as one launch.
std::vector<std::pair<uint32_t, uint32_t>> host_panels(uint32_t n_tiles, uint32_t wave) {
    std::vector<std::pair<uint32_t, uint32_t>> p;
    if (n_tiles <= 4ull * wave) {
        p.emplace_back(0u, n_tiles);
        return p;
    }
    const uint64_t total_w = n_tiles / wave;   // the remainder (< 1 wave) joins the last panel
    const uint64_t cap = std::max<uint64_t>(1, total_w / 24);
    std::vector<uint64_t> head;
    uint64_t used = 0;
    for (uint64_t s = 1; s < cap && used + 2 * s <= total_w / 2; s *= 2) {
        head.push_back(s);
        used += s;
    }
    std::vector<uint64_t> sizes(head);
    for (uint64_t mid = total_w - 2 * used; mid > 0;) {
        const uint64_t s = std::min(cap, mid);
        sizes.push_back(s);
        mid -= s;
    }
    sizes.insert(sizes.end(), head.rbegin(), head.rend());
    uint64_t hi = n_tiles;
    for (size_t k = 0; k < sizes.size(); ++k) {
        const uint64_t lo = (k + 1 == sizes.size()) ? 0 : hi - sizes[k] * wave;
        p.emplace_back((uint32_t)lo, (uint32_t)hi);
        hi = lo;
    }
    return p;
}

uint64_t DenseEngine::run_to_host(const uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits,
                                  uint32_t* d_out, uint32_t* host_out, int kernel_pref, cudaStream_t st,
                                  cudaStream_t copy_st) {
    if (n == 0) {
        log.launches = 0;
        log.last_ms = 0.f;
        return 0;
    }
    const int kind = prepare(n, row_bits, kernel_pref, st);
    return panels_to_host(dX, n, w_pad, kind, d_out, host_out, st, copy_st, 0);
}

uint64_t DenseEngine::run_host_to_host(uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits,
                                       const uint64_t* host_rows, uint32_t host_wpr, uint32_t* d_out,
                                       uint32_t* host_out, int kernel_pref, cudaStream_t st, cudaStream_t copy_st,
                                       cudaStream_t h2d_st) {
    if (n == 0) {
        log.launches = 0;
        log.last_ms = 0.f;
        return 0;
    }
    const int kind = prepare(n, row_bits, kernel_pref, st);
    // What the copies do not cover reads as zero: the row pitch's padding
    // words and the rows [n, n_pad) that whole 128 x 256 tiles read.
    const uint64_t n_pad = round_up(n, 256), pitch = dense_pitch(w_pad);
    if (host_wpr != w_pad)
        SB_CUDA(cudaMemsetAsync(dX, 0, n_pad * pitch * sizeof(uint64_t), h2d_st));
    else if (n_pad > n)
        SB_CUDA(cudaMemsetAsync(dX + n * pitch, 0, (n_pad - n) * pitch * sizeof(uint64_t), h2d_st));
    const uint64_t chunk_rows = round_up(std::max<uint64_t>(1, (n + 31) / 32), 128);
    const uint64_t chunks = (n + chunk_rows - 1) / chunk_rows;
    while (h2d_ev.size() < chunks) {
        cudaEvent_t e;
        SB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h2d_ev.push_back(e);
    }
    // Last rows first: the bottom panels read only them. Event c marks rows
    // [c x chunk_rows, n) (and the zeroing) as resident.
    for (uint64_t c = chunks; c-- > 0;) {
        const uint64_t r0 = c * chunk_rows, r1 = std::min(n, r0 + chunk_rows);
        SB_CUDA(cudaMemcpy2DAsync(dX + r0 * pitch, (size_t)pitch * sizeof(uint64_t), host_rows + r0 * host_wpr,
                                  (size_t)host_wpr * sizeof(uint64_t), (size_t)host_wpr * sizeof(uint64_t),
                                  r1 - r0, cudaMemcpyHostToDevice, h2d_st));
        SB_CUDA(cudaEventRecord(h2d_ev[c], h2d_st));
    }
    uint64_t s = 0;
    try {
        s = panels_to_host(dX, n, w_pad, kind, d_out, host_out, st, copy_st, chunk_rows);
    } catch (...) {
        cudaStreamSynchronize(h2d_st);   // no copy may still read the caller's rows after the return
        throw;
    }
    SB_CUDA(cudaStreamSynchronize(h2d_st));
    return s;
}

// chunk_rows != 0: rows arrive in chunks of chunk_rows on h2d_ev; each panel
// waits for the chunk holding the lowest row its tiles read.
uint64_t DenseEngine::panels_to_host(const uint64_t* dX, uint64_t n, uint32_t w_pad, int kind, uint32_t* d_out,
                                     uint32_t* host_out, cudaStream_t st, cudaStream_t copy_st,
                                     uint64_t chunk_rows) {
    const int sms = require_device();
    const uint64_t bm = tile_rows_a(kind), bn = tile_rows_b(kind);
    const uint32_t wave = kind == STORM_B200_KERNEL_POPC        ? 2u * (uint32_t)sms
                          : kind == STORM_B200_KERNEL_MMA_2CTA ? (uint32_t)sms / 2
                                                               : (uint32_t)sms;
    const auto panels = host_panels(n_tiles, wave);
    // first tile of each A block (the list is ordered by A block)
    std::vector<uint32_t> first_tile((size_t)h_tiles.back().x + 1, 0);
    for (uint32_t t = n_tiles; t-- > 0;) first_tile[h_tiles[t].x] = t;
    while (panel_ev.size() < panels.size()) {
        cudaEvent_t e;
        SB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        panel_ev.push_back(e);
    }
    SB_CUDA(cudaEventRecord(log.ev0, st));
    uint64_t copied_from = n;   // rows [copied_from, n) are on their way to the host
    try {
        for (size_t p = 0; p < panels.size(); ++p) {
            const uint32_t t0 = panels[p].first, t1 = panels[p].second;
            if (chunk_rows) {
                uint64_t need = n;
                for (uint32_t t = t0; t < t1; ++t)
                    need = std::min(need, std::min<uint64_t>(h_tiles[t].x * bm, h_tiles[t].y * bn));
                SB_CUDA(cudaStreamWaitEvent(st, h2d_ev[need / chunk_rows], 0));
            }
            launch(kind, dX, (uint32_t)n, w_pad, t0, t1 - t0, d_out, st);
            SB_CUDA(cudaEventRecord(panel_ev[p], st));
            // Every tile from t0 on is done: the A blocks whose first tile is at
            // or past t0 are complete, and their rows are contiguous in the
            // packed triangle.
            uint64_t b = h_tiles[t0].x;
            if (first_tile[b] != t0) ++b;
            const uint64_t r = std::min<uint64_t>(n, b * bm);
            if (r < copied_from) {
                const uint64_t e0 = r * n - (r * (r - 1)) / 2;   // tri_index(n, r, r)
                const uint64_t e1 = copied_from * n - (copied_from * (copied_from - 1)) / 2;
                SB_CUDA(cudaStreamWaitEvent(copy_st, panel_ev[p], 0));
                SB_CUDA(cudaMemcpyAsync(host_out + e0, d_out + e0, (e1 - e0) * sizeof(uint32_t),
                                        cudaMemcpyDeviceToHost, copy_st));
                copied_from = r;
            }
        }
    } catch (...) {
        // no copy may still write the caller's buffer after the return
        cudaStreamSynchronize(st);
        cudaStreamSynchronize(copy_st);
        throw;
    }
    SB_CUDA(cudaEventRecord(log.ev1, st));
    DeviceFlags f;
    SB_CUDA(cudaMemcpyAsync(&f, d_flags.p, sizeof(f), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    SB_CUDA(cudaStreamSynchronize(copy_st));
    SB_CUDA(cudaEventElapsedTime(&log.last_ms, log.ev0, log.ev1));
    log.launches = (uint32_t)panels.size();
    log.kernel = kind;
    if (f.error) fail(STORM_B200_ETIMEOUT, "bitmap x bitmap kernel: bounded wait expired");
    if (copied_from != 0) fail(STORM_B200_ECUDA, "panel schedule left rows uncopied");
    return f.sum;
}
}  // namespace sb200

// ===================================================================
// Allocation-free entry point.
//
// Some callers cannot allocate device memory at the time they need the
// counts: a service that reserves all of HBM for its own pool at start-up
// and forbids cudaMalloc afterwards (a cudaMalloc on a busy device can
// stall other work and can fail mid-request), or a host framework that owns
// every device buffer through its own allocator.  They hand in the rows and
// the output buffer; this path adds nothing to them.  The tensor-core
// kernel's scratch -- the status / sum words and the tile list -- lives in
// the file-scope array below, sized for at most NOALLOC_MAX_TILES tiles,
// which every GPU that loads the library keeps until the process exits.
// ===================================================================
namespace sb200 {

constexpr uint32_t NOALLOC_MAX_TILES = 32768;   // 256 KiB of (bi, bj) pairs: up to 46080 rows

struct NoAllocScratch {
    DeviceFlags flags;
    uint2 tiles[NOALLOC_MAX_TILES];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// One thread per A block row bi writes its tiles (bi, bj), bj >= bi / 2,
// at offset bi * nbj - sum_{k < bi} floor(k / 2).
__global__ void noalloc_tiles_kernel(NoAllocScratch* s, uint32_t nbi, uint32_t nbj) {
    const uint32_t bi = blockIdx.x * blockDim.x + threadIdx.x;
    if (bi >= nbi) return;
    const uint64_t m = bi / 2;
    const uint64_t below = (bi % 2 == 0) ? m * (m - (m > 0 ? 1 : 0)) : m * m;
    uint64_t t = (uint64_t)bi * nbj - below;
    for (uint32_t bj = bi / 2; bj < nbj; ++bj, ++t) s->tiles[t] = make_uint2(bi, bj);
}

}  // namespace sb200

extern "C" int STORM_contig_pairw_intersect_matrix_noalloc(const uint64_t* d_rows, uint64_t n_rows,
                                                           uint32_t row_pitch_words, uint64_t row_bits,
                                                           uint32_t* d_out, uint64_t out_len, uint64_t* sum,
                                                           void* stream) {
    using namespace sb200;
    if (d_rows == NULL) return STORM_B200_EVALUES;
    if (n_rows == 0 || n_rows > 0xFFFFFFFFull) return STORM_B200_EARG;
    if ((uintptr_t)d_rows % 32 != 0) return STORM_B200_EARG;   // the kernel reads rows 32 bytes at a time
    if (row_pitch_words == 0 || row_pitch_words % 8 != 0 || (uint64_t)row_pitch_words * 64 < row_bits)
        return STORM_B200_EARG;
    if (row_bits > MMA_MAX_BITS) return STORM_B200_ELIMIT;
    const uint64_t need = n_rows * (n_rows + 1) / 2;
    if (d_out != NULL && out_len < need) return STORM_B200_ESIZE;
    const uint32_t nbi = (uint32_t)((n_rows + TS_BM - 1) / TS_BM), nbj = (uint32_t)((n_rows + TS_BN - 1) / TS_BN);
    uint64_t n_tiles = 0;
    for (uint32_t bi = 0; bi < nbi; ++bi) n_tiles += nbj - bi / 2;
    if (n_tiles > NOALLOC_MAX_TILES) return STORM_B200_ELIMIT;

    // Once per device, with that device current: the device address of the
    // scratch array, and the kernel's shared-memory opt-in.
    static std::mutex mu;
    static void* scratch_of[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return STORM_B200_ECUDA;
    NoAllocScratch* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (scratch_of[dev] == nullptr) {
            int major = 0;
            if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major != 10)
                return STORM_B200_ECUDA;
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return STORM_B200_ECUDA;
            if (cudaFuncSetAttribute(bb_mma_ts_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)TS_SMEM_BYTES) != cudaSuccess)
                return STORM_B200_ECUDA;
            scratch_of[dev] = p;
        }
        scratch = static_cast<NoAllocScratch*>(scratch_of[dev]);
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return STORM_B200_ECUDA;
    // A CUDA error still pending from earlier work is reported before
    // anything is queued, so that it cannot be taken for a failed launch here.
    if (cudaPeekAtLastError() != cudaSuccess) return STORM_B200_ECUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(&scratch->flags, 0, sizeof(DeviceFlags), st) != cudaSuccess) return STORM_B200_ECUDA;
    noalloc_tiles_kernel<<<(nbi + 127) / 128, 128, 0, st>>>(scratch, nbi, nbj);
    const uint32_t grid = n_tiles < (uint64_t)sms ? (uint32_t)n_tiles : (uint32_t)sms;
    // The same epilogue rule as the allocating path: rows up to
    // TS_COALESCE_MAX_BITS stage their counts through shared memory.
    const uint32_t smem =
        (uint64_t)row_pitch_words * 64 <= TS_COALESCE_MAX_BITS ? TS_SMEM_BYTES : TS_SMEM_BYTES_LEAN;
    bb_mma_ts_kernel<<<grid, TS_THREADS, smem, st>>>(d_rows, (uint32_t)n_rows, row_pitch_words,
                                                      row_major(row_pitch_words), scratch->tiles,
                                                      (uint32_t)n_tiles, d_out, &scratch->flags, 1u);
    if (cudaGetLastError() != cudaSuccess) {
        cudaStreamSynchronize(st);   // nothing already queued may still write d_out after the return
        return STORM_B200_ECUDA;
    }
    DeviceFlags f;
    if (cudaMemcpyAsync(&f, &scratch->flags, sizeof(f), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return STORM_B200_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return STORM_B200_ECUDA;
    if (f.error) return STORM_B200_ETIMEOUT;
    if (sum) *sum = f.sum;
    return 0;
}

// ===================================================================
// Bounded-wait self-test
//
// The tensor-core kernels bound every mbarrier wait (ts_wait): when a wait
// gives up, the kernel records the site in the status word, stops its other
// roles, frees its tensor memory and returns, and the host call returns
// STORM_B200_ETIMEOUT with the context still usable.  This kernel runs that
// path on purpose, on a barrier nothing ever arrives on, with a short limit:
// warp 1 holds tensor memory as the real kernels do, warp 0's lane 0 waits.
// ===================================================================
namespace sb200 {

constexpr uint32_t ERR_SELFTEST = 0x301;

__global__ void __launch_bounds__(64) wait_selftest_kernel(DeviceFlags* flags, uint64_t limit_ns) {
    __shared__ TsCtl ctl;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&ctl.full[0]), 1);
        ctl.abort = 0;
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(&ctl.tmem_base), 32);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0 && lane == 0) ts_wait(smem_u32(&ctl.full[0]), 0, &ctl, flags, ERR_SELFTEST, false, limit_ns);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(ctl.tmem_base, 32);
    }
}

}  // namespace sb200

extern "C" int STORM_b200_wait_selftest(uint32_t limit_us) {
    using namespace sb200;
    if (limit_us == 0 || limit_us > 10000000u) return STORM_B200_EARG;
    return guard([&]() -> int {
        require_device();
        cudaStream_t st = nullptr;
        SB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        DevBuf<DeviceFlags> f;
        f.reserve(1);
        DeviceFlags h{};
        cudaError_t e = cudaMemsetAsync(f.p, 0, sizeof(DeviceFlags), st);
        if (e == cudaSuccess) {
            wait_selftest_kernel<<<1, 64, 0, st>>>(f.p, (uint64_t)limit_us * 1000ull);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, f.p, sizeof(h), cudaMemcpyDeviceToHost, st);
        const cudaError_t es = cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        SB_CUDA(e);
        SB_CUDA(es);
        return h.error == ERR_SELFTEST ? STORM_B200_ETIMEOUT : 0;
    });
}

// ===================================================================
// Thresholded output
// ===================================================================
namespace sb200 {

// |Xi| of each row: warp per row.
__global__ void row_popcount_kernel(const uint64_t* __restrict__ X, uint64_t n, uint32_t w_pad, uint64_t pitch,
                                    uint32_t* __restrict__ card) {
    const int lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
        uint32_t c = 0;
        for (uint32_t w = lane; w < w_pad; w += 32) c += __popcll(X[r * pitch + w]);
        c = warp_sum_u32(c);
        if (lane == 0) card[r] = c;
    }
}

__global__ void diag_card_kernel(const uint32_t* __restrict__ tri, uint64_t n, uint32_t* __restrict__ card) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x)
        card[r] = tri[tri_index(n, r, r)];
}

// Warp per row i, lanes over j > i; warp-aggregated appends.
__global__ void tri_threshold_kernel(const uint32_t* __restrict__ tri, uint64_t n, const uint32_t* __restrict__ card,
                                     double t, uint2* __restrict__ pairs, uint32_t* __restrict__ cnts,
                                     unsigned long long cap, unsigned long long* __restrict__ found) {
    const int lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const uint64_t base = tri_index(n, i, i) - i;
        const double ci = (double)card[i];
        for (uint64_t j0 = i + 1; j0 < n; j0 += 32) {
            const uint64_t j = j0 + lane;
            bool pass = false;
            uint32_t cnt = 0;
            if (j < n) {
                cnt = tri[base + j];
                if (cnt) {
                    const double u = ci + (double)card[j] - (double)cnt;
                    pass = u > 0.0 && (double)cnt / u >= t;
                }
            }
            const uint32_t m = __ballot_sync(0xffffffffu, pass);
            if (!m) continue;
            const int leader = __ffs(m) - 1;
            unsigned long long b0 = 0;
            if (lane == leader) b0 = atomicAdd(found, (unsigned long long)__popc(m));
            b0 = __shfl_sync(0xffffffffu, b0, leader);
            if (pass) {
                const unsigned long long k = b0 + __popc(m & ((1u << lane) - 1u));
                if (k < cap) {
                    pairs[k] = make_uint2((uint32_t)i, (uint32_t)j);
                    cnts[k] = cnt;
                }
            }
        }
    }
}

uint64_t threshold_from_triangle(const uint32_t* d_tri, uint64_t n, double t, uint32_t* card,
                                 unsigned long long* found, uint2* d_pairs, uint32_t* d_cnts, uint64_t cap,
                                 cudaStream_t st) {
    const int sms = require_device();
    SB_CUDA(cudaMemsetAsync(found, 0, sizeof(unsigned long long), st));
    if (n) {
        diag_card_kernel<<<(uint32_t)std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 8), 256, 0, st>>>(d_tri, n,
                                                                                                          card);
        tri_threshold_kernel<<<(uint32_t)std::min<uint64_t>((n + 7) / 8, (uint64_t)sms * 16), 256, 0, st>>>(
            d_tri, n, card, t, d_pairs, d_cnts, cap, found);
        SB_CUDA(cudaGetLastError());
    }
    unsigned long long h = 0;
    SB_CUDA(cudaMemcpyAsync(&h, found, sizeof(h), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    return h;
}

int threshold_to_host(const uint2* d_pairs, const uint32_t* d_cnts, uint64_t found, uint64_t cap, uint32_t* out_i,
                      uint32_t* out_j, uint32_t* out_count, cudaStream_t st) {
    const uint64_t m = std::min<uint64_t>(found, cap);
    std::vector<uint2> pr(m);
    std::vector<uint32_t> ct(m);
    if (m) {
        SB_CUDA(cudaMemcpyAsync(pr.data(), d_pairs, m * sizeof(uint2), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaMemcpyAsync(ct.data(), d_cnts, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
    }
    std::vector<uint64_t> idx(m);
    for (uint64_t k = 0; k < m; ++k) idx[k] = k;
    std::sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) {
        return pr[a].x != pr[b].x ? pr[a].x < pr[b].x : pr[a].y < pr[b].y;
    });
    for (uint64_t k = 0; k < m; ++k) {
        if (out_i) out_i[k] = pr[idx[k]].x;
        if (out_j) out_j[k] = pr[idx[k]].y;
        if (out_count) out_count[k] = ct[idx[k]];
    }
    return found > cap ? STORM_B200_ESIZE : 0;
}

uint64_t DenseEngine::run_threshold(const uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits,
                                    int kernel_pref, double t, uint2* d_pairs, uint32_t* d_cnts, uint64_t cap,
                                    uint64_t* sum, cudaStream_t st) {
    const int sms = require_device();
    d_found.reserve(1);
    d_card.reserve(n ? n : 1);
    if (n == 0) {
        log.launches = 0;
        log.last_ms = 0.f;
        if (sum) *sum = 0;
        return 0;
    }
    // The thresholded form has its filter fused into the 128 x 256 tensor-core
    // kernel's drain; the double-buffered kernel has none, so rows it would
    // take go to the fused one.
    if ((kernel_pref == STORM_B200_KERNEL_AUTO || kernel_pref == STORM_B200_KERNEL_MMA_DB) &&
        row_bits <= MMA_MAX_BITS_W4)
        kernel_pref = STORM_B200_KERNEL_MMA;
    const int kind = prepare(n, row_bits, kernel_pref, st);
    SB_CUDA(cudaEventRecord(log.ev0, st));
    uint64_t found = 0;
    if (kind == STORM_B200_KERNEL_MMA) {
        static std::atomic<uint64_t> done_a{0}, done_b{0};
        smem_attr_once(bb_mma_ts_thresh_kernel, (int)TS_SMEM_BYTES, done_a);
        smem_attr_once(bb_mma_ts_thresh_long_kernel, (int)TS_SMEM_BYTES, done_b);
        SB_CUDA(cudaMemsetAsync(d_found.p, 0, sizeof(unsigned long long), st));
        row_popcount_kernel<<<(uint32_t)std::min<uint64_t>((n + 7) / 8, (uint64_t)sms * 16), 256, 0, st>>>(
            dX, n, w_pad, dense_pitch(w_pad), d_card.p);
        const TsThresh th{d_card.p, t, d_pairs, d_cnts, (unsigned long long)cap, d_found.p};
        const uint32_t grid = n_tiles < (uint32_t)sms ? n_tiles : (uint32_t)sms;
        const RowLayout lay = row_major(dense_pitch(w_pad));
        if ((uint64_t)w_pad * 64 <= MMA_MAX_BITS)
            bb_mma_ts_thresh_kernel<<<grid, TS_THREADS, TS_SMEM_BYTES_LEAN, st>>>(dX, (uint32_t)n, w_pad, lay, d_tiles.p,
                                                                                   n_tiles, d_flags.p, th);
        else
            bb_mma_ts_thresh_long_kernel<<<grid, TS_THREADS, TS_SMEM_BYTES_LEAN, st>>>(
                dX, (uint32_t)n, w_pad, lay, d_tiles.p, n_tiles, d_flags.p, th);
        SB_CUDA(cudaGetLastError());
        unsigned long long h = 0;
        SB_CUDA(cudaMemcpyAsync(&h, d_found.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        found = h;
        log.launches = 2;
    } else {
        d_scratch_tri.reserve(tri_size(n));
        launch(kind, dX, (uint32_t)n, w_pad, 0, n_tiles, d_scratch_tri.p, st);
        found = threshold_from_triangle(d_scratch_tri.p, n, t, d_card.p, d_found.p, d_pairs, d_cnts, cap, st);
        log.launches = 3;
    }
    SB_CUDA(cudaEventRecord(log.ev1, st));
    DeviceFlags f;
    SB_CUDA(cudaMemcpyAsync(&f, d_flags.p, sizeof(f), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    SB_CUDA(cudaEventElapsedTime(&log.last_ms, log.ev0, log.ev1));
    log.kernel = kind;
    if (f.error) fail(STORM_B200_ETIMEOUT, "bitmap x bitmap kernel: bounded wait expired");
    if (sum) *sum = f.sum;
    return found;
}

}  // namespace sb200

// ===================================================================
// Kernel-layer dense block: the tensor-core kernel over a gathered subset of
// rows, counts scattered into the full row set's triangle.
// ===================================================================
namespace sb200 {

void build_mma_tiles(std::vector<uint2>& t, uint64_t n) { build_tiles(t, n, STORM_B200_KERNEL_MMA); }

void launch_ts_rows(const uint64_t* X, uint32_t n, uint32_t w_pad, RowLayout lay, const uint2* tiles,
                    uint32_t n_tiles, uint32_t* out, DeviceFlags* flags, const uint32_t* row_map, uint64_t n_out, cudaStream_t st,
                    bool out_zeroed) {
    const int sms = require_device();
    if (n_tiles == 0) return;
    static std::atomic<uint64_t> done_a{0}, done_b{0};
    smem_attr_once(bb_mma_ts_rows_kernel, (int)TS_SMEM_BYTES, done_a);
    smem_attr_once(bb_mma_ts_rows_long_kernel, (int)TS_SMEM_BYTES, done_b);
    if ((uint64_t)w_pad * 64 > MMA_MAX_BITS_W4) fail(STORM_B200_ELIMIT, "dense block rows longer than 2^27 bits");
    // With stream-K the partial counts are added into out, so the whole
    // triangle is zeroed first; the other phases write their own pairs after.
    uint32_t grid = 0;
    const uint32_t ks = ts_schedule(n_tiles, sms, w_pad, grid);
    if (ks != 1 && out && !out_zeroed) SB_CUDA(cudaMemsetAsync(out, 0, tri_size(n_out) * sizeof(uint32_t), st));
    const uint32_t smem = (uint64_t)w_pad * 64 <= TS_COALESCE_MAX_BITS ? TS_SMEM_BYTES : TS_SMEM_BYTES_LEAN;
    if ((uint64_t)w_pad * 64 <= MMA_MAX_BITS)
        bb_mma_ts_rows_kernel<<<grid, TS_THREADS, smem, st>>>(X, n, w_pad, lay, tiles, n_tiles, out, flags, row_map, n_out,
                                                              ks);
    else
        bb_mma_ts_rows_long_kernel<<<grid, TS_THREADS, smem, st>>>(X, n, w_pad, lay, tiles, n_tiles, out, flags, row_map,
                                                                   n_out, ks);
    SB_CUDA(cudaGetLastError());
}

}  // namespace sb200
