// contig.cu -- STORM_contiguous_t: dense contiguous rows, all pairs on the GPU.
//
// Mirrors the reference's opaque contiguous container (storm.cpp:1113-1285):
// rows are vector_length bits, ingested through STORM_contig_add (sorted
// positions, duplicates collapsed, storm.cpp:1181-1219) and compared all
// against all.  The reference keeps a sparse list for rows under
// min(len/200, 200) set bits and probes it (storm.cpp:1144-1156); that is a
// CPU speed trick with the same result, so here every pair goes through the
// bitmap x bitmap tile kernels.
//
// HBM layout: [n_pad][pitch] u64, w_pad = roundup(ceil(len/64), 8) words of
// each row read by the kernels, pitch = dense_pitch(w_pad) (64 bytes more
// when w_pad words are a multiple of 4 KiB), n_pad = roundup(n, 256), zero
// padded.  Rows added with STORM_contig_add are
// staged in host memory and flushed in one copy at the next device call;
// STORM_contig_add_bitmaps copies straight into HBM.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dense.cuh"

struct STORM_contiguous_s {
    uint64_t vector_length = 0;
    uint32_t n_words = 0;   // ceil(len / 64)
    uint32_t w_pad = 0;     // words of a row the kernels read
    uint64_t pitch = 0;     // HBM row pitch in words, dense_pitch(w_pad)
    uint64_t n_rows = 0;    // rows on the device + staged
    uint64_t dev_rows = 0;  // rows already in HBM
    uint64_t cap_rows = 0;  // HBM capacity in rows
    std::vector<uint64_t> stage;   // rows added by STORM_contig_add, not yet in HBM
    sb200::DevBuf<uint64_t> d_rows;
    sb200::DevBuf<uint32_t> d_out;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;   // device-to-host copies overlapping the next panel
    cudaStream_t h2d_stream = nullptr;    // host-to-device row copies of the one-call host form
    int kernel_pref = STORM_B200_KERNEL_AUTO;
    sb200::DenseEngine engine;
    sb200::DevBuf<uint2> d_hits;               // thresholded form: reported pairs and counts
    sb200::DevBuf<uint32_t> d_hit_cnt;

    ~STORM_contiguous_s() {
        if (stream) cudaStreamDestroy(stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (h2d_stream) cudaStreamDestroy(h2d_stream);
    }
};

namespace sb200 {

__global__ void mask_tail_kernel(uint64_t* last_word, uint64_t rows, uint64_t pitch, uint64_t keep) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x)
        last_word[r * pitch] &= keep;
}

static cudaStream_t contig_stream(STORM_contiguous_t* c) {
    require_device();
    if (!c->stream) SB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    return c->stream;
}

// Make room for `rows` rows in HBM, preserving the resident ones.
static void contig_grow(STORM_contiguous_t* c, uint64_t rows) {
    const uint64_t need = round_up(rows, 256);
    if (need <= c->cap_rows && c->d_rows.p) return;
    uint64_t cap = std::max<uint64_t>(need, c->cap_rows * 2);
    cudaStream_t st = contig_stream(c);
    uint64_t* np = nullptr;
    cudaError_t e = cudaMalloc((void**)&np, cap * c->pitch * sizeof(uint64_t));
    if (e != cudaSuccess && cap > need) {
        cudaGetLastError();
        cap = need;
        e = cudaMalloc((void**)&np, cap * c->pitch * sizeof(uint64_t));
    }
    SB_CUDA(e);
    if (c->dev_rows)
        SB_CUDA(cudaMemcpyAsync(np, c->d_rows.p, c->dev_rows * c->pitch * sizeof(uint64_t),
                                cudaMemcpyDeviceToDevice, st));
    SB_CUDA(cudaStreamSynchronize(st));
    c->d_rows.release();
    c->d_rows.p = np;
    c->d_rows.n = cap * c->pitch;
    c->cap_rows = cap;
}

// Append `rows` rows of `wpr` words from host memory into HBM (rows zero padded).
static void contig_append_device(STORM_contiguous_t* c, const uint64_t* host, uint64_t rows, uint32_t wpr) {
    if (rows == 0) return;
    contig_grow(c, c->dev_rows + rows);
    cudaStream_t st = contig_stream(c);
    uint64_t* dst = c->d_rows.p + c->dev_rows * c->pitch;
    if (wpr != c->w_pad)
        SB_CUDA(cudaMemsetAsync(dst, 0, rows * c->pitch * sizeof(uint64_t), st));
    SB_CUDA(cudaMemcpy2DAsync(dst, c->pitch * sizeof(uint64_t), host, wpr * sizeof(uint64_t),
                              wpr * sizeof(uint64_t), rows, cudaMemcpyDefault, st));
    SB_CUDA(cudaStreamSynchronize(st));
    c->dev_rows += rows;
}

static void contig_flush(STORM_contiguous_t* c) {
    const uint64_t staged = c->stage.size() / c->n_words;
    if (staged) {
        contig_append_device(c, c->stage.data(), staged, c->n_words);
        c->stage.clear();
    }
    // Rows [n, n_pad) are read by the tile kernels: keep them zero.
    contig_grow(c, c->dev_rows ? c->dev_rows : 1);
    const uint64_t n_pad = round_up(std::max<uint64_t>(c->dev_rows, 1), 256);
    cudaStream_t st = contig_stream(c);
    if (n_pad > c->dev_rows)
        SB_CUDA(cudaMemsetAsync(c->d_rows.p + c->dev_rows * c->pitch, 0,
                                (n_pad - c->dev_rows) * c->pitch * sizeof(uint64_t), st));
}

// Sum over i < j; packed triangle into d_out when non-null.
static uint64_t contig_run(STORM_contiguous_t* c, uint32_t* d_out) {
    contig_flush(c);
    return c->engine.run(c->d_rows.p, c->dev_rows, c->w_pad, c->vector_length, d_out, c->kernel_pref,
                         contig_stream(c));
}

// Runs into the handle's own device buffer and copies to the host.
static uint64_t contig_matrix_host(STORM_contiguous_t* c, uint32_t* out, uint64_t out_len) {
    const uint64_t n = c->n_rows;
    const uint64_t need = tri_size(n);
    if (out_len < need) fail(STORM_B200_ESIZE, "output buffer too small");
    c->d_out.reserve(need ? need : 1);
    contig_flush(c);
    if (!c->copy_stream) SB_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    // Panels of the triangle are copied back while the next panel computes.
    return c->engine.run_to_host(c->d_rows.p, c->dev_rows, c->w_pad, c->vector_length, c->d_out.p, out,
                                 c->kernel_pref, contig_stream(c), c->copy_stream);
}

}  // namespace sb200

using namespace sb200;

extern "C" {

STORM_contiguous_t* STORM_contig_new(size_t vector_length) {
    try {
        STORM_contiguous_t* c = new STORM_contiguous_t();
        c->vector_length = vector_length;
        c->n_words = (uint32_t)((vector_length + 63) / 64);
        c->w_pad = (uint32_t)round_up(c->n_words ? c->n_words : 1, 8);
        c->pitch = dense_pitch(c->w_pad);
        set_last_status(0);
        return c;
    } catch (...) {
        set_last_status(STORM_B200_ENOMEM);
        return NULL;
    }
}

void STORM_contig_free(STORM_contiguous_t* bitmap) { delete bitmap; }

// storm.cpp:1181-1219: -1 NULL handle, -2 NULL values, 0 for n == 0 (no row
// added), n_values on success.  Positions must be < vector_length (the
// reference only asserts this); out-of-range input returns -3 and adds
// nothing.  Duplicates collapse; unsorted input is accepted as a set.
int STORM_contig_add(STORM_contiguous_t* bitmap, const uint32_t* values, const uint32_t n_values) {
    if (bitmap == NULL) return -1;
    if (values == NULL) return -2;
    if (n_values == 0) return 0;
    return guard([&]() -> int {
        for (uint32_t i = 0; i < n_values; ++i)
            if (values[i] >= bitmap->vector_length) return STORM_B200_EARG;
        const size_t off = bitmap->stage.size();
        bitmap->stage.resize(off + bitmap->n_words, 0);
        uint64_t* dst = bitmap->stage.data() + off;
        for (uint32_t i = 0; i < n_values; ++i) dst[values[i] >> 6] |= 1ull << (values[i] & 63);
        ++bitmap->n_rows;
        return (int)n_values;
    });
}

int STORM_contig_add_bitmaps(STORM_contiguous_t* c, const uint64_t* words, uint32_t n_rows,
                             uint32_t words_per_row) {
    if (c == NULL) return STORM_B200_ENULL;
    if (words == NULL && n_rows) return STORM_B200_EVALUES;
    return guard([&]() -> int {
        if (words_per_row != c->n_words) return STORM_B200_EARG;
        cudaPointerAttributes pa;
        const bool on_device = cudaPointerGetAttributes(&pa, words) == cudaSuccess &&
                               (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
        cudaGetLastError();
        // Device input may still be in flight on another stream (the handle's
        // stream does not order against the legacy default stream): wait.
        if (on_device) SB_CUDA(cudaDeviceSynchronize());
        if (c->vector_length % 64 && n_rows && !on_device) {
            const uint64_t tail_mask = ~0ull << (c->vector_length % 64);
            for (uint64_t r = 0; r < n_rows; ++r)
                if (words[r * words_per_row + words_per_row - 1] & tail_mask) return STORM_B200_EARG;
        }
        // Keep row order: staged STORM_contig_add rows go first.
        const uint64_t staged = c->stage.size() / c->n_words;
        if (staged) {
            contig_append_device(c, c->stage.data(), staged, c->n_words);
            c->stage.clear();
        }
        const uint64_t first = c->dev_rows;
        contig_append_device(c, words, n_rows, words_per_row);
        if (on_device && c->vector_length % 64 && n_rows) {
            // Device input is not inspected on the host: clear bits past the row end.
            const uint32_t grid = (uint32_t)std::min<uint64_t>((n_rows + 255) / 256, 65535);
            mask_tail_kernel<<<grid, 256, 0, contig_stream(c)>>>(c->d_rows.p + first * c->pitch + (c->n_words - 1),
                                                                 n_rows, c->pitch,
                                                                 ~0ull >> (64 - c->vector_length % 64));
            SB_CUDA(cudaGetLastError());
            SB_CUDA(cudaStreamSynchronize(contig_stream(c)));
        }
        c->n_rows += n_rows;
        return (int)n_rows;
    });
}

uint64_t STORM_contig_size(const STORM_contiguous_t* c) { return c ? c->n_rows : 0; }

int STORM_contig_clear(STORM_contiguous_t* bitmap) {
    if (bitmap == NULL) return -1;
    bitmap->stage.clear();
    bitmap->n_rows = 0;
    bitmap->dev_rows = 0;   // capacity is kept, as the reference keeps its vectors'
    set_last_status(0);
    return 1;
}

int STORM_contig_set_kernel(STORM_contiguous_t* c, int kernel) {
    if (c == NULL) return STORM_B200_ENULL;
    if (kernel < STORM_B200_KERNEL_AUTO || kernel > STORM_B200_KERNEL_MMA_2CTA) return STORM_B200_EARG;
    c->kernel_pref = kernel;
    return 0;
}

int STORM_contig_set_schedule(STORM_contiguous_t* c, int schedule) {
    if (c == NULL) return STORM_B200_ENULL;
    if (schedule < STORM_B200_SCHED_AUTO || schedule > STORM_B200_SCHED_STREAM_K) return STORM_B200_EARG;
    c->engine.schedule = schedule;
    return 0;
}

int STORM_contig_autotune(STORM_contiguous_t* c, int* best_kernel, int* best_schedule, double* times_ms) {
    if (c == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        const uint64_t n = c->n_rows;
        contig_flush(c);
        c->d_out.reserve(tri_size(n) ? tri_size(n) : 1);
        const uint64_t bits = c->vector_length;
        // tcgen05 (A in TMEM) with 128 x 256 tiles and with 128 x 192 double-
        // buffered tiles, each under both schedules; tcgen05 with both
        // operands in shared memory; CUDA-core POPC; tcgen05 on CTA pairs --
        // each where it is exact.
        constexpr int NK = 7;
        const int kern[NK] = {STORM_B200_KERNEL_MMA,    STORM_B200_KERNEL_MMA,    STORM_B200_KERNEL_MMA_DB,
                              STORM_B200_KERNEL_MMA_DB, STORM_B200_KERNEL_MMA_SS, STORM_B200_KERNEL_POPC,
                              STORM_B200_KERNEL_MMA_2CTA};
        const int sched[NK] = {STORM_B200_SCHED_TILES,    STORM_B200_SCHED_STREAM_K, STORM_B200_SCHED_TILES,
                               STORM_B200_SCHED_STREAM_K, STORM_B200_SCHED_AUTO,     STORM_B200_SCHED_AUTO,
                               STORM_B200_SCHED_TILES};
        const bool ok[NK] = {bits <= TC_MAX_ROW_BITS, bits <= TC_MAX_ROW_BITS,    bits <= TC_MAX_ROW_BITS,
                             bits <= TC_MAX_ROW_BITS, bits <= TC_SS_MAX_ROW_BITS, true,
                             bits <= TC_MAX_ROW_BITS};
        const int keep_sched = c->engine.schedule;
        double best = -1.0;
        int bk = c->kernel_pref, bs = keep_sched;
        for (int k = 0; k < NK; ++k) {
            if (times_ms) times_ms[k] = -1.0;
            if (!ok[k] || n == 0) continue;
            c->engine.schedule = sched[k];
            double ms = -1.0;
            for (int rep = 0; rep < 2; ++rep) {
                c->engine.run(c->d_rows.p, c->dev_rows, c->w_pad, bits, c->d_out.p, kern[k], contig_stream(c));
                const double m = c->engine.log.last_ms;
                ms = ms < 0 ? m : std::min(ms, m);
            }
            if (times_ms) times_ms[k] = ms;
            if (best < 0 || ms < best) {
                best = ms;
                bk = kern[k];
                bs = sched[k];
            }
        }
        c->kernel_pref = bk;
        c->engine.schedule = bs;
        if (best_kernel) *best_kernel = bk;
        if (best_schedule) *best_schedule = bs;
        return 0;
    });
}

int STORM_contig_upload(STORM_contiguous_t* c) {
    if (c == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        contig_flush(c);
        SB_CUDA(cudaStreamSynchronize(contig_stream(c)));
        return 0;
    });
}

// storm.cpp:1232: sum over i < j; 0 for a NULL handle.
uint64_t STORM_contig_pairw_intersect_cardinality(STORM_contiguous_t* bitmap) {
    if (bitmap == NULL) return 0;
    uint64_t s = 0;
    guard([&]() -> int {
        s = contig_run(bitmap, nullptr);
        return 0;
    });
    return s;
}

// The reference's blocked traversal is a CPU cache tiling of the same sum
// (storm.cpp:1248-1281); the GPU tiles on its own, so bsize only affects
// nothing but the call's name.
uint64_t STORM_contig_pairw_intersect_cardinality_blocked(STORM_contiguous_t* bitmap, uint32_t bsize) {
    (void)bsize;
    return STORM_contig_pairw_intersect_cardinality(bitmap);
}
uint64_t STORM_contig_pairw_intersect_cardinality_list(STORM_contiguous_t* bitmap) {
    return STORM_contig_pairw_intersect_cardinality(bitmap);
}
uint64_t STORM_contig_pairw_intersect_cardinality_blocked_list(STORM_contiguous_t* bitmap, uint32_t bsize) {
    (void)bsize;
    return STORM_contig_pairw_intersect_cardinality(bitmap);
}

int STORM_contig_pairw_intersect_matrix(STORM_contiguous_t* c, uint32_t* out, uint64_t out_len,
                                        uint64_t* sum) {
    if (c == NULL) return STORM_B200_ENULL;
    if (out == NULL && c->n_rows) return STORM_B200_EVALUES;
    return guard([&]() -> int {
        const uint64_t s = contig_matrix_host(c, out, out_len);
        if (sum) *sum = s;
        return 0;
    });
}

int STORM_contig_pairw_intersect_matrix_from_host(STORM_contiguous_t* c, const uint64_t* rows, uint32_t n_rows,
                                                  uint32_t words_per_row, uint32_t* out, uint64_t out_len,
                                                  uint64_t* sum) {
    if (c == NULL) return STORM_B200_ENULL;
    if ((rows == NULL || out == NULL) && n_rows) return STORM_B200_EVALUES;
    return guard([&]() -> int {
        if (words_per_row != c->n_words) return STORM_B200_EARG;
        if (out_len < tri_size(n_rows)) return STORM_B200_ESIZE;
        if (n_rows) {
            cudaPointerAttributes pa;
            const bool on_device = cudaPointerGetAttributes(&pa, rows) == cudaSuccess &&
                                   (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
            cudaGetLastError();
            if (on_device) return STORM_B200_EARG;
        }
        if (c->vector_length % 64 && n_rows) {
            const uint64_t tail_mask = ~0ull << (c->vector_length % 64);
            for (uint64_t r = 0; r < n_rows; ++r)
                if (rows[r * words_per_row + words_per_row - 1] & tail_mask) return STORM_B200_EARG;
        }
        c->stage.clear();
        c->n_rows = 0;
        c->dev_rows = 0;
        if (sum) *sum = 0;
        if (n_rows == 0) return 0;
        contig_grow(c, n_rows);
        c->d_out.reserve(tri_size(n_rows));
        if (!c->copy_stream) SB_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        if (!c->h2d_stream) SB_CUDA(cudaStreamCreateWithFlags(&c->h2d_stream, cudaStreamNonBlocking));
        const uint64_t s = c->engine.run_host_to_host(c->d_rows.p, n_rows, c->w_pad, c->vector_length, rows,
                                                      words_per_row, c->d_out.p, out, c->kernel_pref,
                                                      contig_stream(c), c->copy_stream, c->h2d_stream);
        c->n_rows = c->dev_rows = n_rows;
        if (sum) *sum = s;
        return 0;
    });
}

int STORM_contig_pairw_intersect_matrix_device(STORM_contiguous_t* c, uint32_t* d_out, uint64_t out_len,
                                               uint64_t* sum) {
    if (c == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        if (d_out && out_len < tri_size(c->n_rows)) return STORM_B200_ESIZE;
        // The caller's buffer may still be in use by work on other streams.
        if (d_out) SB_CUDA(cudaDeviceSynchronize());
        const uint64_t s = contig_run(c, d_out);
        if (sum) *sum = s;
        return 0;
    });
}

int STORM_contig_pairw_threshold(STORM_contiguous_t* c, double jaccard_min, uint32_t* out_i, uint32_t* out_j,
                                 uint32_t* out_count, uint64_t cap, uint64_t* n_found) {
    if (c == NULL) return STORM_B200_ENULL;
    if (std::isnan(jaccard_min)) return STORM_B200_EARG;
    if (cap && (out_i == NULL || out_j == NULL || out_count == NULL)) return STORM_B200_EVALUES;
    return guard([&]() -> int {
        contig_flush(c);
        cudaStream_t st = contig_stream(c);
        c->d_hits.reserve(cap ? cap : 1);
        c->d_hit_cnt.reserve(cap ? cap : 1);
        const uint64_t found = c->engine.run_threshold(c->d_rows.p, c->dev_rows, c->w_pad, c->vector_length,
                                                       c->kernel_pref, jaccard_min, c->d_hits.p, c->d_hit_cnt.p, cap,
                                                       nullptr, st);
        if (n_found) *n_found = found;
        return threshold_to_host(c->d_hits.p, c->d_hit_cnt.p, found, cap, out_i, out_j, out_count, st);
    });
}

int STORM_contig_pairw_intersect_tiles(STORM_contiguous_t* c, uint32_t tile, STORM_tile_callback cb,
                                       void* ctx) {
    if (c == NULL) return STORM_B200_ENULL;
    if (cb == NULL || tile == 0) return STORM_B200_EARG;
    return guard([&]() -> int {
        const uint64_t n = c->n_rows;
        std::vector<uint32_t> tri(tri_size(n) ? tri_size(n) : 1);
        contig_matrix_host(c, tri.data(), tri.size());
        std::vector<uint32_t> buf((size_t)tile * tile);
        for (uint64_t i0 = 0; i0 < n; i0 += tile) {
            const uint64_t i1 = std::min<uint64_t>(i0 + tile, n);
            for (uint64_t j0 = i0; j0 < n; j0 += tile) {
                const uint64_t j1 = std::min<uint64_t>(j0 + tile, n);
                std::fill(buf.begin(), buf.end(), 0u);
                for (uint64_t i = i0; i < i1; ++i) {
                    const uint64_t base = i * n - (i * (i - 1)) / 2 - i;
                    for (uint64_t j = (j0 == i0 ? i + 1 : j0); j < j1; ++j)
                        buf[(i - i0) * tile + (j - j0)] = tri[base + j];
                }
                cb((uint32_t)i0, (uint32_t)j0, (uint32_t)(i1 - i0), (uint32_t)(j1 - j0), buf.data(), ctx);
            }
        }
        return 0;
    });
}

void* STORM_contig_stream(STORM_contiguous_t* c) {
    if (c == NULL) return NULL;
    void* s = NULL;
    guard([&]() -> int {
        s = (void*)contig_stream(c);
        return 0;
    });
    return s;
}

float STORM_contig_last_kernel_ms(const STORM_contiguous_t* c) { return c ? c->engine.log.last_ms : 0.f; }
uint32_t STORM_contig_last_launches(const STORM_contiguous_t* c) { return c ? c->engine.log.launches : 0; }
int STORM_contig_last_kernel(const STORM_contiguous_t* c) { return c ? c->engine.log.kernel : 0; }

}  // extern "C"
