// storm_t.cu -- the chunked container (STORM_t and its parts) behind the
// reference's public layout.
//
// Ingest builds exactly the host structures the reference builds
// (storm.cpp:396-916): per row a STORM_bitmap_cont_t whose chunks are u16
// lists below STORM_DEFAULT_SCALAR_THRESHOLD values and 1024-word bitmaps
// otherwise, so callers that read the public structs see the same data.
// Differences, all outside the reference's input contract:
//   * the reference's one-past-the-end read in STORM_bitmap_cont_add
//     (storm.cpp:768) and its scalar-buffer overflow when a second add brings
//     more values than the remaining capacity (storm.cpp:513-523) are not
//     reproduced;
//   * values outside a chunk (the reference only asserts) are skipped.
// All counting (every *_intersect_* call) runs on the GPU: the rows are
// packed into HBM on first use and re-packed after STORM_add / STORM_clear.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <memory>
#include <chrono>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cmath>
#include "chunk_engine.cuh"
#include "dense.cuh"
#include "oneshot.cuh"

namespace sb200 {

static void* aligned_alloc64(size_t bytes) {
    void* p = nullptr;
    if (posix_memalign(&p, 64, bytes ? bytes : 64) != 0) return nullptr;
    return p;
}

// Device-side state of a STORM_t, kept beside it (the public struct has no
// room for it).  Invalidated by every mutating call through this library.
struct StormDev {
    ChunkDev dev;
    PinnedStage stage;
    ChunkEngine engine;
    cudaStream_t stream = nullptr;
    DevBuf<uint32_t> d_out;
    DevBuf<uint32_t> d_card, d_hit_cnt;    // thresholded form
    DevBuf<uint2> d_hits;
    DevBuf<unsigned long long> d_found;
    bool valid = false;
    uint64_t shape = 0;    // row_shape() of the rows last packed
    double xfer[4] = {0, 0, 0, 0};   // STORM_last_transfer_ms
    ~StormDev() {
        if (stream) cudaStreamDestroy(stream);
    }
};

static std::mutex g_mu;
static std::unordered_map<const STORM_t*, StormDev*>& table() {
    static std::unordered_map<const STORM_t*, StormDev*> t;
    return t;
}

static StormDev* state_of(const STORM_t* s) {
    std::lock_guard<std::mutex> lock(g_mu);
    auto& t = table();
    auto it = t.find(s);
    if (it != t.end()) return it->second;
    StormDev* d = new StormDev();
    t[s] = d;
    return d;
}

static void invalidate(const STORM_t* s) {
    std::lock_guard<std::mutex> lock(g_mu);
    auto& t = table();
    auto it = t.find(s);
    if (it != t.end()) it->second->valid = false;
}

static void forget(const STORM_t* s) {
    std::lock_guard<std::mutex> lock(g_mu);
    auto& t = table();
    auto it = t.find(s);
    if (it != t.end()) {
        delete it->second;
        t.erase(it);
    }
}

static cudaStream_t stream_of(StormDev* d) {
    require_device();
    if (!d->stream) SB_CUDA(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking));
    return d->stream;
}

// The public struct can also be changed without this library's STORM_add /
// STORM_clear (STORM_bitmap_cont_add on one of s->conts, as the layout
// allows): a hash of each row's chunk count, last inserted value and chunk
// array catches that too, at O(rows) host cost per call.
static uint64_t row_shape(const STORM_t* s) {
    uint64_t h = 0x9E3779B97F4A7C15ull ^ (uint64_t)(uintptr_t)s->conts ^ ((uint64_t)s->n_conts << 1);
    auto mix = [&](uint64_t v) {
        h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
    };
    for (uint32_t r = 0; r < s->n_conts; ++r) {
        const STORM_bitmap_cont_t& c = s->conts[r];
        mix((uint64_t)c.n_bitmaps << 32 | c.prev_inserted_value);
        mix((uint64_t)(uintptr_t)c.bitmaps);
    }
    return h;
}

static double wall_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static void ensure_packed(const STORM_t* s, StormDev* d) {
    const uint64_t shape = row_shape(s);
    for (double& x : d->xfer) x = 0.0;
    if (d->valid && d->shape == shape) return;
    const double t0 = wall_ms();
    d->dev.upload_rows(s->conts, s->n_conts, stream_of(d), d->stage);
    d->xfer[0] = wall_ms() - t0;
    d->xfer[1] = (double)d->dev.payload_bytes;
    d->valid = true;
    d->shape = shape;
}

// This thread's reusable context for the calls that compare a few chunks or
// rows (kept across calls: one stream and the engine's buffers per device).
OneShot& one_shot() {
    require_device();
    int dev = 0;
    SB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) fail(STORM_B200_ECUDA, "device ordinal out of range");
    thread_local std::unique_ptr<OneShot> per_device[64];
    std::unique_ptr<OneShot>& h = per_device[dev];
    if (!h) {
        std::unique_ptr<OneShot> fresh(new OneShot());
        SB_CUDA(cudaStreamCreateWithFlags(&fresh->st, cudaStreamNonBlocking));
        h = std::move(fresh);
    }
    h->pack.clear();
    return *h;
}

}  // namespace sb200

using namespace sb200;

extern "C" {

/* ---------------------------------------------------------------- chunks */

STORM_bitmap_t* STORM_bitmap_new(void) {
    STORM_bitmap_t* b = (STORM_bitmap_t*)malloc(sizeof(STORM_bitmap_t));
    if (!b) return NULL;
    STORM_bitmap_init(b);
    return b;
}

void STORM_bitmap_init(STORM_bitmap_t* b) {
    if (!b) return;
    b->data = NULL;
    b->scalar = NULL;
    b->n_bitmap = 0;
    b->own_data = 1;
    b->own_scalar = 1;
    b->n_bits_set = 0;
    b->n_scalar = 0;
    b->n_scalar_set = 0;
    b->n_missing = 0;
    b->m_scalar = 0;
    b->id = 0;
}

static void bitmap_free_members(STORM_bitmap_t* b) {
    if (!b) return;
    if (b->own_data) free(b->data);
    if (b->own_scalar) free(b->scalar);
    b->data = NULL;
    b->scalar = NULL;
}

void STORM_bitmap_free(STORM_bitmap_t* b) {
    if (!b) return;
    bitmap_free_members(b);
    free(b);
}

static bool ensure_data(STORM_bitmap_t* b) {
    if (b->data == NULL) {
        b->data = (uint64_t*)aligned_alloc64(CHUNK_WORDS * sizeof(uint64_t));
        if (!b->data) return false;
        memset(b->data, 0, CHUNK_WORDS * sizeof(uint64_t));
        b->own_data = 1;
    }
    b->n_bitmap = CHUNK_WORDS;
    return true;
}

static bool ensure_scalar(STORM_bitmap_t* b, uint32_t extra) {
    const uint64_t need = (uint64_t)b->n_scalar + extra;
    if (b->scalar != NULL && need <= b->m_scalar) return true;
    uint64_t m = b->scalar ? need + 1024 : (extra > 256 ? (uint64_t)extra + 256 : 256);
    if (m < need) m = need;
    uint16_t* p = (uint16_t*)aligned_alloc64(m * sizeof(uint16_t));
    if (!p) return false;
    if (b->scalar) {
        memcpy(p, b->scalar, b->n_scalar * sizeof(uint16_t));
        if (b->own_scalar) free(b->scalar);
    }
    b->scalar = p;
    b->m_scalar = (uint32_t)m;
    b->own_scalar = 1;
    return true;
}

// storm.cpp:476-499: -1 / -2 / -3, sets bits of values in this chunk.
int STORM_bitmap_add(STORM_bitmap_t* b, const uint32_t* values, const uint32_t n_values) {
    if (b == NULL) return -1;
    if (values == NULL) return -2;
    if (n_values == 0) return -3;
    if (!ensure_data(b)) return STORM_B200_ENOMEM;
    const uint64_t base = (uint64_t)b->id * STORM_DEFAULT_BLOCK_SIZE;
    // Bits of one word are gathered in a register while consecutive values
    // stay in that word (sorted input: up to 64 per store), and the word's
    // newly set bits are counted when it is written back -- the same bits
    // and the same n_bits_set as setting them one value at a time.
    uint32_t cur = ~0u;
    uint64_t acc = 0;
    for (uint32_t i = 0; i < n_values; ++i) {
        if (values[i] < base || values[i] - base >= STORM_DEFAULT_BLOCK_SIZE) continue;
        const uint32_t v = (uint32_t)(values[i] - base);
        if ((v >> 6) != cur) {
            if (cur != ~0u) {
                b->n_bits_set += (uint32_t)__builtin_popcountll(acc & ~b->data[cur]);
                b->data[cur] |= acc;
            }
            cur = v >> 6;
            acc = 0;
        }
        acc |= 1ull << (v & 63);
    }
    if (cur != ~0u) {
        b->n_bits_set += (uint32_t)__builtin_popcountll(acc & ~b->data[cur]);
        b->data[cur] |= acc;
    }
    return (int)n_values;
}

// storm.cpp:502-553: -1 / -3 / -4; bitmap plus the list of newly set values.
int STORM_bitmap_add_with_scalar(STORM_bitmap_t* b, const uint32_t* values, const uint32_t n_values) {
    if (b == NULL) return -1;
    if (values == NULL) return -3;
    if (n_values == 0) return -4;
    if (!ensure_data(b) || !ensure_scalar(b, n_values)) return STORM_B200_ENOMEM;
    const uint64_t base = (uint64_t)b->id * STORM_DEFAULT_BLOCK_SIZE;
    b->n_scalar_set = 1;
    for (uint32_t i = 0; i < n_values; ++i) {
        if (values[i] < base || values[i] - base >= STORM_DEFAULT_BLOCK_SIZE) continue;
        const uint32_t v = (uint32_t)(values[i] - base);
        const uint64_t bit = 1ull << (v & 63);
        if ((b->data[v >> 6] & bit) == 0) {
            b->data[v >> 6] |= bit;
            b->scalar[b->n_scalar] = (uint16_t)v;
            ++b->n_scalar;
            ++b->n_bits_set;
        }
    }
    return (int)n_values;
}

// storm.cpp:555-592: -1 / -3 / -4; appends values as chunk offsets.
int STORM_bitmap_add_scalar_only(STORM_bitmap_t* b, const uint32_t* values, const uint32_t n_values) {
    if (b == NULL) return -1;
    if (values == NULL) return -3;
    if (n_values == 0) return -4;
    if (!ensure_scalar(b, n_values)) return STORM_B200_ENOMEM;
    const uint64_t base = (uint64_t)b->id * STORM_DEFAULT_BLOCK_SIZE;
    b->n_scalar_set = 1;
    for (uint32_t i = 0; i < n_values; ++i) {
        if (values[i] < base || values[i] - base >= STORM_DEFAULT_BLOCK_SIZE) continue;
        b->scalar[b->n_scalar] = (uint16_t)(values[i] - base);
        ++b->n_scalar;
        ++b->n_bits_set;
    }
    return (int)n_values;
}

int STORM_bitmap_clear(STORM_bitmap_t* b) {
    if (b == NULL) return -1;
    if (b->data != NULL) memset(b->data, 0, sizeof(uint64_t) * b->n_bitmap);
    b->n_scalar = 0;
    b->n_bits_set = 0;
    b->n_bitmap = 0;
    return 1;
}

uint32_t STORM_bitmap_serialized_size(STORM_bitmap_t* b) {
    uint32_t total = (uint32_t)sizeof(uint64_t) * b->n_bitmap;
    if (b->n_scalar_set) total += (uint32_t)sizeof(uint16_t) * b->n_scalar;
    return total + 4 * (uint32_t)sizeof(uint32_t);
}

// storm.cpp:595-650: one chunk pair, 0 for NULL or different chunk ids.
uint64_t STORM_bitmap_intersect_cardinality(STORM_bitmap_t* STORM_RESTRICT b1, STORM_bitmap_t* STORM_RESTRICT b2) {
    if (b1 == NULL || b2 == NULL) return 0;
    if (b1->id != b2->id) return 0;
    uint64_t r = 0;
    guard([&]() -> int {
        OneShot& h = one_shot();
        h.pack.add_chunk(b1->id, *b1);
        h.pack.end_row();
        h.pack.add_chunk(b2->id, *b2);
        h.pack.end_row();
        r = h.rect(1, 1);
        return 0;
    });
    return r;
}

uint64_t STORM_bitmap_intersect_cardinality_func(STORM_bitmap_t* STORM_RESTRICT b1, STORM_bitmap_t* STORM_RESTRICT b2,
                                                 const STORM_compute_func func) {
    (void)func;
    return STORM_bitmap_intersect_cardinality(b1, b2);
}

/* ------------------------------------------------------------ containers */

STORM_bitmap_cont_t* STORM_bitmap_cont_new(void) {
    STORM_bitmap_cont_t* c = (STORM_bitmap_cont_t*)malloc(sizeof(STORM_bitmap_cont_t));
    if (!c) return NULL;
    STORM_bitmap_cont_init(c);
    return c;
}

void STORM_bitmap_cont_init(STORM_bitmap_cont_t* c) {
    if (!c) return;
    c->bitmaps = NULL;
    c->block_ids = NULL;
    c->n_bitmaps = 0;
    c->m_bitmaps = 0;
    c->prev_inserted_value = 0;
}

static void cont_free_members(STORM_bitmap_cont_t* c) {
    if (!c) return;
    if (c->bitmaps) {
        // Entries past n_bitmaps only ever hold buffers that clear() kept.
        for (uint32_t i = 0; i < c->m_bitmaps; ++i) bitmap_free_members(&c->bitmaps[i]);
        free(c->bitmaps);
    }
    free(c->block_ids);
    c->bitmaps = NULL;
    c->block_ids = NULL;
    c->n_bitmaps = 0;
    c->m_bitmaps = 0;
}

void STORM_bitmap_cont_free(STORM_bitmap_cont_t* c) {
    if (!c) return;
    cont_free_members(c);
    free(c);
}

static bool cont_reserve(STORM_bitmap_cont_t* c, uint32_t n) {
    if (n <= c->m_bitmaps && c->bitmaps && c->block_ids) return true;
    uint32_t m = c->m_bitmaps ? c->m_bitmaps : 2;
    while (m < n) m += 8;
    STORM_bitmap_t* nb = (STORM_bitmap_t*)realloc(c->bitmaps, sizeof(STORM_bitmap_t) * m);
    if (!nb) return false;
    for (uint32_t i = c->m_bitmaps; i < m; ++i) STORM_bitmap_init(&nb[i]);
    c->bitmaps = nb;
    uint32_t* ni = (uint32_t*)realloc(c->block_ids, sizeof(uint32_t) * m);
    if (!ni) return false;
    c->block_ids = ni;
    c->m_bitmaps = m;
    return true;
}

// storm.cpp:737-803: split sorted values by chunk; a run of fewer than
// STORM_DEFAULT_SCALAR_THRESHOLD values becomes a u16 list, otherwise a
// bitmap.  -1 NULL container, -2 NULL values, 0 for n == 0, 1 on success.
int STORM_bitmap_cont_add(STORM_bitmap_cont_t* c, const uint32_t* values, const uint32_t n_values) {
    if (c == NULL) return -1;
    if (values == NULL) return -2;
    if (n_values == 0) return 0;
    uint32_t start = 0;
    while (start < n_values) {
        const uint32_t id = values[start] / STORM_DEFAULT_BLOCK_SIZE;
        uint32_t stop = start;
        while (stop < n_values && values[stop] / STORM_DEFAULT_BLOCK_SIZE == id) ++stop;
        if (!cont_reserve(c, c->n_bitmaps + 1)) return STORM_B200_ENOMEM;
        STORM_bitmap_t* x = &c->bitmaps[c->n_bitmaps];
        x->id = id;
        c->block_ids[c->n_bitmaps] = id;
        int rc = (stop - start < STORM_DEFAULT_SCALAR_THRESHOLD)
                     ? STORM_bitmap_add_scalar_only(x, values + start, stop - start)
                     : STORM_bitmap_add(x, values + start, stop - start);
        if (rc < 0) return rc;
        ++c->n_bitmaps;
        c->prev_inserted_value = values[stop - 1];
        start = stop;
    }
    return 1;
}

int STORM_bitmap_cont_clear(STORM_bitmap_cont_t* c) {
    if (c == NULL) return -1;
    for (uint32_t i = 0; i < c->n_bitmaps; ++i) STORM_bitmap_clear(&c->bitmaps[i]);
    c->n_bitmaps = 0;
    c->prev_inserted_value = 0;
    return 1;
}

// storm.cpp:804-833: one row pair.
uint64_t STORM_bitmap_cont_intersect_cardinality(const STORM_bitmap_cont_t* STORM_RESTRICT c1,
                                                 const STORM_bitmap_cont_t* STORM_RESTRICT c2) {
    if (c1 == NULL || c2 == NULL) return 0;
    if (c1->n_bitmaps == 0 || c2->n_bitmaps == 0) return 0;
    uint64_t r = 0;
    guard([&]() -> int {
        OneShot& h = one_shot();
        h.pack.add_row(c1);
        h.pack.add_row(c2);
        r = h.rect(1, 1);
        return 0;
    });
    return r;
}

uint64_t STORM_bitmap_cont_intersect_cardinality_premade(const STORM_bitmap_cont_t* STORM_RESTRICT c1,
                                                         const STORM_bitmap_cont_t* STORM_RESTRICT c2,
                                                         const STORM_compute_func func, uint32_t* out) {
    (void)func;
    if (out == NULL) return 0;
    return STORM_bitmap_cont_intersect_cardinality(c1, c2);
}

uint32_t STORM_bitmap_cont_serialized_size(STORM_bitmap_cont_t* c) {
    uint32_t total = 0;
    if (c->bitmaps != NULL)
        for (uint32_t i = 0; i < c->n_bitmaps; ++i) total += STORM_bitmap_serialized_size(&c->bitmaps[i]);
    return total + (uint32_t)sizeof(uint32_t) * c->n_bitmaps + 3 * (uint32_t)sizeof(uint32_t);
}

/* ----------------------------------------------------------------- STORM_t */

STORM_t* STORM_new(void) {
    STORM_t* s = (STORM_t*)malloc(sizeof(STORM_t));
    if (!s) return NULL;
    s->conts = NULL;
    s->n_conts = 0;
    s->m_conts = 0;
    return s;
}

void STORM_free(STORM_t* s) {
    if (s == NULL) return;
    forget(s);
    if (s->conts)
        for (uint32_t i = 0; i < s->m_conts; ++i) cont_free_members(&s->conts[i]);
    free(s->conts);
    free(s);
}

// storm.cpp:894-916: always appends a row (even for n == 0), returns 1.
int STORM_add(STORM_t* s, const uint32_t* values, const uint32_t n_values) {
    if (s == NULL) return -1;
    invalidate(s);
    if (s->n_conts == s->m_conts) {
        const uint32_t m = s->m_conts + 1024;
        STORM_bitmap_cont_t* nc = (STORM_bitmap_cont_t*)realloc(s->conts, m * sizeof(STORM_bitmap_cont_t));
        if (!nc) return STORM_B200_ENOMEM;
        for (uint32_t i = s->m_conts; i < m; ++i) STORM_bitmap_cont_init(&nc[i]);
        s->conts = nc;
        s->m_conts = m;
    }
    STORM_bitmap_cont_add(&s->conts[s->n_conts++], values, n_values);
    return 1;
}

// n_rows STORM_add calls at once: the row array grows once, then the rows
// are split into chunks on several host threads (each row is its own
// STORM_bitmap_cont_t, so threads never share one).
int64_t STORM_add_rows(STORM_t* s, const uint32_t* values, const uint64_t* offsets, uint64_t n_rows) {
    if (s == NULL) return STORM_B200_ENULL;
    if (n_rows == 0) return 0;
    if (offsets == NULL || (values == NULL && offsets[n_rows] > offsets[0])) return STORM_B200_EVALUES;
    for (uint64_t r = 0; r < n_rows; ++r)
        if (offsets[r + 1] < offsets[r] || offsets[r + 1] - offsets[r] > 0xFFFFFFFFull) return STORM_B200_EARG;
    if ((uint64_t)s->n_conts + n_rows > 0xFFFFFFFFull) return STORM_B200_ELIMIT;
    invalidate(s);
    const uint64_t need = (uint64_t)s->n_conts + n_rows;
    if (need > s->m_conts) {
        const uint64_t m = (need + 1023) / 1024 * 1024;
        if (m > 0xFFFFFFFFull) return STORM_B200_ELIMIT;
        STORM_bitmap_cont_t* nc = (STORM_bitmap_cont_t*)realloc(s->conts, m * sizeof(STORM_bitmap_cont_t));
        if (!nc) return STORM_B200_ENOMEM;
        for (uint64_t i = s->m_conts; i < m; ++i) STORM_bitmap_cont_init(&nc[i]);
        s->conts = nc;
        s->m_conts = (uint32_t)m;
    }
    const uint32_t first = s->n_conts;
    std::atomic<int> failed{0};
    auto fill = [&](uint64_t r0, uint64_t r1) {
        for (uint64_t r = r0; r < r1; ++r) {
            const uint64_t a = offsets[r], b = offsets[r + 1];
            if (STORM_bitmap_cont_add(&s->conts[first + r], b > a ? values + a : values, (uint32_t)(b - a)) < 0)
                failed.store(1);
        }
    };
    const uint64_t total = offsets[n_rows] - offsets[0];
    const unsigned hw = host_threads();
    const uint64_t n_thr = std::min<uint64_t>({(uint64_t)std::min(hw, 64u), n_rows, 1 + total / (1u << 20)});
    if (n_thr <= 1) {
        fill(0, n_rows);
    } else {
        // contiguous row ranges of about equal value counts
        std::vector<uint64_t> cut{0};
        for (uint64_t r = 0; r < n_rows && cut.size() < n_thr; ++r)
            if ((offsets[r + 1] - offsets[0]) * n_thr >= total * cut.size()) cut.push_back(r + 1);
        if (cut.back() != n_rows) cut.push_back(n_rows);
        std::vector<std::thread> th;
        for (size_t t = 0; t + 1 < cut.size(); ++t)
            if (cut[t] < cut[t + 1]) th.emplace_back(fill, cut[t], cut[t + 1]);
        for (auto& t : th) t.join();
    }
    s->n_conts = (uint32_t)need;
    return failed.load() ? STORM_B200_ENOMEM : (int64_t)n_rows;
}

// Rows given as bitmaps: each row's set positions, ascending, through the
// same chunk split as STORM_add, one host thread per range of rows.
int64_t STORM_add_bitmap_rows(STORM_t* s, const uint64_t* words, uint64_t n_rows, uint64_t words_per_row) {
    if (s == NULL) return STORM_B200_ENULL;
    if (n_rows == 0) return 0;
    if (words == NULL) return STORM_B200_EVALUES;
    if (words_per_row == 0 || words_per_row > (1ull << 26)) return STORM_B200_EARG;   // positions < 2^32
    if ((uint64_t)s->n_conts + n_rows > 0xFFFFFFFFull) return STORM_B200_ELIMIT;
    invalidate(s);
    const uint64_t need = (uint64_t)s->n_conts + n_rows;
    if (need > s->m_conts) {
        const uint64_t m = (need + 1023) / 1024 * 1024;
        if (m > 0xFFFFFFFFull) return STORM_B200_ELIMIT;
        STORM_bitmap_cont_t* nc = (STORM_bitmap_cont_t*)realloc(s->conts, m * sizeof(STORM_bitmap_cont_t));
        if (!nc) return STORM_B200_ENOMEM;
        for (uint64_t i = s->m_conts; i < m; ++i) STORM_bitmap_cont_init(&nc[i]);
        s->conts = nc;
        s->m_conts = (uint32_t)m;
    }
    const uint32_t first = s->n_conts;
    std::atomic<int> failed{0};
    // Chunk by chunk, what STORM_bitmap_cont_add builds from the row's set
    // positions: no chunk without a set bit; a list below
    // STORM_DEFAULT_SCALAR_THRESHOLD set bits (their positions); otherwise
    // a bitmap, taken as the words themselves (STORM_bitmap_add on a fresh
    // chunk sets exactly these bits and counts them).
    auto fill = [&](uint64_t r0, uint64_t r1) {
        std::vector<uint32_t> pos;
        for (uint64_t r = r0; r < r1; ++r) {
            const uint64_t* w = words + r * words_per_row;
            STORM_bitmap_cont_t* c = &s->conts[first + r];
            for (uint64_t k0 = 0; k0 < words_per_row; k0 += CHUNK_WORDS) {
                const uint64_t kw = std::min<uint64_t>(CHUNK_WORDS, words_per_row - k0);
                uint64_t cnt = 0, last_k = 0;
                for (uint64_t k = 0; k < kw; ++k)
                    if (w[k0 + k]) {
                        cnt += (uint64_t)__builtin_popcountll(w[k0 + k]);
                        last_k = k;
                    }
                if (cnt == 0) continue;
                const uint32_t id = (uint32_t)(k0 / CHUNK_WORDS);
                if (!cont_reserve(c, c->n_bitmaps + 1)) {
                    failed.store(1);
                    return;
                }
                STORM_bitmap_t* x = &c->bitmaps[c->n_bitmaps];
                x->id = id;
                c->block_ids[c->n_bitmaps] = id;
                if (cnt < STORM_DEFAULT_SCALAR_THRESHOLD) {
                    pos.clear();
                    for (uint64_t k = 0; k < kw; ++k)
                        for (uint64_t y = w[k0 + k]; y; y &= y - 1)
                            pos.push_back((uint32_t)((k0 + k) * 64 + __builtin_ctzll(y)));
                    if (STORM_bitmap_add_scalar_only(x, pos.data(), (uint32_t)pos.size()) < 0) {
                        failed.store(1);
                        return;
                    }
                } else {
                    if (!ensure_data(x)) {
                        failed.store(1);
                        return;
                    }
                    std::memcpy(x->data, w + k0, kw * sizeof(uint64_t));
                    x->n_bits_set += (uint32_t)cnt;
                }
                ++c->n_bitmaps;
                c->prev_inserted_value = (uint32_t)((k0 + last_k) * 64 + 63 - __builtin_clzll(w[k0 + last_k]));
            }
        }
    };
    const unsigned hw = host_threads();
    const uint64_t n_thr = std::min<uint64_t>({(uint64_t)std::min(hw, 64u), n_rows,
                                               1 + n_rows * words_per_row / (1u << 17)});
    if (n_thr <= 1) {
        fill(0, n_rows);
    } else {
        std::vector<std::thread> th;
        for (uint64_t t = 0; t < n_thr; ++t) th.emplace_back(fill, n_rows * t / n_thr, n_rows * (t + 1) / n_thr);
        for (auto& t : th) t.join();
    }
    s->n_conts = (uint32_t)need;
    return failed.load() ? STORM_B200_ENOMEM : (int64_t)n_rows;
}

int STORM_clear(STORM_t* s) {
    if (s == NULL) return -1;
    invalidate(s);
    for (uint32_t i = 0; i < s->n_conts; ++i) STORM_bitmap_cont_clear(&s->conts[i]);
    s->n_conts = 0;
    return 1;
}

int STORM_upload(STORM_t* s) {
    if (s == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        ensure_packed(s, state_of(s));
        return 0;
    });
}

// storm.cpp:927-945: sum over i < j; (uint64_t)-1 for NULL.
uint64_t STORM_pairw_intersect_cardinality(STORM_t* s) {
    if (s == NULL) return (uint64_t)-1;
    uint64_t r = 0;
    guard([&]() -> int {
        StormDev* d = state_of(s);
        ensure_packed(s, d);
        r = d->engine.run(d->dev, PAIRS_TRIANGLE, s->n_conts, 0, nullptr, stream_of(d));
        return 0;
    });
    return r;
}

// storm.cpp:947-1011: the same sum, traversed in CPU cache blocks; the GPU
// path does its own tiling, so bsize does not change the work.
uint64_t STORM_pairw_intersect_cardinality_blocked(STORM_t* s, uint32_t bsize) {
    (void)bsize;
    return STORM_pairw_intersect_cardinality(s);
}

// storm.cpp:1027-1046: sum over all (i in s1, j in s2).
uint64_t STORM_intersect_cardinality_square(const STORM_t* STORM_RESTRICT s1, const STORM_t* STORM_RESTRICT s2) {
    if (s1 == NULL || s2 == NULL) return 0;
    uint64_t r = 0;
    guard([&]() -> int {
        OneShot& h = one_shot();
        h.pack.add_rows(s1->conts, s1->n_conts);
        h.pack.add_rows(s2->conts, s2->n_conts);
        r = h.rect(s1->n_conts, s2->n_conts);
        return 0;
    });
    return r;
}

uint64_t STORM_serialized_size(const STORM_t* s) {
    if (s == NULL) return 0;
    uint64_t tot = 0;
    for (uint32_t i = 0; i < s->n_conts; ++i) tot += STORM_bitmap_cont_serialized_size(&s->conts[i]);
    return tot + 2 * sizeof(uint32_t);
}

int STORM_pairw_intersect_matrix(STORM_t* s, uint32_t* out, uint64_t out_len, uint64_t* sum) {
    if (s == NULL) return STORM_B200_ENULL;
    const uint64_t need = tri_size(s->n_conts);
    if (out == NULL && need) return STORM_B200_EVALUES;
    if (out_len < need) return STORM_B200_ESIZE;
    return guard([&]() -> int {
        StormDev* d = state_of(s);
        ensure_packed(s, d);
        cudaStream_t st = stream_of(d);
        d->d_out.reserve(need ? need : 1);
        const uint64_t r = d->engine.run(d->dev, PAIRS_TRIANGLE, s->n_conts, 0, d->d_out.p, st);
        if (need) {
            const double t0 = wall_ms();
            copy_to_host(out, d->d_out.p, need, st, d->stage);
            d->xfer[2] = wall_ms() - t0;
            d->xfer[3] = (double)need * sizeof(uint32_t);
        }
        if (sum) *sum = r;
        return 0;
    });
}

int STORM_pairw_intersect_matrix_device(STORM_t* s, uint32_t* d_out, uint64_t out_len, uint64_t* sum) {
    if (s == NULL) return STORM_B200_ENULL;
    if (d_out && out_len < tri_size(s->n_conts)) return STORM_B200_ESIZE;
    return guard([&]() -> int {
        StormDev* d = state_of(s);
        ensure_packed(s, d);
        // The caller's buffer may still be in use by work on other streams.
        if (d_out) SB_CUDA(cudaDeviceSynchronize());
        const uint64_t r = d->engine.run(d->dev, PAIRS_TRIANGLE, s->n_conts, 0, d_out, stream_of(d));
        if (sum) *sum = r;
        return 0;
    });
}

int STORM_pairw_threshold(STORM_t* s, double jaccard_min, uint32_t* out_i, uint32_t* out_j, uint32_t* out_count,
                          uint64_t cap, uint64_t* n_found) {
    if (s == NULL) return STORM_B200_ENULL;
    if (std::isnan(jaccard_min)) return STORM_B200_EARG;
    if (cap && (out_i == NULL || out_j == NULL || out_count == NULL)) return STORM_B200_EVALUES;
    return guard([&]() -> int {
        StormDev* d = state_of(s);
        ensure_packed(s, d);
        cudaStream_t st = stream_of(d);
        const uint64_t n = s->n_conts;
        d->d_out.reserve(tri_size(n) ? tri_size(n) : 1);
        d->engine.run(d->dev, PAIRS_TRIANGLE, n, 0, d->d_out.p, st);
        d->d_card.reserve(n ? n : 1);
        d->d_found.reserve(1);
        d->d_hits.reserve(cap ? cap : 1);
        d->d_hit_cnt.reserve(cap ? cap : 1);
        const uint64_t found = threshold_from_triangle(d->d_out.p, n, jaccard_min, d->d_card.p, d->d_found.p,
                                                       d->d_hits.p, d->d_hit_cnt.p, cap, st);
        if (n_found) *n_found = found;
        return threshold_to_host(d->d_hits.p, d->d_hit_cnt.p, found, cap, out_i, out_j, out_count, st);
    });
}

int STORM_pairw_intersect_tiles(STORM_t* s, uint32_t tile, STORM_tile_callback cb, void* ctx) {
    if (s == NULL) return STORM_B200_ENULL;
    if (cb == NULL || tile == 0) return STORM_B200_EARG;
    const uint64_t n = s->n_conts;
    std::vector<uint32_t> tri(tri_size(n) ? tri_size(n) : 1);
    int rc = STORM_pairw_intersect_matrix(s, tri.data(), tri.size(), NULL);
    if (rc < 0) return rc;
    return guard([&]() -> int {
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

float STORM_last_kernel_ms(const STORM_t* s) {
    if (s == NULL) return 0.f;
    return state_of(s)->engine.log.last_ms;
}

int STORM_set_dense_block(STORM_t* s, double min_density, uint64_t budget_bytes) {
    if (s == NULL) return STORM_B200_ENULL;
    if (std::isnan(min_density)) return STORM_B200_EARG;
    StormDev* d = state_of(s);
    d->engine.dense_min_density = min_density;
    d->engine.dense_budget_bytes = budget_bytes;
    return 0;
}

uint64_t STORM_last_dense_rows(const STORM_t* s) { return s ? state_of(s)->engine.last_dense_rows : 0; }
uint64_t STORM_last_dense_panels(const STORM_t* s) { return s ? state_of(s)->engine.last_dense_panels : 0; }

int STORM_autotune(STORM_t* s, double* best_min_density, int* best_postings, double* times_ms) {
    if (s == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        StormDev* d = state_of(s);
        ensure_packed(s, d);
        cudaStream_t st = stream_of(d);
        const uint64_t n = s->n_conts;
        d->d_out.reserve(tri_size(n) ? tri_size(n) : 1);
        // Which engines may take rows: tensor rows by the cost rule or none,
        // postings by cost or none; timed with the per-pair call.
        const double dens[4] = {CHUNK_DENSE_AUTO, CHUNK_DENSE_AUTO, 0.0, 0.0};
        const int post[4] = {-1, 0, -1, 0};
        double best = -1.0;
        double bd = d->engine.dense_min_density;
        int bp = d->engine.postings_mode;
        for (int k = 0; k < 4; ++k) {
            d->engine.dense_min_density = dens[k];
            d->engine.postings_mode = post[k];
            double ms = -1.0;
            for (int rep = 0; rep < 2; ++rep) {
                d->engine.run(d->dev, PAIRS_TRIANGLE, n, 0, d->d_out.p, st);
                const double m = d->engine.log.last_ms;
                ms = ms < 0 ? m : std::min(ms, m);
            }
            if (times_ms) times_ms[k] = ms;
            if (best < 0 || ms < best) {
                best = ms;
                bd = dens[k];
                bp = post[k];
            }
        }
        d->engine.dense_min_density = bd;
        d->engine.postings_mode = bp;
        if (best_min_density) *best_min_density = bd;
        if (best_postings) *best_postings = bp;
        return 0;
    });
}

int STORM_set_sparse_postings(STORM_t* s, int mode) {
    if (s == NULL) return STORM_B200_ENULL;
    if (mode < -1 || mode > 4) return STORM_B200_EARG;
    state_of(s)->engine.postings_mode = mode;
    return 0;
}

uint64_t STORM_last_postings_rows(const STORM_t* s) { return s ? state_of(s)->engine.last_postings_rows : 0; }

int STORM_last_postings_form(const STORM_t* s) {
    if (s == NULL) return STORM_B200_ENULL;
    return state_of(s)->engine.last_postings_form;
}

int STORM_last_engine_ms(const STORM_t* s, double* out12) {
    if (s == NULL) return STORM_B200_ENULL;
    if (out12 == NULL) return STORM_B200_EVALUES;
    const ChunkEngine& e = state_of(s)->engine;
    for (int k = 0; k < 4; ++k) {
        out12[k] = e.last_engine_ms[k];
        out12[4 + k] = e.last_engine_pred_ms[k];
        out12[8 + k] = e.last_engine_work[k];
    }
    return 0;
}

int STORM_last_transfer_ms(const STORM_t* s, double* out4) {
    if (s == NULL) return STORM_B200_ENULL;
    if (out4 == NULL) return STORM_B200_EVALUES;
    const StormDev* d = state_of(s);
    for (int k = 0; k < 4; ++k) out4[k] = d->xfer[k];
    return 0;
}

double STORM_last_plan_ms(const STORM_t* s) {
    if (s == NULL) return -1.0;
    return state_of(s)->engine.last_plan_ms;
}

// The planner's constants fitted to this GPU on a sample of the rows (the
// reference's calibrate_on_rows, storm_cost.cpp:779-895, samples the
// caller's pairs the same way: strided, not the first rows): every plain row
// of the sample on the tensor cores, then in the transposed panel, then the
// list rows by postings; per engine the ratio of measured to predicted
// device time (best of two) scales that engine's constants.
int STORM_calibrate(STORM_t* s, uint32_t sample_rows, double* out) {
    if (s == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        StormDev* d = state_of(s);
        const uint64_t n = s->n_conts;
        const uint64_t m = std::min<uint64_t>(n, sample_rows ? sample_rows : 2048);
        if (m < 2) return STORM_B200_EARG;
        ChunkPack p;
        for (uint64_t k = 0; k < m; ++k) p.add_row(&s->conts[k * n / m]);
        cudaStream_t st = stream_of(d);
        ChunkDev cd;
        cd.upload(p, st);
        ChunkEngine e;
        e.cost = d->engine.cost;
        DevBuf<uint32_t> out_buf;
        out_buf.reserve(tri_size(m));
        // engine k: (dense_min_density, postings_mode, panel_mode) forcing it
        const double dens[3] = {1e-12, 0.0, 0.0};
        const int post[3] = {0, -1, 1}, pan[3] = {0, 2, 0}, eng[3] = {0, 2, 3};
        double scale[3] = {1.0, 1.0, 1.0};
        int post_form = -1;
        for (int k = 0; k < 3; ++k) {
            e.dense_min_density = dens[k];
            e.postings_mode = post[k];
            e.panel_mode = pan[k];
            double meas = -1.0, pred = 0.0;
            for (int rep = 0; rep < 2; ++rep) {
                e.run(cd, PAIRS_TRIANGLE, m, 0, out_buf.p, st);
                const double ms = e.last_engine_ms[eng[k]];
                meas = meas < 0 ? ms : std::min(meas, ms);
                pred = e.last_engine_pred_ms[eng[k]];
            }
            if (pred > 1e-4 && meas > 0) scale[k] = meas / pred;
            if (k == 2) post_form = e.last_postings_form;
        }
        ChunkCostModel& c = d->engine.cost;
        c.ns_per_tensor_bit *= scale[0];
        c.ns_per_panel_value *= scale[1];
        c.ns_per_panel_pair *= scale[1];
        c.ns_per_panel_byte *= scale[1];
        if (post_form == 2) {   // the postings ran as the run sweep: its constant
            c.ns_per_run_check *= scale[2];
        } else {
            c.ns_per_posting_pair *= scale[2];
            c.ns_per_posting_pair_hbm *= scale[2];
            c.ns_per_posting_sweep *= scale[2];
        }
        c.ns_per_sweep_row_pair *= scale[2];
        if (out) {
            out[0] = scale[0];
            out[1] = scale[1];
            out[2] = scale[2];
            out[3] = (double)m;
        }
        return 0;
    });
}

int STORM_reset_cost_model(STORM_t* s) {
    if (s == NULL) return STORM_B200_ENULL;
    state_of(s)->engine.cost = ChunkCostModel{};
    return 0;
}

int STORM_set_panel(STORM_t* s, int mode) {
    if (s == NULL) return STORM_B200_ENULL;
    if (mode < -1 || mode > 2) return STORM_B200_EARG;
    state_of(s)->engine.panel_mode = mode;
    return 0;
}

uint64_t STORM_last_panel_rows(const STORM_t* s) { return s ? state_of(s)->engine.last_panel_rows : 0; }

}  // extern "C"
