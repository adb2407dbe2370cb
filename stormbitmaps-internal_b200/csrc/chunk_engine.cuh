// chunk_engine.cuh -- device layout and kernels for rows split into
// 65536-bit chunks (the STORM_t representation, storm.h:158-178,
// storm.cpp:737-803).
//
// HBM layout (CSR over rows, structure of arrays over chunks):
//   row_off[r] .. row_off[r+1]   the row's chunks, ascending chunk id
//   cid[c]                       chunk id (value >> 16)
//   ckl[c]                       bit 31: bitmap chunk; bit 30: list is not
//                                strictly increasing (a repeated or
//                                out-of-order entry); bits 0..29: words or
//                                entries
//   coff[c]                      offset into bm (words) or lst (entries)
//   bm                           1024-word bitmaps, 16-byte aligned
//   lst                          u16 offsets within the chunk, ascending
//
// A pair of rows is one warp: the chunk-id lists are intersected by binary
// search of the shorter list's ids in the longer one (the same matches as
// the reference's two-pointer STORM_intersect_vector32_unsafe,
// storm.cpp:90-121, including its pairing of repeated ids by rank), then
// each shared chunk is one warp-cooperative cell, chosen by the chunk kinds
// exactly as STORM_bitmap_intersect_cardinality_func does (storm.cpp:652-690):
//   B x B  1024-word AND + POPC, 32 words per lane;
//   B x S  probe: lanes stride over the list, one bit test each;
//   S x S  strictly increasing lists: lanes stride over the shorter list
//          and binary-search the longer; otherwise one lane restates the
//          reference's blocked SSE4.2 count (list16_ref.cuh), which a repeat
//          or an out-of-order entry makes differ from the set size.
#pragma once
#include <memory>
#include <utility>
#include <vector>
#include "common.cuh"

namespace sb200 {

constexpr uint32_t CK_BITMAP = 1u << 31;
constexpr uint32_t CK_DUP = 1u << 30;
constexpr uint32_t CK_LEN = (1u << 30) - 1;
constexpr uint32_t CHUNK_WORDS = 1024;

struct ChunkView {
    const uint64_t* row_off;
    const uint32_t* cid;
    const uint32_t* ckl;
    const uint64_t* coff;
    const uint64_t* bm;
    const uint16_t* lst;
};

// What the dense block needs to know of a row: its value count, chunk
// counts by kind, list entries, and whether it is "plain" (strictly
// ascending chunk ids, no repeated list value, full 1024-word bitmaps -- so
// that its chunks expand to one contiguous bitmap with the same counts).
// Allocator whose resize() leaves new elements unwritten (the bitmap pool is
// filled entirely by the packer, so zeroing it first only costs time).
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U>&) {}
    template <class U>
    void construct(U* p) {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... Args>
    void construct(U* p, Args&&... args) {
        ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
    }
};

struct ChunkRowFacts {
    uint64_t card = 0, list_entries = 0;
    uint64_t runs = 0;   // maximal runs of consecutive values inside the list chunks
    uint32_t chunks = 0, bitmap_chunks = 0;
    bool plain = true;
};

// Host staging of the packed layout, with the per-row facts and the largest
// chunk id.
struct ChunkPack {
    std::vector<uint64_t> row_off{0};
    std::vector<uint32_t> cid, ckl;
    std::vector<uint64_t> coff;
    std::vector<uint64_t, NoInitAlloc<uint64_t>> bm;   // every word is written by the packer
    std::vector<uint16_t> lst;
    std::vector<ChunkRowFacts> facts;
    uint32_t max_cid = 0;
    void clear() {
        row_off.assign(1, 0);
        cid.clear(); ckl.clear(); coff.clear(); bm.clear(); lst.clear();
        facts.clear();
        max_cid = 0;
    }
    uint64_t rows() const { return row_off.size() - 1; }
    void add_chunk(uint32_t id, const STORM_bitmap_t& b);
    void add_row(const STORM_bitmap_cont_t* c);   // c may be NULL (empty row)
    // n rows at once, filled by several host threads; the result is the
    // same as n calls of add_row.
    void add_rows(const STORM_bitmap_cont_t* rows, uint64_t n);
    void end_row() { row_off.push_back(cid.size()); }
};

// Pinned host staging for copies between pageable host memory and the
// device: one lane per host worker thread, each with two pinned buffers
// (one filled or drained by its thread while the other one's copy runs),
// its own stream and two events. Allocated once per handle.
struct PinnedStage {
    static constexpr uint64_t TOTAL = 128ull << 20;   // pinned bytes per handle
    struct Lane {
        unsigned char* buf[2] = {nullptr, nullptr};
        cudaEvent_t done[2] = {nullptr, nullptr};
        cudaStream_t st = nullptr;
    };
    unsigned char* pool = nullptr;
    std::vector<Lane> lanes;
    uint64_t lane_bytes = 0;   // bytes of each of a lane's two buffers
    cudaEvent_t ready = nullptr;
    PinnedStage() = default;
    PinnedStage(const PinnedStage&) = delete;
    PinnedStage& operator=(const PinnedStage&) = delete;
    ~PinnedStage();
    void ensure();   // min(64, host threads) lanes
};

// Copies `count` u32 from device memory to host memory `out` once the work
// already queued on `st` is done, and returns when they are there: one copy
// when `out` is pinned or small, else through the stage's lanes, each host
// worker draining its share of `out` while the next slice of that share
// crosses PCIe.
void copy_to_host(uint32_t* out, const uint32_t* d_src, uint64_t count, cudaStream_t st, PinnedStage& stage);

struct ChunkDev {
    DevBuf<uint64_t> row_off, coff, bm;
    DevBuf<uint32_t> cid, ckl;
    DevBuf<uint16_t> lst;
    uint64_t n_rows = 0;
    std::vector<ChunkRowFacts> facts;   // host copy of the per-row facts
    uint32_t max_cid = 0;
    uint64_t payload_bytes = 0;         // bitmap and list bytes of the last upload
    void upload(const ChunkPack& p, cudaStream_t st);
    // The same layout as upload(ChunkPack::add_rows(rows, n)), without the
    // host copy of the payload: the rows' chunk metadata is built on host
    // threads; their bitmaps and lists are gathered by host workers, each
    // over its own range of chunks, straight into its pinned lane, whose
    // copies to the device run while the worker fills its other buffer; the
    // lists' order (the CK_DUP flag and the rows' "plain" fact) is tested on
    // the device after the upload.
    void upload_rows(const STORM_bitmap_cont_t* rows, uint64_t n, cudaStream_t st, PinnedStage& stage);
    DevBuf<uint8_t> d_row_dup;
    DevBuf<uint32_t> d_row_runs;
    ChunkView view() const {
        return ChunkView{row_off.p, cid.p, ckl.p, coff.p, bm.p, lst.p};
    }
};

struct PostingsStats;   // chunk_engine.cu

// Work item of the transposed-panel engine (panel.cuh): the query row's walk
// position, the range [c_lo, c_hi) of its chunks (indices within the row),
// and its scratch slot (0xFFFFFFFF: the item is the whole row and writes the
// triangle itself).
struct PanelItem {
    uint32_t xw, c_lo, c_hi, slot;
};

// A query row split into work items: its walk position and its scratch
// slots [slot0, slot0 + nslots).
struct PanelSplit {
    uint32_t xw, slot0, nslots, pad;
};

// Pair spaces the chunk kernel walks.
enum PairMode : uint32_t {
    PAIRS_TRIANGLE = 0,   // i <= j < n, packed output
    PAIRS_RECT = 1,       // i < n1, n1 <= j < n1 + n2 (sum only)
};

// Tensor-core dense block of the chunked engine (triangle mode): chosen plain
// rows (universe = 65536 x (largest chunk id + 1), at most 2^27 bits) are
// expanded, panel by panel, into contiguous bitmaps in HBM and compared with
// each other by the tcgen05 kernel; the chunk kernel then walks only the
// pairs with another row.
//
// Which rows: with dense_min_density > 0, those whose value count is at least
// that share of the universe; with dense_min_density < 0 (the default), those
// whose predicted chunk-kernel cost against a copy of themselves exceeds the
// predicted tensor-core cost of one pair. A tensor-core pair costs in
// proportion to the universe; a chunk pair costs per shared chunk (a fixed
// part plus lane iterations: 32 for a bitmap chunk, ceil(e / 32) x
// (log2 e + 1) for lists of e entries -- the binary-search probe), and two
// rows of c chunks each share about c^2 / slots of them. The constants are
// B200 throughput figures (ns per pair with the whole GPU busy) fitted on
// Bernoulli rows at 1e-5 .. 0.17 over 2^24 and run-clustered rows over 2^26.
struct ChunkCostModel {
    double ns_per_shared_chunk = 0.086;
    double ns_per_lane_iteration = 0.0228;
    double ns_per_tensor_bit = 0.7e-6;
    double ns_per_posting_pair = 0.05;       // one (pair, shared value) increment, output in L2
    double ns_per_posting_pair_hbm = 0.042;  // the same, output larger than L2
    double ns_per_posting_sweep = 0.016;     // the same in the row sweep (shared memory)
    double ns_per_sweep_row_pair = 0.0047;   // row sweep: clearing and writing, per (row, row)
    double ns_per_universe_value = 2e-4;     // histogram clear + scan per universe value
    double ns_per_panel_value = 0.05;        // transposed panel: one query value against one 2048-row block
    double ns_per_panel_pair = 0.005;        // transposed panel: one count written
    double ns_per_panel_byte = 1.0 / 6000.0; // transposed panel: expansion and transpose traffic
    double ns_per_run_check = 0.03;          // run sweep: one bin entry read against one piece
};
double chunk_self_pair_ns(const ChunkCostModel& m, const ChunkRowFacts& f, uint64_t slots);
double tensor_pair_ns(const ChunkCostModel& m, uint64_t slots);

constexpr double CHUNK_DENSE_AUTO = -1.0;

// Postings for the sparse rows (plain rows without bitmap chunks, outside the
// dense block): a histogram of their values over the universe gives, per
// value, the rows holding it; each pair of those rows gets one increment
// per shared value, so pairs with nothing in common cost nothing. Used for
// the pairs among these rows when the exact increment count (from the
// histogram) predicts less time than the chunk kernel; sums need only the
// histogram: the sum over those pairs is sum_v C(rows holding v, 2).
constexpr uint64_t POSTINGS_MAX_UNIVERSE = 1ull << 27;
constexpr uint64_t L2_BYTES_B200 = 126ull << 20;

struct ChunkEngine {
    DevBuf<DeviceFlags> d_flags;
    LaunchLog log;
    double dense_min_density = CHUNK_DENSE_AUTO;
    ChunkCostModel cost;
    uint64_t dense_budget_bytes = 0;   // 0: 60 % of free device memory
    int postings_mode = -1;            // -1 by cost, 0 never, 1 always (when the rows qualify);
                                       // 2 / 3 / 4 always, per-pair form list by list / row sweep /
                                       // run sweep
    int panel_mode = -1;               // transposed panel: -1 by cost, 0 never, 1 whenever it can run,
                                       // 2 every plain row in it
    uint64_t last_dense_rows = 0, last_dense_panels = 0, last_postings_rows = 0;
    uint64_t last_panel_rows = 0, last_panel_queries = 0;
    int last_postings_form = -1;       // per-pair form of the last call's postings: 0 list by list,
                                       // 1 row sweep, 2 run sweep (-1: none)
    DevBuf<uint32_t> d_rpieces, d_rbins, d_rstart;
    DevBuf<uint64_t> d_rpoff;
    DevBuf<uint2> d_pieces, d_rlist;
    DevBuf<unsigned long long> d_rstats;
    // Per engine of the last per-pair triangle call -- tensor cores, chunk
    // kernel, transposed panel, postings (with the histograms): device ms
    // (events between the engines on the stream) and the cost model's
    // prediction for the work it gave each.
    double last_engine_ms[4] = {0, 0, 0, 0}, last_engine_pred_ms[4] = {0, 0, 0, 0};
    // ... and the algorithmic work of each: tensor cores in int8 operations
    // (2 x pairs x universe bits), chunk kernel in pairs, the panel and the
    // postings in bytes they must move (panel: one 256-byte transposed line
    // per query value and block, the expanded and transposed blocks, 4 bytes
    // per count written; postings: the histogram and list entries, 8 bytes
    // per increment -- a read and a write of its count).
    double last_engine_work[4] = {0, 0, 0, 0};
    cudaEvent_t ev_eng[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_hist0 = nullptr, ev_hist = nullptr;   // around the postings' histogram
    double last_plan_ms = 0.0;         // time before the first engine that is not the histogram
    DevBuf<uint64_t> d_pX, d_DT;       // panel block: expanded rows, transposed
    DevBuf<PanelItem> d_items;
    DevBuf<PanelSplit> d_splits;
    DevBuf<uint32_t> d_pscratch, d_pmap, d_mrows;
    DevBuf<unsigned long long> d_ctr;
    DevBuf<uint32_t> d_perm, d_map;
    DevBuf<uint32_t> d_qrows, d_counts, d_start, d_post;
    DevBuf<uint2> d_lists;
    DevBuf<PostingsStats> d_pstats;
    DevBuf<uint64_t> d_panel;
    DevBuf<uint2> d_tiles;
    ~ChunkEngine() {
        log.destroy();
        for (cudaEvent_t e : ev_eng)
            if (e) cudaEventDestroy(e);
        if (ev_hist) cudaEventDestroy(ev_hist);
        if (ev_hist0) cudaEventDestroy(ev_hist0);
    }
    // Returns the sum over i < j (triangle) or over all (i, j) (rect).
    uint64_t run(const ChunkDev& d, PairMode mode, uint64_t n1, uint64_t n2, uint32_t* d_out,
                 cudaStream_t st);
};

}  // namespace sb200
