// chunk_engine.cuh -- device layout and kernels for rows split into
// 65536-bit chunks (the STORM_t representation, storm.h:158-178,
// storm.cpp:737-803).
//
// HBM layout (CSR over rows, structure of arrays over chunks):
//   row_off[r] .. row_off[r+1]   the row's chunks, ascending chunk id
//   cid[c]                       chunk id (value >> 16)
//   ckl[c]                       bit 31: bitmap chunk; bit 30: list holds a
//                                repeated value; bits 0..29: words or entries
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
//   S x S  lanes stride over the shorter list and binary-search the longer,
//          matching the k-th copy of a value with the k-th copy (the scalar
//          merge's count, storm.cpp:72-86).
#pragma once
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

// Host staging of the packed layout.
struct ChunkPack {
    std::vector<uint64_t> row_off{0};
    std::vector<uint32_t> cid, ckl;
    std::vector<uint64_t> coff;
    std::vector<uint64_t> bm;
    std::vector<uint16_t> lst;
    void clear() {
        row_off.assign(1, 0);
        cid.clear(); ckl.clear(); coff.clear(); bm.clear(); lst.clear();
    }
    uint64_t rows() const { return row_off.size() - 1; }
    void add_chunk(uint32_t id, const STORM_bitmap_t& b);
    void add_row(const STORM_bitmap_cont_t* c);   // c may be NULL (empty row)
    void end_row() { row_off.push_back(cid.size()); }
};

struct ChunkDev {
    DevBuf<uint64_t> row_off, coff, bm;
    DevBuf<uint32_t> cid, ckl;
    DevBuf<uint16_t> lst;
    uint64_t n_rows = 0;
    void upload(const ChunkPack& p, cudaStream_t st);
    ChunkView view() const {
        return ChunkView{row_off.p, cid.p, ckl.p, coff.p, bm.p, lst.p};
    }
};

// Pair spaces the chunk kernel walks.
enum PairMode : uint32_t {
    PAIRS_TRIANGLE = 0,   // i <= j < n, packed output
    PAIRS_RECT = 1,       // i < n1, n1 <= j < n1 + n2 (sum only)
};

struct ChunkEngine {
    DevBuf<DeviceFlags> d_flags;
    LaunchLog log;
    ~ChunkEngine() { log.destroy(); }
    // Returns the sum over i < j (triangle) or over all (i, j) (rect).
    uint64_t run(const ChunkDev& d, PairMode mode, uint64_t n1, uint64_t n2, uint32_t* d_out,
                 cudaStream_t st);
};

}  // namespace sb200
