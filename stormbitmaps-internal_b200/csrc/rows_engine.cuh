// rows_engine.cuh -- HBM layout of a STORM_rows_t (the reference's
// storm::Row, storm_repr.h:112-276, packed for the GPU) and the engine state.
//
// Every row keeps, in structure-of-arrays pools addressed by per-row offsets:
//   S  sorted u32 positions                         s_off[r] .. s_off[r+1]
//   R  maximal runs [start, end), two u32 streams    r_off[r] .. r_off[r+1]
//   W  EWAH-64 stream (storm_repr.h:28-31)           w_off[r] .. w_off[r+1]
//      + a marker table (stream position, first decoded word) so a warp can
//        jump to the marker covering any word         m_off[r] .. m_off[r+1]
//   B  bitmap, nw words (16-byte aligned), when the row got one   b_off[r]
//   rank9 / zone map under the reference's gates (storm_repr.cpp:186-189)
//   C  complement positions when density > 1/2 (storm_repr.cpp:139-154)
// Absent forms have offset NONE.
#pragma once
#include <vector>
#include "common.cuh"
#include "rows_cost.cuh"

namespace sb200 {

constexpr uint64_t NONE = ~0ull;

struct RowsView {
    uint32_t n, universe, nw, n_occ;
    const RowMetaD* meta;
    const uint64_t* s_off;
    const uint32_t* s_val;
    const uint64_t* r_off;
    const uint32_t* r_start;
    const uint32_t* r_end;
    const uint64_t* w_off;
    const uint64_t* w_buf;
    const uint64_t* m_off;
    const uint2* m_tab;      // (stream position of the marker, first decoded word)
    const uint64_t* b_off;
    const uint64_t* bm;
    const uint64_t* rk_off;
    const uint64_t* rk;
    const uint64_t* oc_off;
    const uint64_t* oc;
    const uint64_t* c_off;
    const uint32_t* c_val;
};

// Host-side packed form (built once per upload).
struct RowsPack {
    std::vector<RowMetaD> meta;
    std::vector<uint64_t> s_off{0}, r_off{0}, w_off{0}, m_off{0}, c_off{0};
    std::vector<uint32_t> s_val, r_start, r_end, c_val;
    std::vector<uint64_t> w_buf, bm, rk, oc;
    std::vector<uint2> m_tab;
    std::vector<uint64_t> b_off, rk_off, oc_off;
};

template <class T>
struct DevVec {
    DevBuf<T> buf;
    void put(const std::vector<T>& h, cudaStream_t st) {
        buf.reserve(h.size() ? h.size() : 1);
        if (!h.empty())
            SB_CUDA(cudaMemcpyAsync(buf.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    }
};

struct RowsDev {
    DevVec<RowMetaD> meta;
    DevVec<uint64_t> s_off, r_off, w_off, m_off, c_off, b_off, rk_off, oc_off, w_buf, bm, rk, oc;
    DevVec<uint32_t> s_val, r_start, r_end, c_val;
    DevVec<uint2> m_tab;
    RowsView view{};
};

// Build every representation of the rows (host, O(total size + bitmap words
// of the rows that get a bitmap)).  `bm_rows` marks the rows that get B.
void pack_rows(const std::vector<uint32_t>& vals, const std::vector<uint64_t>& offs, uint32_t universe,
               const std::vector<uint8_t>& bm_rows, RowsPack& p);
void upload_rows(const RowsPack& p, uint32_t universe, RowsDev& d, cudaStream_t st);

}  // namespace sb200
