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

// Every representation of the rows, in HBM, and a host copy of the
// per-row metadata (the host orders rows and checks policies with it).
struct RowsDev {
    DevBuf<RowMetaD> meta;
    DevBuf<uint64_t> s_off, r_off, w_off, m_off, c_off, b_off, rk_off, oc_off, w_buf, bm, rk, oc;
    DevBuf<uint32_t> s_val, r_start, r_end, c_val;
    DevBuf<uint2> m_tab;
    DevBuf<uint4> counts;              // per-row sizes, scratch of the build
    std::vector<RowMetaD> h_meta;
    RowsView view{};
};

// Uploads the rows' sorted positions and builds every representation from
// them on the device (rows_pack.cu). `bm_rows` marks the rows that get B
// (empty: every row). Synchronous on `st`.
void build_rows(const std::vector<uint32_t>& vals, const std::vector<uint64_t>& offs, uint32_t universe,
                const std::vector<uint8_t>& bm_rows, RowsDev& d, cudaStream_t st);

}  // namespace sb200
