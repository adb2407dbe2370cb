// rows_cost.cuh -- the reference's calibrated cost model (kernels/storm_cost.cpp)
// as host+device code, so selection can run inside the GPU tile driver.
//
// The work functions and the default constants are the reference's own
// (storm_cost.cpp:63-75 bb_expected_bins, :195-333 work_units, :372-420
// predict, :422-465 select_pairing, :482-496 default_model); they are kept
// formula-for-formula because the point of the port is identical decisions
// (tests/test_rows_gpu.py checks select_pairing and predict against the
// reference's golden outputs).  Knobs that the reference reads from the
// environment use their defaults here: probe scale 0.05, B x R orientation
// margin 16, R x R scale 1.0, no excluded cells.
#pragma once
#include <stdint.h>

namespace sb200 {

enum Pairing : int {
    P_BB = 0, P_BS, P_BR, P_BW, P_SS, P_SR, P_SW, P_RR, P_RW, P_WW, P_EMPTY, P_COUNT,
    P_CB = 11,   // complemented pairing, outside the selector's candidate set
};

// RowMeta (storm_repr.h:213-231) plus which representations the row has in HBM.
struct RowMetaD {
    uint32_t card, runs, nw, nnz, first, last;
    uint8_t has_rank, has_occ, has_bm, has_comp;
};

struct CostModelD {
    double ns_per_unit[P_COUNT];
    double ns_fixed, ns_per_occ_word, ns_probe_hot, ns_probe_cold;
    // C x B (|A & B| = |B| - |A' & B|, one probe per complement position):
    // not among the reference's candidates, so 0 (never chosen) in its
    // default model; a calibrated model prices it from its own timings.
    double ns_per_unit_cb;
    // Per-cell fixed cost per pair on top of ns_fixed, indexed by pairing
    // (P_CB included): 0 in the reference's model, fitted by the GPU
    // calibration, where each warp-cooperative cell has its own overhead.
    double ns_fixed_cell[P_CB + 1];
};

// Cells the selectors choose among, as slots: the reference's ten
// (P_BB .. P_WW) and C x B.
constexpr int N_SLOTS = P_EMPTY + 1;
__host__ __device__ inline int slot_cell(int slot) { return slot < P_EMPTY ? slot : P_CB; }
// The default model's price of one complement probe, the unit C x B's
// calibrated constant scales (a probe per entry, as B x S's is).
constexpr double CB_UNIT_REF = 0.30;

__host__ __device__ inline CostModelD default_cost_model() {
    CostModelD m{};
    m.ns_per_unit[P_BB] = 0.116;
    m.ns_per_unit[P_BS] = 0.30;
    m.ns_per_unit[P_BR] = 0.60;
    m.ns_per_unit[P_BW] = 0.55;
    m.ns_per_unit[P_SS] = 0.22;
    m.ns_per_unit[P_SR] = 0.35;
    m.ns_per_unit[P_SW] = 0.40;
    m.ns_per_unit[P_RR] = 0.30;
    m.ns_per_unit[P_RW] = 0.45;
    m.ns_per_unit[P_WW] = 0.50;
    m.ns_per_unit[P_EMPTY] = 0.0;
    m.ns_fixed = 2.0;
    m.ns_per_occ_word = 0.30;
    m.ns_probe_hot = 0.0;
    m.ns_probe_cold = 0.0;
    m.ns_per_unit_cb = 0.0;
    for (int p = 0; p <= P_CB; ++p) m.ns_fixed_cell[p] = 0.0;
    return m;
}

constexpr double BR_ORIENT_MARGIN = 16.0;
constexpr double PROBE_SCALE = 0.05;
constexpr double RR_SCALE = 1.0;

__host__ __device__ inline double dmax(double a, double b) { return a > b ? a : b; }
__host__ __device__ inline double dmin(double a, double b) { return a < b ? a : b; }

__host__ __device__ inline double bb_expected_bins(const RowMetaD& a, const RowMetaD& b) {
    const double bins = dmax(1.0, (double)(a.nw > b.nw ? a.nw : b.nw) / 8.0);
    const double fa = dmin(1.0, (double)a.nnz / (double)(a.nw > 1u ? a.nw : 1u));
    const double fb = dmin(1.0, (double)b.nnz / (double)(b.nw > 1u ? b.nw : 1u));
    const double pa = dmin(1.0, 8.0 * fa), pb = dmin(1.0, 8.0 * fb);
    return dmax(1.0, bins * pa * pb * 8.0);
}

__host__ __device__ inline uint32_t clz32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return (uint32_t)__clz(x);
#else
    return (uint32_t)__builtin_clz(x);
#endif
}

__host__ __device__ inline double work_units(int p, const RowMetaD& a, const RowMetaD& b) {
    const double sa = a.card, sb = b.card, ra = a.runs, rb = b.runs;
    const double wa = 2.0 * ra + 1.0 + (double)a.nnz;
    const double wb = 2.0 * rb + 1.0 + (double)b.nnz;
    const bool a_sparse = sa <= sb;
    const double s_card = a_sparse ? sa : sb;
    const double d_runs = a_sparse ? rb : ra;
    const double d_ewah = a_sparse ? wb : wa;
    switch (p) {
        case P_BB: return bb_expected_bins(a, b);
        case P_BS: return s_card;
        case P_BR: {
            const double dr = a_sparse ? rb : ra, sr = a_sparse ? ra : rb;
            const bool sw = dr * BR_ORIENT_MARGIN <= sr;
            return sw ? dr : sr;
        }
        case P_BW: {
            const double dr = a_sparse ? rb : ra, sr = a_sparse ? ra : rb;
            const bool sw = dr * BR_ORIENT_MARGIN <= sr;
            return sw ? (2.0 * dr + 1.0 + (double)(a_sparse ? b.nnz : a.nnz))
                      : (2.0 * sr + 1.0 + (double)(a_sparse ? a.nnz : b.nnz));
        }
        case P_SS: {
            const double m2 = dmax(2.0, dmax(sa, sb));
            const uint32_t mx = (uint32_t)m2;
            return dmin(sa, sb) * (double)(32u - clz32(mx));
        }
        case P_SR: return s_card + d_runs;
        case P_SW: return s_card + d_ewah;
        case P_RR: return ra + rb;
        case P_RW: return dmin(ra + wb, rb + wa);
        case P_WW: return wa + wb;
        default: return 0.0;
    }
}

// Complement positions of the denser row (the probes of C x B).
__host__ __device__ inline double cb_work(const RowMetaD& a, const RowMetaD& b) {
    const RowMetaD& d = a.card >= b.card ? a : b;
    const double u = (double)d.nw * 64.0;
    return u > (double)d.card ? u - (double)d.card : 0.0;
}

__host__ __device__ inline double predict_cost(const CostModelD& m, int p, const RowMetaD& a, const RowMetaD& b) {
    if (p == P_EMPTY) return 0.0;
    if (p == P_CB) return m.ns_fixed + m.ns_fixed_cell[P_CB] + m.ns_per_unit_cb * cb_work(a, b);
    const double mw = (double)(a.nw > b.nw ? a.nw : b.nw);
    if (p == P_BB && !(a.has_occ && b.has_occ)) return m.ns_fixed + m.ns_fixed_cell[P_BB] + m.ns_per_unit[P_BB] * mw;
    double c = m.ns_fixed + m.ns_fixed_cell[p] + m.ns_per_unit[p] * work_units(p, a, b) * (p == P_RR ? RR_SCALE : 1.0);
    if (p == P_BS && m.ns_probe_cold > m.ns_probe_hot) {
        const double touches = (a.card <= b.card) ? (double)a.nnz : (double)b.nnz;
        c += (m.ns_probe_cold - m.ns_probe_hot) * PROBE_SCALE * touches;
    }
    if (p == P_BB) c += m.ns_per_occ_word * dmax(1.0, mw / 512.0);
    return c;
}

__host__ __device__ inline bool span_disjoint(const RowMetaD& a, const RowMetaD& b) {
    return a.card == 0 || b.card == 0 || a.last < b.first || b.last < a.first;
}

// Can the cell run on this oriented pair (d = denser, s = sparser)?  Cells
// that read a bitmap need one on the side that supplies it.
__host__ __device__ inline bool cell_available(int p, const RowMetaD& d, const RowMetaD& s) {
    switch (p) {
        case P_BB: return d.has_bm && s.has_bm;
        case P_BS: return d.has_bm;
        case P_BR:
        case P_BW: {
            const bool swap = (double)d.runs * BR_ORIENT_MARGIN <= (double)s.runs;
            return swap ? s.has_bm : d.has_bm;
        }
        case P_CB: return d.has_comp && s.has_bm;
        default: return p >= 0 && p < P_EMPTY;
    }
}

// storm_cost.cpp:422-465, restricted to cells whose representations exist.
__host__ __device__ inline int select_pairing_d(const CostModelD& m, const RowMetaD& a, const RowMetaD& b,
                                                double* predicted) {
    if (span_disjoint(a, b)) {
        if (predicted) *predicted = 0.0;
        return P_EMPTY;
    }
    const bool a_dense = a.card >= b.card;
    const RowMetaD& d = a_dense ? a : b;
    const RowMetaD& s = a_dense ? b : a;
    int best = cell_available(P_BB, d, s) ? P_BB : P_SS;
    double bestc = predict_cost(m, best, a, b);
    for (int i = 0; i < P_EMPTY; ++i) {
        if (m.ns_per_unit[i] <= 0.0) continue;
        if (!cell_available(i, d, s)) continue;
        const double c = predict_cost(m, i, a, b);
        if (c < bestc) {
            bestc = c;
            best = i;
        }
    }
    if (m.ns_per_unit_cb > 0.0 && cell_available(P_CB, d, s)) {
        const double c = predict_cost(m, P_CB, a, b);
        if (c < bestc) {
            bestc = c;
            best = P_CB;
        }
    }
    if (predicted) *predicted = bestc;
    return best;
}

}  // namespace sb200
