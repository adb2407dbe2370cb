// rows_engine.cu -- STORM_rows_t: the reference's batched all-pairs driver
// (kernels/storm_allpairs.cpp) on the GPU.
//
// One all-pairs call = three device phases on the handle's stream:
//   1. block_meta_kernel   per row block of the traversal order: the tile
//                          aggregate RowMeta (tile_meta, storm_allpairs.cpp:281-312)
//   2. select_tiles_kernel per tile pair: the policy's cell (cost model, MLP,
//                          or top-2 for Probe/Refine), and for Probe a timed
//                          race of the top two on up to 3 pairs of the tile
//                          (probe_tile, storm_allpairs.cpp:445-482)
//   3. tiles_kernel        the pairs: span test, per-pair choice where the
//                          policy asks for it, the cell, the count written to
//                          the packed triangle in ORIGINAL row order.
// Execution forms: BATCHED = phase 3 as one persistent launch pulling
// (tile, slice) items from a device work queue, the whole call captured once
// in a CUDA graph and replayed; PER_TILE = phase 3 launched once per tile.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/storm_rows.h"
#include "mlp.cuh"
#include "dense.cuh"
#include "rows_cells.cuh"

namespace sb200 {

constexpr int TK_WARPS = 4;
constexpr int TK_THREADS = TK_WARPS * 32;

struct TileDecision {
    int cell, cell2;      // chosen cell; runner-up (Refine) or same
};

struct RowsStatsDev {
    unsigned long long sum, skipped, pairs;
    unsigned long long cell_pairs[STORM_PAIRING_COUNT + 1];
    unsigned int queue_head;
    unsigned int error;
};

// ---------------------------------------------------------------- phase 1
__global__ void block_meta_kernel(RowsView v, const uint32_t* __restrict__ order, uint32_t n, uint32_t T,
                                  RowMetaD* __restrict__ out, uint32_t* __restrict__ het_x1000) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nb = (n + T - 1) / T;
    if (b >= nb) return;
    const uint32_t lo = b * T, hi = min(n, lo + T);
    RowMetaD m{};
    m.first = 0xFFFFFFFFu;
    m.last = 0;
    uint64_t card = 0, runs = 0, nnz = 0;
    uint32_t mx = 0;
    m.has_rank = m.has_occ = m.has_bm = m.has_comp = 1;
    for (uint32_t k = lo; k < hi; ++k) {
        const RowMetaD& r = v.meta[order[k]];
        m.has_rank &= r.has_rank;
        m.has_occ &= r.has_occ;
        m.has_bm &= r.has_bm;
        m.has_comp &= r.has_comp;
        card += r.card;
        runs += r.runs;
        nnz += r.nnz;
        mx = max(mx, r.card);
        m.nw = max(m.nw, r.nw);
        if (r.card) {
            m.first = min(m.first, r.first);
            m.last = max(m.last, r.last);
        }
    }
    const uint32_t cnt = hi - lo;
    m.card = (uint32_t)(card / cnt);
    m.runs = (uint32_t)(runs / cnt);
    m.nnz = (uint32_t)(nnz / cnt);
    if (m.first == 0xFFFFFFFFu) m.first = 0;
    out[b] = m;
    const double mean = (double)card / cnt;
    het_x1000[b] = mean > 0 ? (uint32_t)fmin(4e9, 1000.0 * (double)mx / mean) : 1000u;
}

// Block zone maps (one CTA per row block of the traversal order): a
// superset of the coarse bins holding the block's values -- from each row's
// zone map where it has one (storm_repr.cpp:47-59: 512-value bins), from its
// values when it has at most ZONE_EXACT_MAX of them, else every bin of its
// [first, last] span.  Two blocks whose maps share no bin share no value:
// every pair of their tile is empty (the tile-granular form of the zone-map
// transpose of bench/bench_tile.cpp:224-264); their overlap is also a
// feature of the learned selector.
constexpr uint64_t ZONE_EXACT_MAX = 16384;

__device__ __forceinline__ void zone_set_range(unsigned long long* z, uint64_t c0, uint64_t c1) {
    for (uint64_t cb = c0; cb <= c1; ++cb) atomicOr(&z[cb >> 6], 1ull << (cb & 63));
}

__global__ void __launch_bounds__(256)
block_zone_kernel(RowsView v, const uint32_t* __restrict__ order, uint32_t n, uint32_t T,
                  uint64_t* __restrict__ out) {
    __shared__ unsigned long long z[BZONE_WORDS];
    const uint32_t b = blockIdx.x;
    const uint32_t lo = b * T, hi = min(n, lo + T);
    for (uint32_t k = threadIdx.x; k < BZONE_WORDS; k += blockDim.x) z[k] = 0ull;
    __syncthreads();
    const uint64_t ubits = (uint64_t)v.nw * 64;
    const uint64_t nbins = BZONE_WORDS * 64;
    auto bin_of = [&](uint64_t x) { return x * nbins / ubits; };
    for (uint32_t k = lo; k < hi; ++k) {
        const uint32_t row = order[k];
        const RowMetaD& m = v.meta[row];
        if (m.card == 0) continue;
        const uint64_t s0 = v.s_off[row], len = v.s_off[row + 1] - s0;
        if (v.oc_off[row] != NONE) {
            const uint64_t* oc = v.oc + v.oc_off[row];
            for (uint32_t w = threadIdx.x; w < v.n_occ; w += blockDim.x)
                for (uint64_t x = oc[w]; x; x &= x - 1) {
                    const uint64_t bin = (uint64_t)w * 64 + (uint64_t)(__ffsll((long long)x) - 1);
                    const uint64_t first = bin * 512, last = min(first + 511, ubits - 1);
                    zone_set_range(z, bin_of(first), bin_of(last));
                }
        } else if (len <= ZONE_EXACT_MAX) {
            for (uint64_t e = threadIdx.x; e < len; e += blockDim.x) {
                const uint64_t cb = bin_of(v.s_val[s0 + e]);
                atomicOr(&z[cb >> 6], 1ull << (cb & 63));
            }
        } else {
            const uint64_t c0 = bin_of(m.first), c1 = bin_of(m.last);
            for (uint64_t cb = c0 + threadIdx.x; cb <= c1; cb += blockDim.x) atomicOr(&z[cb >> 6], 1ull << (cb & 63));
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < BZONE_WORDS; k += blockDim.x) out[(uint64_t)b * BZONE_WORDS + k] = z[k];
}

__device__ __forceinline__ bool zones_disjoint(const uint64_t* za, const uint64_t* zb) {
    for (uint32_t k = 0; k < BZONE_WORDS; ++k)
        if (za[k] & zb[k]) return false;
    return true;
}

// Tile (ti, tj), ti <= tj, from a linear index over the block triangle.
__device__ __forceinline__ void tile_decode(uint32_t nb, uint32_t t, uint32_t& ti, uint32_t& tj) {
    // rows of the block triangle: row i holds nb - i tiles
    const double b = 2.0 * nb + 1.0;
    int64_t i = (int64_t)((b - sqrt(b * b - 8.0 * (double)t)) * 0.5);
    if (i < 0) i = 0;
    if (i >= (int64_t)nb) i = nb - 1;
    auto S = [nb](int64_t r) { return (uint64_t)r * nb - (uint64_t)r * (r - 1) / 2; };
    while (i > 0 && S(i) > t) --i;
    while (i + 1 < (int64_t)nb && S(i + 1) <= t) ++i;
    ti = (uint32_t)i;
    tj = (uint32_t)(t - S(i) + i);
}

// ---------------------------------------------------------------- phase 2
__global__ void select_tiles_kernel(const RowMetaD* __restrict__ bmeta, const uint32_t* __restrict__ het,
                                    const uint64_t* __restrict__ bzone, uint32_t nb, int policy, int fixed_cell,
                                    CostModelD model, const float* __restrict__ mlp, MlpShape shape,
                                    TileDecision* __restrict__ dec) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t ntiles = nb * (nb + 1) / 2;
    if (t >= ntiles) return;
    uint32_t ti, tj;
    tile_decode(nb, t, ti, tj);
    const RowMetaD& a = bmeta[ti];
    const RowMetaD& b = bmeta[tj];
    TileDecision d{P_BB, P_BB};
    // Whole-tile rejection: blocks whose zone maps do not meet hold no
    // common value, so every pair of the tile is empty.
    if (policy != STORM_POLICY_ALLBITMAP && bzone != nullptr && ti != tj &&
        zones_disjoint(bzone + (uint64_t)ti * BZONE_WORDS, bzone + (uint64_t)tj * BZONE_WORDS)) {
        dec[t] = TileDecision{P_EMPTY, P_EMPTY};
        return;
    }
    if (policy == STORM_POLICY_ALLBITMAP) {
        d.cell = d.cell2 = P_BB;
    } else if (policy == STORM_POLICY_FIXED) {
        d.cell = d.cell2 = fixed_cell;
    } else if (policy == STORM_POLICY_LEARNED && mlp != nullptr) {
        float x[MLP_MAX_F];
        tile_features(a, b, het[ti], het[tj],
                      zone_overlap(bzone + (uint64_t)ti * BZONE_WORDS, bzone + (uint64_t)tj * BZONE_WORDS), x);
        d.cell = d.cell2 = mlp_argmax_available(mlp, shape, x, a, b);
    } else {
        double best1 = 0.0;
        d.cell = select_pairing_d(model, a, b, &best1);
        if (d.cell == P_EMPTY) d.cell = (a.has_bm && b.has_bm) ? P_BB : P_SS;   // never skip a whole tile
        d.cell2 = d.cell;
        if (policy == STORM_POLICY_REFINE || policy == STORM_POLICY_PROBE) {
            // runner-up (tile_top2, storm_allpairs.cpp:332-347)
            const bool a_dense = a.card >= b.card;
            const RowMetaD& dd = a_dense ? a : b;
            const RowMetaD& ss = a_dense ? b : a;
            double best2 = 1e300;
            for (int p = 0; p < P_EMPTY; ++p) {
                if (p == d.cell || model.ns_per_unit[p] <= 0.0 || !cell_available(p, dd, ss)) continue;
                const double c = predict_cost(model, p, a, b);
                if (c < best2) {
                    best2 = c;
                    d.cell2 = p;
                }
            }
            if (policy == STORM_POLICY_REFINE) {
                // heterogeneity gate 8 and top-2 ratio gate 3 (storm_allpairs.cpp:126-138, 402-411)
                const double h = fmax(het[ti], het[tj]) / 1000.0;
                const double ratio = best1 > 0.0 ? best2 / best1 : 1e300;
                if (!(h >= 8.0 && ratio <= 3.0)) d.cell2 = d.cell;
            }
        }
    }
    dec[t] = d;
}

struct PairCtx {
    RowsView v;
    const uint32_t* order;
    uint32_t n, T, nb;
    int policy;
    CostModelD model;
    uint32_t dense_from = 0xFFFFFFFFu;   // sorted positions >= this form the tensor-core dense block
};

// Gather the bitmaps of the dense block (sorted positions [from, n)) into a
// zero-padded [nd_pad][w_pad] matrix for the tensor-core kernel.
__global__ void gather_dense_kernel(RowsView v, const uint32_t* __restrict__ order, uint32_t from, uint32_t nd,
                                    uint32_t nd_pad, uint64_t pitch, uint64_t* __restrict__ X,
                                    uint32_t* __restrict__ row_map) {
    const uint64_t total = (uint64_t)nd_pad * pitch;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(e / pitch), w = (uint32_t)(e % pitch);
        uint64_t x = 0;
        if (r < nd) {
            const uint32_t row = order[from + r];
            if (w < v.nw) x = v.bm[v.b_off[row] + w];
            if (w == 0) row_map[r] = row;
        }
        X[e] = x;
    }
}

// One pair in the traversal order -> (count, cell used).  Warp-cooperative.
__device__ __forceinline__ uint32_t pair_count(const PairCtx& c, uint32_t oi, uint32_t oj, const TileDecision& td,
                                               int lane, int& used) {
    const uint32_t ri = c.order[oi], rj = c.order[oj];
    const RowMetaD& mi = c.v.meta[ri];
    const RowMetaD& mj = c.v.meta[rj];
    if (ri == rj) {
        used = -1;
        return lane == 0 ? mi.card : 0u;
    }
    if (td.cell == P_EMPTY) {   // the whole tile was rejected by its blocks' zone maps
        used = P_EMPTY;
        return 0;
    }
    const bool i_dense = mi.card >= mj.card;
    const uint32_t d = i_dense ? ri : rj, s = i_dense ? rj : ri;
    const RowMetaD& md = i_dense ? mi : mj;
    const RowMetaD& ms = i_dense ? mj : mi;
    if (c.policy != STORM_POLICY_ALLBITMAP && span_disjoint(md, ms)) {
        used = P_EMPTY;
        return 0;
    }
    int p = td.cell;
    if (c.policy == STORM_POLICY_PERPAIR || c.policy == STORM_POLICY_ORACLE) {
        p = select_pairing_d(c.model, md, ms, nullptr);
    } else if (c.policy == STORM_POLICY_REFINE && td.cell2 != td.cell) {
        p = predict_cost(c.model, td.cell2, md, ms) < predict_cost(c.model, td.cell, md, ms) ? td.cell2 : td.cell;
    }
    if (p == P_EMPTY) {
        used = P_EMPTY;
        return 0;
    }
    if (!cell_available(p, md, ms)) p = select_pairing_d(c.model, md, ms, nullptr);   // a row lacks the form
    if (p == P_EMPTY) {
        used = P_EMPTY;
        return 0;
    }
    used = p;
    return run_cell(c.v, p, d, s, lane, c.policy != STORM_POLICY_ALLBITMAP);
}

// ---------------------------------------------------------------- probe
// One warp per tile: time the top two cells on up to three pairs of the tile
// (clock64 on the SM) and keep the faster (probe_tile).
__global__ void probe_tiles_kernel(PairCtx c, TileDecision* __restrict__ dec, uint32_t ntiles) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= ntiles) return;
    TileDecision td = dec[warp];
    if (td.cell2 == td.cell) return;
    uint32_t ti, tj;
    tile_decode(c.nb, warp, ti, tj);
    const uint32_t i0 = ti * c.T, i1 = min(c.n, i0 + c.T), j0 = tj * c.T, j1 = min(c.n, j0 + c.T);
    const int cand[2] = {td.cell, td.cell2};
    long long best_t = 0x7FFFFFFFFFFFFFFFll;
    int best = td.cell;
    for (int q = 0; q < 2; ++q) {
        const long long t0 = clock64();
        uint32_t sink = 0;
        for (uint32_t k = 0; k < 3; ++k) {
            const uint32_t i = i0 + (uint32_t)((uint64_t)(i1 - i0) * k / 3);
            const uint32_t j = (j0 == i0) ? i + 1 + k : j0 + (uint32_t)((uint64_t)(j1 - j0) * k / 3);
            if (!(i < i1 && j < j1 && i != j)) continue;
            const uint32_t ri = c.order[i], rj = c.order[j];
            const RowMetaD& mi = c.v.meta[ri];
            const RowMetaD& mj = c.v.meta[rj];
            const bool idn = mi.card >= mj.card;
            const RowMetaD& md = idn ? mi : mj;
            const RowMetaD& ms = idn ? mj : mi;
            if (!cell_available(cand[q], md, ms)) continue;
            sink += run_cell(c.v, cand[q], idn ? ri : rj, idn ? rj : ri, lane, true);
        }
        sink = warp_sum_u32(sink);
        const long long dt = clock64() - t0 + (sink == 0xFFFFFFFFu ? 1 : 0);
        if (dt < best_t) {
            best_t = dt;
            best = cand[q];
        }
    }
    if (lane == 0) dec[warp] = TileDecision{best, best};
}

// ---------------------------------------------------------------- phase 3
__global__ void __launch_bounds__(TK_THREADS)
tiles_kernel(PairCtx c, const TileDecision* __restrict__ dec, uint32_t first_tile, uint32_t tile_count,
             uint32_t slices, int use_queue, const uint32_t* __restrict__ tile_list, uint32_t* __restrict__ out,
             RowsStatsDev* __restrict__ st) {
    __shared__ unsigned long long s_cells[STORM_PAIRING_COUNT + 1];
    __shared__ unsigned long long s_sum, s_skip, s_pairs;
    __shared__ uint32_t s_item;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x < STORM_PAIRING_COUNT + 1) s_cells[threadIdx.x] = 0;
    if (threadIdx.x == 0) s_sum = s_skip = s_pairs = 0;
    __syncthreads();
    const uint32_t n_items = tile_count * slices;
    uint32_t item = blockIdx.x;
    unsigned long long my_sum = 0, my_skip = 0, my_pairs = 0;
    uint32_t my_cells[STORM_PAIRING_COUNT + 1];
    for (int k = 0; k <= STORM_PAIRING_COUNT; ++k) my_cells[k] = 0;
    for (;;) {
        if (use_queue) {
            if (threadIdx.x == 0) s_item = atomicAdd(&st->queue_head, 1u);
            __syncthreads();
            item = s_item;
            __syncthreads();
        }
        if (item >= n_items) break;
        const uint32_t t_local = item / slices, slice = item % slices;
        const uint32_t t = tile_list ? tile_list[first_tile + t_local] : first_tile + t_local;
        uint32_t ti, tj;
        tile_decode(c.nb, t, ti, tj);
        const TileDecision td = dec[t];
        const uint32_t i0 = ti * c.T, i1 = min(c.n, i0 + c.T), j0 = tj * c.T, j1 = min(c.n, j0 + c.T);
        const uint32_t nr = i1 - i0, nc = j1 - j0, np = nr * nc;
        for (uint32_t q = slice * TK_WARPS + warp; q < np; q += slices * TK_WARPS) {
            const uint32_t oi = i0 + q / nc, oj = j0 + q % nc;
            if (ti == tj && oj < oi) continue;
            if (oi >= c.dense_from && oj >= c.dense_from) continue;   // the tensor-core block has it
            int used;
            uint32_t cnt = pair_count(c, oi, oj, td, lane, used);
            cnt = warp_sum_u32(cnt);
            if (lane == 0) {
                const uint32_t ri = c.order[oi], rj = c.order[oj];
                const uint32_t lo = min(ri, rj), hi = max(ri, rj);
                if (out) out[tri_index(c.n, lo, hi)] = cnt;
                if (used >= 0) {
                    my_sum += cnt;
                    ++my_pairs;
                    ++my_cells[used];
                    if (used == P_EMPTY) ++my_skip;
                }
            }
        }
        if (!use_queue) item += gridDim.x;
    }
    if (lane == 0) {
        atomicAdd(&s_sum, my_sum);
        atomicAdd(&s_skip, my_skip);
        atomicAdd(&s_pairs, my_pairs);
        for (int k = 0; k <= STORM_PAIRING_COUNT; ++k)
            if (my_cells[k]) atomicAdd(&s_cells[k], (unsigned long long)my_cells[k]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&st->sum, s_sum);
        atomicAdd(&st->skipped, s_skip);
        atomicAdd(&st->pairs, s_pairs);
    }
    if (threadIdx.x < STORM_PAIRING_COUNT + 1 && s_cells[threadIdx.x])
        atomicAdd(&st->cell_pairs[threadIdx.x], s_cells[threadIdx.x]);
}

// One cell on one ordered pair (tests / selector labels).
__global__ void one_cell_kernel(RowsView v, int p, uint32_t a, uint32_t b, unsigned long long* out) {
    const int lane = threadIdx.x & 31;
    uint32_t c = 0;
    switch (p) {
        case P_BB: c = cell_bb(v, a, b, lane, true); break;
        case P_BS: c = cell_bs(v, a, b, lane); break;
        case P_BR: c = cell_br(v, a, b, lane); break;
        case P_BW: c = cell_bw(v, a, b, lane); break;
        case P_SS: c = cell_ss(v, a, b, lane); break;
        case P_SR: c = cell_sr(v, a, b, lane); break;
        case P_SW: c = cell_sw(v, a, b, lane); break;
        case P_RR: c = cell_rr(v, a, b, lane); break;
        case P_RW: c = cell_rw(v, a, b, lane); break;
        case P_WW: c = cell_ww(v, a, b, lane); break;
        case P_CB: c = cell_cb(v, a, b, lane); break;
        default: break;
    }
    c = warp_sum_u32(c);
    if (lane == 0) *out = c;
}

}  // namespace sb200

// ============================================================== handle
using namespace sb200;

struct STORM_rows_s {
    uint32_t universe = 0;
    std::vector<uint32_t> vals;
    std::vector<uint64_t> offs{0};
    uint64_t bitmap_budget = 0;
    bool dirty = true;
    RowsDev dev;
    cudaStream_t stream = nullptr;
    DevBuf<uint32_t> d_order, d_het, d_out, d_tile_list;
    DevBuf<RowMetaD> d_bmeta;
    DevBuf<uint64_t> d_bzone;
    DevBuf<TileDecision> d_dec;
    DevBuf<RowsStatsDev> d_stats;
    // tensor-core dense block
    double dense_min_density = 1.0 / 16384.0;
    uint32_t tuned_tile = 0;      // STORM_rows_autotune's tile (used for calls with tile 0)
    uint32_t trained_tile = 0;    // the tile the learned selector was trained on
    DevBuf<uint64_t> d_dense;
    DevBuf<uint32_t> d_dmap;
    DevBuf<uint2> d_dtiles;
    uint64_t dtiles_n = ~0ull;
    uint32_t n_dtiles = 0;
    DevBuf<DeviceFlags> d_dflags;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // cost model of the cost-model policies and of the untrained learned
    // selector: the reference's defaults until calibrated on this GPU
    CostModelD model = default_cost_model();
    bool calibrated = false;
    double last_training[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    // learned selector
    Mlp mlp;
    // CUDA graph of the batched form, keyed by the call's shape
    cudaGraphExec_t graph = nullptr;
    std::vector<uint64_t> graph_key;
    ~STORM_rows_s() {
        if (graph) cudaGraphExecDestroy(graph);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace sb200 {

static cudaStream_t rows_stream(STORM_rows_t* r) {
    require_device();
    if (!r->stream) SB_CUDA(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
    for (auto& e : r->ev)
        if (!e) SB_CUDA(cudaEventCreate(&e));
    return r->stream;
}

void rows_ensure_uploaded(STORM_rows_t* r) {
    cudaStream_t st = rows_stream(r);
    if (!r->dirty) return;
    const uint64_t n = r->offs.size() - 1;
    const uint32_t nw = (uint32_t)(((uint64_t)r->universe + 63) / 64);
    const uint64_t row_bytes = (uint64_t)((nw + 1) & ~1u) * 8;
    uint64_t budget = r->bitmap_budget;
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        SB_CUDA(cudaMemGetInfo(&fr, &tot));
        budget = fr / 4;
    }
    std::vector<uint8_t> bm_rows(n, 1);
    if (row_bytes * n > budget) {
        // densest rows first get a bitmap (they are the ones B x * serves)
        std::vector<uint64_t> ord(n);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](uint64_t a, uint64_t b) {
            return (r->offs[a + 1] - r->offs[a]) > (r->offs[b + 1] - r->offs[b]);
        });
        std::fill(bm_rows.begin(), bm_rows.end(), 0);
        const uint64_t fit = budget / row_bytes;
        for (uint64_t k = 0; k < n && k < fit; ++k) bm_rows[ord[k]] = 1;
    }
    build_rows(r->vals, r->offs, r->universe, bm_rows, r->dev, st);
    r->dirty = false;
    if (r->graph) {
        cudaGraphExecDestroy(r->graph);
        r->graph = nullptr;
    }
}

static bool sorted_order_policy(int policy) {
    return policy == STORM_POLICY_PERTILE || policy == STORM_POLICY_PROBE || policy == STORM_POLICY_ORACLE ||
           policy == STORM_POLICY_REFINE || policy == STORM_POLICY_LEARNED;
}

// density_order (storm_allpairs.cpp:316-323): stable sort by cardinality.
std::vector<uint32_t> rows_order(const STORM_rows_t* r, int policy) {
    const uint32_t n = (uint32_t)(r->offs.size() - 1);
    std::vector<uint32_t> o(n);
    std::iota(o.begin(), o.end(), 0u);
    if (sorted_order_policy(policy))
        std::stable_sort(o.begin(), o.end(), [&](uint32_t a, uint32_t b) {
            return r->dev.h_meta[a].card < r->dev.h_meta[b].card;
        });
    return o;
}

// Full all-pairs call.  out may be null (sum only).
static void rows_run(STORM_rows_t* r, int policy, uint32_t tile, int fixed_cell, int exec, uint32_t* d_out,
                     STORM_allpairs_stats* st_out) {
    if (policy < 0 || policy > STORM_POLICY_LEARNED) fail(STORM_B200_EARG, "unknown policy");
    if (policy == STORM_POLICY_FIXED && (fixed_cell < 0 || fixed_cell >= P_EMPTY))
        fail(STORM_B200_EARG, "fixed cell must be a pairing below STORM_PAIRING_EMPTY");
    rows_ensure_uploaded(r);
    cudaStream_t st = rows_stream(r);
    const uint32_t n = (uint32_t)(r->offs.size() - 1);
    const uint32_t T = tile ? tile : (r->tuned_tile ? r->tuned_tile : 64);
    STORM_allpairs_stats S{};
    if (policy == STORM_POLICY_ALLBITMAP)
        for (uint32_t i = 0; i < n; ++i)
            if (!r->dev.h_meta[i].has_bm) fail(STORM_B200_ELIMIT, "all-bitmap policy needs a bitmap for every row");
    if (n == 0) {
        if (st_out) *st_out = S;
        return;
    }
    const uint32_t nb = (n + T - 1) / T;
    if ((uint64_t)nb * (nb + 1) / 2 > 0xFFFFFFFFull)
        fail(STORM_B200_ELIMIT, "more than 2^32 tiles: use a larger tile or split the rows");
    const uint32_t ntiles = nb * (nb + 1) / 2;
    const std::vector<uint32_t> order = rows_order(r, policy);
    r->d_order.reserve(n);
    r->d_bmeta.reserve(nb);
    r->d_het.reserve(nb);
    r->d_dec.reserve(ntiles);
    r->d_stats.reserve(1);
    SB_CUDA(cudaMemcpyAsync(r->d_order.p, order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));

    PairCtx c;
    c.v = r->dev.view;
    c.order = r->d_order.p;
    c.n = n;
    c.T = T;
    c.nb = nb;
    c.policy = policy;
    c.model = r->model;
    // Dense block: the suffix of the density order whose rows all have a
    // bitmap and whose smallest sparse form (elements or run bounds) is
    // >= dense_min_density x universe; its pairs run on the tensor
    // cores (exact for universes up to 2^27 bits). A tensor-core pair costs
    // in proportion to the universe, a cell pair to the sparse sizes.
    uint32_t D = n;
    const bool sorted_pol = sorted_order_policy(policy);
    if (sorted_pol && r->dense_min_density > 0.0 && r->universe <= (1u << 27)) {
        const double min_size = r->dense_min_density * (double)r->universe;
        auto joins = [&](uint32_t row) {
            const RowMetaD& m = r->dev.h_meta[row];
            const double sparse = std::min<double>((double)m.card, 2.0 * m.runs);
            return m.has_bm && sparse >= min_size;
        };
        while (D > 0 && joins(order[D - 1])) --D;
        if (n - D < 256) D = n;
    }
    c.dense_from = D;
    const uint32_t nd = n - D;
    const uint32_t w_pad_d = (uint32_t)round_up(((uint64_t)r->universe + 63) / 64, 8);
    const uint32_t nd_pad = (uint32_t)round_up(nd ? nd : 1, 256);
    const uint64_t pitch_d = dense_pitch(w_pad_d);
    if (nd) {
        r->d_dense.reserve((uint64_t)nd_pad * pitch_d);
        r->d_dmap.reserve(nd);
        r->d_dflags.reserve(1);
        if (r->dtiles_n != nd) {
            std::vector<uint2> tl;
            build_mma_tiles(tl, nd);
            r->d_dtiles.reserve(tl.size());
            SB_CUDA(cudaMemcpyAsync(r->d_dtiles.p, tl.data(), tl.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
            SB_CUDA(cudaStreamSynchronize(st));
            r->n_dtiles = (uint32_t)tl.size();
            r->dtiles_n = nd;
        }
    }
    const bool learned = policy == STORM_POLICY_LEARNED && r->mlp.trained;
    if (learned) r->mlp.ensure_device(st);
    const bool zones = policy != STORM_POLICY_ALLBITMAP;   // tile rejection and the learned feature
    if (zones) r->d_bzone.reserve((uint64_t)nb * BZONE_WORDS);

    // slices per tile so the launch has enough CTAs
    const int sms = require_device();
    // Work items of at most 64 pairs: a tile of dense rows can cost thousands
    // of times more than a tile of sparse ones, so the queue hands out slices
    // of tiles, not whole tiles, and no CTA is left holding a heavy tile.
    const uint32_t slices = std::max<uint32_t>(1u, (T * T + 63) / 64);

    auto dense_phase = [&]() {
        if (!nd) return;
        SB_CUDA(cudaMemsetAsync(r->d_dflags.p, 0, sizeof(DeviceFlags), st));
        const uint64_t total = (uint64_t)nd_pad * pitch_d;
        const uint32_t gg = (uint32_t)std::min<uint64_t>((total + 255) / 256, (uint64_t)sms * 32);
        gather_dense_kernel<<<gg, 256, 0, st>>>(c.v, c.order, D, nd, nd_pad, pitch_d, r->d_dense.p, r->d_dmap.p);
        launch_ts_rows(r->d_dense.p, nd, w_pad_d, row_major(pitch_d), r->d_dtiles.p, r->n_dtiles, d_out,
                       r->d_dflags.p, r->d_dmap.p, n, st);
    };
    auto phases_1_2 = [&]() {
        SB_CUDA(cudaMemsetAsync(r->d_stats.p, 0, sizeof(RowsStatsDev), st));
        block_meta_kernel<<<(nb + 127) / 128, 128, 0, st>>>(c.v, c.order, n, T, r->d_bmeta.p, r->d_het.p);
        if (zones) block_zone_kernel<<<nb, 256, 0, st>>>(c.v, c.order, n, T, r->d_bzone.p);
        select_tiles_kernel<<<(ntiles + 127) / 128, 128, 0, st>>>(
            r->d_bmeta.p, r->d_het.p, zones ? r->d_bzone.p : nullptr, nb,
            learned ? policy : (policy == STORM_POLICY_LEARNED ? STORM_POLICY_PERTILE : policy), fixed_cell, c.model,
            learned ? r->mlp.d_params.p : nullptr, r->mlp.shape, r->d_dec.p);
        if (policy == STORM_POLICY_PROBE)
            probe_tiles_kernel<<<(ntiles * 32 + 127) / 128, 128, 0, st>>>(c, r->d_dec.p, ntiles);
    };

    uint32_t launches = 0;
    SB_CUDA(cudaEventRecord(r->ev[0], st));
    if (exec == STORM_EXEC_BATCHED) {
        // Everything the captured launches bake in: the call's shape, the
        // dense block's split, every device buffer they address (a buffer
        // that grew since the capture has moved), and the selector's shape.
        auto ptr = [](const void* p) { return (uint64_t)(uintptr_t)p; };
        const std::vector<uint64_t> key = {(uint64_t)policy,
                                           T,
                                           (uint64_t)fixed_cell,
                                           ptr(d_out),
                                           n,
                                           learned ? 1ull : 0ull,
                                           D,
                                           ptr(r->d_order.p),
                                           ptr(r->d_bmeta.p),
                                           ptr(r->d_het.p),
                                           ptr(r->d_dec.p),
                                           ptr(r->d_stats.p),
                                           nd ? ptr(r->d_dense.p) : 0ull,
                                           nd ? ptr(r->d_dmap.p) : 0ull,
                                           nd ? ptr(r->d_dtiles.p) : 0ull,
                                           nd ? ptr(r->d_dflags.p) : 0ull,
                                           learned ? ptr(r->mlp.d_params.p) : 0ull,
                                           zones ? ptr(r->d_bzone.p) : 0ull,
                                           learned ? ((uint64_t)r->mlp.shape.H << 40 | (uint64_t)r->mlp.shape.F << 20 |
                                                      r->mlp.shape.C)
                                                   : 0ull};
        const bool reuse = r->graph && key == r->graph_key;
        if (!reuse) {
            if (r->graph) {
                cudaGraphExecDestroy(r->graph);
                r->graph = nullptr;
            }
            cudaGraph_t g;
            SB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            phases_1_2();
            const uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)ntiles * slices, (uint64_t)sms * 8);
            dense_phase();
            tiles_kernel<<<grid, TK_THREADS, 0, st>>>(c, r->d_dec.p, 0, ntiles, slices, 1, nullptr, d_out,
                                                      r->d_stats.p);
            SB_CUDA(cudaStreamEndCapture(st, &g));
            SB_CUDA(cudaGraphInstantiate(&r->graph, g, 0));
            cudaGraphDestroy(g);
            r->graph_key = key;
        }
        SB_CUDA(cudaGraphLaunch(r->graph, st));
        launches = 3 + (policy == STORM_POLICY_PROBE ? 1 : 0);
    } else {
        phases_1_2();
        SB_CUDA(cudaEventRecord(r->ev[1], st));
        dense_phase();
        // One launch per tile, spread over the whole GPU (one warp per pair).
        const uint32_t tile_slices =
            (uint32_t)std::min<uint64_t>(((uint64_t)T * T + TK_WARPS - 1) / TK_WARPS, (uint64_t)sms * 8);
        for (uint32_t t = 0; t < ntiles; ++t) {
            tiles_kernel<<<tile_slices, TK_THREADS, 0, st>>>(c, r->d_dec.p, t, 1, tile_slices, 0, nullptr, d_out,
                                                             r->d_stats.p);
        }
        launches = 2 + (policy == STORM_POLICY_PROBE ? 1 : 0) + ntiles;
    }
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaEventRecord(r->ev[2], st));
    DeviceFlags dflags{};
    if (nd) SB_CUDA(cudaMemcpyAsync(&dflags, r->d_dflags.p, sizeof(dflags), cudaMemcpyDeviceToHost, st));
    RowsStatsDev hs;
    SB_CUDA(cudaMemcpyAsync(&hs, r->d_stats.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    float total_ms = 0.f, sel_ms = 0.f;
    SB_CUDA(cudaEventElapsedTime(&total_ms, r->ev[0], r->ev[2]));
    if (exec != STORM_EXEC_BATCHED) SB_CUDA(cudaEventElapsedTime(&sel_ms, r->ev[0], r->ev[1]));
    if (dflags.error) fail(STORM_B200_ETIMEOUT, "dense-block tensor kernel: bounded wait expired");
    hs.sum += dflags.sum;
    hs.pairs += (uint64_t)nd * (nd ? nd - 1 : 0) / 2;
    hs.cell_pairs[P_BB] += (uint64_t)nd * (nd ? nd - 1 : 0) / 2;
    S.sum = hs.sum;
    S.pairs = hs.pairs;
    S.skipped = hs.skipped;
    for (int k = 0; k <= STORM_PAIRING_COUNT; ++k) S.cell_pairs[k] = hs.cell_pairs[k];
    S.decisions = (policy == STORM_POLICY_PERPAIR || policy == STORM_POLICY_ORACLE) ? hs.pairs
                  : (policy == STORM_POLICY_ALLBITMAP || policy == STORM_POLICY_FIXED) ? 0 : ntiles;
    S.ns_total = total_ms * 1e6;
    S.ns_selection = sel_ms * 1e6;
    S.launches = launches;
    if (st_out) *st_out = S;
}

}  // namespace sb200

extern "C" {

STORM_rows_t* STORM_rows_new(uint32_t universe) {
    try {
        STORM_rows_t* r = new STORM_rows_t();
        r->universe = universe;
        return r;
    } catch (...) {
        return NULL;
    }
}

void STORM_rows_free(STORM_rows_t* r) { delete r; }

int STORM_rows_add(STORM_rows_t* r, const uint32_t* positions, uint32_t n) {
    if (r == NULL) return STORM_B200_ENULL;
    if (positions == NULL && n) return STORM_B200_EVALUES;
    return guard([&]() -> int {
        for (uint32_t i = 0; i < n; ++i) {
            if (positions[i] >= r->universe) return STORM_B200_EARG;
            if (i && positions[i] <= positions[i - 1]) return STORM_B200_EARG;
        }
        r->vals.insert(r->vals.end(), positions, positions + n);
        r->offs.push_back(r->vals.size());
        r->dirty = true;
        return (int)n;
    });
}

int STORM_rows_clear(STORM_rows_t* r) {
    if (r == NULL) return STORM_B200_ENULL;
    r->vals.clear();
    r->offs.assign(1, 0);
    r->dirty = true;
    return 1;
}

uint32_t STORM_rows_universe(const STORM_rows_t* r) { return r ? r->universe : 0; }

uint64_t STORM_rows_size(const STORM_rows_t* r) { return r ? r->offs.size() - 1 : 0; }

int STORM_rows_set_bitmap_budget(STORM_rows_t* r, uint64_t bytes) {
    if (r == NULL) return STORM_B200_ENULL;
    r->bitmap_budget = bytes;
    r->dirty = true;
    return 0;
}

int STORM_rows_set_dense_block(STORM_rows_t* r, double min_density) {
    if (r == NULL) return STORM_B200_ENULL;
    if (!(min_density >= 0.0)) return STORM_B200_EARG;
    r->dense_min_density = min_density;
    if (r->graph) {
        cudaGraphExecDestroy(r->graph);
        r->graph = nullptr;
    }
    return 0;
}

int STORM_rows_upload(STORM_rows_t* r) {
    if (r == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        rows_ensure_uploaded(r);
        return 0;
    });
}

int STORM_rows_meta(STORM_rows_t* r, uint64_t row, uint32_t* meta9) {
    if (r == NULL) return STORM_B200_ENULL;
    if (meta9 == NULL) return STORM_B200_EVALUES;
    return guard([&]() -> int {
        rows_ensure_uploaded(r);
        if (row >= r->dev.h_meta.size()) return STORM_B200_EARG;
        const RowMetaD& m = r->dev.h_meta[row];
        const uint32_t w[9] = {m.card, m.runs, m.nw, m.nnz, m.first, m.last, m.has_rank, m.has_occ,
                               (uint32_t)(m.has_bm ? 1 : 0) | (uint32_t)(m.has_comp ? 2 : 0)};
        std::copy(w, w + 9, meta9);
        return 0;
    });
}

int STORM_rows_autotune(STORM_rows_t* r, int policy, int exec, uint32_t* best_tile, double* best_min_density,
                        double* times_ms) {
    if (r == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        // Candidates: tile x dense-block threshold. A trained learned selector
        // keeps the tile it was trained on (its features are per tile).
        const uint32_t tiles[4] = {32, 64, 128, 256};
        const double dens[4] = {0.0, 1.0 / 65536, 1.0 / 16384, 1.0 / 4096};
        const bool fixed_tile = policy == STORM_POLICY_LEARNED && r->mlp.trained && r->trained_tile;
        const double keep_density = r->dense_min_density;
        double best = -1.0;
        uint32_t bt = 64;
        double bd = keep_density;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const int k = a * 4 + b;
                if (times_ms) times_ms[k] = -1.0;
                if (fixed_tile && tiles[a] != r->trained_tile) continue;
                r->dense_min_density = dens[b];
                STORM_allpairs_stats st{};
                double ms = -1.0;
                for (int rep = 0; rep < 2; ++rep) {   // first call builds the launch; keep the faster
                    rows_run(r, policy, tiles[a], STORM_PAIRING_BS, exec, nullptr, &st);
                    const double m = st.ns_total * 1e-6;
                    ms = ms < 0 ? m : std::min(ms, m);
                }
                if (times_ms) times_ms[k] = ms;
                if (best < 0 || ms < best) {
                    best = ms;
                    bt = tiles[a];
                    bd = dens[b];
                }
            }
        r->dense_min_density = bd;
        r->tuned_tile = bt;
        if (r->graph) {
            cudaGraphExecDestroy(r->graph);
            r->graph = nullptr;
        }
        if (best_tile) *best_tile = bt;
        if (best_min_density) *best_min_density = bd;
        return 0;
    });
}

int STORM_rows_allpairs_sum(STORM_rows_t* r, int policy, uint32_t tile, int fixed_cell, int exec,
                            STORM_allpairs_stats* st) {
    if (r == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        rows_run(r, policy, tile, fixed_cell, exec, nullptr, st);
        return 0;
    });
}

int STORM_rows_allpairs_matrix(STORM_rows_t* r, int policy, uint32_t tile, int fixed_cell, int exec, uint32_t* out,
                               uint64_t out_len, STORM_allpairs_stats* st) {
    if (r == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        const uint64_t n = r->offs.size() - 1, need = tri_size(n);
        if (out_len < need) return STORM_B200_ESIZE;
        if (out == NULL && need) return STORM_B200_EVALUES;
        r->d_out.reserve(need ? need : 1);
        rows_run(r, policy, tile, fixed_cell, exec, r->d_out.p, st);
        if (need) {
            SB_CUDA(cudaMemcpyAsync(out, r->d_out.p, need * sizeof(uint32_t), cudaMemcpyDeviceToHost, r->stream));
            SB_CUDA(cudaStreamSynchronize(r->stream));
        }
        return 0;
    });
}

int STORM_rows_allpairs_tiles(STORM_rows_t* r, int policy, uint32_t tile, int exec, STORM_tile_callback cb,
                              void* ctx, STORM_allpairs_stats* st) {
    if (r == NULL) return STORM_B200_ENULL;
    if (cb == NULL) return STORM_B200_EARG;
    const uint64_t n = r->offs.size() - 1;
    const uint32_t T = tile ? tile : 64;   // the callback's tile; the computation may use a tuned one
    std::vector<uint32_t> tri(tri_size(n) ? tri_size(n) : 1);
    int rc = STORM_rows_allpairs_matrix(r, policy, tile, STORM_PAIRING_BS, exec, tri.data(), tri.size(), st);
    if (rc < 0) return rc;
    return guard([&]() -> int {
        std::vector<uint32_t> buf((size_t)T * T);
        for (uint64_t i0 = 0; i0 < n; i0 += T) {
            const uint64_t i1 = std::min<uint64_t>(i0 + T, n);
            for (uint64_t j0 = i0; j0 < n; j0 += T) {
                const uint64_t j1 = std::min<uint64_t>(j0 + T, n);
                std::fill(buf.begin(), buf.end(), 0u);
                for (uint64_t i = i0; i < i1; ++i) {
                    const uint64_t base = i * n - (i * (i - 1)) / 2 - i;
                    for (uint64_t j = (j0 == i0 ? i + 1 : j0); j < j1; ++j) buf[(i - i0) * T + (j - j0)] = tri[base + j];
                }
                cb((uint32_t)i0, (uint32_t)j0, (uint32_t)(i1 - i0), (uint32_t)(j1 - j0), buf.data(), ctx);
            }
        }
        return 0;
    });
}

static RowMetaD meta_from8(const uint32_t* m) {
    RowMetaD r{};
    r.card = m[0]; r.runs = m[1]; r.nw = m[2]; r.nnz = m[3]; r.first = m[4]; r.last = m[5];
    r.has_rank = m[6] != 0; r.has_occ = m[7] != 0; r.has_bm = 1; r.has_comp = 0;
    return r;
}

int STORM_select_pairing(const uint32_t* ma, const uint32_t* mb, double* predicted) {
    if (ma == NULL || mb == NULL) return STORM_B200_EVALUES;
    const CostModelD m = default_cost_model();
    return select_pairing_d(m, meta_from8(ma), meta_from8(mb), predicted);
}

double STORM_predict(int pairing, const uint32_t* ma, const uint32_t* mb) {
    if (ma == NULL || mb == NULL || pairing < 0 || pairing > P_EMPTY) return -1.0;
    const CostModelD m = default_cost_model();
    return predict_cost(m, pairing, meta_from8(ma), meta_from8(mb));
}

int64_t STORM_rows_cell(STORM_rows_t* r, int pairing, uint64_t a, uint64_t b) {
    if (r == NULL) return STORM_B200_ENULL;
    int64_t res = 0;
    int rc = guard([&]() -> int {
        rows_ensure_uploaded(r);
        const uint64_t n = r->offs.size() - 1;
        if (a >= n || b >= n || pairing < 0 || pairing > P_CB || pairing == P_EMPTY) return STORM_B200_EARG;
        const RowMetaD& ma = r->dev.h_meta[a];
        const RowMetaD& mb = r->dev.h_meta[b];
        const bool need_a_bm = pairing == P_BB || pairing == P_BS || pairing == P_BR || pairing == P_BW;
        if ((need_a_bm && !ma.has_bm) || (pairing == P_BB && !mb.has_bm)) return STORM_B200_ELIMIT;
        if (pairing == P_CB && (!ma.has_comp || !mb.has_bm)) return STORM_B200_ELIMIT;
        cudaStream_t st = rows_stream(r);
        DevBuf<unsigned long long> d;
        d.reserve(1);
        one_cell_kernel<<<1, 32, 0, st>>>(r->dev.view, pairing, (uint32_t)a, (uint32_t)b, d.p);
        SB_CUDA(cudaGetLastError());
        unsigned long long h = 0;
        SB_CUDA(cudaMemcpyAsync(&h, d.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        res = (int64_t)h;
        return 0;
    });
    return rc < 0 ? rc : res;
}

int64_t STORM_rows_repr(STORM_rows_t* r, uint64_t row, int kind, void* out, uint64_t cap) {
    if (r == NULL) return STORM_B200_ENULL;
    int64_t res = 0;
    int rc = guard([&]() -> int {
        rows_ensure_uploaded(r);
        const uint64_t n = r->offs.size() - 1;
        if (row >= n || kind < STORM_REPR_RUN_START || kind > STORM_REPR_COMPLEMENT) return STORM_B200_EARG;
        const RowMetaD& m = r->dev.h_meta[row];
        const RowsDev& d = r->dev;
        const uint32_t nblk = (m.nw + 7) / 8;
        auto span = [&](const DevBuf<uint64_t>& off) {
            uint64_t h[2];
            SB_CUDA(cudaMemcpy(h, off.p + row, sizeof(h), cudaMemcpyDeviceToHost));
            return std::make_pair(h[0], h[1] - h[0]);
        };
        auto start = [&](const DevBuf<uint64_t>& off) {
            uint64_t h = 0;
            SB_CUDA(cudaMemcpy(&h, off.p + row, sizeof(h), cudaMemcpyDeviceToHost));
            return h;
        };
        const void* src = nullptr;
        size_t elem = 0;
        uint64_t count = 0;
        switch (kind) {
            case STORM_REPR_RUN_START:
            case STORM_REPR_RUN_END: {
                const auto s = span(d.r_off);
                src = (kind == STORM_REPR_RUN_START ? d.r_start.p : d.r_end.p) + s.first;
                elem = 4;
                count = s.second;
                break;
            }
            case STORM_REPR_EWAH: {
                const auto s = span(d.w_off);
                src = d.w_buf.p + s.first;
                elem = 8;
                count = s.second;
                break;
            }
            case STORM_REPR_MARKERS: {
                const auto s = span(d.m_off);
                src = d.m_tab.p + s.first;
                elem = 8;
                count = s.second;
                break;
            }
            case STORM_REPR_BITMAP:
                if (m.has_bm) {
                    src = d.bm.p + start(d.b_off);
                    elem = 8;
                    count = m.nw;
                }
                break;
            case STORM_REPR_RANK:
                if (m.has_rank) {
                    src = d.rk.p + start(d.rk_off);
                    elem = 8;
                    count = 2 * (uint64_t)(nblk + 1);
                }
                break;
            case STORM_REPR_OCC:
                if (m.has_occ) {
                    src = d.oc.p + start(d.oc_off);
                    elem = 8;
                    count = r->dev.view.n_occ;
                }
                break;
            default: {   // complement
                const auto s = span(d.c_off);
                src = d.c_val.p + s.first;
                elem = 4;
                count = s.second;
                break;
            }
        }
        if (out && count && cap)
            SB_CUDA(cudaMemcpy(out, src, std::min<uint64_t>(count, cap) * elem, cudaMemcpyDeviceToHost));
        res = (int64_t)count;
        return 0;
    });
    return rc < 0 ? rc : res;
}

}  // extern "C"

// ======================================================= selector training
namespace sb200 {

// Labels for the learned selector: every cell on (a sample of the pairs of)
// each sampled tile, timed with the SM clock.  One CTA per (tile, cell);
// cycles = ~0 when some pair of the tile lacks a form the cell needs.
__global__ void __launch_bounds__(TK_THREADS)
time_cells_kernel(PairCtx c, const uint32_t* __restrict__ tiles, uint32_t n_samples, uint32_t max_pairs,
                  unsigned long long* __restrict__ cycles) {
    const uint32_t sample = blockIdx.x / N_SLOTS, slot = blockIdx.x % N_SLOTS;
    const int cell = slot_cell((int)slot);
    if (sample >= n_samples) return;
    __shared__ int s_missing;
    __shared__ long long s_t0;
    __shared__ unsigned int s_sink;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t ti, tj;
    tile_decode(c.nb, tiles[sample], ti, tj);
    const uint32_t i0 = ti * c.T, i1 = min(c.n, i0 + c.T), j0 = tj * c.T, j1 = min(c.n, j0 + c.T);
    const uint32_t nr = i1 - i0, nc = j1 - j0, np = nr * nc;
    const uint32_t step = np > max_pairs ? np / max_pairs : 1;
    if (threadIdx.x == 0) {
        s_missing = 0;
        s_sink = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) s_t0 = clock64();
    __syncthreads();
    uint32_t sink = 0;
    for (uint32_t q = warp * step; q < np; q += TK_WARPS * step) {
        const uint32_t oi = i0 + q / nc, oj = j0 + q % nc;
        if (ti == tj && oj <= oi) continue;
        const uint32_t ri = c.order[oi], rj = c.order[oj];
        const RowMetaD& mi = c.v.meta[ri];
        const RowMetaD& mj = c.v.meta[rj];
        const bool idn = mi.card >= mj.card;
        const RowMetaD& md = idn ? mi : mj;
        const RowMetaD& ms = idn ? mj : mi;
        if (span_disjoint(md, ms)) continue;
        if (!cell_available(cell, md, ms)) {
            s_missing = 1;
            continue;
        }
        sink += run_cell(c.v, cell, idn ? ri : rj, idn ? rj : ri, lane, true);
    }
    sink = warp_sum_u32(sink);
    if (lane == 0) atomicAdd(&s_sink, sink);
    __syncthreads();
    if (threadIdx.x == 0) {
        const long long dt = clock64() - s_t0;
        cycles[(uint64_t)sample * N_SLOTS + slot] =
            s_missing ? ~0ull : (unsigned long long)dt + (s_sink == 0xFFFFFFFFu ? 1ull : 0ull);
    }
}

// What the cost model sees of the pairs time_cells_kernel times (the same
// pair sample of each tile): per (tile, cell) the reference default model's
// predicted cost above its fixed term, summed, and the number of pairs.
__global__ void __launch_bounds__(TK_THREADS)
cell_predict_kernel(PairCtx c, const uint32_t* __restrict__ tiles, uint32_t n_samples, uint32_t max_pairs,
                    double* __restrict__ pred, uint32_t* __restrict__ npairs) {
    const uint32_t sample = blockIdx.x / N_SLOTS, slot = blockIdx.x % N_SLOTS;
    const int cell = slot_cell((int)slot);
    if (sample >= n_samples) return;
    __shared__ double s_pred;
    __shared__ unsigned int s_np;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t ti, tj;
    tile_decode(c.nb, tiles[sample], ti, tj);
    const uint32_t i0 = ti * c.T, i1 = min(c.n, i0 + c.T), j0 = tj * c.T, j1 = min(c.n, j0 + c.T);
    const uint32_t nr = i1 - i0, nc = j1 - j0, np = nr * nc;
    const uint32_t step = np > max_pairs ? np / max_pairs : 1;
    if (threadIdx.x == 0) {
        s_pred = 0.0;
        s_np = 0;
    }
    __syncthreads();
    // the default model without the per-pair terms the fitted model drops
    // (its fixed term, and the B x S probe's cold/hot difference)
    CostModelD m = default_cost_model();
    m.ns_probe_cold = m.ns_probe_hot = 0.0;
    double acc = 0.0;
    uint32_t cnt = 0;
    if (lane == 0) {
        for (uint32_t q = warp * step; q < np; q += TK_WARPS * step) {
            const uint32_t oi = i0 + q / nc, oj = j0 + q % nc;
            if (ti == tj && oj <= oi) continue;
            const RowMetaD& mi = c.v.meta[c.order[oi]];
            const RowMetaD& mj = c.v.meta[c.order[oj]];
            if (span_disjoint(mi, mj)) continue;
            // C x B, absent from the default model, priced as a probe per complement position
            acc += cell == P_CB ? CB_UNIT_REF * cb_work(mi, mj) : predict_cost(m, cell, mi, mj) - m.ns_fixed;
            ++cnt;
        }
        atomicAdd(&s_pred, acc);
        atomicAdd(&s_np, cnt);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        pred[(uint64_t)sample * N_SLOTS + slot] = s_pred;
        npairs[(uint64_t)sample * N_SLOTS + slot] = s_np;
    }
}

// Timings of every cell on sampled tiles of r's density order, with the
// tile aggregates and the cost model's view of the same pairs.
struct TileTimings {
    uint32_t T = 64, nb = 0;
    std::vector<uint32_t> pick;                 // sampled tile indices
    std::vector<unsigned long long> cyc;        // [sample][slot] min of three, ~0 = cell unavailable
    std::vector<double> pred;                   // [sample][slot] default model, above its fixed term
    std::vector<uint32_t> npairs;               // [sample][slot]
    std::vector<RowMetaD> bmeta;
    std::vector<uint32_t> het;
    std::vector<uint64_t> bzone;                // [block][BZONE_WORDS]
    void tile_of(uint32_t k, uint32_t& ti, uint32_t& tj) const {
        uint64_t t = pick[k], i = 0;
        auto S = [this](uint64_t q) { return q * nb - q * (q - 1) / 2; };
        while (i + 1 < nb && S(i + 1) <= t) ++i;
        ti = (uint32_t)i;
        tj = (uint32_t)(t - S(i) + i);
    }
};

static TileTimings time_tiles(STORM_rows_t* r, uint32_t T, uint32_t samples, uint64_t seed) {
    rows_ensure_uploaded(r);
    cudaStream_t st = rows_stream(r);
    const uint32_t n = (uint32_t)(r->offs.size() - 1);
    if (n < 2) fail(STORM_B200_EARG, "fewer than two rows");
    TileTimings tt;
    tt.T = T;
    const uint32_t nb = (n + T - 1) / T;
    tt.nb = nb;
    if ((uint64_t)nb * (nb + 1) / 2 > 0xFFFFFFFFull) fail(STORM_B200_ELIMIT, "more than 2^32 tiles");
    const uint32_t ntiles = nb * (nb + 1) / 2;
    const std::vector<uint32_t> order = rows_order(r, STORM_POLICY_PERTILE);
    r->d_order.reserve(n);
    r->d_bmeta.reserve(nb);
    r->d_het.reserve(nb);
    r->d_bzone.reserve((size_t)nb * BZONE_WORDS);
    SB_CUDA(cudaMemcpyAsync(r->d_order.p, order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    PairCtx c;
    c.v = r->dev.view;
    c.order = r->d_order.p;
    c.n = n;
    c.T = T;
    c.nb = nb;
    c.policy = STORM_POLICY_PERTILE;
    c.model = r->model;
    block_meta_kernel<<<(nb + 127) / 128, 128, 0, st>>>(c.v, c.order, n, T, r->d_bmeta.p, r->d_het.p);
    block_zone_kernel<<<nb, 256, 0, st>>>(c.v, c.order, n, T, r->d_bzone.p);
    SB_CUDA(cudaGetLastError());
    tt.bmeta.resize(nb);
    tt.het.resize(nb);
    tt.bzone.resize((size_t)nb * BZONE_WORDS);
    SB_CUDA(cudaMemcpyAsync(tt.bmeta.data(), r->d_bmeta.p, nb * sizeof(RowMetaD), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(tt.het.data(), r->d_het.p, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(tt.bzone.data(), r->d_bzone.p, tt.bzone.size() * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, st));
    // sample tiles (all of them when there are few)
    uint64_t s = seed ? seed : 0x5E1EC7;
    auto rnd = [&s]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    if (samples == 0 || samples >= ntiles) {
        tt.pick.resize(ntiles);
        std::iota(tt.pick.begin(), tt.pick.end(), 0u);
    } else {
        std::vector<uint32_t> all(ntiles);
        std::iota(all.begin(), all.end(), 0u);
        for (uint32_t k = 0; k < samples; ++k) std::swap(all[k], all[k + rnd() % (ntiles - k)]);
        tt.pick.assign(all.begin(), all.begin() + samples);
    }
    const uint32_t ns = (uint32_t)tt.pick.size();
    DevBuf<uint32_t> dpick, dnp;
    DevBuf<unsigned long long> dcyc;
    DevBuf<double> dpred;
    dpick.reserve(ns);
    dcyc.reserve((size_t)ns * N_SLOTS);
    dpred.reserve((size_t)ns * N_SLOTS);
    dnp.reserve((size_t)ns * N_SLOTS);
    SB_CUDA(cudaMemcpyAsync(dpick.p, tt.pick.data(), ns * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    tt.cyc.assign((size_t)ns * N_SLOTS, ~0ull);
    std::vector<unsigned long long> tmp((size_t)ns * N_SLOTS);
    for (int rep = 0; rep < 3; ++rep) {   // min of three timings per (tile, cell)
        time_cells_kernel<<<ns * N_SLOTS, TK_THREADS, 0, st>>>(c, dpick.p, ns, 256, dcyc.p);
        SB_CUDA(cudaGetLastError());
        SB_CUDA(cudaMemcpyAsync(tmp.data(), dcyc.p, tmp.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                st));
        SB_CUDA(cudaStreamSynchronize(st));
        for (size_t k = 0; k < tt.cyc.size(); ++k) tt.cyc[k] = std::min(tt.cyc[k], tmp[k]);
    }
    cell_predict_kernel<<<ns * N_SLOTS, TK_THREADS, 0, st>>>(c, dpick.p, ns, 256, dpred.p, dnp.p);
    SB_CUDA(cudaGetLastError());
    tt.pred.resize((size_t)ns * N_SLOTS);
    tt.npairs.resize((size_t)ns * N_SLOTS);
    SB_CUDA(cudaMemcpyAsync(tt.pred.data(), dpred.p, tt.pred.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(tt.npairs.data(), dnp.p, tt.npairs.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            st));
    SB_CUDA(cudaStreamSynchronize(st));
    return tt;
}

// The reference's calibration (calibrate / calibrate_on_rows,
// storm_cost.cpp:556-769, 779-895) fits, per cell, time / work on pairs it
// times, plus a per-pair fixed term; here the timings are this GPU's, of the
// container's own sampled tiles (time_cells_kernel), and the model keeps the
// reference's work formulas: per cell slot, cycles(tile) ~ a x (the default
// model's prediction above its fixed term) + f x pairs, a weighted
// least-squares fit (relative error) of both, because each warp-cooperative
// cell has its own per-pair overhead on the GPU.  Returns the fitted model
// in SM cycles (the selector compares predictions, so the unit is free) and
// the fit's relative RMS error.
static CostModelD fit_cost_model(const TileTimings& tt, const std::vector<uint32_t>& use, double* rms_out) {
    double a[N_SLOTS], f[N_SLOTS];
    bool fitted[N_SLOTS];
    for (int cl = 0; cl < N_SLOTS; ++cl) {
        double sxx = 0, sxp = 0, spp = 0, sxy = 0, spy = 0, sy = 0, sx = 0;
        int cnt = 0;
        for (uint32_t k : use) {
            const size_t e = (size_t)k * N_SLOTS + cl;
            if (tt.cyc[e] == ~0ull || tt.npairs[e] == 0 || tt.pred[e] <= 0.0) continue;
            const double y = (double)tt.cyc[e], w = 1.0 / (y * y);
            const double x = tt.pred[e], q = (double)tt.npairs[e];
            sxx += w * x * x;
            sxp += w * x * q;
            spp += w * q * q;
            sxy += w * x * y;
            spy += w * q * y;
            sy += y;
            sx += x;
            ++cnt;
        }
        fitted[cl] = cnt > 0;
        a[cl] = f[cl] = 0.0;
        if (!cnt) continue;
        // The least-squares optimum under a > 0, f >= 0: the free optimum if
        // it is inside, else the best point on the boundary -- f = 0 (time
        // in proportion to work) or a at a floor (time per pair).
        const double a_only = sxx > 0 ? sxy / sxx : 0.0;
        const double det = sxx * spp - sxp * sxp;
        bool inside = false;
        if (cnt >= 3 && det > 1e-12 * sxx * spp) {
            a[cl] = (sxy * spp - spy * sxp) / det;
            f[cl] = (sxx * spy - sxp * sxy) / det;
            inside = a[cl] > 0.0 && f[cl] >= 0.0;
        }
        if (!inside) {
            auto err = [&](double aa, double ff) {   // sum of squared relative errors
                double e2 = 0;
                for (uint32_t k : use) {
                    const size_t e = (size_t)k * N_SLOTS + cl;
                    if (tt.cyc[e] == ~0ull || tt.npairs[e] == 0 || tt.pred[e] <= 0.0) continue;
                    const double y = (double)tt.cyc[e];
                    const double r = (aa * tt.pred[e] + ff * (double)tt.npairs[e] - y) / y;
                    e2 += r * r;
                }
                return e2;
            };
            const double a_floor = 1e-6 * (a_only > 0 ? a_only : (sx > 0 ? sy / sx : 1.0));
            const double f_only = spp > 0 ? std::max(0.0, (spy - a_floor * sxp) / spp) : 0.0;
            if (a_only > 0 && err(a_only, 0.0) <= err(a_floor, f_only)) {
                a[cl] = a_only;
                f[cl] = 0.0;
            } else {
                a[cl] = a_floor;
                f[cl] = f_only;
            }
        }
    }
    // reference cells with no sample take the mean scale of the others;
    // C x B stays unpriced (never chosen) without one
    double mean = 0;
    int nf = 0;
    for (int cl = 0; cl < P_EMPTY; ++cl)
        if (fitted[cl] && a[cl] > 0) {
            mean += a[cl];
            ++nf;
        }
    mean = nf ? mean / nf : 1.0;
    const CostModelD d = default_cost_model();
    CostModelD m = d;
    m.ns_fixed = 0.0;
    for (int cl = 0; cl < P_EMPTY; ++cl) {
        if (!fitted[cl] || !(a[cl] > 0)) {
            a[cl] = mean;
            f[cl] = 0.0;
        }
        m.ns_per_unit[cl] = a[cl] * d.ns_per_unit[cl];
        m.ns_fixed_cell[cl] = f[cl];
    }
    const bool cb = fitted[P_EMPTY] && a[P_EMPTY] > 0;
    m.ns_per_unit_cb = cb ? a[P_EMPTY] * CB_UNIT_REF : 0.0;
    m.ns_fixed_cell[P_CB] = cb ? f[P_EMPTY] : 0.0;
    m.ns_per_occ_word = a[P_BB] * d.ns_per_occ_word;
    m.ns_probe_hot = m.ns_probe_cold = 0.0;
    double se = 0;
    size_t cnt = 0;
    for (uint32_t k : use)
        for (int cl = 0; cl < N_SLOTS; ++cl) {
            const size_t e = (size_t)k * N_SLOTS + cl;
            if (tt.cyc[e] == ~0ull || tt.npairs[e] == 0 || tt.pred[e] <= 0.0) continue;
            const double y = (double)tt.cyc[e];
            const double p = a[cl] * tt.pred[e] + f[cl] * tt.npairs[e];
            se += (p - y) * (p - y) / (y * y);
            ++cnt;
        }
    if (rms_out) *rms_out = cnt ? std::sqrt(se / cnt) : 0.0;
    return m;
}

static void drop_graph(STORM_rows_t* r) {
    if (r->graph) {
        cudaGraphExecDestroy(r->graph);
        r->graph = nullptr;
    }
}

}  // namespace sb200

extern "C" {

int STORM_rows_calibrate(STORM_rows_t* r, uint32_t tile, uint32_t samples, uint64_t seed, double* model_out) {
    if (r == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        const TileTimings tt = time_tiles(r, tile ? tile : 64, samples, seed);
        std::vector<uint32_t> use(tt.pick.size());
        std::iota(use.begin(), use.end(), 0u);
        double rms = 0;
        r->model = fit_cost_model(tt, use, &rms);
        r->calibrated = true;
        drop_graph(r);
        if (model_out) {
            for (int cl = 0; cl < P_COUNT; ++cl) model_out[cl] = r->model.ns_per_unit[cl];
            model_out[P_COUNT] = r->model.ns_fixed;
            model_out[P_COUNT + 1] = r->model.ns_per_occ_word;
            model_out[P_COUNT + 2] = r->model.ns_per_unit_cb;
            for (int p = 0; p <= P_CB; ++p) model_out[P_COUNT + 3 + p] = r->model.ns_fixed_cell[p];
            model_out[P_COUNT + 3 + P_CB + 1] = rms;
        }
        return 0;
    });
}

int STORM_rows_cost_model(STORM_rows_t* r, double* model, int set) {
    if (r == NULL) return STORM_B200_ENULL;
    if (set) {
        if (model == NULL) {
            r->model = default_cost_model();
            r->calibrated = false;
        } else {
            for (int cl = 0; cl < P_COUNT; ++cl) r->model.ns_per_unit[cl] = model[cl];
            r->model.ns_fixed = model[P_COUNT];
            r->model.ns_per_occ_word = model[P_COUNT + 1];
            r->model.ns_per_unit_cb = model[P_COUNT + 2];
            for (int p = 0; p <= P_CB; ++p) r->model.ns_fixed_cell[p] = model[P_COUNT + 3 + p];
            r->model.ns_probe_hot = r->model.ns_probe_cold = 0.0;
            r->calibrated = true;
        }
        drop_graph(r);
        return 0;
    }
    if (model == NULL) return STORM_B200_EVALUES;
    for (int cl = 0; cl < P_COUNT; ++cl) model[cl] = r->model.ns_per_unit[cl];
    model[P_COUNT] = r->model.ns_fixed;
    model[P_COUNT + 1] = r->model.ns_per_occ_word;
    model[P_COUNT + 2] = r->model.ns_per_unit_cb;
    for (int p = 0; p <= P_CB; ++p) model[P_COUNT + 3 + p] = r->model.ns_fixed_cell[p];
    return r->calibrated ? 1 : 0;
}

int STORM_rows_train_selector(STORM_rows_t* r, uint32_t tile, uint32_t samples, uint32_t epochs, uint64_t seed,
                              double* stats) {
    if (r == NULL) return STORM_B200_ENULL;
    return guard([&]() -> int {
        const uint32_t T = tile ? tile : 64;
        const TileTimings tt = time_tiles(r, T, samples, seed);
        r->trained_tile = T;
        const uint32_t ns = (uint32_t)tt.pick.size();
        // features, labels
        const MlpShape sh = r->mlp.shape;
        std::vector<float> X;
        std::vector<int32_t> Y;
        std::vector<uint32_t> idx;
        for (uint32_t k = 0; k < ns; ++k) {
            uint32_t best = N_SLOTS;
            unsigned long long bc = ~0ull;
            for (uint32_t cl = 0; cl < (uint32_t)N_SLOTS; ++cl)
                if (tt.cyc[(size_t)k * N_SLOTS + cl] < bc) {
                    bc = tt.cyc[(size_t)k * N_SLOTS + cl];
                    best = cl;
                }
            if (best == (uint32_t)N_SLOTS) continue;
            uint32_t ti, tj;
            tt.tile_of(k, ti, tj);
            float x[MLP_MAX_F];
            tile_features(tt.bmeta[ti], tt.bmeta[tj], tt.het[ti], tt.het[tj],
                          zone_overlap(tt.bzone.data() + (size_t)ti * BZONE_WORDS,
                                       tt.bzone.data() + (size_t)tj * BZONE_WORDS),
                          x);
            X.insert(X.end(), x, x + sh.F);
            Y.push_back((int32_t)best);
            idx.push_back(k);
        }
        const uint32_t nl = (uint32_t)Y.size();
        if (nl < 4) return STORM_B200_EARG;
        // 80 / 20 split, deterministic by sample position
        std::vector<float> Xtr, Xte;
        std::vector<int32_t> Ytr, Yte;
        std::vector<uint32_t> tr_idx, te_idx;
        for (uint32_t k = 0; k < nl; ++k) {
            const bool test = (k % 5) == 4;
            (test ? Xte : Xtr).insert((test ? Xte : Xtr).end(), X.begin() + (size_t)k * sh.F,
                                      X.begin() + (size_t)(k + 1) * sh.F);
            (test ? Yte : Ytr).push_back(Y[k]);
            (test ? te_idx : tr_idx).push_back(idx[k]);
        }
        // Regret of a cost model on a set of sampled tiles: the measured
        // cycles of the cell it picks (from the tile's block meta, as the
        // per-tile policy does), summed, over the sum of the best cell's - 1.
        auto model_regret = [&](const CostModelD& mm, const std::vector<uint32_t>& tiles) {
            double best_sum = 0, got_sum = 0;
            for (uint32_t k : tiles) {
                uint32_t ti, tj;
                tt.tile_of(k, ti, tj);
                const unsigned long long* cy = tt.cyc.data() + (size_t)k * N_SLOTS;
                int y = 0;
                for (int cl = 1; cl < N_SLOTS; ++cl)
                    if (cy[cl] < cy[y]) y = cl;
                const RowMetaD& a = tt.bmeta[ti];
                const RowMetaD& b = tt.bmeta[tj];
                int cl = select_pairing_d(mm, a, b, nullptr);
                if (cl == P_EMPTY) cl = (a.has_bm && b.has_bm) ? P_BB : P_SS;
                const int sl = cl == P_CB ? P_EMPTY : cl;
                best_sum += (double)cy[y];
                got_sum += cy[sl] == ~0ull ? (double)cy[y] * 4.0 : (double)cy[sl];
            }
            return best_sum > 0 ? got_sum / best_sum - 1.0 : 0.0;
        };
        // The cost model calibrated on the training tiles' timings, or the
        // reference's default model where that picks better cells on the
        // same tiles, becomes this container's model: the fallback of the
        // learned policy and the model of the cost-model policies.
        double rms = 0;
        const CostModelD fitted = fit_cost_model(tt, tr_idx, &rms);
        const bool keep_fit = model_regret(fitted, tr_idx) <= model_regret(default_cost_model(), tr_idx);
        r->model = keep_fit ? fitted : default_cost_model();
        r->calibrated = keep_fit;
        mlp_init(r->mlp, seed ^ 0xA5A5A5A5ull);
        r->mlp.dirty = true;
        const float loss = mlp_train(r->mlp, Xtr, Ytr, epochs ? epochs : 400, rows_stream(r));
        r->mlp.trained = true;
        // accuracy on the training split
        uint32_t correct = 0;
        for (size_t k = 0; k < Ytr.size(); ++k) {
            float h[MLP_MAX_H], lg[MLP_MAX_C];
            mlp_forward(r->mlp.params.data(), sh, Xtr.data() + k * sh.F, h, lg);
            uint32_t am = 0;
            for (uint32_t cl = 1; cl < sh.C; ++cl)
                if (lg[cl] > lg[am]) am = cl;
            correct += (am == (uint32_t)Ytr[k]);
        }
        // regret on the held-out tiles: sum of chosen cycles / sum of best - 1,
        // for the MLP, the calibrated model and the reference's default model
        const CostModelD dflt = default_cost_model();
        double best_sum = 0, mlp_sum = 0, cal_sum = 0, def_sum = 0;
        for (size_t q = 0; q < te_idx.size(); ++q) {
            const uint32_t k = te_idx[q];
            uint32_t ti, tj;
            tt.tile_of(k, ti, tj);
            const unsigned long long* cy = tt.cyc.data() + (size_t)k * N_SLOTS;
            const int y = Yte[q];
            const RowMetaD& a = tt.bmeta[ti];
            const RowMetaD& b = tt.bmeta[tj];
            const int m_cell = mlp_argmax_available(r->mlp.params.data(), sh, Xte.data() + q * sh.F, a, b);
            auto model_cell = [&](const CostModelD& mm) {
                int cl = select_pairing_d(mm, a, b, nullptr);
                if (cl == P_EMPTY) cl = (a.has_bm && b.has_bm) ? P_BB : P_SS;
                return cl;
            };
            auto cost = [&](int cl) {   // a cell's timed slot (C x B is the last)
                const int sl = cl == P_CB ? P_EMPTY : cl;
                return cy[sl] == ~0ull ? (double)cy[y] * 4.0 : (double)cy[sl];
            };
            best_sum += (double)cy[y];
            mlp_sum += cost(m_cell);
            cal_sum += cost(model_cell(fitted));
            def_sum += cost(model_cell(dflt));
        }
        const double reg_mlp = best_sum > 0 ? mlp_sum / best_sum - 1.0 : 0.0;
        const double reg_cal = best_sum > 0 ? cal_sum / best_sum - 1.0 : 0.0;
        const double reg_def = best_sum > 0 ? def_sum / best_sum - 1.0 : 0.0;
        if (stats) {
            stats[0] = ns;
            stats[1] = epochs ? epochs : 400;
            stats[2] = loss;
            stats[3] = Ytr.empty() ? 0.0 : (double)correct / Ytr.size();
            stats[4] = reg_mlp;
            stats[5] = reg_cal;
        }
        double fixed_mean = 0.0;
        for (int cl = 0; cl < P_EMPTY; ++cl) fixed_mean += r->model.ns_fixed_cell[cl] / P_EMPTY;
        const double rep[9] = {reg_mlp, reg_cal, reg_def, (double)te_idx.size(), (double)tr_idx.size(), rms,
                               r->model.ns_fixed + fixed_mean, (double)ns, keep_fit ? 1.0 : 0.0};
        std::copy(rep, rep + 9, r->last_training);
        drop_graph(r);
        return 0;
    });
}

int STORM_rows_last_training(const STORM_rows_t* r, double* out9) {
    if (r == NULL) return STORM_B200_ENULL;
    if (out9 == NULL) return STORM_B200_EVALUES;
    std::copy(r->last_training, r->last_training + 9, out9);
    return 0;
}

int STORM_rows_reset_selector(STORM_rows_t* r) {
    if (r == NULL) return STORM_B200_ENULL;
    r->mlp.trained = false;
    if (r->graph) {
        cudaGraphExecDestroy(r->graph);
        r->graph = nullptr;
    }
    return 0;
}

int64_t STORM_rows_selector_params(STORM_rows_t* r, float* params, uint64_t n_params, int load) {
    if (r == NULL) return STORM_B200_ENULL;
    const uint64_t np = r->mlp.shape.n_params();
    if (params == NULL) return (int64_t)np;
    if (n_params < np) return STORM_B200_ESIZE;
    if (load) {
        r->mlp.params.assign(params, params + np);
        r->mlp.trained = true;
        r->mlp.dirty = true;
        if (r->graph) {
            cudaGraphExecDestroy(r->graph);
            r->graph = nullptr;
        }
    } else {
        if (r->mlp.params.size() != np) return STORM_B200_EARG;
        std::copy(r->mlp.params.begin(), r->mlp.params.end(), params);
    }
    return (int64_t)np;
}

}  // extern "C"
