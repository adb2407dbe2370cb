// mlp.cuh -- the learned cell selector: a two-layer MLP over tile features.
//
//   x (16 tile features) -> h = relu(W1 x + b1) (32) -> logits = W2 h + b2 (11 cell slots:
//   the reference's ten cells and C x B)
//
// The features are the tile aggregates the cost model reads (storm_cost.cpp:
// work_units inputs: cardinality, runs, non-zero words, universe words, the
// index flags) on a log scale, plus what the cost model cannot see: the span
// overlap of the two row blocks, their cardinality spread (max / mean) and
// the overlap of their zone maps.
// Inference runs inside the tile-selection kernel (one thread per tile) and
// takes the best-scoring cell among those whose representations exist.
// Training (mlp.cu) uses device forward/backward kernels and labels timed on
// this GPU.
#pragma once
#include <vector>
#include "common.cuh"
#include "rows_cost.cuh"

namespace sb200 {

constexpr int MLP_MAX_F = 16;
constexpr int MLP_MAX_H = 64;
constexpr int MLP_MAX_C = 16;

struct MlpShape {
    uint32_t F = 16, H = 32, C = 11;   // C: cell slots (slot_cell)
    __host__ __device__ uint32_t n_params() const { return H * F + H + C * H + C; }
};

// Parameter layout: W1 [H x F] row-major, b1 [H], W2 [C x H], b2 [C].
struct Mlp {
    MlpShape shape;
    std::vector<float> params;
    DevBuf<float> d_params;
    bool trained = false;
    bool dirty = true;
    void ensure_device(cudaStream_t st) {
        if (!dirty && d_params.p) return;
        d_params.reserve(params.size() ? params.size() : 1);
        if (!params.empty())
            SB_CUDA(cudaMemcpyAsync(d_params.p, params.data(), params.size() * sizeof(float), cudaMemcpyHostToDevice, st));
        dirty = false;
    }
};

__host__ __device__ inline float flog2(double v) {
#ifdef __CUDA_ARCH__
    return (float)log2(v);
#else
    return (float)std::log2(v);
#endif
}

// Zone map of a row block: BZONE_WORDS x 64 coarse bins over the universe,
// a bin set when some row of the block holds a value in it (the OR of the
// rows' zone maps, storm_repr.cpp:47-59, at a coarser grain).
constexpr uint32_t BZONE_WORDS = 64;

// Overlap of two block zone maps: bins both hold / bins either holds (the
// zone-map test the reference's B x B plans from, cell_bb.cpp:522-550).
__host__ __device__ inline float zone_overlap(const uint64_t* za, const uint64_t* zb) {
    uint32_t both = 0, any = 0;
    for (uint32_t k = 0; k < BZONE_WORDS; ++k) {
#ifdef __CUDA_ARCH__
        both += __popcll(za[k] & zb[k]);
        any += __popcll(za[k] | zb[k]);
#else
        both += (uint32_t)__builtin_popcountll(za[k] & zb[k]);
        any += (uint32_t)__builtin_popcountll(za[k] | zb[k]);
#endif
    }
    return any ? (float)both / (float)any : 0.0f;
}

// 16 features of a tile pair from the two row blocks' aggregate metadata
// and the overlap of their zone maps.
__host__ __device__ inline void tile_features(const RowMetaD& a, const RowMetaD& b, uint32_t het_a_x1000,
                                              uint32_t het_b_x1000, float zone, float* x) {
    const float s = 1.0f / 32.0f;
    x[0] = flog2(1.0 + a.card) * s;
    x[1] = flog2(1.0 + b.card) * s;
    x[2] = flog2(1.0 + a.runs) * s;
    x[3] = flog2(1.0 + b.runs) * s;
    x[4] = flog2(1.0 + a.nnz) * s;
    x[5] = flog2(1.0 + b.nnz) * s;
    x[6] = flog2(1.0 + (a.nw > b.nw ? a.nw : b.nw)) * s;
    x[7] = (flog2(1.0 + a.card) - flog2(1.0 + a.runs)) * s * 4.0f;   // log mean run length
    x[8] = (flog2(1.0 + b.card) - flog2(1.0 + b.runs)) * s * 4.0f;
    x[9] = (a.has_occ && b.has_occ) ? 1.0f : 0.0f;
    x[10] = (a.has_rank || b.has_rank) ? 1.0f : 0.0f;
    x[11] = (a.has_bm && b.has_bm) ? 1.0f : 0.0f;
    const double lo = a.first > b.first ? a.first : b.first, hi = a.last < b.last ? a.last : b.last;
    const double span = (double)(a.nw > b.nw ? a.nw : b.nw) * 64.0;
    x[12] = (hi > lo && span > 0) ? (float)((hi - lo) / span) : 0.0f;
    x[13] = flog2(het_a_x1000 / 1000.0 + 1e-3) * 0.25f;
    x[14] = flog2(het_b_x1000 / 1000.0 + 1e-3) * 0.25f;
    x[15] = zone;
}

__host__ __device__ inline void mlp_forward(const float* p, const MlpShape& sh, const float* x, float* h,
                                            float* logits) {
    const float* W1 = p;
    const float* b1 = W1 + sh.H * sh.F;
    const float* W2 = b1 + sh.H;
    const float* b2 = W2 + sh.C * sh.H;
    for (uint32_t j = 0; j < sh.H; ++j) {
        float acc = b1[j];
        for (uint32_t f = 0; f < sh.F; ++f) acc += W1[j * sh.F + f] * x[f];
        h[j] = acc > 0.f ? acc : 0.f;
    }
    for (uint32_t c = 0; c < sh.C; ++c) {
        float acc = b2[c];
        for (uint32_t j = 0; j < sh.H; ++j) acc += W2[c * sh.H + j] * h[j];
        logits[c] = acc;
    }
}

void mlp_init(Mlp& m, uint64_t seed);
float mlp_train(Mlp& m, const std::vector<float>& X, const std::vector<int32_t>& Y, uint32_t epochs,
                cudaStream_t st);

// Best-scoring cell whose representations exist on the tile (tile metas are
// AND-ed over rows, so has_bm means every row has a bitmap).
__host__ __device__ inline int mlp_argmax_available(const float* p, const MlpShape& sh, const float* x,
                                                    const RowMetaD& a, const RowMetaD& b) {
    float h[MLP_MAX_H], lg[MLP_MAX_C];
    mlp_forward(p, sh, x, h, lg);
    const bool a_dense = a.card >= b.card;
    const RowMetaD& d = a_dense ? a : b;
    const RowMetaD& s = a_dense ? b : a;
    int best = P_SS;
    float bs = -3.0e38f;
    for (uint32_t c = 0; c < sh.C && c < (uint32_t)N_SLOTS; ++c) {
        if (!cell_available(slot_cell((int)c), d, s)) continue;
        if (lg[c] > bs) {
            bs = lg[c];
            best = slot_cell((int)c);
        }
    }
    return best;
}

}  // namespace sb200
