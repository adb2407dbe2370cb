/*
 * storm_rows.h -- the reference's kernel layer (kernels/storm_allpairs.h,
 * storm_cost.h, storm_repr.h) behind a C ABI, on the GPU.
 *
 * A STORM_rows_t holds rows of one universe, each given as sorted distinct
 * positions (storm::build_row's contract, storm_repr.h:280-291).  Every row is
 * kept in HBM in the reference's representations -- sorted list (S), maximal
 * runs (R), EWAH-64 (W), and where memory allows bitmap (B, with the rank9
 * index and the zone map under the reference's own gates, storm_repr.cpp:186-
 * 189) and complement (C, density > 1/2).  The all-pairs calls traverse the
 * upper triangle in tiles exactly like storm::allpairs_sum / allpairs_tiles
 * (storm_allpairs.cpp:486-732): optional density order, a cell chosen per
 * pair or per tile by a policy, the O(1) span test per pair, and a cell
 * kernel per pair.  Counts do not depend on the policy; only the time does.
 *
 * Extra policies beyond the reference's:
 *   STORM_POLICY_LEARNED   a small MLP over tile features picks the cell; it
 *                          is trained on this GPU's own cell timings
 *                          (STORM_rows_train_selector) and falls back to the
 *                          cost model when untrained.
 * Execution forms:
 *   STORM_EXEC_PER_TILE    one kernel launch per tile (the plain GPU form)
 *   STORM_EXEC_BATCHED     every tile in one persistent work-queue launch,
 *                          captured in a CUDA graph and replayed
 */
#ifndef STORM_B200_ROWS_H_
#define STORM_B200_ROWS_H_

#include <stdint.h>
#include <stddef.h>
#include "storm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct STORM_rows_s STORM_rows_t;

/* storm::Policy (storm_allpairs.h:42-123), plus LEARNED. */
#define STORM_POLICY_ALLBITMAP 0
#define STORM_POLICY_PERPAIR   1
#define STORM_POLICY_PERTILE   2
#define STORM_POLICY_ORACLE    3
#define STORM_POLICY_FIXED     4
#define STORM_POLICY_PROBE     5
#define STORM_POLICY_REFINE    6
#define STORM_POLICY_LEARNED   7

/* storm::Pairing (storm_cost.h:47-49). */
#define STORM_PAIRING_BB 0
#define STORM_PAIRING_BS 1
#define STORM_PAIRING_BR 2
#define STORM_PAIRING_BW 3
#define STORM_PAIRING_SS 4
#define STORM_PAIRING_SR 5
#define STORM_PAIRING_SW 6
#define STORM_PAIRING_RR 7
#define STORM_PAIRING_RW 8
#define STORM_PAIRING_WW 9
#define STORM_PAIRING_EMPTY 10
#define STORM_PAIRING_COUNT 11
/* Complemented pairing (kernels/cell_comp.cpp): |A & B| = |B| - |A' & B|. */
#define STORM_PAIRING_CB 11

#define STORM_EXEC_PER_TILE 0
#define STORM_EXEC_BATCHED  1

/* storm::AllPairsStats (storm_allpairs.h:127-144). ns_* are device times. */
typedef struct {
    uint64_t sum;
    uint64_t pairs;
    uint64_t decisions;
    uint64_t skipped;
    double   ns_total;
    double   ns_selection;
    uint64_t cell_pairs[STORM_PAIRING_COUNT + 1];
    uint32_t launches;
} STORM_allpairs_stats;

STORM_rows_t* STORM_rows_new(uint32_t universe);
void STORM_rows_free(STORM_rows_t* r);
/* Append one row: sorted, distinct positions < universe (-3 otherwise). */
int STORM_rows_add(STORM_rows_t* r, const uint32_t* positions, uint32_t n);
int STORM_rows_clear(STORM_rows_t* r);
uint64_t STORM_rows_size(const STORM_rows_t* r);
uint32_t STORM_rows_universe(const STORM_rows_t* r);
/* HBM budget for the bitmap form (bytes, 0 = automatic: a quarter of free
 * memory).  Rows that do not get a bitmap behave like the reference's
 * sparse_only rows (storm_repr.h:280-291): no B, no rank, no zone map. */
int STORM_rows_set_bitmap_budget(STORM_rows_t* r, uint64_t bytes);
/* Copies the rows' positions to the device and builds every representation
 * there (storm::build_row's rules, storm_repr.cpp:25-207); the all-pairs
 * calls do it themselves after rows change. */
int STORM_rows_upload(STORM_rows_t* r);
/* A new STORM_rows_t (universe = the file's n_bits) holding the rows of a
 * STORMBIN corpus file; same format, stride and max_rows rules and errors
 * as STORM_load_stormbin.  Returns the rows loaded; *out is NULL on error. */
int64_t STORM_rows_load_stormbin(const char* path, uint32_t max_rows, uint32_t stride, STORM_rows_t** out);
/* The same for a STORMPACK file (every row, empty ones included). */
int64_t STORM_rows_load_stormpack(const char* path, STORM_rows_t** out);
/* Tensor-core dense block: under the density-ordered policies (per-tile,
 * probe, oracle, refine, learned), the densest rows -- the suffix of the
 * density order whose rows all have a bitmap and whose smallest sparse form
 * min(cardinality, 2 x runs) is >= min_density * universe --
 * are compared with each other by the tcgen05 bitmap kernel (the
 * tensor-core form of dense B x B tiles), everything else by the cells.
 * The tensor cores pay per pair in proportion to the universe, the cells in
 * proportion to the sparse sizes, so a row joins only when its sparse form
 * is a large enough share of the universe: run-clustered rows with few runs
 * stay on the run cells.  Universes up to 2^27 bits; at least 256 rows.
 * 0 disables; the default is 2^-14. */
int STORM_rows_set_dense_block(STORM_rows_t* r, double min_density);
/* RowMeta of one row (storm_repr.h:213-231) as 8 words: cardinality,
 * n_runs, n_words, n_nonzero_w, first_set, last_set, has_rank, has_occ;
 * plus a 9th word of representation flags (bit 0 bitmap, 1 complement). */
int STORM_rows_meta(STORM_rows_t* r, uint64_t row, uint32_t* meta9);

/* Forms of one row's stored representation, as STORM_rows_repr copies them
 * (storm::Row, storm_repr.h:112-276, built on the device by
 * storm::build_row's rules, storm_repr.cpp:25-207). */
#define STORM_REPR_RUN_START  0   /* u32 run starts, ascending */
#define STORM_REPR_RUN_END    1   /* u32 run ends (exclusive) */
#define STORM_REPR_EWAH       2   /* u64 EWAH-64 stream (storm_repr.h:28-31) */
#define STORM_REPR_MARKERS    3   /* u32 pairs: stream position of each marker, first word it decodes */
#define STORM_REPR_BITMAP     4   /* u64 words, n_words of them */
#define STORM_REPR_RANK       5   /* u64 rank9 directory, 2 x (n_words / 8 rounded up + 1) */
#define STORM_REPR_OCC        6   /* u64 zone map, one bit per 8 words */
#define STORM_REPR_COMPLEMENT 7   /* u32 positions not in the row, ascending */
/* Copies one form of one row to host memory (no counterpart in the
 * reference, whose Row is a host struct the caller reads directly): returns
 * the form's element count (pairs for STORM_REPR_MARKERS; 0 for a form the
 * row does not have) and, when out is non-NULL, copies min(count, cap)
 * elements into it. */
int64_t STORM_rows_repr(STORM_rows_t* r, uint64_t row, int kind, void* out, uint64_t cap);

/* Autotuner (no counterpart in the reference, which fixes its tile at 64):
 * times this container's own all-pairs sum on the GPU for every tile in
 * {32, 64, 128, 256} x tensor dense-block threshold in {0, 2^-16, 2^-14,
 * 2^-12} under the given policy and execution form (best of two calls each;
 * a trained learned selector keeps its training tile), then keeps the
 * fastest: the threshold becomes the container's dense block and the tile
 * is used by later calls that pass tile 0.  times_ms (16 entries, tile-major,
 * -1 for a skipped candidate) and the choice are reported when non-NULL.
 * Counts do not depend on the choice. */
int STORM_rows_autotune(STORM_rows_t* r, int policy, int exec, uint32_t* best_tile, double* best_min_density,
                        double* times_ms);

/* storm::allpairs_sum: sum over i < j (plus stats). fixed_cell is used by
 * STORM_POLICY_FIXED.  tile 0 means 64 (storm_allpairs.h:152-201), or the
 * tile STORM_rows_autotune chose. */
int STORM_rows_allpairs_sum(STORM_rows_t* r, int policy, uint32_t tile, int fixed_cell, int exec,
                            STORM_allpairs_stats* st);
/* Per-pair counts, packed upper triangle in ORIGINAL row order. */
int STORM_rows_allpairs_matrix(STORM_rows_t* r, int policy, uint32_t tile, int fixed_cell, int exec,
                               uint32_t* out, uint64_t out_len, STORM_allpairs_stats* st);
/* storm::allpairs_tiles: tile visitor over ORIGINAL row indices (the
 * reference hands out density-sorted positions and drops the permutation,
 * storm_allpairs.cpp:689,725; this call keeps original order). */
int STORM_rows_allpairs_tiles(STORM_rows_t* r, int policy, uint32_t tile, int exec,
                              STORM_tile_callback cb, void* ctx, STORM_allpairs_stats* st);

/* storm::select_pairing / storm::predict with the reference's default model
 * (storm_cost.cpp:372-496), on two 8-word RowMeta records. */
int STORM_select_pairing(const uint32_t* meta_a, const uint32_t* meta_b, double* predicted);
double STORM_predict(int pairing, const uint32_t* meta_a, const uint32_t* meta_b);

/* One cell on one pair of rows (both orders are valid); for tests and the
 * per-cell timing the selector is trained on.  Returns the count, or a
 * negative status when a representation the cell needs is absent. */
int64_t STORM_rows_cell(STORM_rows_t* r, int pairing, uint64_t row_a, uint64_t row_b);

/* ---- learned selector ---------------------------------------------------
 * Features per tile pair (row tiles of the density-sorted order) -> scores
 * per cell (the reference's ten and C x B); argmax is the cell.  STORM_rows_train_selector times every
 * applicable cell on sampled tiles of `r` on the GPU (the labels), trains the
 * MLP with the device forward/backward kernels, and installs it in `r`.
 * Returns 0; stats[0..5] = samples, epochs, final loss, train accuracy,
 * regret of the MLP on held-out tiles, regret of the cost model there. */
int STORM_rows_train_selector(STORM_rows_t* r, uint32_t tile, uint32_t samples, uint32_t epochs,
                              uint64_t seed, double* stats);
/* The selector's training also fits a cost model to the cell timings of
 * its training tiles (as STORM_rows_calibrate does) and keeps, as this
 * container's model from then on (the cost-model policies and the
 * untrained/fallback selector), whichever of that fitted model and the
 * reference's default model has the lower regret on the training tiles;
 * stats[5] is the regret of the fitted model on the held-out tiles.
 * STORM_rows_last_training reports the last training: out9 = regret of the
 * MLP, of the fitted model and of the reference's default model on the
 * held-out tiles, held-out and training tile counts, the fit's relative RMS
 * error, the kept model's mean fixed cost per pair over the reference's ten
 * cells, sampled tiles, and 1 if the fitted model was kept (0: the default
 * model). */
int STORM_rows_last_training(const STORM_rows_t* r, double* out9);
/* Reset to the untrained (cost-model fallback) selector. */
int STORM_rows_reset_selector(STORM_rows_t* r);

/* GPU calibration of the cost model (the reference's calibrate /
 * calibrate_on_rows, storm_cost.cpp:556-769, 779-895, which time each cell
 * on the host CPU): every cell is timed on this GPU (SM clock) on sampled
 * tiles of r's own rows -- tile rows of the density order, `samples` tiles
 * (0: all), seeded -- and the model keeps the reference's work formulas with
 * constants fitted to those timings: per cell, cycles(tile) ~ a x (the
 * reference default model's prediction above its fixed term) + f x pairs,
 * a weighted least-squares fit (relative error) giving the cell's
 * ns_per_unit and its own fixed cost per pair.  The result replaces r's cost
 * model (the cost-model policies and the untrained learned policy use it;
 * counts never depend on it).  The complement cell C x B
 * (STORM_PAIRING_CB, kernels/cell_comp.cpp), which the reference never
 * selects, is timed too and becomes a candidate of the calibrated model
 * (priced per complement position) when it was timed.  model_out (27
 * entries, may be NULL): the model as STORM_rows_cost_model lays it out,
 * then the fit's relative RMS error.  No counterpart in the reference's C
 * ABI. */
int STORM_rows_calibrate(STORM_rows_t* r, uint32_t tile, uint32_t samples, uint64_t seed, double* model_out);
/* r's cost model: set = 0 copies it into model[26] -- ns_per_unit[11]
 * (by pairing, STORM_PAIRING_EMPTY's unused), the fixed and zone-map-word
 * terms, C x B's price per complement position (0: never chosen), then the
 * fixed cost per pair of each pairing 0 .. STORM_PAIRING_CB (12 entries, 0
 * in the reference's model) -- and returns 1 when calibrated, 0 for the
 * reference default; set = 1 installs model[26], or the reference default
 * when model is NULL.  Units are those of the model (SM cycles once
 * calibrated). */
int STORM_rows_cost_model(STORM_rows_t* r, double* model, int set);
/* Parameters out/in (so a trained selector can be saved and loaded):
 * n_params floats.  Returns the parameter count when params is NULL. */
int64_t STORM_rows_selector_params(STORM_rows_t* r, float* params, uint64_t n_params, int load);

/* MLP kernels exposed for gradient checks against the CPU oracle:
 * a 2-layer MLP  logits = W2 relu(W1 x + b1) + b2 over a batch, softmax
 * cross-entropy against integer labels; grads in the same layout as params
 * (W1 [H x F], b1 [H], W2 [C x H], b2 [C]).  Device run, host buffers. */
int STORM_mlp_forward_backward(const float* params, uint32_t F, uint32_t H, uint32_t Cn,
                               const float* x, const int32_t* labels, uint32_t batch,
                               float* logits, float* loss, float* grads);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* STORM_B200_ROWS_H_ */
