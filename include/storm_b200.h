/*
 * storm_b200.h -- extensions of the drop-in interface.
 *
 * The reference interface (storm.h) only returns the SUM of |Xi & Xj| over
 * i < j.  An all-pairs user almost always wants the individual counts, which
 * the reference's C++ kernel layer hands out tile by tile
 * (kernels/storm_allpairs.h:206-214, `allpairs_tiles` + `TileCallback`).
 * The entry points below expose that per-pair output through the C ABI, plus
 * bulk ingest and device-resident variants used for measurement.
 *
 * Conventions shared by every entry point in this file:
 *   - int returns: 0 (or a count) on success, a negative STORM_B200_E* code
 *     on failure; STORM_b200_strerror() names it.
 *   - "matrix" outputs are the packed upper triangle INCLUDING the diagonal,
 *     in original row order: entry (i, j), i <= j, lives at
 *     STORM_tri_index(n, i, j); n*(n+1)/2 entries in total.  The diagonal is
 *     the row cardinality.
 *   - the optional `sum` out-parameter receives the reference's own result,
 *     the sum over i < j (storm.cpp:1232-1240, 927-945).
 *   - every call is synchronous: results are on the host (or, for *_device
 *     calls, complete in device memory) when it returns.
 */
#ifndef STORM_B200_EXT_H_
#define STORM_B200_EXT_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct STORM_s STORM_t;
typedef struct STORM_contiguous_s STORM_contiguous_t;

/* ---- status codes ----------------------------------------------------- */
#define STORM_B200_OK          0
#define STORM_B200_ENULL      (-1)   /* NULL handle (reference code -1)            */
#define STORM_B200_EVALUES    (-2)   /* NULL values pointer (reference code -2)    */
#define STORM_B200_EARG       (-3)   /* argument out of range / unsorted input     */
#define STORM_B200_ENOMEM     (-4)   /* host or device allocation failed (ref -4)  */
#define STORM_B200_ECUDA      (-5)   /* no usable sm_100 device, or a CUDA error   */
#define STORM_B200_ETIMEOUT   (-6)   /* a bounded device-side wait gave up         */
#define STORM_B200_ESIZE      (-7)   /* output buffer smaller than required        */
#define STORM_B200_ELIMIT     (-8)   /* problem exceeds a documented size limit    */

const char* STORM_b200_strerror(int status);
/* Status of the last call on this thread that returned a sentinel instead of
 * a status (the uint64_t-returning reference calls return 0, or (uint64_t)-1
 * for a NULL STORM_t, exactly as the reference does). */
int STORM_b200_last_status(void);

/* Failure detection, exercised without a fault (no counterpart in the
 * reference): runs the bounded mbarrier wait of the tensor-core kernels on a
 * barrier nothing arrives on, with a limit of limit_us microseconds (1 ..
 * 10,000,000), in a kernel that holds tensor memory as they do.  When the
 * wait gives up the kernel records where, frees its tensor memory and
 * returns, and this call returns STORM_B200_ETIMEOUT -- the status every
 * all-pairs call returns when one of its waits gives up -- with the context
 * still usable.  Returns 0 if the wait did not give up. */
int STORM_b200_wait_selftest(uint32_t limit_us);

/* Packed upper-triangle index of pair (i, j), i <= j < n. */
static inline uint64_t STORM_tri_index(uint64_t n, uint64_t i, uint64_t j) {
    /* rows 0..i-1 hold n, n-1, ..., n-i+1 entries; i*(i-1) is even */
    return i * n - (i * (i - 1)) / 2 + (j - i);
}
static inline uint64_t STORM_tri_size(uint64_t n) { return n * (n + 1) / 2; }

/* Tile visitor, shaped like storm::TileCallback (storm_allpairs.h:206-208):
 * `counts` is a tile x tile buffer, row stride `tile`, of which the nr x nc
 * block is live.  On diagonal tiles only j > i is filled (the reference's
 * allpairs_tiles convention, storm_allpairs.cpp:709); other entries are 0.
 * Rows/columns are ORIGINAL row indices i0.., j0.. */
typedef void (*STORM_tile_callback)(uint32_t i0, uint32_t j0, uint32_t nr, uint32_t nc,
                                    const uint32_t* counts, void* ctx);

/* ---- STORM_contiguous_t extensions ------------------------------------ */
/* Bitmap x bitmap kernel used by the contiguous all-pairs calls. */
#define STORM_B200_KERNEL_AUTO  0   /* MMA_DB for rows <= 2^17 bits, MMA up to
                                       2^27, POPC beyond                         */
#define STORM_B200_KERNEL_POPC  1   /* CUDA-core AND + POPC tiles                  */
#define STORM_B200_KERNEL_MMA   2   /* tcgen05 kind::i8, A operand in TMEM         */
#define STORM_B200_KERNEL_MMA_SS 3  /* tcgen05 kind::i8, both operands in smem     */
#define STORM_B200_KERNEL_MMA_DB 4  /* tcgen05 kind::i8, A in TMEM, 128 x 192 tiles
                                       with two accumulators drained by their own
                                       warps while the next tile computes        */
#define STORM_B200_KERNEL_MMA_2CTA 5 /* tcgen05 kind::i8 on CTA pairs (cta_group::2):
                                       256 x 256 tiles, each CTA expanding half of
                                       the B rows                                */

/* Append n_rows rows given as packed little-endian bitmaps of
 * words_per_row 64-bit words each, in host memory or (unified addressing)
 * device memory (bit b of row r = word b/64, bit b%64).  Device input is
 * read after all work queued on the device so far has finished.
 * words_per_row must equal ceil(vector_length/64).  Bits at or above
 * vector_length must be zero (STORM_B200_EARG otherwise).  Equivalent to one
 * STORM_contig_add per row with that row's set positions, except that empty
 * rows are kept (STORM_contig_add drops n_values == 0 calls).  Returns
 * n_rows. */
int STORM_contig_add_bitmaps(STORM_contiguous_t* c, const uint64_t* words,
                             uint32_t n_rows, uint32_t words_per_row);
/* Number of rows held. */
uint64_t STORM_contig_size(const STORM_contiguous_t* c);
int STORM_contig_set_kernel(STORM_contiguous_t* c, int kernel);
/* Work schedule of the tensor-core kernel: STORM_B200_SCHED_AUTO picks per
 * launch (stream-K when the last wave of whole tiles would be less than
 * 98.5 % full and rows have at least 32768 bits), _TILES deals whole tiles
 * round robin, _STREAM_K always
 * splits the (tile, K stage) space evenly over the SMs. Counts are the same
 * under every schedule. */
#define STORM_B200_SCHED_AUTO     0
#define STORM_B200_SCHED_TILES    1
#define STORM_B200_SCHED_STREAM_K 2
int STORM_contig_set_schedule(STORM_contiguous_t* c, int schedule);
/* Autotuner (no counterpart in the reference): times this container's own
 * all-pairs call on the GPU with each bitmap x bitmap kernel that is exact
 * for its row length -- tcgen05 with A in tensor memory (128 x 256 tiles,
 * then 128 x 192 double-buffered tiles), each under whole-tile and stream-K
 * schedules; tcgen05 with both operands in shared memory; CUDA-core POPC;
 * tcgen05 on CTA pairs (whole tiles) -- best of two calls each, and keeps
 * the fastest kernel and schedule for later calls.  times_ms (7 entries in
 * that order, -1 when skipped) and the choice are reported when non-NULL.
 * Counts do not depend on it. */
int STORM_contig_autotune(STORM_contiguous_t* c, int* best_kernel, int* best_schedule, double* times_ms);
/* Pack the rows into HBM now (otherwise done by the first all-pairs call). */
int STORM_contig_upload(STORM_contiguous_t* c);
/* Per-pair counts into a HOST buffer of out_len >= n*(n+1)/2 entries. */
int STORM_contig_pairw_intersect_matrix(STORM_contiguous_t* c, uint32_t* out,
                                        uint64_t out_len, uint64_t* sum);
/* STORM_contig_clear + STORM_contig_add_bitmaps + STORM_contig_pairw_intersect_matrix
 * in one call, so that the three overlap: n_rows rows of words_per_row (=
 * ceil(vector_length / 64)) words in HOST memory -- pinned memory lets the
 * copies run asynchronously -- replace the container's rows and are copied
 * to the device last rows first, while the tiles that read only those rows
 * already run (from the bottom of the triangle up) and the finished rows of
 * the triangle are copied back into out (out_len >= n*(n+1)/2).  Same checks
 * and codes as the three calls; device-memory rows get STORM_B200_EARG (use
 * STORM_contig_add_bitmaps).  Afterwards the container holds the rows; on an
 * error it is left empty.  Counts are those of the three calls. */
int STORM_contig_pairw_intersect_matrix_from_host(STORM_contiguous_t* c, const uint64_t* rows, uint32_t n_rows,
                                                  uint32_t words_per_row, uint32_t* out, uint64_t out_len,
                                                  uint64_t* sum);
/* Same, into a DEVICE buffer on the current device (d_out may be NULL to
 * compute only the sum).  Work already queued on other streams is waited for
 * before d_out is written. */
int STORM_contig_pairw_intersect_matrix_device(STORM_contiguous_t* c, uint32_t* d_out,
                                               uint64_t out_len, uint64_t* sum);
int STORM_contig_pairw_intersect_tiles(STORM_contiguous_t* c, uint32_t tile,
                                       STORM_tile_callback cb, void* ctx);
/* CUDA stream the handle launches on (a cudaStream_t), for event timing. */
void* STORM_contig_stream(STORM_contiguous_t* c);
/* Device time of the kernels of the last all-pairs call (CUDA events on the
 * handle's stream) and how many kernels it launched. */
float STORM_contig_last_kernel_ms(const STORM_contiguous_t* c);
uint32_t STORM_contig_last_launches(const STORM_contiguous_t* c);
/* Which kernel the last call ran (STORM_B200_KERNEL_POPC, _MMA, _MMA_SS or
 * _MMA_DB). */
int STORM_contig_last_kernel(const STORM_contiguous_t* c);

/* All pairs of rows that are already in device memory, into a device buffer,
 * without allocating anything.  No counterpart in the reference: it is for
 * callers that cannot allocate device memory when they need the counts -- a
 * service that reserves all of HBM for its own pool at start-up and forbids
 * cudaMalloc afterwards, or a framework whose allocator owns every device
 * buffer.  The caller owns both buffers:
 *   d_rows  32-byte aligned (STORM_B200_EARG otherwise; any cudaMalloc
 *           pointer is), row r at d_rows + r * row_pitch_words (pitch a
 *           multiple of 8 words); ceil(n_rows / 256) * 256 rows must be readable, the
 *           rows from n_rows on must be zero, and so must every bit of a row
 *           at or past row_bits (up to the pitch);
 *   d_out   n_rows*(n_rows+1)/2 u32, packed upper triangle (may be NULL for
 *           the sum only).
 * Runs the tensor-core kernel (row_bits <= 2^23) on `stream` (a
 * cudaStream_t; NULL = the default stream) and waits for that stream before
 * returning, so the counts and the sum are complete on return.  Its scratch
 * (status/sum words and a tile list of at most 32768 tiles of 128 x 256
 * pairs: n_rows up to 46080) is a 256 KiB array in the library that every
 * GPU holding the library keeps until exit; larger problems return
 * STORM_B200_ELIMIT.  The first call on a device looks that array up (and
 * opts the kernel into its shared memory), so make the first call before any
 * stream capture.  A CUDA error still pending from earlier work on the
 * thread is returned as STORM_B200_ECUDA before anything is launched.  All
 * calls share the one array: calls that overlap on the GPU race and must not
 * be issued. */
int STORM_contig_pairw_intersect_matrix_noalloc(const uint64_t* d_rows, uint64_t n_rows,
                                                uint32_t row_pitch_words, uint64_t row_bits,
                                                uint32_t* d_out, uint64_t out_len, uint64_t* sum,
                                                void* stream);

/* Thresholded all-pairs: the opt-in contract of the reference's thresholded
 * mode (bench/bench_threshold.cpp:129-132, README.md "Thresholded mode"): only
 * the pairs i < j whose exact count v = |Xi & Xj| is > 0 and whose Jaccard
 * v / (|Xi| + |Xj| - v) >= jaccard_min (compared in double precision) are
 * reported, with v; the counts are exact, only the set of reported pairs is
 * restricted.  No per-pair triangle reaches the host: on the tensor-core
 * kernel the filter runs in the epilogue and nothing else is written.
 * out_i / out_j / out_count receive min(found, cap) pairs sorted by (i, j);
 * *n_found = how many passed.  Returns 0, or STORM_B200_ESIZE when more than
 * cap passed (the arrays then hold cap of them, not necessarily the first).
 * No counterpart in storm.h (the reference's thresholded mode is a bench). */
int STORM_contig_pairw_threshold(STORM_contiguous_t* c, double jaccard_min, uint32_t* out_i, uint32_t* out_j,
                                 uint32_t* out_count, uint64_t cap, uint64_t* n_found);

/* ---- STORM_t extensions ----------------------------------------------- */
/* n_rows STORM_add calls in one (no counterpart in the reference, whose
 * callers loop over STORM_add, storm.cpp:894-916): row r is values
 * [offsets[r], offsets[r+1]) (offsets has n_rows + 1 entries, ascending),
 * appended with exactly the chunks STORM_add builds -- empty rows included --
 * while the rows are split into chunks on several host threads.  Returns
 * n_rows; STORM_B200_EARG for offsets that decrease or a row of 2^32 values
 * or more, STORM_B200_ENOMEM when a chunk could not be allocated (the rows
 * are then appended with what fit). */
int64_t STORM_add_rows(STORM_t* s, const uint32_t* values, const uint64_t* offsets, uint64_t n_rows);
/* The same for rows given as little-endian bitmaps in host memory: row r is
 * words [r * words_per_row, (r + 1) * words_per_row), bit b = word b / 64,
 * bit b % 64 (words_per_row <= 2^26), appended as STORM_add appends the
 * row's set positions in ascending order.  Returns n_rows; errors as
 * STORM_add_rows. */
int64_t STORM_add_bitmap_rows(STORM_t* s, const uint64_t* words, uint64_t n_rows, uint64_t words_per_row);
/* Append the rows of a STORMBIN corpus file (the reference's on-disk format:
 * "STORMBIN", u32 version 1, n_rows, n_bits, pad, then per row a u32 count
 * and that many strictly ascending u32 positions < n_bits;
 * bench/bench_allpairs.cpp:44-72) to s with STORM_add.  As the reference's
 * loaders do, empty rows are skipped and every stride-th row (0 or 1: all)
 * is kept, up to max_rows (0: all).  Returns the rows added and sets
 * *n_bits (may be NULL); STORM_B200_EARG if the file cannot be opened,
 * STORM_B200_EVALUES for a bad header, a truncated row or positions out of
 * order or range. */
int64_t STORM_load_stormbin(STORM_t* s, const char* path, uint32_t max_rows, uint32_t stride, uint32_t* n_bits);
/* Append the rows of a STORMPACK file (the reference's packed format with one
 * stored representation per row -- bitmap, u16 array, u16 runs, full, empty;
 * tools/pack.cpp:100-145) to s, every row including empty ones.  Returns the
 * rows added and sets *n_bits; errors as STORM_load_stormbin. */
int64_t STORM_load_stormpack(STORM_t* s, const char* path, uint32_t* n_bits);
/* Thresholded all-pairs over STORM_t rows: as STORM_contig_pairw_threshold;
 * |Xi| is row i's count against itself. */
int STORM_pairw_threshold(STORM_t* s, double jaccard_min, uint32_t* out_i, uint32_t* out_j, uint32_t* out_count,
                          uint64_t cap, uint64_t* n_found);
int STORM_upload(STORM_t* s);
int STORM_pairw_intersect_matrix(STORM_t* s, uint32_t* out, uint64_t out_len, uint64_t* sum);
/* Same, into a DEVICE buffer on the current device (d_out may be NULL to
 * compute only the sum).  Work already queued on other streams is waited for
 * before d_out is written. */
int STORM_pairw_intersect_matrix_device(STORM_t* s, uint32_t* d_out, uint64_t out_len, uint64_t* sum);
int STORM_pairw_intersect_tiles(STORM_t* s, uint32_t tile, STORM_tile_callback cb, void* ctx);
float STORM_last_kernel_ms(const STORM_t* s);
/* Tensor-core dense block of the STORM_t all-pairs calls (no counterpart in
 * the reference, which compares chunk by chunk): rows with strictly
 * ascending chunk ids, no repeated list value and full 1024-word bitmap
 * chunks are candidates (universe = 65536 x (largest chunk id + 1), at most
 * 2^27 bits).  The chosen ones are expanded into contiguous bitmaps and
 * compared with each other by the tcgen05 kernel; pairs with any other row
 * stay on the chunk kernel.  Counts are identical either way.
 * min_density < 0 (the default): a candidate joins when its predicted chunk-
 * kernel cost against a row like itself exceeds the tensor-core cost of a
 * pair (which grows with the universe); min_density > 0: when its value
 * count is >= min_density x universe; 0 disables the block.
 * budget_bytes bounds the expanded rows held at once (0: 60 % of free device
 * memory), each row taking (universe / 65536) x 8256 bytes (its 8 KiB
 * chunk slots 64 bytes apart); larger sets run in panels.  Applies to later
 * all-pairs calls. */
int STORM_set_dense_block(STORM_t* s, double min_density, uint64_t budget_bytes);
/* Rows / panels the last all-pairs call on s gave to the dense block. */
uint64_t STORM_last_dense_rows(const STORM_t* s);
uint64_t STORM_last_dense_panels(const STORM_t* s);
/* Postings for the sparse rows of the STORM_t all-pairs calls (no
 * counterpart in the reference): plain rows without bitmap chunks outside
 * the dense block are indexed by value (a histogram over the universe, at
 * most 2^27 values), and each pair of them gets one increment per shared
 * value -- pairs with nothing in common cost nothing.  mode -1 (default):
 * used when the exact increment count predicts less time than the chunk
 * kernel; 1: whenever rows qualify; 0: never.  Per-pair counts take one of
 * two forms: the increments go list by list into the output, or -- for
 * outputs larger than L2, and when predicted faster from the exact
 * increment count -- a row sweep counts each row's partners in shared
 * memory (in blocks of 51200 partner rows, reading the row's lists once per
 * block) and writes its slice once.  A third per-pair form indexes runs
 * instead of values: the universe is cut into bins of a power of two near
 * the rows' mean run
 * length, each row's maximal runs into pieces per bin, and a row sweep adds
 * the overlaps of a row's pieces with the pieces of later rows in the same
 * bins -- rows made of long runs then cost per run, not per value; it is
 * used when its exact entry count (from a histogram of pieces per bin)
 * predicts less time than the value form.  Modes 2, 3 and 4 force the rows
 * in and pick the list-by-list, the row-sweep or the run-sweep form.
 * Counts are identical. */
int STORM_set_sparse_postings(STORM_t* s, int mode);
/* The per-pair form the last all-pairs call on s used for its postings
 * rows: 0 list by list, 1 row sweep, 2 run sweep, -1 none (no postings
 * rows, or a sum-only call). */
int STORM_last_postings_form(const STORM_t* s);
/* Autotuner (no counterpart in the reference): times the per-pair all-pairs
 * call on the GPU with the tensor-core rows on (cost rule) or off, crossed
 * with the postings on (cost rule) or off, best of two calls each, and keeps
 * the fastest settings for later calls (as STORM_set_dense_block(s, -1 or 0,
 * budget unchanged) and STORM_set_sparse_postings(s, -1 or 0)).  times_ms (4
 * entries: both on, postings off, tensor rows off, both off) and the choice
 * are reported when non-NULL.  Counts do not depend on the choice. */
int STORM_autotune(STORM_t* s, double* best_min_density, int* best_postings, double* times_ms);
uint64_t STORM_last_postings_rows(const STORM_t* s);
/* Transposed panel of the STORM_t per-pair calls (no counterpart in the
 * reference): plain rows below the tensor-core rows in value count are
 * queried, value by value, against blocks of up to 2048 denser rows stored
 * transposed in HBM (per value, one bit per panel row), so that a pair of a
 * sparse row x and a dense row costs |x| bits of traffic instead of the
 * universe's.  The planner then splits plain rows three ways -- postings
 * rows (pairs among themselves by value postings), panel rows, tensor rows
 * (pairs among themselves on the tensor cores) -- by predicted time.
 * mode -1 (default): when predicted faster than the plan without it; 1:
 * whenever the rows and device memory allow (universe up to 2^26 values);
 * 2: every plain row in the panel (all their pairs by it); 0: never.  Applies with the automatic dense block and postings
 * (STORM_set_dense_block(s, -1, ...), STORM_set_sparse_postings(s, -1)).
 * Counts are identical. */
int STORM_set_panel(STORM_t* s, int mode);
/* Rows the last per-pair call stored in the transposed panel. */
uint64_t STORM_last_panel_rows(const STORM_t* s);
/* Per engine of the last per-pair call -- out12[0..3]: device ms of the
 * tensor cores, the chunk kernel, the transposed panel and the postings
 * (with their histogram); out12[4..7]: the planner's predicted ms for the
 * work it gave each (0 for the chunk kernel, which it does not price);
 * out12[8..11]: that work -- tensor cores in int8 operations (2 x pairs x
 * universe bits), chunk kernel in pairs, panel and postings in the bytes
 * they must move (panel: a 256-byte transposed line per query value and
 * 2048-row block, the expanded and transposed blocks, 4 bytes per count;
 * postings: 8 bytes per value, per list entry and per increment, and the
 * universe-sized histogram). */
int STORM_last_engine_ms(const STORM_t* s, double* out12);
/* The rest of the last per-pair call's device time before its first engine:
 * the planner's host work while the GPU waits (before the postings'
 * histogram and after its statistics are read back), the row order's upload
 * and the output's clearing, in ms; -1.0 for a NULL handle. */
double STORM_last_plan_ms(const STORM_t* s);
/* Host-side transfers of the last all-pairs call (no counterpart in the
 * reference, which has no device): out4[0] wall ms of packing and uploading
 * the rows (0 when they were already on the device), out4[1] the payload
 * bytes uploaded (bitmaps and lists), out4[2] wall ms of copying the
 * per-pair triangle into the caller's host buffer (0 for calls without
 * one), out4[3] its bytes. */
int STORM_last_transfer_ms(const STORM_t* s, double* out4);
/* GPU calibration of the planner (no counterpart in the reference's C ABI;
 * its calibrate_on_rows fits the kernel layer's constants on the host,
 * storm_cost.cpp:779-895): on a strided sample of up to sample_rows rows (0:
 * 2048) every plain row is counted on the tensor cores, then in the
 * transposed panel, then the list rows by postings; each engine's constants
 * are scaled by its measured / predicted device time, and later plans of s
 * use them.  out (4 entries, may be NULL): the tensor, panel and postings
 * scales and the sample's row count.  Counts never depend on it. */
int STORM_calibrate(STORM_t* s, uint32_t sample_rows, double* out);
/* Back to the planner's built-in constants. */
int STORM_reset_cost_model(STORM_t* s);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* STORM_B200_EXT_H_ */
