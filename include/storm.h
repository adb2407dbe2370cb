/*
 * storm.h -- drop-in C interface of the B200 all-pairs intersection library.
 *
 * Every declaration below keeps the name, argument list, return type and
 * error convention of the StormBitmaps C interface (reference storm.h), so a
 * program written against that header recompiles and relinks against
 * libstorm_b200.so unchanged.  The two public container layouts
 * (STORM_bitmap_t / STORM_bitmap_cont_t / STORM_t) are byte-compatible with
 * the reference (storm.h:158-178) because callers may read them directly.
 * STORM_contiguous_t stays opaque (storm.h:180-190).
 *
 * What changes is where the all-pairs work runs: every *_pairw_* call packs
 * the rows into HBM and runs hand-written sm_100a kernels; nothing on that
 * path falls back to the CPU.  If the CUDA device or the kernels are missing
 * the call fails with a negative status (see storm_b200.h) instead of
 * computing on the host.
 *
 * Reference correspondence (file:line in the StormBitmaps tree):
 *   low-level kernels        storm.h:56-61      storm.cpp:15-151
 *   example wrappers         storm.h:95-148     storm.cpp:156-393
 *   STORM_bitmap_* / cont_*  storm.h:192-212    storm.cpp:396-873
 *   STORM_t container        storm.h:214-221    storm.cpp:875-1046
 *   STORM_contiguous_t       storm.h:224-231    storm.cpp:1048-1285
 */
#ifndef STORM_B200_STORM_H_
#define STORM_B200_STORM_H_

#include <stdint.h>
#include <stddef.h>

#if defined(__cplusplus)
#  define STORM_RESTRICT __restrict__
#elif defined(__STDC_VERSION__) && __STDC_VERSION__ >= 199901L
#  define STORM_RESTRICT restrict
#else
#  define STORM_RESTRICT
#endif

#if defined(_MSC_VER)
#  define STORM_ALIGN(n) __declspec(align(n))
#else
#  define STORM_ALIGN(n) __attribute__((aligned(n)))
#endif

/* Width of one STORM_t chunk in bits and the per-chunk list/bitmap switch.
 * Same compile-time defaults as the reference (storm.h:35-47). */
#ifndef STORM_CACHE_BLOCK_SIZE
#define STORM_CACHE_BLOCK_SIZE 256e3
#endif
#ifndef STORM_DEFAULT_BLOCK_SIZE
#define STORM_DEFAULT_BLOCK_SIZE 65536
#endif
#ifndef STORM_DEFAULT_SCALAR_THRESHOLD
#define STORM_DEFAULT_SCALAR_THRESHOLD 4096
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Pointer to a "popcount(A & B) over n words" kernel.  In the reference this
 * type comes from libalgebra.h:3045 and selects a CPU SIMD routine.  Here the
 * all-pairs loops run on the GPU, so wrappers accept the pointer only for
 * source compatibility and never call it (NULL is allowed). */
typedef uint64_t (*STORM_compute_func)(const uint64_t*, const uint64_t*, const size_t);
typedef uint64_t (*STORM_compute_lfunc)(const uint64_t*, const uint64_t*,
                                         const uint32_t*, const uint32_t*,
                                         const size_t, const size_t);

/* ---- low-level single-pair kernels (reference storm.h:56-61) ---------- */
uint64_t STORM_intersect_vector16_cardinality(const uint16_t* STORM_RESTRICT v1,
                                              const uint16_t* STORM_RESTRICT v2,
                                              const uint32_t len1, const uint32_t len2);
uint64_t STORM_intersect_vector32_unsafe(const uint32_t* STORM_RESTRICT v1,
                                         const uint32_t* STORM_RESTRICT v2,
                                         const uint32_t len1, const uint32_t len2,
                                         uint32_t* STORM_RESTRICT out);
uint64_t STORM_intersect_bitmaps_scalar_list(const uint64_t* STORM_RESTRICT b1,
                                             const uint64_t* STORM_RESTRICT b2,
                                             const uint32_t* l1, const uint32_t* l2,
                                             const uint32_t n1, const uint32_t n2);

/* ---- example wrappers (reference storm.h:95-148) ----------------------
 * Sum of popcount(A & B) over all pairs of n_vectors bitmaps of n_ints words
 * each, packed back to back in `vals`.  Computed on the GPU. */
uint64_t STORM_wrapper_diag(const uint32_t n_vectors, const uint64_t* vals,
                            const uint32_t n_ints, const STORM_compute_func f);
uint64_t STORM_wrapper_square(const uint32_t n_vectors1, const uint64_t* STORM_RESTRICT vals1,
                              const uint32_t n_vectors2, const uint64_t* STORM_RESTRICT vals2,
                              const uint32_t n_ints, const STORM_compute_func f);
uint64_t STORM_wrapper_diag_list(const uint32_t n_vectors, const uint64_t* STORM_RESTRICT vals,
                                 const uint32_t n_ints,
                                 const uint32_t* STORM_RESTRICT n_alts,
                                 const uint32_t* STORM_RESTRICT alt_positions,
                                 const uint32_t* STORM_RESTRICT alt_offsets,
                                 const STORM_compute_func f, const STORM_compute_lfunc fl,
                                 const uint32_t cutoff);
uint64_t STORM_wrapper_diag_blocked(const uint32_t n_vectors, const uint64_t* vals,
                                    const uint32_t n_ints, const STORM_compute_func f,
                                    uint32_t block_size);
uint64_t STORM_wrapper_diag_list_blocked(const uint32_t n_vectors,
                                         const uint64_t* STORM_RESTRICT vals,
                                         const uint32_t n_ints,
                                         const uint32_t* STORM_RESTRICT n_alts,
                                         const uint32_t* STORM_RESTRICT alt_positions,
                                         const uint32_t* STORM_RESTRICT alt_offsets,
                                         const STORM_compute_func f, const STORM_compute_lfunc fl,
                                         const uint32_t cutoff, uint32_t block_size);

/* ---- canonical (chunked) representation: PUBLIC layouts -------------- */
typedef struct STORM_bitmap_s STORM_bitmap_t;
typedef struct STORM_bitmap_cont_s STORM_bitmap_cont_t;
typedef struct STORM_s STORM_t;
typedef struct STORM_contiguous_bitmap_s STORM_contiguous_bitmap_t;
typedef struct STORM_contiguous_s STORM_contiguous_t;

/* One 65536-bit chunk of one row: either a 1024-word bitmap (n_bitmap != 0)
 * or a u16 offset list (n_bitmap == 0).  Field order, widths and the 64-byte
 * member alignment reproduce the reference layout (storm.h:158-166): the
 * struct is 128 bytes with `scalar` at offset 64. */
struct STORM_bitmap_s {
    STORM_ALIGN(64) uint64_t* data;
    STORM_ALIGN(64) uint16_t* scalar;
    uint32_t n_bitmap: 30, own_data: 1, own_scalar: 1;
    uint32_t n_bits_set;
    uint32_t n_scalar: 31, n_scalar_set: 1, n_missing;
    uint32_t m_scalar;
    uint32_t id;            /* chunk index = value / STORM_DEFAULT_BLOCK_SIZE */
};

/* One row: its non-empty chunks in ascending chunk order (storm.h:168-173). */
struct STORM_bitmap_cont_s {
    STORM_bitmap_t* bitmaps;
    uint32_t* block_ids;
    uint32_t n_bitmaps, m_bitmaps;
    uint32_t prev_inserted_value;
};

/* A set of rows (storm.h:175-178). */
struct STORM_s {
    STORM_bitmap_cont_t* conts;
    uint32_t n_conts, m_conts;
};

/* ---- chunk-level calls (reference storm.h:192-212) -------------------- */
STORM_bitmap_t* STORM_bitmap_new(void);
void STORM_bitmap_init(STORM_bitmap_t* all);
void STORM_bitmap_free(STORM_bitmap_t* bitmap);
int STORM_bitmap_add(STORM_bitmap_t* bitmap, const uint32_t* values, const uint32_t n_values);
int STORM_bitmap_add_with_scalar(STORM_bitmap_t* bitmap, const uint32_t* values, const uint32_t n_values);
int STORM_bitmap_add_scalar_only(STORM_bitmap_t* bitmap, const uint32_t* values, const uint32_t n_values);
uint64_t STORM_bitmap_intersect_cardinality(STORM_bitmap_t* STORM_RESTRICT bitmap1,
                                            STORM_bitmap_t* STORM_RESTRICT bitmap2);
uint64_t STORM_bitmap_intersect_cardinality_func(STORM_bitmap_t* STORM_RESTRICT bitmap1,
                                                 STORM_bitmap_t* STORM_RESTRICT bitmap2,
                                                 const STORM_compute_func func);
int STORM_bitmap_clear(STORM_bitmap_t* bitmap);
uint32_t STORM_bitmap_serialized_size(STORM_bitmap_t* bitmap);

STORM_bitmap_cont_t* STORM_bitmap_cont_new(void);
void STORM_bitmap_cont_init(STORM_bitmap_cont_t* bitmap);
void STORM_bitmap_cont_free(STORM_bitmap_cont_t* bitmap);
int STORM_bitmap_cont_add(STORM_bitmap_cont_t* bitmap, const uint32_t* values, const uint32_t n_values);
int STORM_bitmap_cont_clear(STORM_bitmap_cont_t* bitmap);
uint64_t STORM_bitmap_cont_intersect_cardinality(const STORM_bitmap_cont_t* STORM_RESTRICT bitmap1,
                                                 const STORM_bitmap_cont_t* STORM_RESTRICT bitmap2);
uint64_t STORM_bitmap_cont_intersect_cardinality_premade(const STORM_bitmap_cont_t* STORM_RESTRICT bitmap1,
                                                         const STORM_bitmap_cont_t* STORM_RESTRICT bitmap2,
                                                         const STORM_compute_func func, uint32_t* out);
uint32_t STORM_bitmap_cont_serialized_size(STORM_bitmap_cont_t* bitmap);

/* ---- STORM_t container (reference storm.h:214-221) -------------------- */
STORM_t* STORM_new(void);
void STORM_free(STORM_t* bitmap);
int STORM_add(STORM_t* bitmap, const uint32_t* values, const uint32_t n_values);
int STORM_clear(STORM_t* bitmap);
uint64_t STORM_pairw_intersect_cardinality(STORM_t* bitmap);
uint64_t STORM_pairw_intersect_cardinality_blocked(STORM_t* bitmap, uint32_t bsize);
uint64_t STORM_intersect_cardinality_square(const STORM_t* STORM_RESTRICT bitmap1,
                                            const STORM_t* STORM_RESTRICT bitmap2);
uint64_t STORM_serialized_size(const STORM_t* bitmap);

/* ---- contiguous rows (reference storm.h:224-231) ---------------------- */
STORM_contiguous_t* STORM_contig_new(size_t vector_length);
void STORM_contig_free(STORM_contiguous_t* bitmap);
int STORM_contig_add(STORM_contiguous_t* bitmap, const uint32_t* values, const uint32_t n_values);
int STORM_contig_clear(STORM_contiguous_t* bitmap);
uint64_t STORM_contig_pairw_intersect_cardinality(STORM_contiguous_t* bitmap);
uint64_t STORM_contig_pairw_intersect_cardinality_blocked(STORM_contiguous_t* bitmap, uint32_t bsize);
uint64_t STORM_contig_pairw_intersect_cardinality_list(STORM_contiguous_t* bitmap);
uint64_t STORM_contig_pairw_intersect_cardinality_blocked_list(STORM_contiguous_t* bitmap, uint32_t bsize);

#ifdef __cplusplus
} /* extern "C" */
#endif

#include "storm_b200.h"

#endif /* STORM_B200_STORM_H_ */
