// list16_ref.cuh -- |v1 & v2| of two u16 chunk lists exactly as the
// reference's STORM_intersect_vector16_cardinality counts it in its SSE4.2
// build (storm.cpp:15-88), for lists that are not strictly increasing.
//
// For strictly increasing lists that count is the size of the intersection,
// and the warp-parallel cells compute it. With a repeated value (STORM_add
// does not deduplicate list chunks) or an unsorted list the reference's
// answer depends on its blocking, so it is restated step by step here:
//   * while both lists have a whole block of 8 entries left, the current
//     blocks are compared: every entry of v1's block that equals any entry
//     of v2's block counts once (an "equal any" string compare with v1's
//     block as the string). As long as either block starts with 0 both
//     blocks have their full 8 entries; otherwise each block ends at its
//     first 0 entry (the implicit-length compare). Then the block with the
//     smaller last entry advances (both on a tie); the blocked phase stops
//     as soon as either list has no whole block left;
//   * the remaining entries are merged by the scalar two-pointer loop (equal
//     entries count once and both advance).
// Host and device: the host build is what the tests compare with the
// reference library; the chunk kernel runs the same code on one lane.
#pragma once
#include <stdint.h>

namespace sb200 {

// Entries of an 8-entry block before its first 0 (8 when there is none).
__host__ __device__ __forceinline__ uint32_t list16_block_len(const uint16_t* b) {
    uint32_t n = 0;
    while (n < 8 && b[n] != 0) ++n;
    return n;
}

// Entries i < la of a that equal some entry k < lb of b.
__host__ __device__ __forceinline__ uint32_t list16_block_any(const uint16_t* a, uint32_t la, const uint16_t* b,
                                                              uint32_t lb) {
    uint32_t c = 0;
    for (uint32_t i = 0; i < la; ++i) {
        bool hit = false;
        for (uint32_t k = 0; k < lb; ++k) hit |= a[i] == b[k];
        c += hit ? 1u : 0u;
    }
    return c;
}

__host__ __device__ inline uint64_t list16_blocked_count(const uint16_t* v1, const uint16_t* v2, uint32_t len1,
                                                         uint32_t len2) {
    uint64_t count = 0;
    uint32_t ia = 0, ib = 0;
    const uint32_t sta = len1 / 8 * 8, stb = len2 / 8 * 8;
    if (ia < sta && ib < stb) {
        bool done = false;
        // blocks that start with 0: full-length compares
        while (v1[ia] == 0 || v2[ib] == 0) {
            count += list16_block_any(v1 + ia, 8, v2 + ib, 8);
            const uint16_t a_max = v1[ia + 7], b_max = v2[ib + 7];
            if (a_max <= b_max) {
                ia += 8;
                if (ia == sta) {
                    done = true;
                    break;
                }
            }
            if (b_max <= a_max) {
                ib += 8;
                if (ib == stb) {
                    done = true;
                    break;
                }
            }
        }
        // then compares that end each block at its first 0
        if (!done && ia < sta && ib < stb) {
            for (;;) {
                count += list16_block_any(v1 + ia, list16_block_len(v1 + ia), v2 + ib, list16_block_len(v2 + ib));
                const uint16_t a_max = v1[ia + 7], b_max = v2[ib + 7];
                if (a_max <= b_max) {
                    ia += 8;
                    if (ia == sta) break;
                }
                if (b_max <= a_max) {
                    ib += 8;
                    if (ib == stb) break;
                }
            }
        }
    }
    while (ia < len1 && ib < len2) {
        const uint16_t a = v1[ia], b = v2[ib];
        if (a < b) {
            ++ia;
        } else if (b < a) {
            ++ib;
        } else {
            ++count;
            ++ia;
            ++ib;
        }
    }
    return count;
}

}  // namespace sb200
