// run_pieces.cuh -- the piece rules of the run postings (chunk_engine.cu):
// the universe is cut into bins of 2^wlog values (16 .. 32768, so that no bin
// straddles a 65536-value chunk), and a piece is a maximal run of a row's
// values inside one bin. Host and device share these rules (the host checks
// them without a GPU, tests/run_pieces_check.cu).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define SB_RUN_FN __host__ __device__ __forceinline__
#else
#define SB_RUN_FN inline
#endif

namespace sb200 {

// Entry e of a strictly increasing list chunk (chunk-local u16 values)
// starts a piece: the first entry, after a gap, or at a bin's first value.
SB_RUN_FN bool run_piece_start(const uint16_t* l, uint32_t e, uint32_t wmask) {
    return e == 0 || l[e] != l[e - 1] + 1 || (l[e] & wmask) == 0;
}

// Entry e ends a piece: the last entry, before a gap, or at a bin's last value.
SB_RUN_FN bool run_piece_last(const uint16_t* l, uint32_t e, uint32_t nl, uint32_t wmask) {
    return e + 1 == nl || l[e + 1] != l[e] + 1 || ((l[e] + 1u) & wmask) == 0;
}

// In a bitmap chunk, per word (index `word` inside the chunk): the bits
// where a bin starts and where one ends.
SB_RUN_FN uint64_t run_bin_first_bits(uint32_t word, uint32_t wlog) {
    if (wlog >= 6) return ((word << 6) & ((1u << wlog) - 1u)) == 0 ? 1ull : 0ull;
    return wlog == 4 ? 0x0001000100010001ull : 0x0000000100000001ull;
}

SB_RUN_FN uint64_t run_bin_last_bits(uint32_t word, uint32_t wlog) {
    if (wlog >= 6) return (((word + 1) << 6) & ((1u << wlog) - 1u)) == 0 ? (1ull << 63) : 0ull;
    return wlog == 4 ? 0x8000800080008000ull : 0x8000000080000000ull;
}

// Word `word` of a bitmap chunk holding x, with cin = bit 63 of the word
// before it and nin = bit 0 of the word after it (0 at the chunk's edges):
// the set bits that start a piece and the set bits that end one.
SB_RUN_FN void run_word_masks(uint64_t x, uint64_t cin, uint64_t nin, uint32_t word,
                                                        uint32_t wlog, uint64_t& starts, uint64_t& lasts) {
    starts = (x & ~((x << 1) | cin)) | (x & run_bin_first_bits(word, wlog));
    lasts = (x & ~((x >> 1) | (nin << 63))) | (x & run_bin_last_bits(word, wlog));
}

}  // namespace sb200
