// Host-only check (no GPU) of the tcgen05 descriptor encoders in
// csrc/tc_ptx.cuh, field by field against the PTX ISA layouts for sm_100a:
//   instruction descriptor, kind::i8 (32 bit): sparsity/saturate bits 0-3
//     zero, D format bits 4-5 (2 = s32), A format bits 7-9 and B format
//     bits 10-12 (0 = u8), negate bits 13-14 zero, A major bit 15 and B major
//     bit 16 (0 = K-major), N >> 3 in bits 17-22, bit 23 reserved, M >> 4 in
//     bits 24-28, bits 29-31 zero;
//   shared-memory matrix descriptor (64 bit): start address >> 4 in bits
//     0-13, leading byte offset >> 4 in bits 16-29, stride byte offset >> 4
//     in bits 32-45, version 1 in bits 46-47, base offset bits 49-51 zero,
//     leading-offset mode bit 52 zero, swizzle mode in bits 61-63
//     (2 = 128-byte swizzle).
// Every shape and address pattern the kernels issue is checked, and the
// shapes against the kind::i8 rules (M = 128: N a multiple of 16, 16..256).
// Built and run by test_descriptors_cpu.py.
#include <cstdint>
#include <cstdio>

#include "tc_ptx.cuh"
#include "bb_mma.cuh"
#include "bb_mma_ts.cuh"
#include "bb_mma_ts2.cuh"

static int g_fail = 0;
#define CHECK(c, ...)                 \
    do {                              \
        if (!(c)) {                   \
            std::printf(__VA_ARGS__); \
            std::printf("\n");        \
            ++g_fail;                 \
        }                             \
    } while (0)

static uint64_t bits(uint64_t v, int lo, int hi) {   // [lo, hi] inclusive
    return (v >> lo) & ((1ull << (hi - lo + 1)) - 1ull);
}

static void check_idesc(uint32_t m, uint32_t n) {
    const uint32_t d = sb200::umma_idesc_u8_s32(m, n);
    CHECK(bits(d, 0, 3) == 0, "idesc %ux%u: sparsity/saturate bits set", m, n);
    CHECK(bits(d, 4, 5) == 2, "idesc %ux%u: D format %llu, want 2 (s32)", m, n,
          (unsigned long long)bits(d, 4, 5));
    CHECK(bits(d, 6, 6) == 0, "idesc %ux%u: reserved bit 6", m, n);
    CHECK(bits(d, 7, 9) == 0 && bits(d, 10, 12) == 0, "idesc %ux%u: A/B format not u8", m, n);
    CHECK(bits(d, 13, 14) == 0, "idesc %ux%u: negate bits set", m, n);
    CHECK(bits(d, 15, 15) == 0 && bits(d, 16, 16) == 0, "idesc %ux%u: operands not K-major", m, n);
    CHECK(bits(d, 17, 22) == n / 8, "idesc %ux%u: N field %llu", m, n, (unsigned long long)bits(d, 17, 22));
    CHECK(bits(d, 23, 23) == 0, "idesc %ux%u: reserved bit 23", m, n);
    CHECK(bits(d, 24, 28) == m / 16, "idesc %ux%u: M field %llu", m, n, (unsigned long long)bits(d, 24, 28));
    CHECK(bits(d, 29, 31) == 0, "idesc %ux%u: high bits set", m, n);
    // kind::i8, cta_group::1, M = 128: N in 16..256, a multiple of 16
    CHECK(m == 128 && n % 16 == 0 && n >= 16 && n <= 256, "shape %ux%u not valid for kind::i8", m, n);
}

static void check_sdesc(uint32_t addr, uint32_t sbo) {
    const uint64_t d = sb200::umma_desc_sw128(addr, sbo);
    CHECK(bits(d, 0, 13) == ((addr & 0x3FFFFu) >> 4), "sdesc addr %u: start field", addr);
    CHECK(bits(d, 14, 15) == 0, "sdesc addr %u: reserved bits 14-15", addr);
    CHECK(bits(d, 16, 29) == 1, "sdesc addr %u: leading byte offset field", addr);
    CHECK(bits(d, 30, 31) == 0, "sdesc addr %u: reserved bits 30-31", addr);
    CHECK(bits(d, 32, 45) == sbo / 16, "sdesc addr %u: stride byte offset field", addr);
    CHECK(bits(d, 46, 47) == 1, "sdesc addr %u: version", addr);
    CHECK(bits(d, 48, 48) == 0 && bits(d, 49, 51) == 0 && bits(d, 52, 52) == 0,
          "sdesc addr %u: base offset / mode bits", addr);
    CHECK(bits(d, 53, 60) == 0, "sdesc addr %u: reserved bits 53-60", addr);
    CHECK(bits(d, 61, 63) == 2, "sdesc addr %u: swizzle mode", addr);
    // 128-byte swizzle atoms: 8 rows x 128 bytes, start 16-byte aligned
    CHECK(addr % 16 == 0, "sdesc addr %u not 16-byte aligned", addr);
}

int main() {
    check_idesc(sb200::MMA_BM, sb200::MMA_BN);
    check_idesc(sb200::TS_BM, sb200::TS_BN);
    check_idesc(sb200::T2_BM, sb200::T2_BN);
    // Every B operand address the TS kernels form: ring base (1024-aligned,
    // anywhere in 227 KB) + stage + K atom + 32-byte K step.
    for (uint32_t base = 0; base < 232448; base += 1024)
        for (uint32_t s = 0; s < (uint32_t)sb200::TS_STAGES; ++s)
            for (uint32_t kk = 0; kk < 8; ++kk) {
                const uint32_t a = base + s * sb200::TS_B_STAGE_BYTES + (kk >> 2) * sb200::TS_B_ATOM_BYTES + (kk & 3) * 32u;
                if (a < 232448) check_sdesc(a, 1024);
            }
    for (uint32_t s = 0; s < (uint32_t)sb200::T2_STAGES; ++s)
        for (uint32_t kk = 0; kk < 8; ++kk)
            check_sdesc(s * sb200::T2_B_STAGE_BYTES + (kk >> 2) * sb200::T2_B_ATOM_BYTES + (kk & 3) * 32u, 1024);
    // the SS kernel's A and B stages (32-byte K steps)
    for (uint32_t s = 0; s < (uint32_t)sb200::MMA_STAGES; ++s)
        for (uint32_t kk = 0; kk < 4; ++kk) {
            check_sdesc(s * sb200::MMA_STAGE_BYTES + 32u * kk, 1024);
            check_sdesc(s * sb200::MMA_STAGE_BYTES + sb200::MMA_A_BYTES + 32u * kk, 1024);
        }
    if (g_fail) {
        std::printf("%d failures\n", g_fail);
        return 1;
    }
    std::printf("descriptors ok\n");
    return 0;
}
