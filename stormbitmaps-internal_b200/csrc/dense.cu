// dense.cu -- launchers for the B x B kernels (POPC and tcgen05).
#include "dense.cuh"
#include "bb_popc.cuh"
#include "bb_mma.cuh"
#include "bb_mma_ts.cuh"

namespace sb200 {

static void build_tiles(std::vector<uint2>& t, uint64_t n, int kind) {
    t.clear();
    if (kind == STORM_B200_KERNEL_MMA || kind == STORM_B200_KERNEL_MMA_SS) {
        const uint64_t nbi = (n + MMA_BM - 1) / MMA_BM, nbj = (n + MMA_BN - 1) / MMA_BN;
        // Tile (bi, bj) holds a pair with i <= j iff 128 bi <= 256 bj + 255,
        // i.e. bj >= floor(bi / 2).
        for (uint64_t bi = 0; bi < nbi; ++bi)
            for (uint64_t bj = bi / 2; bj < nbj; ++bj) t.push_back(make_uint2((uint32_t)bi, (uint32_t)bj));
    } else {
        const uint64_t nb = (n + POPC_BM - 1) / POPC_BM;
        for (uint64_t bi = 0; bi < nb; ++bi)
            for (uint64_t bj = bi; bj < nb; ++bj) t.push_back(make_uint2((uint32_t)bi, (uint32_t)bj));
    }
}

uint64_t DenseEngine::run(const uint64_t* dX, uint64_t n, uint32_t w_pad, uint64_t row_bits,
                          uint32_t* d_out, int kernel_pref, cudaStream_t st) {
    const int sms = require_device();
    if (n == 0) {
        log.launches = 0;
        log.last_ms = 0.f;
        return 0;
    }
    if (n > 0xFFFFFFFFull) fail(STORM_B200_ELIMIT, "more than 2^32 rows");
    int kind = kernel_pref;
    if (kind == STORM_B200_KERNEL_AUTO) kind = row_bits <= MMA_MAX_BITS ? STORM_B200_KERNEL_MMA : STORM_B200_KERNEL_POPC;
    if ((kind == STORM_B200_KERNEL_MMA || kind == STORM_B200_KERNEL_MMA_SS) && row_bits > MMA_MAX_BITS)
        fail(STORM_B200_ELIMIT, "tensor-core kernel is exact only for rows of at most 2^23 bits");

    if (tiles_n != n || tiles_kind != kind) {
        std::vector<uint2> t;
        build_tiles(t, n, kind);
        d_tiles.reserve(t.size());
        SB_CUDA(cudaMemcpyAsync(d_tiles.p, t.data(), t.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
        n_tiles = (uint32_t)t.size();
        tiles_n = n;
        tiles_kind = kind;
    }
    d_flags.reserve(1);
    SB_CUDA(cudaMemsetAsync(d_flags.p, 0, sizeof(DeviceFlags), st));
    log.ensure();

    SB_CUDA(cudaEventRecord(log.ev0, st));
    if (kind == STORM_B200_KERNEL_MMA) {
        static bool attr_set = false;
        if (!attr_set) {
            SB_CUDA(cudaFuncSetAttribute(bb_mma_ts_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)TS_SMEM_BYTES));
            attr_set = true;
        }
        const uint32_t grid = n_tiles < (uint32_t)sms ? n_tiles : (uint32_t)sms;
        bb_mma_ts_kernel<<<grid, TS_THREADS, TS_SMEM_BYTES, st>>>(dX, (uint32_t)n, w_pad, d_tiles.p, n_tiles,
                                                                   d_out, d_flags.p);
    } else if (kind == STORM_B200_KERNEL_MMA_SS) {
        static bool attr_set = false;
        if (!attr_set) {
            SB_CUDA(cudaFuncSetAttribute(bb_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)MMA_SMEM_BYTES));
            attr_set = true;
        }
        const uint32_t grid = n_tiles < (uint32_t)sms ? n_tiles : (uint32_t)sms;
        bb_mma_kernel<<<grid, MMA_THREADS, MMA_SMEM_BYTES, st>>>(dX, (uint32_t)n, w_pad, d_tiles.p, n_tiles,
                                                                  d_out, d_flags.p);
    } else {
        const size_t smem = sizeof(PopcSmem);
        static bool attr_set = false;
        if (!attr_set) {
            SB_CUDA(cudaFuncSetAttribute(bb_popc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_set = true;
        }
        const uint32_t cap = (uint32_t)sms * 2;
        const uint32_t grid = n_tiles < cap ? n_tiles : cap;
        bb_popc_kernel<<<grid, POPC_THREADS, smem, st>>>(dX, (uint32_t)n, w_pad, d_tiles.p, n_tiles, d_out,
                                                          d_flags.p);
    }
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaEventRecord(log.ev1, st));
    DeviceFlags f;
    SB_CUDA(cudaMemcpyAsync(&f, d_flags.p, sizeof(f), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    SB_CUDA(cudaEventElapsedTime(&log.last_ms, log.ev0, log.ev1));
    log.launches = 1;
    log.kernel = kind;
    if (f.error) fail(STORM_B200_ETIMEOUT, "bitmap x bitmap kernel: bounded wait expired");
    return f.sum;
}

}  // namespace sb200
