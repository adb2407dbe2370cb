// oneshot.cuh -- this host thread's reusable context for the calls that
// compare a few chunks, rows or lists (the reference's per-pair and
// low-level entry points: STORM_bitmap_intersect_cardinality,
// STORM_bitmap_cont_intersect_cardinality, STORM_intersect_cardinality_square,
// STORM_intersect_vector16/32, STORM_intersect_bitmaps_scalar_list, the
// STORM_wrapper_* calls).  One non-blocking stream, the chunk engine, a dense
// engine and scratch buffers per device, created on the thread's first call
// and kept until the thread exits, so that a caller looping over pairs the
// reference's way (storm.cpp:936-940) pays one copy in, one launch and one
// copy out per call -- not a stream creation and device allocations.
#pragma once
#include "chunk_engine.cuh"
#include "dense.cuh"

namespace sb200 {

struct OneShot {
    cudaStream_t st = nullptr;
    ChunkPack pack;
    ChunkDev cdev;
    ChunkEngine engine;
    DenseEngine dense;
    DevBuf<uint64_t> w64;
    DevBuf<uint32_t> u32a, u32b, tri;
    DevBuf<int64_t> i64;
    DevBuf<DeviceFlags> flags;
    ~OneShot() {
        if (st) cudaStreamDestroy(st);
    }
    uint64_t read_sum(DeviceFlags* d) {
        DeviceFlags f;
        SB_CUDA(cudaMemcpyAsync(&f, d, sizeof(f), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        return f.sum;
    }
    // Sum over all (i < n1, n1 <= j < n1 + n2) of the rows in `pack`.
    uint64_t rect(uint64_t n1, uint64_t n2) {
        cdev.upload(pack, st);
        return engine.run(cdev, PAIRS_RECT, n1, n2, nullptr, st);
    }
};

// The calling thread's context on the current device (must be sm_100).
OneShot& one_shot();

}  // namespace sb200
