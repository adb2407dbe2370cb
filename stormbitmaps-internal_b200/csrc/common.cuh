// common.cuh -- shared host/device plumbing of libstorm_b200.
//
// Error model: every CUDA call made on behalf of a C-ABI entry point is
// checked; a failure becomes a negative STORM_B200_E* status that the entry
// point returns (or records for STORM_b200_last_status when its reference
// signature returns a count).  No C++ exception crosses the C ABI: each entry
// point wraps its body in guard() (the same firewall idea as the reference's
// contiguous entry points, storm.cpp:1160-1169).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <new>
#include <stdexcept>
#include <atomic>
#include <string>

#include "../../include/storm.h"

namespace sb200 {

// Thrown inside the library only; converted to a status at the ABI edge.
struct Status : std::exception {
    int code;
    std::string what_;
    Status(int c, std::string w) : code(c), what_(std::move(w)) {}
    const char* what() const noexcept override { return what_.c_str(); }
};

void set_last_status(int s);
int last_status();

[[noreturn]] inline void fail(int code, const std::string& what) { throw Status(code, what); }

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? STORM_B200_ENOMEM : STORM_B200_ECUDA;
        fail(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
#define SB_CUDA(x) ::sb200::cuda_check((x), #x)

// Run `body` and turn any failure into a status code.
template <class F>
int guard(F&& body) {
    try {
        const int r = body();
        set_last_status(r < 0 ? r : STORM_B200_OK);
        return r;
    } catch (const Status& s) {
        set_last_status(s.code);
        return s.code;
    } catch (const std::bad_alloc&) {
        set_last_status(STORM_B200_ENOMEM);
        return STORM_B200_ENOMEM;
    } catch (...) {
        set_last_status(STORM_B200_ECUDA);
        return STORM_B200_ECUDA;
    }
}

// Host threads this process may run on (its CPU affinity set; at least 1):
// the width of the library's host-side packing and copying.
unsigned host_threads();

// Current device must be an sm_100 part (the kernels are built for sm_100a
// only).  Returns its SM count; throws ECUDA otherwise.
int require_device();

// Device buffer with RAII ownership.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // Grow to at least `count` elements (contents not preserved).
    void reserve(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) return;
        SB_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
        n = count;
    }
};

// Per-launch bookkeeping a handle keeps for measurement.
struct LaunchLog {
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    uint32_t launches = 0;
    int kernel = 0;
    void ensure() {
        if (!ev0) SB_CUDA(cudaEventCreate(&ev0));
        if (!ev1) SB_CUDA(cudaEventCreate(&ev1));
    }
    void destroy() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        ev0 = ev1 = nullptr;
    }
};

// Device error word the kernels write when a bounded wait gives up.
// Values: 0 ok, else (role << 16) | site.
struct DeviceFlags {
    unsigned int error;
    unsigned int pad;
    unsigned long long sum;   // sum over i < j accumulated by the epilogues
};

inline uint64_t tri_size(uint64_t n) { return n * (n + 1) / 2; }

// Raises a kernel's dynamic shared-memory limit once per device (the
// attribute is per device; `done` holds one bit per device ordinal).
template <class K>
inline void smem_attr_once(K* kernel, int bytes, std::atomic<uint64_t>& done) {
    int dev = 0;
    SB_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load() & bit) return;
    SB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    done.fetch_or(bit);
}

// Where the rows of an all-pairs launch are in device memory: word k of row
// r at X[r * pitch + (k >> 10) * kstride + (k & 1023)].  Row-major rows have
// kstride = 1024 (a row's 1024-word blocks follow each other); block-major
// panels keep block b of every row together (kstride = the words one block
// of all the panel's rows takes), so that the rows a tile reads at one K
// stage lie within a few pages instead of one page per row.
struct RowLayout {
    uint64_t pitch = 0;
    uint64_t kstride = 1024;
};
inline RowLayout row_major(uint64_t pitch) { return RowLayout{pitch, 1024}; }

}  // namespace sb200

// ---------------------------------------------------------------------------
// Device-side helpers shared by the kernels.
// ---------------------------------------------------------------------------
#ifdef __CUDACC__
namespace sb200 {

// The first word of 256-bit stage kb (4 words, never across a 1024-word
// block) of the row that starts at `row`.
__device__ __forceinline__ const uint64_t* stage_ptr(const uint64_t* row, uint32_t kb, uint64_t kstride) {
    return row + (uint64_t)(kb >> 8) * kstride + ((kb & 255u) << 2);
}

// Packed upper-triangle index, i <= j.
__device__ __forceinline__ uint64_t tri_index(uint64_t n, uint64_t i, uint64_t j) {
    return i * n - (i * (i - 1)) / 2 + (j - i);
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ uint32_t warp_sum_u32(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace sb200
#endif
