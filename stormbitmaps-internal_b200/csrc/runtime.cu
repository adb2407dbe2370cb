// runtime.cu -- device discovery, status strings, thread-local status.
#include "common.cuh"

#include <sched.h>

#include <mutex>
#include <thread>

namespace sb200 {

static thread_local int g_last_status = 0;
void set_last_status(int s) { g_last_status = s; }
int last_status() { return g_last_status; }

unsigned host_threads() {
    static const unsigned n = [] {
        cpu_set_t set;
        CPU_ZERO(&set);
        if (sched_getaffinity(0, sizeof(set), &set) == 0) {
            const int c = CPU_COUNT(&set);
            if (c > 0) return (unsigned)c;
        }
        const unsigned h = std::thread::hardware_concurrency();
        return h ? h : 1u;
    }();
    return n;
}

int require_device() {
    int dev = 0;
    SB_CUDA(cudaGetDevice(&dev));
    static std::mutex mu;
    static int cached_dev = -1, cached_sms = 0, cached_major = 0;
    std::lock_guard<std::mutex> lock(mu);
    if (cached_dev != dev) {
        cudaDeviceProp p;
        SB_CUDA(cudaGetDeviceProperties(&p, dev));
        cached_dev = dev;
        cached_sms = p.multiProcessorCount;
        cached_major = p.major;
    }
    if (cached_major != 10)
        fail(STORM_B200_ECUDA, "device is not an sm_100 (Blackwell B200) part; the kernels target sm_100a only");
    return cached_sms;
}

}  // namespace sb200

extern "C" {

const char* STORM_b200_strerror(int status) {
    switch (status) {
        case STORM_B200_OK: return "ok";
        case STORM_B200_ENULL: return "NULL handle";
        case STORM_B200_EVALUES: return "NULL values pointer";
        case STORM_B200_EARG: return "argument out of range or unsorted input";
        case STORM_B200_ENOMEM: return "host or device allocation failed";
        case STORM_B200_ECUDA: return "no usable sm_100 device, or a CUDA error";
        case STORM_B200_ETIMEOUT: return "a bounded device-side wait gave up";
        case STORM_B200_ESIZE: return "output buffer smaller than required";
        case STORM_B200_ELIMIT: return "problem exceeds a documented size limit";
        default: return status >= 0 ? "ok" : "unknown error";
    }
}

int STORM_b200_last_status(void) { return sb200::last_status(); }

}  // extern "C"
