// Host-only check (no GPU): sb200::list16_blocked_count, the restatement of
// the reference's SSE4.2 list x list count that the chunk kernel runs for
// lists that are not strictly increasing, against the reference's own
// STORM_intersect_vector16_cardinality (oracle/_ref/libstorm_ref.so, built
// from the reference sources, loaded with dlopen). Seeded lists: sorted with
// repeats, unsorted, leading zeros, runs of one value, lengths around the
// 8-entry blocks. Prints "skip" when the reference library is not built.
// Built and run by test_list16_cpu.py with the library path as argv[1].
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

#include "list16_ref.cuh"

typedef uint64_t (*ref_fn)(const uint16_t*, const uint16_t*, uint32_t, uint32_t);

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    void* h = dlopen(argv[1], RTLD_NOW | RTLD_LOCAL);
    if (!h) {
        std::printf("skip\n");
        return 0;
    }
    ref_fn ref = (ref_fn)dlsym(h, "STORM_intersect_vector16_cardinality");
    if (!ref) {
        std::printf("skip\n");
        return 0;
    }
    std::mt19937_64 g(20261204);
    auto list = [&](uint32_t n, int kind) {
        std::vector<uint16_t> v(n);
        const uint32_t span = 1u + (uint32_t)(g() % 65536);
        for (auto& x : v) x = (uint16_t)(g() % span);
        if (kind == 0) std::sort(v.begin(), v.end());                 // sorted, repeats likely
        if (kind == 1) {                                                // sorted, each value 1-3 times
            std::sort(v.begin(), v.end());
            v.erase(std::unique(v.begin(), v.end()), v.end());
            std::vector<uint16_t> w;
            for (uint16_t x : v)
                for (uint32_t k = 0, r = 1 + (uint32_t)(g() % 3); k < r && w.size() < n; ++k) w.push_back(x);
            v = w;
        }
        if (kind == 3) {                                                // leading zeros, then sorted
            std::sort(v.begin(), v.end());
            for (uint32_t k = 0, z = (uint32_t)(g() % 20); k < z && k < v.size(); ++k) v[k] = 0;
            std::sort(v.begin(), v.end());
        }
        if (kind == 4) std::fill(v.begin(), v.end(), (uint16_t)(g() % 4));   // one value repeated
        return v;                                                       // kind 2: unsorted
    };
    uint64_t cases = 0, bad = 0;
    for (int it = 0; it < 20000; ++it) {
        const uint32_t n1 = (uint32_t)(g() % (it % 10 == 0 ? 4000 : 70)), n2 = (uint32_t)(g() % (it % 7 == 0 ? 4000 : 70));
        const int k1 = (int)(g() % 5), k2 = (int)(g() % 5);
        const std::vector<uint16_t> a = list(n1, k1), b = list(n2, k2);
        const uint16_t* pa = a.empty() ? nullptr : a.data();
        const uint16_t* pb = b.empty() ? nullptr : b.data();
        if (!pa || !pb) continue;
        const uint64_t want = ref(pa, pb, (uint32_t)a.size(), (uint32_t)b.size());
        const uint64_t got = sb200::list16_blocked_count(pa, pb, (uint32_t)a.size(), (uint32_t)b.size());
        ++cases;
        if (want != got) {
            if (bad < 5)
                std::printf("n1 %zu kind %d, n2 %zu kind %d: reference %llu, restatement %llu\n", a.size(), k1,
                            b.size(), k2, (unsigned long long)want, (unsigned long long)got);
            ++bad;
        }
    }
    std::printf("%llu cases, %llu differ\n", (unsigned long long)cases, (unsigned long long)bad);
    if (bad) return 1;
    std::printf("identical\n");
    return 0;
}
