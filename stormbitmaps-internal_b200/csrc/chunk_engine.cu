// chunk_engine.cu -- packing and the warp-per-pair kernel over 65536-bit
// chunks (layout and cell rules: chunk_engine.cuh).
#include <cmath>
#include "chunk_engine.cuh"

namespace sb200 {

void ChunkPack::add_chunk(uint32_t id, const STORM_bitmap_t& b) {
    cid.push_back(id);
    if (b.n_bitmap) {
        const uint32_t nw = b.n_bitmap < CHUNK_WORDS ? b.n_bitmap : CHUNK_WORDS;
        coff.push_back(bm.size());
        ckl.push_back(CK_BITMAP | nw);
        const size_t off = bm.size();
        bm.resize(off + CHUNK_WORDS, 0);
        if (b.data) std::copy(b.data, b.data + nw, bm.begin() + off);
    } else {
        const uint32_t ns = b.scalar ? b.n_scalar : 0;
        // Lists start on a 16-byte boundary.
        while (lst.size() % 8) lst.push_back(0);
        coff.push_back(lst.size());
        uint32_t flags = ns & CK_LEN;
        for (uint32_t e = 1; e < ns; ++e)
            if (b.scalar[e] == b.scalar[e - 1]) { flags |= CK_DUP; break; }
        ckl.push_back(flags);
        lst.insert(lst.end(), b.scalar, b.scalar + ns);
    }
}

void ChunkPack::add_row(const STORM_bitmap_cont_t* c) {
    if (c && c->bitmaps && c->block_ids)
        for (uint32_t k = 0; k < c->n_bitmaps; ++k) add_chunk(c->block_ids[k], c->bitmaps[k]);
    end_row();
}

template <class T>
static void put(DevBuf<T>& d, const std::vector<T>& h, cudaStream_t st) {
    d.reserve(h.size() ? h.size() : 1);
    if (!h.empty()) SB_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

void ChunkDev::upload(const ChunkPack& p, cudaStream_t st) {
    put(row_off, p.row_off, st);
    put(cid, p.cid, st);
    put(ckl, p.ckl, st);
    put(coff, p.coff, st);
    put(bm, p.bm, st);
    put(lst, p.lst, st);
    n_rows = p.rows();
    SB_CUDA(cudaStreamSynchronize(st));
}

template <class T>
__device__ __forceinline__ uint32_t lower_bound_dev(const T* a, uint32_t n, T x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// This lane's share of |chunk ca & chunk cb| (warp-cooperative; every lane
// must call it with the same ca, cb).
__device__ __forceinline__ uint32_t chunk_cell_lane(const ChunkView& v, uint64_t ca, uint64_t cb, int lane) {
    const uint32_t ka = v.ckl[ca], kb = v.ckl[cb];
    const bool ba = (ka & CK_BITMAP) != 0, bb = (kb & CK_BITMAP) != 0;
    uint32_t cnt = 0;
    if (ba && bb) {
        const uint64_t* wa = v.bm + v.coff[ca];
        const uint64_t* wb = v.bm + v.coff[cb];
        const uint32_t nw = ka & CK_LEN;   // the reference counts bitmap1->n_bitmap words
        for (uint32_t w = lane; w < nw; w += 32) cnt += __popcll(wa[w] & wb[w]);
    } else if (ba || bb) {
        const uint64_t* w = v.bm + v.coff[ba ? ca : cb];
        const uint32_t kl = ba ? kb : ka;
        const uint16_t* l = v.lst + v.coff[ba ? cb : ca];
        const uint32_t nl = kl & CK_LEN;
        for (uint32_t e = lane; e < nl; e += 32) {
            const uint32_t x = l[e];
            cnt += (uint32_t)(w[x >> 6] >> (x & 63)) & 1u;
        }
    } else {
        const uint32_t la = ka & CK_LEN, lb = kb & CK_LEN;
        const bool a_short = la <= lb;
        const uint16_t* s = v.lst + v.coff[a_short ? ca : cb];
        const uint16_t* g = v.lst + v.coff[a_short ? cb : ca];
        const uint32_t ns = a_short ? la : lb, ng = a_short ? lb : la;
        const bool sdup = ((a_short ? ka : kb) & CK_DUP) != 0;
        for (uint32_t e = lane; e < ns; e += 32) {
            const uint16_t x = s[e];
            const uint32_t r = sdup ? e - lower_bound_dev<uint16_t>(s, e, x) : 0;
            const uint32_t p = lower_bound_dev<uint16_t>(g, ng, x) + r;
            cnt += (p < ng && g[p] == x) ? 1u : 0u;
        }
    }
    return cnt;
}

// Row start S(i) = i*n - i(i-1)/2 of the packed triangle; p -> (i, j).
__device__ __forceinline__ void tri_decode(uint64_t n, uint64_t p, uint64_t& i, uint64_t& j) {
    const double b = 2.0 * (double)n + 1.0;
    double x = (b - sqrt(b * b - 8.0 * (double)p)) * 0.5;
    int64_t ii = (int64_t)x;
    if (ii < 0) ii = 0;
    if ((uint64_t)ii >= n) ii = (int64_t)n - 1;
    auto S = [n](uint64_t r) { return r * n - (r * (r - 1)) / 2; };
    while (ii > 0 && S((uint64_t)ii) > p) --ii;
    while ((uint64_t)ii + 1 < n && S((uint64_t)ii + 1) <= p) ++ii;
    i = (uint64_t)ii;
    j = p - S(i) + i;
}

__global__ void __launch_bounds__(256)
chunk_pairs_kernel(ChunkView v, uint32_t mode, uint64_t n1, uint64_t n2, uint64_t n_pairs,
                   uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags) {
    const int lane = threadIdx.x & 31;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long local = 0;
    for (uint64_t p = wid; p < n_pairs; p += nwarps) {
        uint64_t i, j;
        if (mode == PAIRS_TRIANGLE) tri_decode(n1, p, i, j);
        else {
            i = p / n2;
            j = n1 + p % n2;
        }
        const uint64_t a0 = v.row_off[i], b0 = v.row_off[j];
        const uint32_t na = (uint32_t)(v.row_off[i + 1] - a0), nb = (uint32_t)(v.row_off[j + 1] - b0);
        const bool a_short = na <= nb;
        const uint64_t s0 = a_short ? a0 : b0, l0 = a_short ? b0 : a0;
        const uint32_t ns = a_short ? na : nb, nl = a_short ? nb : na;
        uint32_t cnt = 0;
        for (uint32_t base = 0; base < ns; base += 32) {
            const uint32_t e = base + lane;
            int32_t match = -1;
            if (e < ns) {
                const uint32_t id = v.cid[s0 + e];
                uint32_t r = 0;
                if (e > 0 && v.cid[s0 + e - 1] == id) r = e - lower_bound_dev<uint32_t>(v.cid + s0, e, id);
                const uint32_t q = lower_bound_dev<uint32_t>(v.cid + l0, nl, id) + r;
                if (q < nl && v.cid[l0 + q] == id) match = (int32_t)q;
            }
            uint32_t mask = __ballot_sync(0xffffffffu, match >= 0);
            while (mask) {
                const int src = __ffs(mask) - 1;
                mask &= mask - 1;
                const uint32_t q = (uint32_t)__shfl_sync(0xffffffffu, match, src);
                const uint64_t cs = s0 + base + (uint32_t)src, cl = l0 + q;
                // Row i's chunk is the first argument, as in the reference.
                cnt += a_short ? chunk_cell_lane(v, cs, cl, lane) : chunk_cell_lane(v, cl, cs, lane);
            }
        }
        cnt = warp_sum_u32(cnt);
        if (lane == 0) {
            if (mode == PAIRS_TRIANGLE) {
                if (out) out[tri_index(n1, i, j)] = cnt;
                if (j > i) local += cnt;
            } else {
                local += cnt;
            }
        }
    }
    if (lane == 0 && local) atomicAdd(&flags->sum, local);
}

uint64_t ChunkEngine::run(const ChunkDev& d, PairMode mode, uint64_t n1, uint64_t n2, uint32_t* d_out,
                          cudaStream_t st) {
    const int sms = require_device();
    const uint64_t n_pairs = mode == PAIRS_TRIANGLE ? tri_size(n1) : n1 * n2;
    log.launches = 0;
    log.last_ms = 0.f;
    if (n_pairs == 0) return 0;
    d_flags.reserve(1);
    SB_CUDA(cudaMemsetAsync(d_flags.p, 0, sizeof(DeviceFlags), st));
    log.ensure();
    const uint64_t want_blocks = (n_pairs + 7) / 8;
    const uint32_t grid = (uint32_t)(want_blocks < (uint64_t)sms * 16 ? want_blocks : (uint64_t)sms * 16);
    SB_CUDA(cudaEventRecord(log.ev0, st));
    chunk_pairs_kernel<<<grid, 256, 0, st>>>(d.view(), (uint32_t)mode, n1, n2, n_pairs, d_out, d_flags.p);
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaEventRecord(log.ev1, st));
    DeviceFlags f;
    SB_CUDA(cudaMemcpyAsync(&f, d_flags.p, sizeof(f), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    SB_CUDA(cudaEventElapsedTime(&log.last_ms, log.ev0, log.ev1));
    log.launches = 1;
    return f.sum;
}

}  // namespace sb200
