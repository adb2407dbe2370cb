// chunk_engine.cu -- packing and the warp-per-pair kernel over 65536-bit
// chunks (layout and cell rules: chunk_engine.cuh).
#include <cmath>
#include <algorithm>
#include "chunk_engine.cuh"
#include "dense.cuh"

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
    ChunkRowFacts f;
    if (c && c->bitmaps && c->block_ids) {
        for (uint32_t k = 0; k < c->n_bitmaps; ++k) {
            const STORM_bitmap_t& b = c->bitmaps[k];
            const uint32_t id = c->block_ids[k];
            add_chunk(id, b);
            ++f.chunks;
            if (k > 0 && id <= c->block_ids[k - 1]) f.plain = false;
            if (b.n_bitmap) {
                if (b.n_bitmap != CHUNK_WORDS || b.data == NULL) f.plain = false;
                f.card += b.n_bits_set;
                ++f.bitmap_chunks;
            } else {
                if (ckl.back() & CK_DUP) f.plain = false;
                const uint32_t ns = b.scalar ? b.n_scalar : 0;
                f.card += ns;
                f.list_entries += ns;
            }
            if (id > max_cid) max_cid = id;
        }
    }
    facts.push_back(f);
    end_row();
}

double chunk_self_pair_ns(const ChunkCostModel& m, const ChunkRowFacts& f, uint64_t slots) {
    if (f.chunks == 0 || slots == 0) return 0.0;
    const uint32_t lists = f.chunks - f.bitmap_chunks;
    double iters = 32.0 * f.bitmap_chunks;
    if (lists) {
        const double e = std::max(1.0, (double)f.list_entries / lists);
        iters += lists * std::ceil(e / 32.0) * (std::log2(e) + 1.0);
    }
    const double shared = (double)f.chunks * f.chunks / (double)slots;
    return shared * (m.ns_per_shared_chunk + m.ns_per_lane_iteration * iters / f.chunks);
}

double tensor_pair_ns(const ChunkCostModel& m, uint64_t slots) { return m.ns_per_tensor_bit * 65536.0 * slots; }

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
    facts = p.facts;
    max_cid = p.max_cid;
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

// Expands plain rows into contiguous bitmaps: local row r of X (W words,
// W = 1024 x chunk slots) is row rows[r]. One CTA per row, a warp per chunk
// slot: absent chunks become zeros, bitmap chunks are copied, list chunks
// are set bit by bit in a shared-memory copy of the chunk and written out.
constexpr int EXPAND_WARPS = 4;

__global__ void __launch_bounds__(EXPAND_WARPS * 32)
expand_rows_kernel(ChunkView v, const uint32_t* __restrict__ rows, uint32_t m, uint32_t W,
                   uint64_t* __restrict__ X) {
    __shared__ __align__(16) unsigned long long chunk[EXPAND_WARPS][CHUNK_WORDS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t slots = W / CHUNK_WORDS;
    for (uint32_t r = blockIdx.x; r < m; r += gridDim.x) {
        const uint32_t row = rows[r];
        const uint64_t c0 = v.row_off[row], c1 = v.row_off[row + 1];
        uint4* dst_row = reinterpret_cast<uint4*>(X + (uint64_t)r * W);
        uint64_t pos = c0;
        for (uint32_t s = warp; s < slots; s += EXPAND_WARPS) {
            while (pos < c1 && v.cid[pos] < s) ++pos;   // ids ascend: a forward walk
            uint4* dst = dst_row + (uint64_t)s * (CHUNK_WORDS / 2);
            if (pos >= c1 || v.cid[pos] != s) {
                for (uint32_t q = lane; q < CHUNK_WORDS / 2; q += 32) dst[q] = make_uint4(0, 0, 0, 0);
                continue;
            }
            const uint32_t k = v.ckl[pos];
            if (k & CK_BITMAP) {
                const uint4* src = reinterpret_cast<const uint4*>(v.bm + v.coff[pos]);
                for (uint32_t q = lane; q < CHUNK_WORDS / 2; q += 32) dst[q] = __ldg(src + q);
            } else {
                unsigned long long* cw = chunk[warp];
                for (uint32_t q = lane; q < CHUNK_WORDS; q += 32) cw[q] = 0ull;
                __syncwarp();
                const uint16_t* l = v.lst + v.coff[pos];
                const uint32_t nl = k & CK_LEN;
                for (uint32_t e = lane; e < nl; e += 32) {
                    const uint32_t x = l[e];
                    atomicOr(&cw[x >> 6], 1ull << (x & 63));
                }
                __syncwarp();
                const uint4* src = reinterpret_cast<const uint4*>(cw);
                for (uint32_t q = lane; q < CHUNK_WORDS / 2; q += 32) dst[q] = src[q];
                __syncwarp();
            }
        }
    }
}

// perm (optional) maps the walk's row index to the stored row: with the
// dense block on, the sparse rows come first and the walk stops after the
// pairs whose first row is sparse.
__global__ void __launch_bounds__(256)
chunk_pairs_kernel(ChunkView v, uint32_t mode, uint64_t n1, uint64_t n2, uint64_t n_pairs,
                   const uint32_t* __restrict__ perm, uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags) {
    const int lane = threadIdx.x & 31;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long local = 0;
    for (uint64_t p = wid; p < n_pairs; p += nwarps) {
        uint64_t i, j;
        if (mode == PAIRS_TRIANGLE) {
            tri_decode(n1, p, i, j);
            if (perm) {
                const uint64_t a = perm[i], b = perm[j];
                i = a < b ? a : b;
                j = a < b ? b : a;
            }
        } else {
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
    const uint64_t n_pairs_all = mode == PAIRS_TRIANGLE ? tri_size(n1) : n1 * n2;
    log.launches = 0;
    log.last_ms = 0.f;
    last_dense_rows = last_dense_panels = 0;
    if (n_pairs_all == 0) return 0;
    d_flags.reserve(1);
    SB_CUDA(cudaMemsetAsync(d_flags.p, 0, sizeof(DeviceFlags), st));
    log.ensure();

    // ---- dense block plan (triangle walks only)
    std::vector<uint32_t> dense;
    const uint64_t slots = (uint64_t)d.max_cid + 1;
    const uint64_t W = slots * CHUNK_WORDS;               // words per expanded row
    uint64_t P = 0;                                        // rows per panel
    bool single = false;
    if (mode == PAIRS_TRIANGLE && dense_min_density != 0.0 && slots * 65536 <= TC_MAX_ROW_BITS &&
        n1 >= 256 && d.facts.size() == n1) {
        const double min_card = dense_min_density * (double)(slots * 65536);
        const double tc_ns = tensor_pair_ns(cost, slots);
        for (uint32_t r = 0; r < n1; ++r) {
            const ChunkRowFacts& f = d.facts[r];
            if (!f.plain) continue;
            const bool joins = dense_min_density > 0.0 ? (double)f.card >= min_card
                                                       : chunk_self_pair_ns(cost, f, slots) >= tc_ns;
            if (joins) dense.push_back(r);
        }
        if (dense.size() >= 256) {
            uint64_t budget = dense_budget_bytes;
            if (!budget) {
                size_t fr = 0, tot = 0;
                SB_CUDA(cudaMemGetInfo(&fr, &tot));
                budget = (uint64_t)(0.6 * (double)(fr + d_panel.n * sizeof(uint64_t)));
            }
            const uint64_t cap_rows = budget / (W * sizeof(uint64_t));
            if (round_up(dense.size(), 256) <= cap_rows) {
                single = true;
                P = round_up(dense.size(), 256);
            } else {
                P = cap_rows / 2 / 256 * 256;
            }
        }
        if (P == 0) dense.clear();
    }
    const uint64_t nd = dense.size();

    SB_CUDA(cudaEventRecord(log.ev0, st));
    uint32_t launches = 0;
    const uint32_t* perm = nullptr;
    uint64_t n_pairs = n_pairs_all;
    if (nd) {
        // Walk order: sparse rows first, then the dense rows; the chunk
        // kernel stops after the pairs whose first row is sparse.
        std::vector<uint32_t> h_perm;
        h_perm.reserve(n1);
        std::vector<uint8_t> is_dense(n1, 0);
        for (uint32_t r : dense) is_dense[r] = 1;
        for (uint32_t r = 0; r < n1; ++r)
            if (!is_dense[r]) h_perm.push_back(r);
        const uint64_t ns = h_perm.size();
        h_perm.insert(h_perm.end(), dense.begin(), dense.end());
        d_perm.reserve(n1);
        SB_CUDA(cudaMemcpyAsync(d_perm.p, h_perm.data(), n1 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        perm = d_perm.p;
        n_pairs = ns * n1 - (ns * (ns - 1)) / 2 * (ns ? 1 : 0);

        const uint64_t rows_alloc = single ? P : 2 * P;
        d_panel.reserve(rows_alloc * W);
        d_map.reserve(rows_alloc);
        // every tile list below fits: (P / 128) row blocks x (2P / 256) column blocks
        d_tiles.reserve((P / 128) * (2 * P / 256 + 1));
        // Split-K tensor launches add partial counts: zero the triangle once.
        if (d_out) SB_CUDA(cudaMemsetAsync(d_out, 0, tri_size(n1) * sizeof(uint32_t), st));
        const uint64_t npan = single ? 1 : (nd + P - 1) / P;
        std::vector<uint2> tl;
        auto expand = [&](uint64_t first, uint64_t m, uint64_t slot) {
            SB_CUDA(cudaMemcpyAsync(d_map.p + slot, dense.data() + first, m * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice, st));
            const uint32_t grid = (uint32_t)std::min<uint64_t>(m, (uint64_t)sms * 16);
            expand_rows_kernel<<<grid, EXPAND_WARPS * 32, 0, st>>>(d.view(), d_map.p + slot, (uint32_t)m,
                                                                   (uint32_t)W, d_panel.p + slot * W);
            SB_CUDA(cudaGetLastError());
            ++launches;
        };
        auto tensor = [&](uint64_t n_local) {
            SB_CUDA(cudaMemcpyAsync(d_tiles.p, tl.data(), tl.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
            launch_ts_rows(d_panel.p, (uint32_t)n_local, (uint32_t)W, d_tiles.p, (uint32_t)tl.size(), d_out,
                           d_flags.p, d_map.p, n1, st, /*out_zeroed=*/true);
            ++launches;
        };
        for (uint64_t I = 0; I < npan; ++I) {
            const uint64_t mI = std::min<uint64_t>(P, nd - I * P);
            expand(I * P, mI, 0);
            build_mma_tiles(tl, mI);                       // I x I triangle
            tensor(mI);
            for (uint64_t J = I + 1; J < npan; ++J) {        // I x J rectangle (I is a full panel)
                const uint64_t mJ = std::min<uint64_t>(P, nd - J * P);
                expand(J * P, mJ, P);
                tl.clear();
                for (uint32_t bi = 0; bi < P / 128; ++bi)
                    for (uint32_t bj = (uint32_t)(P / 256); bj < (uint32_t)((P + mJ + 255) / 256); ++bj)
                        tl.push_back(make_uint2(bi, bj));
                tensor(P + mJ);
            }
        }
        last_dense_rows = nd;
        last_dense_panels = npan;
    }
    if (n_pairs) {
        const uint64_t want_blocks = (n_pairs + 7) / 8;
        const uint32_t grid = (uint32_t)(want_blocks < (uint64_t)sms * 16 ? want_blocks : (uint64_t)sms * 16);
        chunk_pairs_kernel<<<grid, 256, 0, st>>>(d.view(), (uint32_t)mode, n1, n2, n_pairs, perm, d_out,
                                                  d_flags.p);
        SB_CUDA(cudaGetLastError());
        ++launches;
    }
    SB_CUDA(cudaEventRecord(log.ev1, st));
    DeviceFlags f;
    SB_CUDA(cudaMemcpyAsync(&f, d_flags.p, sizeof(f), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    if (f.error) fail(STORM_B200_ETIMEOUT, "tensor-core dense block: a pipeline wait timed out");
    SB_CUDA(cudaEventElapsedTime(&log.last_ms, log.ev0, log.ev1));
    log.launches = launches;
    return f.sum;
}

}  // namespace sb200
