// chunk_engine.cu -- packing and the warp-per-pair kernel over 65536-bit
// chunks (layout and cell rules: chunk_engine.cuh).
#include <cmath>
#include <cstring>
#include <algorithm>
#include <exception>
#include <mutex>
#include <thread>
#include "chunk_engine.cuh"
#include "dense.cuh"
#include "list16_ref.cuh"
#include "panel.cuh"
#include "run_pieces.cuh"

namespace sb200 {

// Maximal runs of set bits of a bitmap chunk (its words as stored).
static uint64_t bitmap_runs(const STORM_bitmap_t& b) {
    if (!b.data) return 0;
    const uint32_t nw = b.n_bitmap < CHUNK_WORDS ? b.n_bitmap : CHUNK_WORDS;
    uint64_t runs = 0, carry = 0;
    for (uint32_t w = 0; w < nw; ++w) {
        const uint64_t x = b.data[w];
        runs += (uint64_t)__builtin_popcountll(x & ~((x << 1) | carry));
        carry = x >> 63;
    }
    return runs;
}

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
            if (b.scalar[e] <= b.scalar[e - 1]) { flags |= CK_DUP; break; }
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
                f.runs += bitmap_runs(b);
            } else {
                if (ckl.back() & CK_DUP) f.plain = false;
                const uint32_t ns = b.scalar ? b.n_scalar : 0;
                f.card += ns;
                f.list_entries += ns;
                for (uint32_t e = 0; e < ns; ++e) f.runs += e == 0 || b.scalar[e] != b.scalar[e - 1] + 1;
            }
            if (id > max_cid) max_cid = id;
        }
    }
    facts.push_back(f);
    end_row();
}

void ChunkPack::add_rows(const STORM_bitmap_cont_t* rows, uint64_t n) {
    if (n == 0) return;
    auto live = [&](uint64_t r) { return rows[r].bitmaps && rows[r].block_ids ? rows[r].n_bitmaps : 0u; };
    // Pass 1: every row's chunk count, bitmap chunks and list slots (each
    // list starts on a multiple of 8 entries, as add_chunk places them).
    std::vector<uint64_t> c_base(n + 1), b_base(n + 1), l_base(n + 1);
    std::vector<uint64_t> l_used(n);
    std::vector<uint8_t> has_list(n);
    for (uint64_t r = 0; r < n; ++r) {
        const uint32_t k_n = live(r);
        uint64_t nb = 0, pos = 0;
        bool lists = false;
        for (uint32_t k = 0; k < k_n; ++k) {
            const STORM_bitmap_t& b = rows[r].bitmaps[k];
            if (b.n_bitmap) {
                ++nb;
            } else {
                pos = (pos + 7) / 8 * 8 + (b.scalar ? b.n_scalar : 0);
                lists = true;
            }
        }
        c_base[r + 1] = c_base[r] + k_n;
        b_base[r + 1] = b_base[r] + nb * CHUNK_WORDS;
        l_used[r] = pos;
        has_list[r] = lists;
        l_base[r + 1] = l_base[r] + (pos + 7) / 8 * 8;
    }
    // Global placement: appended after what the pack already holds.
    const uint64_t c0 = cid.size(), b0 = bm.size();
    uint64_t last_list_row = n;
    for (uint64_t r = n; r-- > 0;)
        if (has_list[r]) {
            last_list_row = r;
            break;
        }
    const uint64_t l0 = last_list_row < n ? (lst.size() + 7) / 8 * 8 : lst.size();
    const uint64_t l_end = last_list_row < n ? l0 + l_base[last_list_row] + l_used[last_list_row] : lst.size();
    cid.resize(c0 + c_base[n]);
    ckl.resize(c0 + c_base[n]);
    coff.resize(c0 + c_base[n]);
    bm.resize(b0 + b_base[n]);
    lst.resize(l_end, 0);   // padding between lists stays zero
    std::vector<ChunkRowFacts> fr(n);
    std::vector<uint32_t> row_max(n, 0);
    // Pass 2: fill, rows split over threads by the bytes they copy.
    auto fill = [&](uint64_t r0, uint64_t r1) {
        for (uint64_t r = r0; r < r1; ++r) {
            ChunkRowFacts f;
            uint32_t mx = 0;
            uint64_t c = c0 + c_base[r], w = b0 + b_base[r], pos = 0;
            const uint64_t lb = l0 + l_base[r];
            const uint32_t k_n = live(r);
            for (uint32_t k = 0; k < k_n; ++k, ++c) {
                const STORM_bitmap_t& b = rows[r].bitmaps[k];
                const uint32_t id = rows[r].block_ids[k];
                cid[c] = id;
                ++f.chunks;
                if (k > 0 && id <= rows[r].block_ids[k - 1]) f.plain = false;
                if (b.n_bitmap) {
                    const uint32_t nw = b.n_bitmap < CHUNK_WORDS ? b.n_bitmap : CHUNK_WORDS;
                    coff[c] = w;
                    ckl[c] = CK_BITMAP | nw;
                    uint64_t* dst = bm.data() + w;
                    const uint32_t copied = b.data ? nw : 0;
                    if (copied) std::memcpy(dst, b.data, copied * sizeof(uint64_t));
                    std::memset(dst + copied, 0, (CHUNK_WORDS - copied) * sizeof(uint64_t));
                    w += CHUNK_WORDS;
                    if (b.n_bitmap != CHUNK_WORDS || b.data == NULL) f.plain = false;
                    f.card += b.n_bits_set;
                    ++f.bitmap_chunks;
                    f.runs += bitmap_runs(b);
                } else {
                    const uint32_t ns = b.scalar ? b.n_scalar : 0;
                    pos = (pos + 7) / 8 * 8;
                    coff[c] = lb + pos;
                    uint32_t flags = ns & CK_LEN;
                    for (uint32_t e = 0; e < ns; ++e) {
                        if (e && b.scalar[e] <= b.scalar[e - 1]) flags |= CK_DUP;
                        f.runs += e == 0 || b.scalar[e] != b.scalar[e - 1] + 1;
                    }
                    ckl[c] = flags;
                    if (ns) std::memcpy(lst.data() + lb + pos, b.scalar, ns * sizeof(uint16_t));
                    pos += ns;
                    if (flags & CK_DUP) f.plain = false;
                    f.card += ns;
                    f.list_entries += ns;
                }
                if (id > mx) mx = id;
            }
            fr[r] = f;
            row_max[r] = mx;
        }
    };
    const uint64_t work = b_base[n] * 8 + l_base[n] * 2 + c_base[n] * 16;
    const unsigned hw = host_threads();
    const uint64_t n_thr = std::min<uint64_t>({(uint64_t)std::min(hw, 32u), n, 1 + work / (8u << 20)});
    if (n_thr <= 1) {
        fill(0, n);
    } else {
        // contiguous row ranges of about equal bytes
        std::vector<uint64_t> cut{0};
        uint64_t acc = 0;
        for (uint64_t r = 0; r < n && cut.size() < n_thr; ++r) {
            acc += (b_base[r + 1] - b_base[r]) * 8 + (l_base[r + 1] - l_base[r]) * 2 +
                   (c_base[r + 1] - c_base[r]) * 16;
            if (acc * n_thr >= work * cut.size()) cut.push_back(r + 1);
        }
        if (cut.back() != n) cut.push_back(n);
        std::vector<std::thread> th;
        for (size_t t = 0; t + 1 < cut.size(); ++t)
            if (cut[t] < cut[t + 1]) th.emplace_back(fill, cut[t], cut[t + 1]);
        for (auto& t : th) t.join();
    }
    for (uint64_t r = 0; r < n; ++r) {
        facts.push_back(fr[r]);
        row_off.push_back(c0 + c_base[r + 1]);
        if (row_max[r] > max_cid) max_cid = row_max[r];
    }
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

template <class T, class A>
static void put(DevBuf<T>& d, const std::vector<T, A>& h, cudaStream_t st) {
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

PinnedStage::~PinnedStage() {
    for (Lane& l : lanes) {
        if (l.st) {
            cudaStreamSynchronize(l.st);
            cudaStreamDestroy(l.st);
        }
        for (cudaEvent_t e : l.done)
            if (e) cudaEventDestroy(e);
    }
    if (ready) cudaEventDestroy(ready);
    if (pool) cudaFreeHost(pool);
}

void PinnedStage::ensure() {
    if (pool) return;
    const unsigned w = std::max(1u, std::min(64u, host_threads()));
    SB_CUDA(cudaHostAlloc((void**)&pool, TOTAL, cudaHostAllocDefault));
    lane_bytes = TOTAL / (2 * w) / 4096 * 4096;   // >= 1 MiB: any chunk's payload fits
    lanes.resize(w);
    for (unsigned t = 0; t < w; ++t) {
        Lane& l = lanes[t];
        l.buf[0] = pool + (2 * (uint64_t)t) * lane_bytes;
        l.buf[1] = l.buf[0] + lane_bytes;
        SB_CUDA(cudaStreamCreateWithFlags(&l.st, cudaStreamNonBlocking));
        for (cudaEvent_t& e : l.done) SB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    SB_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
}

// Waits for a lane's stream when a worker leaves, also by an exception, so
// that no copy of a failed call still reads or writes the lane's buffers
// when the next call fills them.
struct LaneSync {
    cudaStream_t st;
    ~LaneSync() { cudaStreamSynchronize(st); }
};

// Runs fn(t) for t in [0, workers) on that many host threads (t = 0 on the
// calling thread) and rethrows the first failure after all have ended.
template <class F>
static void run_workers(unsigned workers, F fn) {
    std::mutex mu;
    std::exception_ptr first;
    auto body = [&](unsigned t) {
        try {
            fn(t);
        } catch (...) {
            std::lock_guard<std::mutex> lock(mu);
            if (!first) first = std::current_exception();
        }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < workers; ++t) th.emplace_back(body, t);
    body(0);
    for (auto& t : th) t.join();
    if (first) std::rethrow_exception(first);
}

// Splits [0, n) into at most `parts` contiguous ranges of about equal weight
// (prefix[r] = weight of rows before r) and runs fn(r0, r1) on each, one
// host thread per range.
template <class F>
static void parallel_rows(uint64_t n, const std::vector<uint64_t>& prefix, unsigned parts, F fn) {
    if (n == 0) return;
    const uint64_t total = prefix[n];
    const uint64_t k = std::max<uint64_t>(1, std::min<uint64_t>({(uint64_t)parts, n, 1 + total / (4u << 20)}));
    if (k <= 1) {
        fn((uint64_t)0, n);
        return;
    }
    std::vector<uint64_t> cut{0};
    for (uint64_t r = 0; r < n && cut.size() < k; ++r)
        if (prefix[r + 1] * k >= total * cut.size()) cut.push_back(r + 1);
    if (cut.back() != n) cut.push_back(n);
    run_workers((unsigned)(cut.size() - 1), [&](unsigned t) { fn(cut[t], cut[t + 1]); });
}

// Lists are not necessarily strictly increasing in the public layout (a
// repeated value, or values added out of order): one warp per chunk tests a
// list's entries, flags the chunk CK_DUP and marks its row; and counts the
// chunk's maximal runs of consecutive values into its row.
__global__ void list_order_kernel(const uint64_t* __restrict__ row_off, uint64_t n_rows, uint32_t* __restrict__ ckl,
                                  const uint64_t* __restrict__ coff, const uint16_t* __restrict__ lst,
                                  const uint64_t* __restrict__ bm, uint64_t nc, uint8_t* __restrict__ row_dup,
                                  uint32_t* __restrict__ row_runs) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t c = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nc; c += warps) {
        const uint32_t k = ckl[c];
        const uint32_t len = k & CK_LEN;
        if (len == 0) continue;
        bool bad = false;
        uint32_t runs = 0;   // maximal runs of consecutive values (the run sweep's pieces)
        if (k & CK_BITMAP) {
            // run starts: set bits whose lower neighbour is clear
            const uint64_t* wd = bm + coff[c];
            uint64_t carry = 0;
            for (uint32_t w0 = 0; w0 < len; w0 += 32) {
                const uint32_t wi = w0 + lane;
                const uint64_t x = wi < len ? wd[wi] : 0ull;
                const uint64_t prev = __shfl_up_sync(0xffffffffu, x, 1);
                const uint64_t cin = lane ? prev >> 63 : carry;
                carry = __shfl_sync(0xffffffffu, x, 31) >> 63;
                runs += warp_sum_u32((uint32_t)__popcll(x & ~((x << 1) | cin)));
            }
        } else {
            const uint16_t* l = lst + coff[c];
            for (uint32_t e0 = 0; e0 < len; e0 += 32) {
                const uint32_t e = e0 + lane;
                const bool in = e < len;
                bad |= __any_sync(0xffffffffu, in && e > 0 && l[e] <= l[e - 1]);
                runs += __popc(__ballot_sync(0xffffffffu, in && (e == 0 || l[e] != l[e - 1] + 1)));
            }
        }
        if (lane == 0) {
            uint64_t lo = 0, hi = n_rows;   // the row r with row_off[r] <= c < row_off[r + 1]
            while (lo + 1 < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (row_off[mid] <= c) lo = mid;
                else hi = mid;
            }
            if (bad) {
                ckl[c] = k | CK_DUP;
                row_dup[lo] = 1;
            }
            atomicAdd(&row_runs[lo], runs);
        }
    }
}

void ChunkDev::upload_rows(const STORM_bitmap_cont_t* rows, uint64_t n, cudaStream_t st, PinnedStage& stage) {
    const unsigned hw = std::max(1u, std::min(64u, host_threads()));
    auto live = [&](uint64_t r) { return rows[r].bitmaps && rows[r].block_ids ? rows[r].n_bitmaps : 0u; };
    // Pass 1: per row its chunk count, bitmap words, list slots (each list on
    // a multiple of 8 entries, as ChunkPack places them) and facts; the
    // lists' order is tested on the device below.
    std::vector<uint64_t> c_base(n + 1, 0), b_base(n + 1, 0), l_base(n + 1, 0), w1(n + 1, 0);
    std::vector<uint32_t> row_max(n, 0);
    facts.assign(n, ChunkRowFacts{});
    for (uint64_t r = 0; r < n; ++r) w1[r + 1] = w1[r] + 1 + live(r);
    parallel_rows(n, w1, hw, [&](uint64_t r0, uint64_t r1) {
        for (uint64_t r = r0; r < r1; ++r) {
            ChunkRowFacts f;
            uint64_t nb = 0, pos = 0;
            uint32_t mx = 0;
            const uint32_t k_n = live(r);
            for (uint32_t k = 0; k < k_n; ++k) {
                const STORM_bitmap_t& b = rows[r].bitmaps[k];
                const uint32_t id = rows[r].block_ids[k];
                ++f.chunks;
                if (k > 0 && id <= rows[r].block_ids[k - 1]) f.plain = false;
                if (b.n_bitmap) {
                    ++nb;
                    if (b.n_bitmap != CHUNK_WORDS || b.data == NULL) f.plain = false;
                    f.card += b.n_bits_set;
                    ++f.bitmap_chunks;
                } else {
                    const uint32_t ns = b.scalar ? b.n_scalar : 0;
                    pos = (pos + 7) / 8 * 8 + ns;
                    f.card += ns;
                    f.list_entries += ns;
                }
                if (id > mx) mx = id;
            }
            facts[r] = f;
            row_max[r] = mx;
            c_base[r + 1] = k_n;
            b_base[r + 1] = nb * CHUNK_WORDS;
            l_base[r + 1] = (pos + 7) / 8 * 8;
        }
    });
    max_cid = 0;
    for (uint64_t r = 0; r < n; ++r) {
        c_base[r + 1] += c_base[r];
        b_base[r + 1] += b_base[r];
        l_base[r + 1] += l_base[r];
        max_cid = std::max(max_cid, row_max[r]);
    }
    n_rows = n;
    const uint64_t nc = c_base[n], nbw = b_base[n], nl = l_base[n];
    payload_bytes = nbw * 8 + nl * 2;
    // Pass 2: chunk metadata on host threads, then to the device.
    std::vector<uint64_t> h_row_off(n + 1);
    std::vector<uint32_t, NoInitAlloc<uint32_t>> h_cid(nc), h_ckl(nc);
    std::vector<uint64_t, NoInitAlloc<uint64_t>> h_coff(nc);
    for (uint64_t r = 0; r <= n; ++r) h_row_off[r] = c_base[r];
    parallel_rows(n, w1, hw, [&](uint64_t r0, uint64_t r1) {
        for (uint64_t r = r0; r < r1; ++r) {
            uint64_t c = c_base[r], w = b_base[r], pos = 0;
            const uint32_t k_n = live(r);
            for (uint32_t k = 0; k < k_n; ++k, ++c) {
                const STORM_bitmap_t& b = rows[r].bitmaps[k];
                h_cid[c] = rows[r].block_ids[k];
                if (b.n_bitmap) {
                    h_coff[c] = w;
                    h_ckl[c] = CK_BITMAP | (b.n_bitmap < CHUNK_WORDS ? b.n_bitmap : CHUNK_WORDS);
                    w += CHUNK_WORDS;
                } else {
                    const uint32_t ns = b.scalar ? b.n_scalar : 0;
                    pos = (pos + 7) / 8 * 8;
                    h_coff[c] = l_base[r] + pos;
                    h_ckl[c] = ns & CK_LEN;
                    pos += ns;
                }
            }
        }
    });
    row_off.reserve(n + 1);
    cid.reserve(nc ? nc : 1);
    ckl.reserve(nc ? nc : 1);
    coff.reserve(nc ? nc : 1);
    bm.reserve(nbw ? nbw : 1);
    lst.reserve(nl ? nl : 1);
    SB_CUDA(cudaMemcpyAsync(row_off.p, h_row_off.data(), (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    if (nc) {
        SB_CUDA(cudaMemcpyAsync(cid.p, h_cid.data(), nc * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        SB_CUDA(cudaMemcpyAsync(ckl.p, h_ckl.data(), nc * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        SB_CUDA(cudaMemcpyAsync(coff.p, h_coff.data(), nc * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    }
    // Pass 3: the payload. Each worker takes a range of rows of about equal
    // bytes and moves it in slices of whole chunks: bitmaps (1024 words,
    // short ones zero-filled) at the front of its buffer, list slots (the
    // list, zero padding to a multiple of 8 entries) behind them, two copies
    // per slice on the worker's stream while it fills its other buffer.
    stage.ensure();
    std::vector<uint64_t> pb(n + 1, 0);   // payload bytes of rows before r
    for (uint64_t r = 0; r < n; ++r)
        pb[r + 1] = pb[r] + (b_base[r + 1] - b_base[r]) * 8 + (l_base[r + 1] - l_base[r]) * 2;
    const unsigned workers =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>({(uint64_t)stage.lanes.size(), n, 1 + pb[n] / (4u << 20)}));
    std::vector<uint64_t> cut{0};
    for (uint64_t r = 0; r < n && cut.size() < workers; ++r)
        if (pb[r + 1] * workers >= pb[n] * cut.size()) cut.push_back(r + 1);
    while (cut.size() <= workers) cut.push_back(n);
    SB_CUDA(cudaEventRecord(stage.ready, st));   // the metadata copies and earlier work on st
    const uint64_t cap = stage.lane_bytes;
    run_workers(workers, [&](unsigned t) {
        PinnedStage::Lane& L = stage.lanes[t];
        const LaneSync lane_sync{L.st};
        SB_CUDA(cudaStreamWaitEvent(L.st, stage.ready, 0));
        uint64_t r = cut[t], k = 0;
        const uint64_t r_end = cut[t + 1];
        bool used[2] = {false, false};
        int which = 0;
        auto advance = [&]() {
            ++k;
            while (r < r_end && k >= live(r)) {
                ++r;
                k = 0;
            }
        };
        while (r < r_end && k >= live(r)) {
            ++r;
            k = 0;
        }
        while (r < r_end) {
            // the slice: whole chunks from (r, k) while they fit
            uint64_t sr = r, sk = k, bw = 0, ls = 0;
            uint64_t b0 = ~0ull, l0 = ~0ull;
            while (r < r_end) {
                const STORM_bitmap_t& b = rows[r].bitmaps[k];
                const uint64_t c = c_base[r] + k;
                uint64_t nb = 0, nls = 0;
                if (b.n_bitmap) nb = CHUNK_WORDS;
                else nls = ((uint64_t)(h_ckl[c] & CK_LEN) + 7) / 8 * 8;
                if ((bw + nb) * 8 + (ls + nls) * 2 > cap) {
                    if (bw || ls) break;
                    // a list longer than a buffer (the public layout allows
                    // any length): straight from its own memory
                    const uint64_t ns = h_ckl[c] & CK_LEN;
                    if (ns) SB_CUDA(cudaMemcpyAsync(lst.p + h_coff[c], b.scalar, ns * 2, cudaMemcpyHostToDevice, L.st));
                    if (nls > ns) SB_CUDA(cudaMemsetAsync(lst.p + h_coff[c] + ns, 0, (nls - ns) * 2, L.st));
                    advance();
                    sr = r;
                    sk = k;
                    continue;
                }
                if (nb && b0 == ~0ull) b0 = h_coff[c];
                if (nls && l0 == ~0ull) l0 = h_coff[c];
                bw += nb;
                ls += nls;
                advance();
            }
            if (used[which]) SB_CUDA(cudaEventSynchronize(L.done[which]));
            uint64_t* sbm = reinterpret_cast<uint64_t*>(L.buf[which]);
            uint16_t* slst = reinterpret_cast<uint16_t*>(L.buf[which] + bw * 8);
            uint64_t w = 0, p = 0;
            for (uint64_t q = sr, qk = sk; q < r || (q == r && qk < k);) {
                const STORM_bitmap_t& b = rows[q].bitmaps[qk];
                if (b.n_bitmap) {
                    const uint32_t nw = b.n_bitmap < CHUNK_WORDS ? b.n_bitmap : CHUNK_WORDS;
                    const uint32_t copied = b.data ? nw : 0;
                    if (copied) std::memcpy(sbm + w, b.data, copied * sizeof(uint64_t));
                    std::memset(sbm + w + copied, 0, (CHUNK_WORDS - copied) * sizeof(uint64_t));
                    w += CHUNK_WORDS;
                } else {
                    const uint32_t ns = b.scalar ? b.n_scalar : 0;
                    const uint64_t slot = ((uint64_t)ns + 7) / 8 * 8;
                    if (ns) std::memcpy(slst + p, b.scalar, ns * sizeof(uint16_t));
                    std::memset(slst + p + ns, 0, (slot - ns) * sizeof(uint16_t));
                    p += slot;
                }
                ++qk;
                while (q < r_end && qk >= live(q)) {
                    ++q;
                    qk = 0;
                }
            }
            if (bw) SB_CUDA(cudaMemcpyAsync(bm.p + b0, sbm, bw * 8, cudaMemcpyHostToDevice, L.st));
            if (ls) SB_CUDA(cudaMemcpyAsync(lst.p + l0, slst, ls * 2, cudaMemcpyHostToDevice, L.st));
            SB_CUDA(cudaEventRecord(L.done[which], L.st));
            used[which] = true;
            which ^= 1;
        }
        SB_CUDA(cudaStreamSynchronize(L.st));
    });
    // The lists' order and runs, on the device.
    d_row_dup.reserve(n ? n : 1);
    d_row_runs.reserve(n ? n : 1);
    SB_CUDA(cudaMemsetAsync(d_row_dup.p, 0, n ? n : 1, st));
    SB_CUDA(cudaMemsetAsync(d_row_runs.p, 0, (n ? n : 1) * sizeof(uint32_t), st));
    if (nc) {
        const uint64_t blocks = std::min<uint64_t>((nc + 7) / 8, 148ull * 16);
        list_order_kernel<<<(unsigned)blocks, 256, 0, st>>>(row_off.p, n, ckl.p, coff.p, lst.p, bm.p, nc,
                                                            d_row_dup.p, d_row_runs.p);
        SB_CUDA(cudaGetLastError());
    }
    std::vector<uint8_t> dup(n ? n : 1);
    std::vector<uint32_t> runs(n ? n : 1);
    SB_CUDA(cudaMemcpyAsync(dup.data(), d_row_dup.p, n ? n : 1, cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(runs.data(), d_row_runs.p, (n ? n : 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    for (uint64_t r = 0; r < n; ++r) {
        if (dup[r]) facts[r].plain = false;
        facts[r].runs = runs[r];
    }
}

void copy_to_host(uint32_t* out, const uint32_t* d_src, uint64_t count, cudaStream_t st, PinnedStage& stage) {
    const uint64_t bytes = count * sizeof(uint32_t);
    if (bytes == 0) return;
    cudaPointerAttributes a{};
    const bool known = cudaPointerGetAttributes(&a, out) == cudaSuccess;
    cudaGetLastError();   // an attribute query of plain host memory may leave an error behind
    if (known && a.type == cudaMemoryTypeDevice) fail(STORM_B200_EARG, "the host output buffer is device memory");
    const bool pinned = known && a.type == cudaMemoryTypeHost;
    if (pinned || bytes < (32u << 20)) {
        SB_CUDA(cudaMemcpyAsync(out, d_src, bytes, cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        return;
    }
    stage.ensure();
    const uint64_t cap = stage.lane_bytes / sizeof(uint32_t);
    const unsigned workers =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(stage.lanes.size(), bytes / (8u << 20)));
    SB_CUDA(cudaEventRecord(stage.ready, st));
    run_workers(workers, [&](unsigned t) {
        PinnedStage::Lane& L = stage.lanes[t];
        const LaneSync lane_sync{L.st};
        SB_CUDA(cudaStreamWaitEvent(L.st, stage.ready, 0));
        const uint64_t lo = count * t / workers, hi = count * (t + 1) / workers;
        auto issue = [&](uint64_t x, int b) {
            const uint64_t len = std::min(cap, hi - x);
            SB_CUDA(cudaMemcpyAsync(L.buf[b], d_src + x, len * sizeof(uint32_t), cudaMemcpyDeviceToHost, L.st));
            SB_CUDA(cudaEventRecord(L.done[b], L.st));
        };
        if (lo < hi) issue(lo, 0);
        int b = 0;
        for (uint64_t x = lo; x < hi; x += cap, b ^= 1) {
            if (x + cap < hi) issue(x + cap, b ^ 1);   // its buffer was drained in the last round
            SB_CUDA(cudaEventSynchronize(L.done[b]));
            std::memcpy(out + x, L.buf[b], std::min(cap, hi - x) * sizeof(uint32_t));
        }
    });
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
    } else if ((ka | kb) & CK_DUP) {
        // A list with a repeated or out-of-order entry: the reference's
        // blocked SSE4.2 count, which then differs from the set size, on
        // one lane (ca is row i's chunk: the reference's first list).
        if (lane == 0)
            cnt = (uint32_t)list16_blocked_count(v.lst + v.coff[ca], v.lst + v.coff[cb], ka & CK_LEN, kb & CK_LEN);
    } else {
        // Strictly increasing lists: each entry of the shorter one is
        // searched in the longer one.
        const uint32_t la = ka & CK_LEN, lb = kb & CK_LEN;
        const bool a_short = la <= lb;
        const uint16_t* s = v.lst + v.coff[a_short ? ca : cb];
        const uint16_t* g = v.lst + v.coff[a_short ? cb : ca];
        const uint32_t ns = a_short ? la : lb, ng = a_short ? lb : la;
        for (uint32_t e = lane; e < ns; e += 32) {
            const uint16_t x = s[e];
            const uint32_t p = lower_bound_dev<uint16_t>(g, ng, x);
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
// W = 1024 x chunk slots, in layout `lay`: chunk slot s of row r -- one
// 1024-word block -- at X + r x pitch + s x kstride) is row rows[r]. One CTA
// per row, a warp per chunk slot: absent chunks and padding rows (~0) become
// zeros, bitmap chunks are copied, list chunks are set bit by bit in a
// shared-memory copy of the chunk and written out.
constexpr int EXPAND_WARPS = 4;

// Expanded rows for the tensor cores are stored block-major: chunk slot s of
// all the panel's rows together, rows PANEL_PITCH words (8 KiB + 64 bytes)
// apart within it.  A tile's 384 rows at one K stage then lie in about 3 MiB
// instead of on 384 pages of 2 MiB (rows of 2^24 bits row-major), and no two
// rows share a pitch that is a power of two.
constexpr uint64_t PANEL_PITCH = CHUNK_WORDS + 8;
inline uint64_t panel_row_words(uint64_t W) { return W / CHUNK_WORDS * PANEL_PITCH; }

__global__ void __launch_bounds__(EXPAND_WARPS * 32)
expand_rows_kernel(ChunkView v, const uint32_t* __restrict__ rows, uint32_t m, uint32_t W, RowLayout lay,
                   uint64_t* __restrict__ X) {
    __shared__ __align__(16) unsigned long long chunk[EXPAND_WARPS][CHUNK_WORDS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t slots = W / CHUNK_WORDS;
    for (uint32_t r = blockIdx.x; r < m; r += gridDim.x) {
        const uint32_t row = rows[r];
        uint64_t* dst_row = X + (uint64_t)r * lay.pitch;
        const uint64_t c0 = row == ~0u ? 0 : v.row_off[row], c1 = row == ~0u ? 0 : v.row_off[row + 1];
        uint64_t pos = c0;
        for (uint32_t s = warp; s < slots; s += EXPAND_WARPS) {
            while (pos < c1 && v.cid[pos] < s) ++pos;   // ids ascend: a forward walk
            uint4* dst = reinterpret_cast<uint4*>(dst_row + (uint64_t)s * lay.kstride);
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

// Pair p of the walk -> rows (i, j), i < j or i == j, as stored:
//   PAIRS_TRIANGLE  p-th entry of the packed triangle of n1 walk rows (a
//                   prefix of it when n_pairs < n1 (n1 + 1) / 2);
//   PAIRS_RECT      walk rows ib + p / n2 and jb + p % n2.
// perm (optional) maps walk rows to stored rows. Counts land at the packed
// index of (i, j) in the triangle of n_out rows when out is given; the sum
// over i != j accumulates into flags->sum.
__global__ void __launch_bounds__(256)
chunk_pairs_kernel(ChunkView v, uint32_t mode, uint64_t n1, uint64_t n2, uint64_t n_pairs,
                   const uint32_t* __restrict__ perm, uint64_t ib, uint64_t jb, uint64_t n_out,
                   uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags) {
    const int lane = threadIdx.x & 31;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long local = 0;
    for (uint64_t p = wid; p < n_pairs; p += nwarps) {
        uint64_t i, j;
        if (mode == PAIRS_TRIANGLE) {
            tri_decode(n1, p, i, j);
        } else {
            i = ib + p / n2;
            j = jb + p % n2;
        }
        if (perm) {
            const uint64_t a = perm[i], b = perm[j];
            i = a < b ? a : b;
            j = a < b ? b : a;
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
            if (out) out[tri_index(n_out, i, j)] = cnt;
            if (j != i) local += cnt;
        }
    }
    if (lane == 0 && local) atomicAdd(&flags->sum, local);
}

// ---- postings: pairs of plain rows without bitmap chunks ----------------
// value of entry e of list chunk c: cid << 16 | entry (universe <= 2^27)

// rows == nullptr: rows [0, nq). Bitmap chunks count every set bit (only the
// rectangle sums send rows that have them).
__global__ void postings_hist_kernel(ChunkView v, const uint32_t* __restrict__ rows, uint32_t nq,
                                     uint32_t* __restrict__ counts) {
    const int lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nq; r += nw) {
        const uint32_t row = rows ? rows[r] : r;
        for (uint64_t c = v.row_off[row]; c < v.row_off[row + 1]; ++c) {
            const uint32_t base = v.cid[c] << 16;
            const uint32_t k = v.ckl[c];
            if (k & CK_BITMAP) {
                const uint64_t* wd = v.bm + v.coff[c];
                for (uint32_t w = lane; w < CHUNK_WORDS; w += 32)
                    for (uint64_t x = wd[w]; x; x &= x - 1)
                        atomicAdd(&counts[base | (w << 6) | (uint32_t)__ffsll((long long)x) - 1u], 1u);
            } else {
                const uint16_t* l = v.lst + v.coff[c];
                const uint32_t nl = k & CK_LEN;
                for (uint32_t e = lane; e < nl; e += 32) atomicAdd(&counts[base | l[e]], 1u);
            }
        }
    }
}

// sum over values of a[x] * b[x] into flags->sum: the rectangle sum of two
// sets of plain rows.
__global__ void counts_dot_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint64_t U,
                                  DeviceFlags* __restrict__ flags) {
    unsigned long long acc = 0;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < U; x += (uint64_t)gridDim.x * blockDim.x)
        acc += (unsigned long long)a[x] * b[x];
    acc = warp_sum_u64(acc);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(&flags->sum, acc);
}

struct PostingsStats {
    unsigned long long pairs;     // sum over values of C(rows holding it, 2)
    unsigned long long lists;     // values held by >= 2 rows
    unsigned long long entries;   // their rows, summed
    unsigned long long cursor[2]; // allocation cursors (entries, lists)
};

__global__ void postings_stats_kernel(const uint32_t* __restrict__ counts, uint64_t U, PostingsStats* st) {
    unsigned long long p = 0, l = 0, e = 0;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < U; x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = counts[x];
        if (c >= 2) {
            p += (unsigned long long)c * (c - 1) / 2;
            l += 1;
            e += c;
        }
    }
    p = warp_sum_u64(p);
    l = warp_sum_u64(l);
    e = warp_sum_u64(e);
    if ((threadIdx.x & 31) == 0 && l) {
        atomicAdd(&st->pairs, p);
        atomicAdd(&st->lists, l);
        atomicAdd(&st->entries, e);
    }
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    return x;
}

// Gives every value held by >= 2 rows a slot range in the postings array
// (start) and, when `lists` is given, a list record; other values get
// start = ~0. One atomic per warp per 32 values. (The run postings use it
// for bins.)
__global__ void postings_alloc_kernel(const uint32_t* __restrict__ counts, uint64_t U, uint32_t* __restrict__ start,
                                      uint2* __restrict__ lists, PostingsStats* st) {
    const int lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t x0 = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; x0 < U; x0 += nw * 32) {
        const uint64_t x = x0 + lane;
        const uint32_t c = x < U ? counts[x] : 0u;
        const bool want = c >= 2;
        const uint32_t n_incl = warp_incl_scan(want ? c : 0u, lane);
        const uint32_t b = __ballot_sync(0xffffffffu, want);
        unsigned long long e0 = 0, l0 = 0;
        if (lane == 31 && b) {
            e0 = atomicAdd(&st->cursor[0], (unsigned long long)n_incl);
            l0 = atomicAdd(&st->cursor[1], (unsigned long long)__popc(b));
        }
        e0 = __shfl_sync(0xffffffffu, e0, 31);
        l0 = __shfl_sync(0xffffffffu, l0, 31);
        if (x < U) {
            if (want) {
                const uint32_t s = (uint32_t)(e0 + n_incl - c);
                start[x] = s;
                if (lists) lists[l0 + __popc(b & ((1u << lane) - 1u))] = make_uint2(s, c);
            } else {
                start[x] = ~0u;
            }
        }
    }
}

// Writes each Q row's position in the Q list (its local index) into the
// lists of its values; start[x] advances to the end of x's list.
__global__ void postings_scatter_kernel(ChunkView v, const uint32_t* __restrict__ rows, uint32_t nq,
                                        uint32_t* __restrict__ start, uint32_t* __restrict__ post) {
    const int lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nq; r += nw) {
        const uint32_t row = rows[r];
        for (uint64_t c = v.row_off[row]; c < v.row_off[row + 1]; ++c) {
            const uint32_t base = v.cid[c] << 16;
            const uint16_t* l = v.lst + v.coff[c];
            const uint32_t nl = v.ckl[c] & CK_LEN;
            for (uint32_t e = lane; e < nl; e += 32) {
                const uint32_t x = base | l[e];
                if (start[x] != ~0u) post[atomicAdd(&start[x], 1u)] = r;
            }
        }
    }
}

// One increment per (pair of rows, shared value): thread per list for lists
// of up to POST_THREAD_MAX rows, warp per list beyond.
constexpr uint32_t POST_THREAD_MAX = 64;

__global__ void postings_pairs_kernel(const uint2* __restrict__ lists, uint64_t n_lists,
                                      const uint32_t* __restrict__ post, const uint32_t* __restrict__ qrows,
                                      uint64_t n, uint32_t* __restrict__ out) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t li = tid; li < n_lists; li += nt) {
        const uint2 L = lists[li];
        if (L.y > POST_THREAD_MAX) continue;
        for (uint32_t a = 0; a + 1 < L.y; ++a) {
            const uint32_t ra = qrows[post[L.x + a]];
            for (uint32_t b = a + 1; b < L.y; ++b) {
                const uint32_t rb = qrows[post[L.x + b]];
                atomicAdd(&out[ra < rb ? tri_index(n, ra, rb) : tri_index(n, rb, ra)], 1u);
            }
        }
    }
    const int lane = threadIdx.x & 31;
    for (uint64_t li = tid >> 5; li < n_lists; li += nt >> 5) {
        const uint2 L = lists[li];
        if (L.y <= POST_THREAD_MAX) continue;
        for (uint32_t a = 0; a + 1 < L.y; ++a) {
            const uint32_t ra = qrows[post[L.x + a]];
            for (uint32_t b = a + 1 + lane; b < L.y; b += 32) {
                const uint32_t rb = qrows[post[L.x + b]];
                atomicAdd(&out[ra < rb ? tri_index(n, ra, rb) : tri_index(n, rb, ra)], 1u);
            }
        }
    }
}

// Row sweep: CTA per Q row a; for every value of a, the rows b > a on that
// value's list get one shared-memory increment; then a's slice of the
// triangle (its Q partners b > a and its diagonal) is written once, in
// ascending order. The row's entries are split evenly over the threads (a
// shared-memory prefix of its chunk lengths maps entry -> chunk), so rows of
// one long chunk and rows of many short ones both keep every thread busy.
// Partners are counted for one block of local indices [pb0, pb0 + pbn) per
// launch (at most POST_SWEEP_MAX_ROWS, the counters shared memory holds):
// more postings rows take one launch per block, each reading a row's lists
// again; the launch of block 0 writes the diagonal.
// Shared memory: pbn counters, then up to POST_SWEEP_MAX_CHUNKS + 1 prefix
// words. Lists hold local indices, list x is [end[x] - counts[x], end[x]).
constexpr uint32_t POST_SWEEP_THREADS = 256;
constexpr uint32_t POST_SWEEP_MAX_CHUNKS = 2048;  // universe <= 2^27
constexpr uint32_t POST_SWEEP_MAX_ROWS = 51200;   // 200 KiB of counters + 8 KiB of prefix

__global__ void __launch_bounds__(POST_SWEEP_THREADS)
postings_rows_kernel(ChunkView v, const uint32_t* __restrict__ qrows, uint32_t nq, const uint32_t* __restrict__ counts,
                     const uint32_t* __restrict__ end, const uint32_t* __restrict__ post, uint64_t n,
                     uint32_t* __restrict__ out, uint32_t pb0, uint32_t pbn) {
    extern __shared__ uint32_t cnt[];
    uint32_t* pref = cnt + pbn;                // pref[k] = entries of the row's chunks before chunk k
    const uint32_t pb1 = pb0 + pbn;
    for (uint32_t a = blockIdx.x; a < nq; a += gridDim.x) {
        if (a + 1 >= pb1 && pb0 > 0) continue;     // no partner after a in this block, diagonal not here
        const uint32_t row = qrows[a];
        const uint64_t c0 = v.row_off[row];
        const uint32_t nc = (uint32_t)(v.row_off[row + 1] - c0);   // <= POST_SWEEP_MAX_CHUNKS (plain rows)
        for (uint32_t b = threadIdx.x; b < pbn; b += blockDim.x) cnt[b] = 0;
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
            for (uint32_t k = 0; k < nc; ++k) {
                pref[k] = acc;
                acc += v.ckl[c0 + k] & CK_LEN;
            }
            pref[nc] = acc;
        }
        __syncthreads();
        const uint32_t total = pref[nc];
        const uint32_t work = a + 1 < pb1 ? total : 0u;   // no partner in the block: the diagonal only
        for (uint32_t e = threadIdx.x; e < work; e += blockDim.x) {
            uint32_t lo = 0, hi = nc;              // last chunk k with pref[k] <= e
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (pref[mid] <= e) lo = mid;
                else hi = mid;
            }
            const uint64_t c = c0 + lo;
            const uint32_t x = (v.cid[c] << 16) | v.lst[v.coff[c] + (e - pref[lo])];
            const uint32_t len = counts[x];
            if (len < 2) continue;
            const uint32_t e1 = end[x];
            for (uint32_t k = e1 - len; k < e1; ++k) {
                const uint32_t b = post[k];
                if (b > a && b >= pb0 && b < pb1) atomicAdd(&cnt[b - pb0], 1u);
            }
        }
        __syncthreads();
        const uint64_t base = tri_index(n, row, row) - row;   // out index of (row, j) is base + j
        for (uint32_t b = (a + 1 > pb0 ? a + 1 : pb0) + threadIdx.x; b < pb1; b += blockDim.x) {
            const uint32_t gb = qrows[b];   // ascending: gb > row (the other order kept exact too)
            out[gb > row ? base + gb : tri_index(n, gb, row)] = cnt[b - pb0];
        }
        if (threadIdx.x == 0 && pb0 == 0) out[base + row] = total;
        __syncthreads();
    }
}

// ---- run postings: L x L by overlaps of runs, bin by bin ----------------
// The universe is cut into bins of 2^wlog values (16 .. 32768, so that no
// bin straddles a chunk); a piece is a maximal run of a row's values inside
// one bin. A row's pieces are disjoint, so |Xa & Xb| is the sum over bins of
// the overlaps of a's pieces with b's pieces there: rows made of long runs
// cost per piece instead of per value. Each bin held by >= 2 pieces gets a
// list of (row, start, end) entries (offsets inside the bin), built like the
// value postings (histogram, allocation, scatter); then a row sweep: a CTA
// per row, for each of its pieces the entries of the piece's bin, overlaps
// with rows after it added in shared memory, its triangle slice written once.
// The piece rules: run_pieces.cuh.
constexpr uint32_t RUN_SWEEP_BATCH = 2048;   // pieces prefixed in shared memory at once

// Word wi of a bitmap chunk held by this lane (a warp walks the chunk 32
// words at a time, `carry` = bit 63 of the word before the warp's first):
// the bits that start a piece and the bits that end one.
__device__ __forceinline__ void run_bitmap_word(const uint64_t* wd, uint32_t nwc, uint32_t w0, int lane,
                                                uint32_t wlog, uint64_t& carry, uint64_t& starts, uint64_t& lasts) {
    const uint32_t wi = w0 + lane;
    const uint64_t x = wi < nwc ? wd[wi] : 0ull;
    const uint64_t prev = __shfl_up_sync(0xffffffffu, x, 1);
    const uint64_t next = __shfl_down_sync(0xffffffffu, x, 1);
    const uint64_t cin = lane ? prev >> 63 : carry;
    const uint64_t nin = lane < 31 ? next & 1ull : (w0 + 32 < nwc ? wd[w0 + 32] & 1ull : 0ull);
    carry = __shfl_sync(0xffffffffu, x, 31) >> 63;
    run_word_masks(x, cin, nin, wi, wlog, starts, lasts);
}

// Pieces per row and per bin; warp per row.
__global__ void run_count_kernel(ChunkView v, const uint32_t* __restrict__ rows, uint32_t nq, uint32_t wlog,
                                 uint32_t* __restrict__ pieces, uint32_t* __restrict__ bins) {
    const int lane = threadIdx.x & 31;
    const uint32_t wmask = (1u << wlog) - 1u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nq; r += nw) {
        const uint32_t row = rows[r];
        uint32_t cnt = 0;
        for (uint64_t c = v.row_off[row]; c < v.row_off[row + 1]; ++c) {
            const uint32_t base = v.cid[c] << 16;
            const uint32_t k = v.ckl[c];
            if (k & CK_BITMAP) {
                const uint64_t* wd = v.bm + v.coff[c];
                const uint32_t nwc = k & CK_LEN;
                uint64_t carry = 0, starts, lasts;
                for (uint32_t w0 = 0; w0 < nwc; w0 += 32) {
                    run_bitmap_word(wd, nwc, w0, lane, wlog, carry, starts, lasts);
                    cnt += __popcll(starts);
                    for (uint64_t x = starts; x; x &= x - 1)
                        atomicAdd(&bins[(base + ((w0 + lane) << 6) + (uint32_t)(__ffsll((long long)x) - 1)) >> wlog],
                                  1u);
                }
            } else {
                const uint16_t* l = v.lst + v.coff[c];
                const uint32_t nl = k & CK_LEN;
                for (uint32_t e = lane; e < nl; e += 32)
                    if (run_piece_start(l, e, wmask)) {
                        ++cnt;
                        atomicAdd(&bins[(base | l[e]) >> wlog], 1u);
                    }
            }
        }
        cnt = warp_sum_u32(cnt);
        if (lane == 0) pieces[r] = cnt;
    }
}

// Over the bins held by >= 2 pieces: st[0] += their pieces (list entries),
// st[1] += pieces^2 (the sweep's entry reads).
__global__ void run_stats_kernel(const uint32_t* __restrict__ bins, uint64_t nb, unsigned long long* __restrict__ st) {
    unsigned long long e = 0, q = 0;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < nb; x += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long c = bins[x];
        if (c >= 2) {
            e += c;
            q += c * c;
        }
    }
    e = warp_sum_u64(e);
    q = warp_sum_u64(q);
    if ((threadIdx.x & 31) == 0 && e) {
        atomicAdd(&st[0], e);
        atomicAdd(&st[1], q);
    }
}

// The rows' pieces in row order: pieces[poff[r] + k] = (first value, end),
// the k-th start and the k-th last value of the row paired by rank (list
// entries, or set bits of bitmap chunks).
__global__ void run_fill_kernel(ChunkView v, const uint32_t* __restrict__ rows, uint32_t nq, uint32_t wlog,
                                const uint64_t* __restrict__ poff, uint2* __restrict__ pieces) {
    const int lane = threadIdx.x & 31;
    const uint32_t wmask = (1u << wlog) - 1u;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nq; r += nw) {
        const uint32_t row = rows[r];
        uint2* out = pieces + poff[r];
        uint32_t ks = 0, kl = 0;
        for (uint64_t c = v.row_off[row]; c < v.row_off[row + 1]; ++c) {
            const uint32_t base = v.cid[c] << 16;
            const uint32_t k = v.ckl[c];
            if (k & CK_BITMAP) {
                const uint64_t* wd = v.bm + v.coff[c];
                const uint32_t nwc = k & CK_LEN;
                uint64_t carry = 0, starts, lasts;
                for (uint32_t w0 = 0; w0 < nwc; w0 += 32) {
                    run_bitmap_word(wd, nwc, w0, lane, wlog, carry, starts, lasts);
                    const uint32_t ns = (uint32_t)__popcll(starts), nls = (uint32_t)__popcll(lasts);
                    uint32_t xs = ns, xl = nls;   // inclusive scans over the lanes (words in order)
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t ys = __shfl_up_sync(0xffffffffu, xs, o), yl = __shfl_up_sync(0xffffffffu, xl, o);
                        if (lane >= o) {
                            xs += ys;
                            xl += yl;
                        }
                    }
                    const uint32_t at = base + ((w0 + lane) << 6);
                    uint32_t j = ks + xs - ns;
                    for (uint64_t x = starts; x; x &= x - 1) out[j++].x = at + (uint32_t)(__ffsll((long long)x) - 1);
                    j = kl + xl - nls;
                    for (uint64_t x = lasts; x; x &= x - 1) out[j++].y = at + (uint32_t)__ffsll((long long)x);
                    ks += __shfl_sync(0xffffffffu, xs, 31);
                    kl += __shfl_sync(0xffffffffu, xl, 31);
                }
            } else {
                const uint16_t* l = v.lst + v.coff[c];
                const uint32_t nl = k & CK_LEN;
                for (uint32_t e0 = 0; e0 < nl; e0 += 32) {
                    const uint32_t e = e0 + lane;
                    const bool in = e < nl;
                    const bool st = in && run_piece_start(l, e, wmask);
                    const bool la = in && run_piece_last(l, e, nl, wmask);
                    const uint32_t bs = __ballot_sync(0xffffffffu, st), bl = __ballot_sync(0xffffffffu, la);
                    if (st) out[ks + __popc(bs & lt)].x = base | l[e];
                    if (la) out[kl + __popc(bl & lt)].y = (base | l[e]) + 1u;
                    ks += __popc(bs);
                    kl += __popc(bl);
                }
            }
        }
    }
}

// Each piece of a bin held by >= 2 pieces into the bin's list: (row, start
// | end << 16), offsets inside the bin; start[b] advances to the list's end.
__global__ void run_scatter_kernel(uint32_t nq, uint32_t wlog, const uint64_t* __restrict__ poff,
                                   const uint2* __restrict__ pieces, uint32_t* __restrict__ start,
                                   uint2* __restrict__ list) {
    const int lane = threadIdx.x & 31;
    const uint32_t wmask = (1u << wlog) - 1u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nq; r += nw)
        for (uint64_t p = poff[r] + lane; p < poff[r + 1]; p += 32) {
            const uint2 pc = pieces[p];
            const uint32_t bin = pc.x >> wlog;
            if (start[bin] == ~0u) continue;
            list[atomicAdd(&start[bin], 1u)] = make_uint2(r, (pc.x & wmask) | ((pc.y - (bin << wlog)) << 16));
        }
}

// The row sweep over pieces: CTA per row a; the (piece, bin entry) pairs of
// a batch of a's pieces are split evenly over the threads (a shared-memory
// prefix of the pieces' bin lengths maps work index -> piece). Partners in
// one block of local indices [pb0, pb0 + pbn) per launch, as in
// postings_rows_kernel. Shared memory: pbn counters, then RUN_SWEEP_BATCH + 1
// prefix words. Bin b's list is [end[b] - bins[b], end[b]). Adds the sum
// over a's partners after it (in the block) to flags->sum.
__global__ void __launch_bounds__(POST_SWEEP_THREADS)
run_sweep_kernel(const uint32_t* __restrict__ qrows, uint32_t nq, const uint64_t* __restrict__ poff,
                 const uint2* __restrict__ pieces, uint32_t wlog, const uint32_t* __restrict__ bins,
                 const uint32_t* __restrict__ end, const uint2* __restrict__ list, uint64_t n,
                 uint32_t* __restrict__ out, DeviceFlags* __restrict__ flags, uint32_t pb0, uint32_t pbn) {
    extern __shared__ uint32_t cnt[];
    uint32_t* pref = cnt + pbn;
    const uint32_t pb1 = pb0 + pbn;
    __shared__ uint32_t warp_tot[POST_SWEEP_THREADS / 32];
    __shared__ unsigned long long row_card;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint32_t a = blockIdx.x; a < nq; a += gridDim.x) {
        if (a + 1 >= pb1 && pb0 > 0) continue;     // no partner after a in this block, diagonal not here
        const uint32_t row = qrows[a];
        for (uint32_t b = threadIdx.x; b < pbn; b += blockDim.x) cnt[b] = 0;
        if (threadIdx.x == 0) row_card = 0;
        const uint64_t p0 = poff[a], np = poff[a + 1] - p0;
        unsigned long long card = 0;
        for (uint64_t pb = 0; pb < np; pb += RUN_SWEEP_BATCH) {
            const uint32_t m = (uint32_t)(np - pb < RUN_SWEEP_BATCH ? np - pb : RUN_SWEEP_BATCH);
            // pref[k] = entries of the bins of pieces pb .. pb + k - 1: each
            // thread sums a contiguous segment, then a block scan of the sums
            const uint32_t seg = (m + POST_SWEEP_THREADS - 1) / POST_SWEEP_THREADS;
            const uint32_t k0 = threadIdx.x * seg, k1 = k0 + seg < m ? k0 + seg : m;
            uint32_t mine = 0;
            for (uint32_t k = k0; k < k1; ++k) {
                const uint2 pc = pieces[p0 + pb + k];
                card += pc.y - pc.x;
                const uint32_t c = bins[pc.x >> wlog];
                mine += c >= 2 ? c : 0u;
            }
            uint32_t inc = mine;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            __syncthreads();   // the previous batch is done with pref and warp_tot
            if (lane == 31) warp_tot[wid] = inc;
            __syncthreads();
            uint32_t before = 0, total = 0;
            for (int w = 0; w < POST_SWEEP_THREADS / 32; ++w) {
                if (w < wid) before += warp_tot[w];
                total += warp_tot[w];
            }
            uint32_t acc = before + inc - mine;
            for (uint32_t k = k0; k < k1; ++k) {
                pref[k] = acc;
                const uint32_t c = bins[pieces[p0 + pb + k].x >> wlog];
                acc += c >= 2 ? c : 0u;
            }
            if (threadIdx.x == 0) pref[m] = total;
            __syncthreads();
            const uint32_t work = a + 1 < pb1 ? total : 0u;   // no partner in the block: the diagonal only
            for (uint32_t t = threadIdx.x; t < work; t += blockDim.x) {
                uint32_t lo = 0, hi = m;           // last piece k with pref[k] <= t
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (pref[mid] <= t) lo = mid;
                    else hi = mid;
                }
                const uint2 pc = pieces[p0 + pb + lo];
                const uint32_t bin = pc.x >> wlog;
                const uint2 E = list[end[bin] - bins[bin] + (t - pref[lo])];
                if (E.x > a && E.x >= pb0 && E.x < pb1) {
                    const uint32_t b0 = bin << wlog;
                    const uint32_t s2 = b0 + (E.y & 0xFFFFu), e2 = b0 + (E.y >> 16);
                    const uint32_t s = pc.x > s2 ? pc.x : s2, e = pc.y < e2 ? pc.y : e2;
                    if (e > s) atomicAdd(&cnt[E.x - pb0], e - s);
                }
            }
        }
        card = warp_sum_u64(card);
        if (lane == 0 && card) atomicAdd(&row_card, card);
        __syncthreads();
        const uint64_t base = tri_index(n, row, row) - row;   // out index of (row, j) is base + j
        unsigned long long sum = 0;
        for (uint32_t b = (a + 1 > pb0 ? a + 1 : pb0) + threadIdx.x; b < pb1; b += blockDim.x) {
            const uint32_t gb = qrows[b];
            out[gb > row ? base + gb : tri_index(n, gb, row)] = cnt[b - pb0];
            sum += cnt[b - pb0];
        }
        sum = warp_sum_u64(sum);
        if (lane == 0 && sum) atomicAdd(&flags->sum, sum);
        if (threadIdx.x == 0 && pb0 == 0) out[base + row] = (uint32_t)row_card;
        __syncthreads();
    }
}

// Diagonal of rows with bitmap chunks too (warp per row): each row's value
// count, set bits of its bitmap chunks plus its list entries.
__global__ void row_card_diag_kernel(ChunkView v, const uint32_t* __restrict__ rows, uint32_t m, uint64_t n,
                                     uint32_t* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
        const uint32_t row = rows[r];
        uint32_t card = 0;
        for (uint64_t c = v.row_off[row]; c < v.row_off[row + 1]; ++c) {
            const uint32_t k = v.ckl[c];
            if (k & CK_BITMAP) {
                const uint64_t* wd = v.bm + v.coff[c];
                for (uint32_t w = lane; w < (k & CK_LEN); w += 32) card += __popcll(wd[w]);
            } else if (lane == 0) {
                card += k & CK_LEN;
            }
        }
        card = warp_sum_u32(card);
        if (lane == 0) out[tri_index(n, row, row)] = card;
    }
}

// Diagonal of the postings rows: their value count.
__global__ void postings_diag_kernel(ChunkView v, const uint32_t* __restrict__ rows, uint32_t nq, uint64_t n,
                                     uint32_t* __restrict__ out) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nq; r += gridDim.x * blockDim.x) {
        const uint32_t row = rows[r];
        uint32_t card = 0;
        for (uint64_t c = v.row_off[row]; c < v.row_off[row + 1]; ++c) card += v.ckl[c] & CK_LEN;
        out[tri_index(n, row, row)] = card;
    }
}

uint64_t ChunkEngine::run(const ChunkDev& d, PairMode mode, uint64_t n1, uint64_t n2, uint32_t* d_out,
                          cudaStream_t st) {
    const int sms = require_device();
    const uint64_t n_pairs_all = mode == PAIRS_TRIANGLE ? tri_size(n1) : n1 * n2;
    log.launches = 0;
    log.last_ms = 0.f;
    last_dense_rows = last_dense_panels = last_postings_rows = 0;
    last_panel_rows = last_panel_queries = 0;
    last_postings_form = -1;
    for (int k = 0; k < 4; ++k) last_engine_ms[k] = last_engine_pred_ms[k] = last_engine_work[k] = 0.0;
    if (n_pairs_all == 0) return 0;
    d_flags.reserve(1);
    SB_CUDA(cudaMemsetAsync(d_flags.p, 0, sizeof(DeviceFlags), st));
    log.ensure();
    uint32_t launches = 0;
    auto chunk_launch = [&](uint32_t m, uint64_t np, const uint32_t* perm, uint64_t ib, uint64_t jb, uint64_t nn1,
                            uint64_t nn2) {
        if (np == 0) return;
        const uint64_t want_blocks = (np + 7) / 8;
        const uint32_t grid = (uint32_t)(want_blocks < (uint64_t)sms * 16 ? want_blocks : (uint64_t)sms * 16);
        chunk_pairs_kernel<<<grid, 256, 0, st>>>(d.view(), m, nn1, nn2, np, perm, ib, jb, n1, d_out, d_flags.p);
        SB_CUDA(cudaGetLastError());
        ++launches;
    };
    if (mode == PAIRS_RECT) {   // the rectangle of rows [0, n1) x [n1, n1 + n2): sums only
        SB_CUDA(cudaEventRecord(log.ev0, st));
        // All rows plain: sum over values of (rows of the first set holding
        // it) x (rows of the second set holding it), from two histograms.
        const uint64_t U = ((uint64_t)d.max_cid + 1) * 65536;
        bool plain = postings_mode != 0 && U <= POSTINGS_MAX_UNIVERSE && d.facts.size() == n1 + n2 &&
                     n_pairs_all >= 1024;
        for (uint64_t r = 0; plain && r < n1 + n2; ++r) plain = d.facts[r].plain;
        if (plain) {
            d_counts.reserve(U);
            d_start.reserve(U);
            SB_CUDA(cudaMemsetAsync(d_counts.p, 0, U * sizeof(uint32_t), st));
            SB_CUDA(cudaMemsetAsync(d_start.p, 0, U * sizeof(uint32_t), st));
            d_qrows.reserve(n2);
            std::vector<uint32_t> second(n2);
            for (uint64_t r = 0; r < n2; ++r) second[r] = (uint32_t)(n1 + r);
            SB_CUDA(cudaMemcpyAsync(d_qrows.p, second.data(), n2 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
            postings_hist_kernel<<<(uint32_t)std::min<uint64_t>((n1 + 7) / 8, (uint64_t)sms * 16), 256, 0, st>>>(
                d.view(), nullptr, (uint32_t)n1, d_counts.p);
            postings_hist_kernel<<<(uint32_t)std::min<uint64_t>((n2 + 7) / 8, (uint64_t)sms * 16), 256, 0, st>>>(
                d.view(), d_qrows.p, (uint32_t)n2, d_start.p);
            counts_dot_kernel<<<sms * 8, 256, 0, st>>>(d_counts.p, d_start.p, U, d_flags.p);
            SB_CUDA(cudaGetLastError());
            launches += 3;
            last_postings_rows = n1 + n2;
        } else {
            uint32_t* keep = d_out;
            d_out = nullptr;
            chunk_launch(PAIRS_RECT, n_pairs_all, nullptr, 0, n1, n1, n2);
            d_out = keep;
        }
        SB_CUDA(cudaEventRecord(log.ev1, st));
        DeviceFlags f;
        SB_CUDA(cudaMemcpyAsync(&f, d_flags.p, sizeof(f), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        SB_CUDA(cudaEventElapsedTime(&log.last_ms, log.ev0, log.ev1));
        log.launches = launches;
        return f.sum;
    }

    // ---- row classes, in walk order [C | L | M | H]:
    //   C  chunk kernel: every pair with a C row (rows with a repeated list
    //      value, or anything the other engines cannot take);
    //   L  postings rows (plain, no bitmap chunk): L x L by value postings;
    //   M  panel rows queried and stored: (L u M) x (M u H) pairs by the
    //      transposed-panel engine (panel.cuh), each pair once;
    //   H  tensor rows: H x H on the tensor cores -- and, in the plan without
    //      a panel, H x L too (the L rows expanded behind the H rows).
    const uint64_t n = n1;
    const uint64_t slots = (uint64_t)d.max_cid + 1;
    const uint64_t U = slots * 65536;                      // universe of the rows' values
    const uint64_t W = slots * CHUNK_WORDS;                // words per expanded row
    const bool facts_ok = d.facts.size() == n;
    const bool tc_ok = dense_min_density != 0.0 && U <= TC_MAX_ROW_BITS && facts_ok;
    const bool post_ok = postings_mode != 0 && U <= POSTINGS_MAX_UNIVERSE && facts_ok;
    const double tc_ns = tensor_pair_ns(cost, slots);
    std::vector<uint8_t> cls(n, 0);                        // 0 C, 1 L, 2 M, 3 H
    if (!ev_hist) SB_CUDA(cudaEventCreate(&ev_hist));
    if (!ev_hist0) SB_CUDA(cudaEventCreate(&ev_hist0));
    bool hist_ran = false;
    last_panel_rows = last_panel_queries = 0;

    SB_CUDA(cudaEventRecord(log.ev0, st));
    PostingsStats ps{};
    auto histogram = [&](const std::vector<uint32_t>& rows) {
        d_qrows.reserve(rows.size());
        SB_CUDA(cudaEventRecord(ev_hist0, st));
        SB_CUDA(cudaMemcpyAsync(d_qrows.p, rows.data(), rows.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        d_counts.reserve(U);
        d_pstats.reserve(1);
        SB_CUDA(cudaMemsetAsync(d_counts.p, 0, U * sizeof(uint32_t), st));
        SB_CUDA(cudaMemsetAsync(d_pstats.p, 0, sizeof(PostingsStats), st));
        const uint32_t gq = (uint32_t)std::min<uint64_t>((rows.size() + 7) / 8, (uint64_t)sms * 16);
        postings_hist_kernel<<<gq, 256, 0, st>>>(d.view(), d_qrows.p, (uint32_t)rows.size(), d_counts.p);
        postings_stats_kernel<<<sms * 8, 256, 0, st>>>(d_counts.p, U, d_pstats.p);
        SB_CUDA(cudaGetLastError());
        SB_CUDA(cudaEventRecord(ev_hist, st));
        hist_ran = true;
        launches += 2;
        PostingsStats h{};
        SB_CUDA(cudaMemcpyAsync(&h, d_pstats.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        return h;
    };
    // Run postings (run_sweep_kernel): bins of 2^rwlog values, the mean run
    // length of the plain list rows rounded to a power of two in [16, 32768]
    // (a run of length l spans about 1 + l / bin bins; the sweep's entry
    // reads, pieces^2 x bin / U for uniform rows, are least at bin = l).
    uint32_t rwlog = 4;
    if (facts_ok) {
        double sc = 0.0, sr = 0.0;
        for (uint64_t r = 0; r < n; ++r) {
            const ChunkRowFacts& f = d.facts[r];
            if (f.plain && f.bitmap_chunks == 0) {
                sc += (double)f.card;
                sr += (double)f.runs;
            }
        }
        const double ml = sr > 0.0 ? sc / sr : 1.0;
        rwlog = (uint32_t)std::min(15.0, std::max(4.0, std::round(std::log2(std::max(ml, 1.0)))));
    }
    const double RW = (double)(1u << rwlog);
    const uint64_t n_bins = U >> rwlog;
    auto pieces_est = [&](const ChunkRowFacts& f) { return (double)f.runs + (double)f.card / RW; };
    unsigned long long run_entries = 0, run_checks = 0;   // exact, from the piece histogram
    std::vector<uint32_t> h_rpieces;
    bool use_run = false;
    auto run_histogram = [&](const std::vector<uint32_t>& rows) {
        const uint64_t q = rows.size();
        d_qrows.reserve(q);
        SB_CUDA(cudaEventRecord(ev_hist0, st));
        SB_CUDA(cudaMemcpyAsync(d_qrows.p, rows.data(), q * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        d_rbins.reserve(n_bins);
        d_rpieces.reserve(q);
        d_rstats.reserve(2);
        SB_CUDA(cudaMemsetAsync(d_rbins.p, 0, n_bins * sizeof(uint32_t), st));
        SB_CUDA(cudaMemsetAsync(d_rstats.p, 0, 2 * sizeof(unsigned long long), st));
        const uint32_t gq = (uint32_t)std::min<uint64_t>((q + 7) / 8, (uint64_t)sms * 16);
        run_count_kernel<<<gq, 256, 0, st>>>(d.view(), d_qrows.p, (uint32_t)q, rwlog, d_rpieces.p, d_rbins.p);
        run_stats_kernel<<<sms * 8, 256, 0, st>>>(d_rbins.p, n_bins, d_rstats.p);
        SB_CUDA(cudaGetLastError());
        SB_CUDA(cudaEventRecord(ev_hist, st));
        hist_ran = true;
        launches += 2;
        unsigned long long h[2] = {0, 0};
        h_rpieces.resize(q);
        SB_CUDA(cudaMemcpyAsync(h, d_rstats.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaMemcpyAsync(h_rpieces.data(), d_rpieces.p, q * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        run_entries = h[0];
        run_checks = h[1];
    };
    auto finish = [&](uint64_t extra_sum) {
        SB_CUDA(cudaEventRecord(log.ev1, st));
        DeviceFlags f;
        SB_CUDA(cudaMemcpyAsync(&f, d_flags.p, sizeof(f), cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        if (f.error) fail(STORM_B200_ETIMEOUT, "tensor-core dense block: a pipeline wait timed out");
        SB_CUDA(cudaEventElapsedTime(&log.last_ms, log.ev0, log.ev1));
        log.launches = launches;
        return f.sum + extra_sum;
    };

    // Sum-only calls: over every pair of plain rows the sum is
    // sum_v C(rows holding v, 2) -- one value histogram, no pair touched
    // (bitmap chunks count every set bit); pairs with another row run on the
    // chunk kernel.
    if (!d_out && post_ok) {
        std::vector<uint32_t> plain;
        for (uint32_t r = 0; r < n; ++r)
            if (d.facts[r].plain) plain.push_back(r);
        uint64_t q_sum = 0;
        if (plain.size() >= 2) {
            q_sum = histogram(plain).pairs;
            last_postings_rows = plain.size();
        }
        const uint64_t nc = n - plain.size();
        if (nc) {
            for (uint32_t r : plain) cls[r] = 1;
            std::vector<uint32_t> h_perm;
            h_perm.reserve(n);
            for (int k = 0; k < 2; ++k)
                for (uint32_t r = 0; r < n; ++r)
                    if (cls[r] == k) h_perm.push_back(r);
            d_perm.reserve(n);
            SB_CUDA(cudaMemcpyAsync(d_perm.p, h_perm.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
            chunk_launch(PAIRS_TRIANGLE, nc * n - (nc * (nc - 1)) / 2, d_perm.p, 0, 0, n, 0);
        }
        return finish(q_sum);
    }

    // Per-pair form of the postings: list by list into the output while the
    // triangle fits in L2 (its atomics stay on chip), else the row sweep
    // (partners counted in shared memory, each output written once).
    const bool big_out = tri_size(n) * sizeof(uint32_t) > L2_BYTES_B200;
    const double c_list = big_out ? cost.ns_per_posting_pair_hbm : cost.ns_per_posting_pair;
    // The row sweeps count partners in blocks of POST_SWEEP_MAX_ROWS rows,
    // reading each row's lists (or bins) once per block.
    auto sweep_blocks = [&](uint64_t q) { return (double)((q + POST_SWEEP_MAX_ROWS - 1) / POST_SWEEP_MAX_ROWS); };
    auto sweep_ns = [&](double incr, uint64_t q) {
        return (double)q * (double)q * cost.ns_per_sweep_row_pair + incr * cost.ns_per_posting_sweep * sweep_blocks(q);
    };
    auto sweep_form = [&](double incr, uint64_t q) {
        if (postings_mode == 2) return false;
        return postings_mode == 3 || (big_out && sweep_ns(incr, q) < incr * c_list);
    };
    // ns of the postings for a set of q rows with incr increments (sums need
    // only the histogram)
    auto post_ns = [&](double incr, uint64_t q) {
        const double per_pair = sweep_form(incr, q) ? sweep_ns(incr, q) : incr * c_list;
        return (d_out ? per_pair : 0.0) + (double)U * cost.ns_per_universe_value;
    };
    // ns of the run sweep with `checks` entry reads for q rows (per pair only)
    auto run_ns = [&](double checks, uint64_t q) {
        return (double)q * (double)q * cost.ns_per_sweep_row_pair + checks * cost.ns_per_run_check * sweep_blocks(q) +
               (double)n_bins * cost.ns_per_universe_value;
    };
    auto run_ok = [&](uint64_t q) {
        return d_out != nullptr && q >= 2 && postings_mode != 2 && postings_mode != 3;
    };
    std::vector<uint32_t> qrows, dense, mrows;             // L, H, M
    // L x L for `rest` (plain rows without bitmap chunks) by postings when
    // predicted faster than `alt` ns (or when forced): the run sweep when its
    // estimate beats the value postings' and its exact count (the piece
    // histogram) beats `alt`, else the value postings on their exact count
    // (the value histogram).
    auto decide = [&](const std::vector<uint32_t>& rest, double alt) -> bool {
        const uint64_t q = rest.size();
        if (q < 2) return false;
        bool lists_only = true;   // the value postings index list chunks only
        for (uint32_t r : rest) lists_only = lists_only && d.facts[r].bitmap_chunks == 0;
        if (run_ok(q)) {
            double P = 0.0, C1 = 0.0, C2 = 0.0;
            for (uint32_t r : rest) {
                const ChunkRowFacts& f = d.facts[r];
                P += pieces_est(f);
                C1 += (double)f.card;
                C2 += (double)f.card * (double)f.card;
            }
            const double run_e = run_ns(P * P * RW / (double)U, q);
            const double val_e = post_ns((C1 * C1 - C2) / (2.0 * (double)U), q);
            if (postings_mode == 4 || run_e < val_e || !lists_only) {
                run_histogram(rest);
                if (postings_mode == 4 || postings_mode == 1 || run_ns((double)run_checks, q) < alt) {
                    use_run = true;
                    qrows = rest;
                    return true;
                }
            }
        }
        if (!lists_only) return false;
        ps = histogram(rest);
        if (ps.entries < (1ull << 32) && (postings_mode > 0 || post_ns((double)ps.pairs, q) < alt)) {
            qrows = rest;
            return true;
        }
        return false;
    };
    bool panel_plan = false;
    // The panel needs a block of expanded rows and its transpose in HBM.
    const uint64_t panel_bytes = 2ull * PANEL_ROWS * W * sizeof(uint64_t);
    auto panel_fits = [&]() {
        if (!facts_ok || panel_mode == 0 || U > PANEL_MAX_UNIVERSE) return false;
        size_t fr = 0, tot = 0;
        SB_CUDA(cudaMemGetInfo(&fr, &tot));
        return (double)panel_bytes < 0.5 * ((double)fr + (double)(d_pX.n + d_DT.n) * sizeof(uint64_t));
    };

    if (panel_mode == 2 && facts_ok && U <= PANEL_MAX_UNIVERSE) {
        // Every plain row in the panel: all their pairs by the transposed
        // panel, rows queried against the blocks after them.
        for (uint32_t r = 0; r < n; ++r)
            if (d.facts[r].plain) mrows.push_back(r);
        panel_plan = true;
    } else if (tc_ok && dense_min_density > 0.0) {
        // Explicit threshold: plain rows with value count >= min_density x U.
        const double min_card = dense_min_density * (double)U;
        std::vector<uint32_t> rest;
        double chunk_rest = 0.0;
        for (uint32_t r = 0; r < n; ++r) {
            const ChunkRowFacts& f = d.facts[r];
            if (!f.plain) continue;
            if ((double)f.card >= min_card) {
                dense.push_back(r);
            } else if (post_ok && f.bitmap_chunks == 0) {
                rest.push_back(r);
                chunk_rest += chunk_self_pair_ns(cost, f, slots);
            }
        }
        if (rest.size() >= 2) decide(rest, 0.5 * ((double)rest.size() - 1.0) * chunk_rest);
    } else if (tc_ok && post_ok) {
        // Plain rows, heaviest first.  Plan A (no panel): rows with bitmap
        // chunks go to H, list rows join H while that lowers tensor time (H x
        // everything) + postings time (increments estimated as for
        // independent uniform rows, sum_{i<j} c_i c_j / U).  Plan B (panel):
        // the top h rows H, the next m rows M, the rest L; every row with a
        // bitmap chunk in H u M.  The cheaper predicted plan runs.
        std::vector<uint32_t> pl;
        for (uint32_t r = 0; r < n; ++r)
            if (d.facts[r].plain) pl.push_back(r);
        std::stable_sort(pl.begin(), pl.end(),
                         [&](uint32_t x, uint32_t y) { return d.facts[x].card > d.facts[y].card; });
        const uint64_t np = pl.size();
        std::vector<double> S1(np + 1, 0.0), S2(np + 1, 0.0), S3(np + 1, 0.0);
        uint64_t lb = 0;                                   // rows [0, lb) hold every bitmap-chunk row
        for (uint64_t t = 0; t < np; ++t) {
            const double c = (double)d.facts[pl[t]].card;
            S1[t + 1] = S1[t] + c;
            S2[t + 1] = S2[t] + c * c;
            S3[t + 1] = S3[t] + pieces_est(d.facts[pl[t]]);
            if (d.facts[pl[t]].bitmap_chunks) lb = t + 1;
        }
        // postings ns of the rows [from, np): the value form (rows without
        // bitmap chunks: from >= lb) or the run form (any plain rows)
        auto post_est = [&](uint64_t from) {
            const uint64_t q = np - from;
            if (q < 2) return 0.0;
            const double r1 = S1[np] - S1[from], r2 = S2[np] - S2[from];
            double v = from >= lb ? post_ns((r1 * r1 - r2) / (2.0 * (double)U), q) : HUGE_VAL;
            if (run_ok(q)) {
                const double P = S3[np] - S3[from];
                v = std::min(v, run_ns(P * P * RW / (double)U, q));
            }
            return v;
        };
        // Plan A: H = [0, k); the rows below k by postings.
        uint64_t best_k = lb;
        double best_a = -1.0;
        for (uint64_t k = 0; k <= np; ++k) {
            const double kk = (double)k;
            const double v = tc_ns * (kk * (kk - 1.0) / 2.0 + kk * (double)(np - k)) + post_est(k);
            if (best_a < 0 || v < best_a) {
                best_a = v;
                best_k = k;
            }
        }
        if (postings_mode == 4) best_k = 0;                // forced: every plain row to the run sweep
        else if (postings_mode > 0) best_k = lb;           // forced: every list row to the postings
        // Plan B over candidate cuts (h, m).
        uint64_t best_h = 0, best_m = 0;
        double best_b = -1.0;
        if (postings_mode < 0 && panel_mode != 0 && panel_fits()) {
            std::vector<uint64_t> cand{0, lb, np};
            for (double x = 1.0; x < (double)np; x *= 1.12) cand.push_back((uint64_t)x);
            std::sort(cand.begin(), cand.end());
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
            const double build_ns = 3.0 * (double)PANEL_ROWS * (double)W * 8.0 * cost.ns_per_panel_byte;
            for (uint64_t h : cand) {
                for (uint64_t e : cand) {                  // e = h + m
                    if (e < h || e > np || e == 0) continue;   // rows past e: postings (value or run form)
                    if (panel_mode > 0 && e == h) continue;    // forced: some rows in M
                    const double m = (double)(e - h), hh = (double)h, nl = (double)(np - e);
                    const double nb = std::ceil((double)e / PANEL_ROWS);
                    const double nbh = hh / PANEL_ROWS, nbm = m / PANEL_ROWS;
                    const double sl = S1[np] - S1[e], sm = S1[e] - S1[h];
                    const double panel = cost.ns_per_panel_value * (sl * nb + sm * (nbh + 0.5 * nbm + 0.5)) +
                                         cost.ns_per_panel_pair * (nl * (double)e + m * (m - 1.0) / 2.0 + m * hh) +
                                         nb * build_ns;
                    const double v = tc_ns * hh * (hh - 1.0) / 2.0 + panel + post_est(e);
                    if (best_b < 0 || v < best_b) {
                        best_b = v;
                        best_h = h;
                        best_m = e - h;
                    }
                }
            }
        }
        panel_plan = best_b >= 0 && (panel_mode > 0 || best_b < best_a);
        std::vector<uint32_t> rest;
        if (panel_plan) {
            dense.assign(pl.begin(), pl.begin() + best_h);
            mrows.assign(pl.begin() + best_h, pl.begin() + best_h + best_m);
            rest.assign(pl.begin() + best_h + best_m, pl.end());
        } else {
            dense.assign(pl.begin(), pl.begin() + best_k);
            rest.assign(pl.begin() + best_k, pl.end());
        }
        std::sort(rest.begin(), rest.end());               // stored order: ascending output writes
        if (rest.size() >= 2) {
            // The estimate assumes independent rows; correlated rows share
            // more. With the exact count, keep the postings only if they beat
            // the alternative on these pairs: the panel (the rows queried
            // against themselves) or the tensor cores.
            const double q = (double)rest.size();
            const double alt = panel_plan ? cost.ns_per_panel_value * (S1[np] - S1[np - rest.size()]) *
                                                (0.5 * std::ceil(q / PANEL_ROWS) + 0.5) +
                                                cost.ns_per_panel_pair * q * (q - 1.0) / 2.0
                                          : tc_ns * (q * (q - 1.0) / 2.0);
            if (decide(rest, alt)) {
            } else if (panel_plan) {
                mrows.insert(mrows.end(), rest.begin(), rest.end());
            } else {
                dense.insert(dense.end(), rest.begin(), rest.end());
            }
        } else if (panel_plan) {
            mrows.insert(mrows.end(), rest.begin(), rest.end());
        } else {
            dense.insert(dense.end(), rest.begin(), rest.end());
        }
    } else if (tc_ok) {
        // Per-row rule: plain rows whose chunk-kernel cost against a row
        // like themselves exceeds a tensor-core pair.
        for (uint32_t r = 0; r < n; ++r) {
            const ChunkRowFacts& f = d.facts[r];
            if (f.plain && chunk_self_pair_ns(cost, f, slots) >= tc_ns) dense.push_back(r);
        }
    } else if (post_ok) {
        std::vector<uint32_t> rest;
        double chunk_rest = 0.0;
        for (uint32_t r = 0; r < n; ++r) {
            const ChunkRowFacts& f = d.facts[r];
            if (f.plain && f.bitmap_chunks == 0) {
                rest.push_back(r);
                chunk_rest += chunk_self_pair_ns(cost, f, slots);
            }
        }
        if (rest.size() >= 2) decide(rest, 0.5 * ((double)rest.size() - 1.0) * chunk_rest);
    }
    if (panel_plan && mrows.empty() && dense.empty()) panel_plan = false;
    // Rows the tensor cores expand behind the H rows: the L rows in the plan
    // without a panel (H x L on the tensor cores), none with it.
    const std::vector<uint32_t> none;
    const std::vector<uint32_t>& tq = panel_plan ? none : qrows;
    // The tensor cores take H x H (and H x tq): expanded rows in the order
    // [H | padding to a multiple of 256 | tq], so that every 128-row and
    // 256-row block is all H or all tq and the tq x tq blocks can be left out.
    // Panels of P rows when they do not all fit the budget.
    if (panel_plan) {
        d_pX.reserve(PANEL_ROWS * W);
        d_DT.reserve(PANEL_ROWS * W);
    }
    const uint64_t nd0 = dense.size();
    const uint64_t nd_pad = round_up(nd0, 256);
    const uint64_t ne = nd0 ? nd_pad + tq.size() : 0;
    uint64_t P = 0;
    if (ne) {
        uint64_t budget = dense_budget_bytes;
        if (!budget) {
            size_t fr = 0, tot = 0;
            SB_CUDA(cudaMemGetInfo(&fr, &tot));
            budget = (uint64_t)(0.6 * (double)(fr + d_panel.n * sizeof(uint64_t)));
        }
        const uint64_t cap_rows = budget / (panel_row_words(W) * sizeof(uint64_t));
        P = round_up(ne, 256) <= cap_rows ? round_up(ne, 256) : cap_rows / 2 / 256 * 256;
        if (P == 0) {   // not even two panels fit: the H rows go to the chunk kernel (or the panel)
            if (panel_plan) mrows.insert(mrows.end(), dense.begin(), dense.end());
            dense.clear();
        }
    }
    for (uint32_t r : qrows) cls[r] = 1;
    for (uint32_t r : mrows) cls[r] = 2;
    for (uint32_t r : dense) cls[r] = 3;
    // Walk order: C, L, M, H rows.
    std::vector<uint32_t> h_perm;
    h_perm.reserve(n);
    for (int k = 0; k < 4; ++k)
        for (uint32_t r = 0; r < n; ++r)
            if (cls[r] == k) h_perm.push_back(r);
    const uint64_t nd = dense.size(), nq = qrows.size(), nm = mrows.size(), nc = n - nd - nq - nm;
    const uint32_t* perm = nullptr;
    if (nd || nq || nm) {
        d_perm.reserve(n);
        SB_CUDA(cudaMemcpyAsync(d_perm.p, h_perm.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        perm = d_perm.p;
        // The tensor cores (stream-K) and the postings add into the triangle.
        if (d_out) SB_CUDA(cudaMemsetAsync(d_out, 0, tri_size(n) * sizeof(uint32_t), st));
    }

    // ---- predicted device time of each engine for this plan
    for (int k = 0; k < 4; ++k) last_engine_ms[k] = last_engine_pred_ms[k] = last_engine_work[k] = 0.0;
    for (cudaEvent_t& e : ev_eng)
        if (!e) SB_CUDA(cudaEventCreate(&e));
    {
        const double dd = (double)nd, tqn = (double)tq.size();
        last_engine_pred_ms[0] = 1e-6 * tc_ns * (dd * (dd + 1.0) / 2.0 + dd * tqn);
        last_engine_work[0] = 2.0 * (dd * (dd + 1.0) / 2.0 + dd * tqn) * (double)U;
        last_engine_work[1] = (double)(nc * n - (nc * (nc - 1)) / 2 * (nc ? 1 : 0));
        if (panel_plan && (nm || nd) && (nq + nm)) {
            const double npw = (double)(nm + nd), nb = std::ceil(npw / PANEL_ROWS);
            double vb = 0.0, pairs = 0.0;
            for (uint64_t w = nc; w < nc + nq + nm; ++w) {
                const double after = (double)(n - 1 - w) < npw ? (double)(n - 1 - w) : npw;   // panel rows after it
                vb += (double)d.facts[h_perm[w]].card * std::ceil(after / PANEL_ROWS);
                pairs += after;
            }
            last_engine_pred_ms[2] = 1e-6 * (cost.ns_per_panel_value * vb + cost.ns_per_panel_pair * pairs +
                                             nb * 3.0 * PANEL_ROWS * (double)W * 8.0 * cost.ns_per_panel_byte);
            last_engine_work[2] = 256.0 * vb + 4.0 * pairs + nb * 3.0 * PANEL_ROWS * (double)W * 8.0;
        }
        if (nq && use_run) {
            // run sweep: the pieces (8 B each, written and read), the bin
            // entries each piece reads (8 B), 4 B per count of the slice
            last_engine_pred_ms[3] = 1e-6 * run_ns((double)run_checks, nq);
            double pcs = 0.0;
            for (uint32_t k : h_rpieces) pcs += (double)k;
            last_engine_work[3] = 16.0 * pcs + 8.0 * (double)run_entries + 8.0 * (double)run_checks +
                                  4.0 * (double)nq * ((double)nq + 1.0) / 2.0 + 4.0 * (double)n_bins;
        } else if (nq) {
            last_engine_pred_ms[3] = 1e-6 * post_ns((double)ps.pairs, nq);
            double vals = 0.0;
            for (uint32_t r : qrows) vals += (double)d.facts[r].card;
            last_engine_work[3] = 8.0 * vals + 8.0 * (double)ps.entries + 8.0 * (double)ps.pairs + 8.0 * (double)U;
        }
    }
    SB_CUDA(cudaEventRecord(ev_eng[0], st));   // the postings' histogram and the set-up precede it

    // ---- tensor cores: H x H and H x tq, panel by panel
    if (nd) {
        std::vector<uint32_t> emap(nd_pad + tq.size(), ~0u);   // expanded row -> stored row (~0: padding)
        std::copy(dense.begin(), dense.end(), emap.begin());
        std::copy(tq.begin(), tq.end(), emap.begin() + nd_pad);
        const uint64_t ne2 = emap.size();
        const bool single = P >= round_up(ne2, 256);
        const uint64_t rows_alloc = single ? P : 2 * P;
        // Block-major panels: chunk slot s of every expanded row together,
        // rows PANEL_PITCH words apart within it (see panel_row_words).
        const RowLayout lay{PANEL_PITCH, rows_alloc * PANEL_PITCH};
        d_panel.reserve(rows_alloc * panel_row_words(W));
        d_map.reserve(rows_alloc);
        d_tiles.reserve((P / 128) * (2 * P / 256 + 1));
        const uint64_t npan = single ? 1 : (ne2 + P - 1) / P;
        auto is_q = [&](uint64_t global_row) { return global_row >= nd_pad; };
        std::vector<uint2> tl;
        auto expand = [&](uint64_t first, uint64_t m, uint64_t slot) {
            SB_CUDA(cudaMemcpyAsync(d_map.p + slot, emap.data() + first, m * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice, st));
            const uint32_t grid = (uint32_t)std::min<uint64_t>(m, (uint64_t)sms * 16);
            expand_rows_kernel<<<grid, EXPAND_WARPS * 32, 0, st>>>(d.view(), d_map.p + slot, (uint32_t)m,
                                                                   (uint32_t)W, lay, d_panel.p + slot * lay.pitch);
            SB_CUDA(cudaGetLastError());
            ++launches;
        };
        auto tensor = [&](uint64_t n_local) {
            if (tl.empty()) return;
            SB_CUDA(cudaMemcpyAsync(d_tiles.p, tl.data(), tl.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
            launch_ts_rows(d_panel.p, (uint32_t)n_local, (uint32_t)W, lay, d_tiles.p, (uint32_t)tl.size(), d_out,
                           d_flags.p, d_map.p, n, st, /*out_zeroed=*/true);
            ++launches;
        };
        for (uint64_t I = 0; I < npan; ++I) {
            const uint64_t gI = I * P, mI = std::min<uint64_t>(P, ne2 - gI);
            if (is_q(gI)) break;                          // this and later panels are all tq
            expand(gI, mI, 0);
            std::vector<uint2> tri;
            build_mma_tiles(tri, mI);                      // I x I triangle, tq x tq blocks left out
            tl.clear();
            for (const uint2& t : tri)
                if (!(is_q(gI + (uint64_t)t.x * 128) && is_q(gI + (uint64_t)t.y * 256))) tl.push_back(t);
            tensor(mI);
            for (uint64_t J = I + 1; J < npan; ++J) {      // I x J rectangle (I is a full panel)
                const uint64_t gJ = J * P, mJ = std::min<uint64_t>(P, ne2 - gJ);
                expand(gJ, mJ, P);
                tl.clear();
                for (uint32_t bi = 0; bi < P / 128; ++bi) {
                    if (is_q(gI + (uint64_t)bi * 128) && is_q(gJ)) continue;
                    for (uint32_t bj = (uint32_t)(P / 256); bj < (uint32_t)((P + mJ + 255) / 256); ++bj)
                        if (!(is_q(gI + (uint64_t)bi * 128) && is_q(gJ + (uint64_t)bj * 256 - P)))
                            tl.push_back(make_uint2(bi, bj));
                }
                tensor(P + mJ);
            }
        }
        last_dense_rows = nd;
        last_dense_panels = npan;
    }
    SB_CUDA(cudaEventRecord(ev_eng[1], st));
    // ---- chunk kernel: every pair with a C row (the walk's triangle prefix)
    chunk_launch(PAIRS_TRIANGLE, nc * n - (nc * (nc - 1)) / 2 * (nc ? 1 : 0), perm, 0, 0, n, 0);
    SB_CUDA(cudaEventRecord(ev_eng[2], st));
    // ---- transposed panel: (L u M) x (M u H), blocks of PANEL_ROWS panel rows
    if (panel_plan && (nm || nd) && (nq + nm)) {
        const uint64_t pw0 = nc + nq;                      // walk position of the first panel row
        const uint64_t npw = nm + nd;
        // Work items over the query rows (walk positions of L and M),
        // heaviest first: a row with more than `seg` values is split into
        // ranges of its chunks (about seg values each), so that the warps
        // finish together; seg is sized for ~64 items per SM and at least
        // PANEL_MIN_SEG values (the per-item epilogue costs about as much as
        // a few hundred values), and doubled until the split rows' scratch
        // slots fit PANEL_MAX_SLOTS.
        uint64_t max_card = 0;
        double total = 0.0;
        for (uint64_t w = nc; w < nc + nq + nm; ++w) {
            const uint64_t c = d.facts[h_perm[w]].card;
            max_card = std::max<uint64_t>(max_card, c);
            total += (double)c;
        }
        std::vector<PanelItem> items;
        std::vector<PanelSplit> splits;
        std::vector<double> weight;
        uint32_t nslots = 0;
        for (uint64_t seg = std::max<uint64_t>(PANEL_MIN_SEG, (uint64_t)(total / (64.0 * sms)));; seg *= 2) {
            items.clear();
            splits.clear();
            weight.clear();
            nslots = 0;
            for (uint64_t w = nc; w < nc + nq + nm; ++w) {
                const ChunkRowFacts& f = d.facts[h_perm[w]];
                const uint32_t ns =
                    f.card > seg && f.chunks > 1 ? (uint32_t)std::min<uint64_t>(f.chunks, (f.card + seg - 1) / seg) : 1u;
                if (ns == 1) {
                    items.push_back(PanelItem{(uint32_t)w, 0u, f.chunks, PANEL_NO_VALUE});
                    weight.push_back((double)f.card);
                    continue;
                }
                splits.push_back(PanelSplit{(uint32_t)w, nslots, ns, 0u});
                for (uint32_t k = 0; k < ns; ++k) {
                    const uint32_t lo = (uint32_t)((uint64_t)f.chunks * k / ns);
                    const uint32_t hi = (uint32_t)((uint64_t)f.chunks * (k + 1) / ns);
                    items.push_back(PanelItem{(uint32_t)w, lo, hi, nslots + k});
                    weight.push_back((double)f.card * (double)(hi - lo) / (double)f.chunks);
                }
                nslots += ns;
            }
            if (nslots <= PANEL_MAX_SLOTS) break;
        }
        {
            std::vector<uint32_t> ord(items.size());
            for (uint32_t k = 0; k < ord.size(); ++k) ord[k] = k;
            std::stable_sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return weight[x] > weight[y]; });
            std::vector<PanelItem> sorted(items.size());
            for (uint32_t k = 0; k < ord.size(); ++k) sorted[k] = items[ord[k]];
            items.swap(sorted);
        }
        d_items.reserve(items.size());
        d_ctr.reserve(1);
        d_pmap.reserve(PANEL_ROWS);
        SB_CUDA(cudaMemcpyAsync(d_items.p, items.data(), items.size() * sizeof(PanelItem), cudaMemcpyHostToDevice, st));
        if (!splits.empty()) {
            d_splits.reserve(splits.size());
            d_pscratch.reserve((uint64_t)nslots * PANEL_ROWS);
            SB_CUDA(cudaMemcpyAsync(d_splits.p, splits.data(), splits.size() * sizeof(PanelSplit),
                                    cudaMemcpyHostToDevice, st));
        }
        static std::atomic<uint64_t> t_done{0};
        smem_attr_once(panel_transpose_kernel, (int)PANEL_T_SMEM, t_done);
        std::vector<uint32_t> bmap(PANEL_ROWS);
        const uint32_t qgrid = (uint32_t)sms * 8;
        for (uint64_t b0 = 0; b0 < npw; b0 += PANEL_ROWS) {
            const uint32_t prows = (uint32_t)std::min<uint64_t>(PANEL_ROWS, npw - b0);
            for (uint32_t t = 0; t < PANEL_ROWS; ++t) bmap[t] = t < prows ? h_perm[pw0 + b0 + t] : ~0u;
            SB_CUDA(cudaMemcpyAsync(d_pmap.p, bmap.data(), PANEL_ROWS * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
            expand_rows_kernel<<<(uint32_t)std::min<uint64_t>(PANEL_ROWS, (uint64_t)sms * 16), EXPAND_WARPS * 32, 0,
                                 st>>>(d.view(), d_pmap.p, PANEL_ROWS, (uint32_t)W, row_major(W), d_pX.p);
            panel_transpose_kernel<<<(uint32_t)(W / PANEL_T_WORDS), 1024, PANEL_T_SMEM, st>>>(d_pX.p, W, d_DT.p);
            SB_CUDA(cudaMemsetAsync(d_ctr.p, 0, sizeof(unsigned long long), st));
            const uint32_t ni = (uint32_t)items.size();
            uint32_t* scr = splits.empty() ? nullptr : d_pscratch.p;
#define SB_PANEL_QUERY(NP)                                                                                      \
    panel_query_kernel<NP><<<qgrid, PANEL_Q_WARPS * 32, 0, st>>>(d.view(), perm, d_items.p, ni, pw0 + b0, prows, \
                                                                 d_DT.p, n, d_out, scr, d_flags.p, d_ctr.p)
            if (max_card < (1ull << 11)) SB_PANEL_QUERY(8);
            else if (max_card < (1ull << 15)) SB_PANEL_QUERY(12);
            else if (max_card < (1ull << 19)) SB_PANEL_QUERY(16);
            else if (max_card < (1ull << 23)) SB_PANEL_QUERY(20);
            else SB_PANEL_QUERY(24);
#undef SB_PANEL_QUERY
            launches += 3;
            if (scr && d_out) {
                panel_reduce_kernel<<<(uint32_t)std::min<uint64_t>(splits.size(), (uint64_t)sms * 8), 256, 0, st>>>(
                    perm, d_splits.p, (uint32_t)splits.size(), pw0 + b0, prows, scr, n, d_out);
                ++launches;
            }
            SB_CUDA(cudaGetLastError());
        }
        last_panel_rows = npw;
        last_panel_queries = nq + nm;
    }
    SB_CUDA(cudaEventRecord(ev_eng[3], st));
    // ---- L x L by postings
    uint64_t q_sum = 0;
    last_postings_form = -1;
    if (nq && use_run) {
        // run sweep (the sum over these pairs is added by the kernel)
        last_postings_form = 2;
        std::vector<uint64_t> poff(nq + 1, 0);
        for (uint64_t k = 0; k < nq; ++k) poff[k + 1] = poff[k] + h_rpieces[k];
        d_rpoff.reserve(nq + 1);
        SB_CUDA(cudaMemcpyAsync(d_rpoff.p, poff.data(), (nq + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        d_pieces.reserve(poff[nq] ? poff[nq] : 1);
        d_rstart.reserve(n_bins);
        d_rlist.reserve(run_entries ? run_entries : 1);
        d_pstats.reserve(1);
        SB_CUDA(cudaMemsetAsync(d_pstats.p, 0, sizeof(PostingsStats), st));
        const uint32_t gq = (uint32_t)std::min<uint64_t>((nq + 7) / 8, (uint64_t)sms * 16);
        run_fill_kernel<<<gq, 256, 0, st>>>(d.view(), d_qrows.p, (uint32_t)nq, rwlog, d_rpoff.p, d_pieces.p);
        postings_alloc_kernel<<<sms * 8, 256, 0, st>>>(d_rbins.p, n_bins, d_rstart.p, nullptr, d_pstats.p);
        run_scatter_kernel<<<gq, 256, 0, st>>>((uint32_t)nq, rwlog, d_rpoff.p, d_pieces.p, d_rstart.p, d_rlist.p);
        static std::atomic<uint64_t> done{0};
        smem_attr_once(run_sweep_kernel, (int)((POST_SWEEP_MAX_ROWS + RUN_SWEEP_BATCH + 1) * sizeof(uint32_t)), done);
        const uint32_t gr = (uint32_t)std::min<uint64_t>(nq, (uint64_t)sms * 8);
        for (uint64_t pb0 = 0; pb0 < nq; pb0 += POST_SWEEP_MAX_ROWS) {
            const uint32_t pbn = (uint32_t)std::min<uint64_t>(POST_SWEEP_MAX_ROWS, nq - pb0);
            const uint32_t smem = (uint32_t)((pbn + RUN_SWEEP_BATCH + 1) * sizeof(uint32_t));
            run_sweep_kernel<<<gr, POST_SWEEP_THREADS, smem, st>>>(d_qrows.p, (uint32_t)nq, d_rpoff.p, d_pieces.p,
                                                                   rwlog, d_rbins.p, d_rstart.p, d_rlist.p, n, d_out,
                                                                   d_flags.p, (uint32_t)pb0, pbn);
            ++launches;
        }
        SB_CUDA(cudaGetLastError());
        launches += 3;
        last_postings_rows = nq;
    } else if (nq) {
        q_sum = ps.pairs;
        const bool sweep = sweep_form((double)ps.pairs, nq);
        last_postings_form = sweep ? 1 : 0;
        if (d_out) {
            d_start.reserve(U);
            d_lists.reserve(ps.lists ? ps.lists : 1);
            d_post.reserve(ps.entries ? ps.entries : 1);
            postings_alloc_kernel<<<sms * 8, 256, 0, st>>>(d_counts.p, U, d_start.p, d_lists.p, d_pstats.p);
            const uint32_t gq = (uint32_t)std::min<uint64_t>((nq + 7) / 8, (uint64_t)sms * 16);
            postings_scatter_kernel<<<gq, 256, 0, st>>>(d.view(), d_qrows.p, (uint32_t)nq, d_start.p, d_post.p);
            if (sweep) {
                static std::atomic<uint64_t> done{0};
                smem_attr_once(postings_rows_kernel,
                               (int)((POST_SWEEP_MAX_ROWS + POST_SWEEP_MAX_CHUNKS + 1) * sizeof(uint32_t)), done);
                const uint32_t gr = (uint32_t)std::min<uint64_t>(nq, (uint64_t)sms * 8);
                for (uint64_t pb0 = 0; pb0 < nq; pb0 += POST_SWEEP_MAX_ROWS) {
                    const uint32_t pbn = (uint32_t)std::min<uint64_t>(POST_SWEEP_MAX_ROWS, nq - pb0);
                    const uint32_t smem = (uint32_t)((pbn + POST_SWEEP_MAX_CHUNKS + 1) * sizeof(uint32_t));
                    postings_rows_kernel<<<gr, POST_SWEEP_THREADS, smem, st>>>(
                        d.view(), d_qrows.p, (uint32_t)nq, d_counts.p, d_start.p, d_post.p, n, d_out, (uint32_t)pb0, pbn);
                    ++launches;
                }
                launches += 2;
            } else {
                const uint32_t gp = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((ps.lists + 255) / 256,
                                                                                       (uint64_t)sms * 16));
                postings_pairs_kernel<<<gp, 256, 0, st>>>(d_lists.p, ps.lists, d_post.p, d_qrows.p, n, d_out);
                postings_diag_kernel<<<(uint32_t)std::min<uint64_t>((nq + 255) / 256, (uint64_t)sms * 4), 256, 0,
                                       st>>>(d.view(), d_qrows.p, (uint32_t)nq, n, d_out);
                launches += 4;
            }
            SB_CUDA(cudaGetLastError());
        }
        last_postings_rows = nq;
    }
    // ---- diagonal of the M rows (no other engine pairs them with themselves)
    if (nm && d_out) {
        d_mrows.reserve(nm);
        SB_CUDA(cudaMemcpyAsync(d_mrows.p, h_perm.data() + nc + nq, nm * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        row_card_diag_kernel<<<(uint32_t)std::min<uint64_t>((nm + 7) / 8, (uint64_t)sms * 16), 256, 0, st>>>(
            d.view(), d_mrows.p, (uint32_t)nm, n, d_out);
        SB_CUDA(cudaGetLastError());
        ++launches;
    }
    const uint64_t total = finish(q_sum);
    float t_pre = 0, t_hist = 0, t_tc = 0, t_ch = 0, t_pa = 0, t_po = 0;
    SB_CUDA(cudaEventElapsedTime(&t_pre, log.ev0, ev_eng[0]));
    if (hist_ran) SB_CUDA(cudaEventElapsedTime(&t_hist, ev_hist0, ev_hist));
    SB_CUDA(cudaEventElapsedTime(&t_tc, ev_eng[0], ev_eng[1]));
    SB_CUDA(cudaEventElapsedTime(&t_ch, ev_eng[1], ev_eng[2]));
    SB_CUDA(cudaEventElapsedTime(&t_pa, ev_eng[2], ev_eng[3]));
    SB_CUDA(cudaEventElapsedTime(&t_po, ev_eng[3], log.ev1));
    last_engine_ms[0] = t_tc;
    last_engine_ms[1] = t_ch;
    last_engine_ms[2] = t_pa;
    last_engine_ms[3] = t_po + (nq ? t_hist : 0.f);
    // the rest of the time before the engines: planning on the host while
    // the GPU waits (before the histogram and after its statistics are read
    // back), the row order's upload and the output's clearing
    last_plan_ms = nq ? t_pre - t_hist : t_pre;
    return total;
}

}  // namespace sb200
