"""STORM_contiguous_t on the GPU against the oracle and the reference's
golden vectors: both bitmap x bitmap kernels (CUDA-core POPC and tcgen05),
bit-exact, on the reference's own cases, edge shapes and the full-size
dense configurations (sampled pairs + size-independent identities)."""
import os

import numpy as np
import pytest

import gen
import oracle_lib as ol

pytestmark = pytest.mark.gpu

KERNELS = ("popc", "mma", "mma_ss", "mma_db", "mma_2cta")


def _kernel(sb, name):
    return {"popc": sb.KERNEL_POPC, "mma": sb.KERNEL_MMA, "mma_ss": sb.KERNEL_MMA_SS, "mma_db": sb.KERNEL_MMA_DB,
            "mma_2cta": sb.KERNEL_MMA_2CTA}[name]


def contig_from_words(sb, words, m, kernel):
    c = sb.StormContig(m)
    c.set_kernel(_kernel(sb, kernel))
    c.add_bitmaps(words)
    return c


@pytest.mark.parametrize("kernel", KERNELS)
def test_golden_contig_cases(sb, golden, kernel):
    names = sorted({k.split("/")[1] for k in golden.files if k.startswith("contig/")})
    for name in names:
        words = golden[f"contig/{name}/words"]
        m = int(golden[f"contig/{name}/m"][0])
        c = contig_from_words(sb, words, m, kernel)
        mat, s = c.matrix()
        assert s == int(golden[f"contig/{name}/sum"][0]), name
        np.testing.assert_array_equal(mat, golden[f"contig/{name}/matrix"], err_msg=f"{name}/{kernel}")
        assert c.pairw_intersect_cardinality() == s
        assert c.last_kernel() == _kernel(sb, kernel)


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("n,m,p", [
    (1, 64, 0.5), (2, 65, 0.5), (3, 640, 0.9), (127, 1000, 0.3), (128, 4096, 0.5), (129, 4097, 0.2),
    (255, 512, 0.5), (256, 128, 0.7), (257, 8192, 0.01), (300, 2048 + 64, 0.5), (513, 256, (0.0, 1.0)),
    (300, (1 << 17) + 64, 0.3),   # long rows: the tensor kernel's lean (unstaged) epilogue
])
def test_edge_shapes_match_oracle(sb, kernel, n, m, p):
    words = gen.bernoulli_rows(n, m, p, seed=1000 + n + m)
    c = contig_from_words(sb, words, m, kernel)
    mat, s = c.matrix()
    want, ws = ol.contig_matrix(words)
    assert s == ws
    np.testing.assert_array_equal(mat, want)


@pytest.mark.parametrize("kernel", ("mma", "mma_db", "mma_2cta"))
def test_long_rows_tensor_kernel(sb, kernel):
    """Rows past 2^23 bits take the 4-byte weight cycle (D = 8 x count):
    random rows, and all-ones rows of 2^26 bits (count 2^26, D = 2^29)."""
    m = (1 << 23) + 4096
    words = gen.bernoulli_rows(40, m, 0.3, 4242)
    c = contig_from_words(sb, words, m, kernel)
    mat, s = c.matrix()
    want, ws = ol.contig_matrix(words)
    assert s == ws
    np.testing.assert_array_equal(mat, want)
    m = 1 << 26
    ones = np.full((3, m // 64), np.uint64(0xFFFFFFFFFFFFFFFF), dtype=np.uint64)
    ones[1, ::2] = 0
    c = contig_from_words(sb, ones, m, kernel)
    mat, s = c.matrix()
    want, ws = ol.contig_matrix(ones)
    assert s == ws and mat[0] == m
    np.testing.assert_array_equal(mat, want)


def test_all_ones_and_empty_rows(sb):
    m = 4096
    words = np.zeros((260, m // 64), dtype=np.uint64)
    words[::3] = np.uint64(0xFFFFFFFFFFFFFFFF)
    words[1::7, 5] = np.uint64(1)
    for kernel in KERNELS:
        c = contig_from_words(sb, words, m, kernel)
        mat, s = c.matrix()
        want, ws = ol.contig_matrix(words)
        assert s == ws
        np.testing.assert_array_equal(mat, want)


def test_add_positions_with_duplicates_matches_set_semantics(sb):
    g = gen.rng(7)
    m = 8192
    c = sb.StormContig(m)
    sets = []
    for r in range(70):
        v = np.sort(g.integers(0, m, size=int(g.integers(1, 300)))).astype(np.uint32)  # duplicates kept
        assert c.add(v) == v.size
        sets.append(np.unique(v))
    assert c.add(np.zeros(0, np.uint32)) == 0       # reference: n == 0 adds no row
    assert len(c) == 70
    mat, s = c.matrix()
    want, ws = ol.contig_matrix(gen.sets_to_rows(sets, m))
    assert s == ws
    np.testing.assert_array_equal(mat, want)


def test_mixed_ingest_order_clear_and_reuse(sb):
    m = 1000
    a = gen.bernoulli_rows(40, m, 0.2, 3)
    b = gen.bernoulli_rows(50, m, 0.4, 4)
    c = sb.StormContig(m)
    for row in gen.rows_to_sets(a, m):
        c.add(row) if row.size else None
    c.add_bitmaps(b)
    rows = np.concatenate([np.stack([r for r, s in zip(a, gen.rows_to_sets(a, m)) if s.size]), b])
    mat, s = c.matrix()
    want, ws = ol.contig_matrix(rows)
    np.testing.assert_array_equal(mat, want)
    assert c.clear() == 1 and len(c) == 0
    c.add_bitmaps(b)
    mat, s = c.matrix()
    want, ws = ol.contig_matrix(b)
    np.testing.assert_array_equal(mat, want)


def test_device_input_tail_bits_are_masked(sb):
    torch = pytest.importorskip("torch")
    m = 100   # 2 words, 36 tail bits
    words = gen.bernoulli_rows(33, 128, 0.5, 9)   # random bits beyond m
    d = torch.from_numpy(words.view(np.int64)).cuda()
    c = sb.StormContig(m)
    rc = sb.lib().STORM_contig_add_bitmaps(c.h, sb.C.cast(d.data_ptr(), sb.u64p), 33, 2)
    assert rc == 33
    mat, _ = c.matrix()
    masked = words.copy()
    masked[:, 1] &= np.uint64((1 << 36) - 1)
    want, _ = ol.contig_matrix(masked)
    np.testing.assert_array_equal(mat, want)


@pytest.mark.parametrize("tile", [8, 64, 100])
def test_tiles_callback_matches_matrix(sb, tile):
    words = gen.bernoulli_rows(150, 2048, 0.3, 77)
    c = contig_from_words(sb, words, 2048, "mma")
    mat, s = c.matrix()
    col = c.tiles(tile)
    n = 150
    iu = np.triu_indices(n)
    strict = iu[0] != iu[1]
    np.testing.assert_array_equal(col.out[strict], mat[strict])
    assert sum(x[4] for x in col.calls) == s
    # every tile of the triangle visited once, diagonal tiles included
    nt = (n + tile - 1) // tile
    assert len(col.calls) == nt * (nt + 1) // 2


def test_wrappers_and_lowlevel_match_reference(sb, golden):
    w = golden["wrapper_diag/words"]
    assert sb.wrapper_diag(w) == golden["wrapper_diag/sum"][0]
    assert sb.wrapper_diag(w, blocked=4) == golden["wrapper_diag/sum"][1]
    v1, v2 = w[:10], w[10:]
    want = sum(ol.and_popcount(x, y) for x in v1 for y in v2)
    assert sb.wrapper_square(v1, v2) == want


def _cfg_rows_gpu(n, m, p, seed):
    torch = pytest.importorskip("torch")
    import bench
    return bench.bernoulli_rows_gpu(n, m, p, seed, torch.device("cuda"))


def _check_full_size(sb, n, m, p, seed, kernels, every_pair=False):
    """Full-size dense configuration: device-resident output, checked by
    (a) oracle on every pair of a row sample -- or, with every_pair, the whole
    triangle against the reference's own AND+popcount kernel on all host
    threads (the oracle where the reference was not built), (b) diagonal = row
    popcounts, (c) kernel-vs-kernel identity, (d) sum identity."""
    import torch
    rows = _cfg_rows_gpu(n, m, p, seed)           # int64 [n, w] on device
    host = rows.cpu().numpy().view(np.uint64)
    tri = n * (n + 1) // 2
    results = {}
    for k in kernels:
        c = sb.StormContig(m)
        c.set_kernel(_kernel(sb, k))
        c.add_bitmaps(host)
        out = torch.empty(tri, dtype=torch.int32, device="cuda")
        s = c.matrix_device(out.data_ptr(), tri)
        results[k] = (out, s)
    out, s = results[kernels[0]]
    # (a) sampled rows, every pair of each: oracle on the host.
    g = gen.rng(seed)
    sample = np.unique(np.concatenate([[0, n - 1], g.integers(0, n, size=6)]))
    for i in sample:
        want = ol.contig_row(host, int(i))
        base = int(sb.tri_index(n, i, i))
        got = out[base: base + (n - i)].cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, want, err_msg=f"row {i}")
    if every_pair:
        want = np.zeros(tri, np.uint32)
        R = ol.reference()
        if R is not None:
            ws = R.ref_contig_matrix_mt(host.ctypes.data_as(ol.u64p), n, host.shape[1], 0, n,
                                        want.ctypes.data_as(ol.u32p), os.cpu_count() or 1)
        else:
            want, ws = ol.contig_matrix(host)
        assert ws == s
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), want)
    # (b) diagonal
    ii = np.arange(n, dtype=np.uint64)
    diag_idx = torch.from_numpy(sb.tri_index(n, ii, ii).astype(np.int64)).cuda()
    diag = out[diag_idx].cpu().numpy().view(np.uint32)
    pc = ol.row_popcounts(host).astype(np.int64)
    np.testing.assert_array_equal(diag, pc)
    # (c) kernels agree bit for bit
    for k in kernels[1:]:
        assert torch.equal(results[k][0], out), k
        assert results[k][1] == s
    # (d) sum over i < j = total - trace
    total = int(out.view(torch.int32).to(torch.int64).bitwise_and(0xFFFFFFFF).sum().item())
    assert s == total - int(pc.sum())


def test_config1_full_size_every_pair(sb):
    """4096 rows x 65536 bits, Bernoulli(0.5): all 8,390,656 pairs against the
    reference's own kernel, and the four bitmap x bitmap kernels bit for bit."""
    _check_full_size(sb, 4096, 65536, 0.5, 101, ["mma", "mma_db", "mma_ss", "mma_2cta", "popc"], every_pair=True)


def test_config5a_haplotypes_full_size(sb):
    """200,000 sites x 20,000 haplotypes, 1/k allele counts in 32-haplotype
    blocks: 2.0e10 pairs, 80 GB of counts kept in HBM.  Checked on sampled
    whole rows against the oracle, the diagonal and the sum identity."""
    import torch
    import bench
    n, m = 200000, 20000
    rows = bench.haplotype_rows_gpu(n, m, 32, 55, torch.device("cuda"))
    host = rows.cpu().numpy().view(np.uint64)
    pc = ol.row_popcounts(host).astype(np.int64)
    assert pc.min() >= 1 and pc.max() <= m - 1
    c = sb.StormContig(m)
    c.add_bitmaps(host)
    tri = n * (n + 1) // 2
    out = torch.empty(tri, dtype=torch.int32, device="cuda")
    s = c.matrix_device(out.data_ptr(), tri)
    assert c.last_kernel() == sb.KERNEL_MMA_DB   # the automatic choice for 20000-bit rows
    g = gen.rng(5)
    for i in np.unique(np.concatenate([[0, n - 1], g.integers(0, n, size=5)])):
        base = int(sb.tri_index(n, i, i))
        got = out[base: base + (n - i)].cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, ol.contig_row(host, int(i)), err_msg=f"row {i}")
    ii = np.arange(n, dtype=np.uint64)
    diag = out[torch.from_numpy(sb.tri_index(n, ii, ii).astype(np.int64)).cuda()].cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(diag, pc)
    total = 0
    step = 1 << 30
    for a in range(0, tri, step):
        total += int(out[a: a + step].to(torch.int64).bitwise_and(0xFFFFFFFF).sum().item())
    assert s == total - int(pc.sum())


def test_config2_full_size_tensor_and_popc_kernels(sb):
    """65536 rows x 262144 bits, p ~ U[0.05, 0.5] (2 GiB in, 8.6 GB out): the
    tensor-core kernel against the CUDA-core AND + POPC kernel -- an
    independent code path -- on all 2,147,516,416 pairs, plus sampled rows
    against the oracle, the diagonal and the sum identity."""
    _check_full_size(sb, 65536, 262144, (0.05, 0.5), 202, ["mma", "mma_2cta", "popc"])


def test_device_pointer_ingest_orders_after_producer(sb):
    """Rows generated on torch's stream and handed over as a device pointer
    right away must be read only after the generator finished."""
    import torch
    import bench
    n, m = 4096, 65536
    rows = bench.bernoulli_rows_gpu(n, m, (0.05, 0.5), 31, torch.device("cuda"))
    c = sb.StormContig(m)
    assert sb.lib().STORM_contig_add_bitmaps(c.h, sb.C.cast(rows.data_ptr(), sb.u64p), n, m // 64) == n
    host = rows.cpu().numpy().view(np.uint64)
    ref = sb.StormContig(m)
    ref.add_bitmaps(host)
    assert c.pairw_intersect_cardinality() == ref.pairw_intersect_cardinality()
    want = ol.contig_row(host, 5)
    mat, _ = c.matrix()
    base = int(sb.tri_index(n, 5, 5))
    np.testing.assert_array_equal(mat[base: base + n - 5], want)


@pytest.mark.parametrize("n,m", [(200, (1 << 20) + 64), (130, (1 << 23) + 256), (5, 1 << 22), (300, 1 << 16)])
def test_split_k_few_tiles(sb, n, m):
    """Fewer tiles than SMs: each tile's K range is cut into slices whose
    partial counts are added into the zeroed triangle. Exact through the host
    matrix, the sum-only call, and a device buffer that held garbage."""
    import torch
    g = gen.rng(77 + n)
    words = g.integers(0, 1 << 63, size=(n, (m + 63) // 64), dtype=np.uint64) & g.integers(
        0, 1 << 63, size=(n, (m + 63) // 64), dtype=np.uint64)        # p = 1/4, top bit clear
    if m % 64:
        words[:, -1] &= np.uint64((1 << (m % 64)) - 1)
    c = contig_from_words(sb, words, m, "mma")
    mat, s = c.matrix()
    want, ws = ol.contig_matrix(words)
    assert s == ws
    np.testing.assert_array_equal(mat, want)
    assert c.pairw_intersect_cardinality() == ws
    d = torch.full((want.size,), -1, dtype=torch.int32, device="cuda")
    assert c.matrix_device(d.data_ptr(), want.size) == ws
    np.testing.assert_array_equal(d.cpu().numpy().view(np.uint32), want)


@pytest.mark.parametrize("kernel", ("mma", "mma_db"))
@pytest.mark.parametrize("n,m", [(300, (1 << 17) + 64), (700, 16384), (129, 4097), (1000, 1 << 15)])
def test_every_schedule_is_exact(sb, kernel, n, m):
    """Whole tiles round robin and stream-K (partial tiles added with atomics
    into the zeroed triangle) give the oracle's counts; the automatic choice
    too -- for both tensor-core tile shapes."""
    words = gen.bernoulli_rows(n, m, (0.05, 0.6), seed=500 + n)
    want, ws = ol.contig_matrix(words)
    c = contig_from_words(sb, words, m, kernel)
    for sched in (sb.SCHED_TILES, sb.SCHED_STREAM_K, sb.SCHED_AUTO):
        c.set_schedule(sched)
        mat, s = c.matrix()
        assert s == ws, sched
        np.testing.assert_array_equal(mat, want, err_msg=str(sched))


@pytest.mark.parametrize("kernel", ("mma", "popc"))
@pytest.mark.parametrize("n,m", [(300, (1 << 17) + 64), (700, 16384), (129, 4097)])
def test_threshold_matches_oracle(sb, kernel, n, m):
    """Thresholded form (pairs with v > 0 and Jaccard >= t, exact v): fused in
    the tensor-core epilogue, and by compaction of the triangle for POPC."""
    words = gen.bernoulli_rows(n, m, (0.05, 0.6), seed=800 + n)
    tri, _ = ol.contig_matrix(words)
    c = contig_from_words(sb, words, m, kernel)
    for t in (0.0, 0.2, 0.35, 1.0):
        wi, wj, wc = ol.threshold_pairs(tri, n, t)
        gi, gj, gc, found = c.threshold(t, cap=n * n)
        assert found == len(wi), t
        np.testing.assert_array_equal(gi, wi)
        np.testing.assert_array_equal(gj, wj)
        np.testing.assert_array_equal(gc, wc)


def test_threshold_long_rows_and_small_cap(sb):
    """Rows past 2^23 bits (4-byte weight cycle), and an output capacity
    smaller than the hit count: STORM_B200_ESIZE, the true count, and cap
    hits that all belong to the answer."""
    m = (1 << 23) + 4096
    g = gen.rng(4343)
    words = g.integers(0, 1 << 63, size=(40, (m + 63) // 64), dtype=np.uint64)
    words[:, -1] &= np.uint64((1 << (m % 64)) - 1)
    tri, _ = ol.contig_matrix(words)
    c = contig_from_words(sb, words, m, "mma")
    wi, wj, wc = ol.threshold_pairs(tri, 40, 0.3)
    gi, gj, gc, found = c.threshold(0.3, cap=2000)
    assert found == len(wi) and len(wi) > 10
    np.testing.assert_array_equal(gi, wi)
    np.testing.assert_array_equal(gc, wc)
    oi = np.zeros(5, np.uint32)
    oj = np.zeros(5, np.uint32)
    oc = np.zeros(5, np.uint32)
    f = sb.C.c_uint64(0)
    rc = sb.lib().STORM_contig_pairw_threshold(c.h, 0.3, sb._p(oi, sb.u32p), sb._p(oj, sb.u32p),
                                               sb._p(oc, sb.u32p), 5, sb.C.byref(f))
    assert rc == sb.ESIZE and f.value == len(wi)
    want = {(a, b, v) for a, b, v in zip(wi.tolist(), wj.tolist(), wc.tolist())}
    assert all((a, b, v) in want for a, b, v in zip(oi.tolist(), oj.tolist(), oc.tolist()))


def test_autotune_keeps_the_fastest_exact_kernel(sb):
    """The autotuner times every kernel/schedule exact for the row length on
    these rows, keeps the fastest, and later calls stay exact."""
    n, m = 700, 16384
    words = gen.bernoulli_rows(n, m, (0.05, 0.6), seed=901)
    want, ws = ol.contig_matrix(words)
    c = contig_from_words(sb, words, m, "mma")
    k, sched, times = c.autotune()
    assert all(t > 0 for t in times)
    cands = [(sb.KERNEL_MMA, sb.SCHED_TILES), (sb.KERNEL_MMA, sb.SCHED_STREAM_K), (sb.KERNEL_MMA_DB, sb.SCHED_TILES),
             (sb.KERNEL_MMA_DB, sb.SCHED_STREAM_K), (sb.KERNEL_MMA_SS, sb.SCHED_AUTO), (sb.KERNEL_POPC, sb.SCHED_AUTO)]
    assert (k, sched) == cands[int(np.argmin(times))]
    mat, s = c.matrix()
    assert s == ws and c.last_kernel() == k
    np.testing.assert_array_equal(mat, want)
    # rows past 2^23 bits: only the tensor-core kernel in the 4-byte cycle and POPC qualify
    m = (1 << 23) + 64
    g = gen.rng(902)
    words = g.integers(0, 1 << 63, size=(20, (m + 63) // 64), dtype=np.uint64)
    words[:, -1] &= np.uint64((1 << (m % 64)) - 1)
    c = contig_from_words(sb, words, m, "mma")
    k, sched, times = c.autotune()
    assert times[4] == -1.0 and times[0] > 0 and times[2] > 0 and times[5] > 0
    assert c.matrix()[1] == ol.contig_matrix(words)[1]


@pytest.mark.parametrize("kernel", ("auto",) + KERNELS)
def test_matrix_from_host_overlapped(sb, kernel):
    """The one-call host form (rows in from host memory, triangle out to host
    memory, upload / tiles / copy-back overlapped in panels from the bottom of
    the triangle up) equals the oracle; the container then holds the rows and
    the two-call host form (bottom-up panels too) gives the same counts.
    9000 rows: 8 to 11 panels, whichever kernel."""
    n, m = 9000, 512
    words = gen.bernoulli_rows(n, m, (0.05, 0.5), 71)
    want, ws = ol.contig_matrix(words)
    c = sb.StormContig(m)
    if kernel != "auto":
        c.set_kernel(_kernel(sb, kernel))
    got, s = c.matrix_from_host(words)
    assert s == ws
    np.testing.assert_array_equal(got, want)
    assert len(c) == n
    got2, s2 = c.matrix()
    assert s2 == ws
    np.testing.assert_array_equal(got2, want)
    c.close()


def test_matrix_from_host_ragged_rows(sb):
    """Row length not a multiple of 64 or of the 512-bit pitch (zeroed pitch
    padding), a repeated call replacing the rows, and 0 / 1 rows."""
    m = 4100
    c = sb.StormContig(m)
    for n, seed in ((7000, 72), (300, 73), (1, 74), (0, 75), (5000, 76)):
        words = gen.bernoulli_rows(n, m, (0.05, 0.5), seed) if n else np.zeros((0, 65), dtype=np.uint64)
        got, s = c.matrix_from_host(words)
        assert len(c) == n
        if n == 0:
            assert s == 0
            continue
        want, ws = ol.contig_matrix(words)
        assert s == ws, n
        np.testing.assert_array_equal(got, want, err_msg=str(n))
    c.close()
