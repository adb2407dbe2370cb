"""STORM_t (65536-bit chunks) and the reference's single-pair kernels on the
GPU, against the reference's golden vectors and the oracle."""
import os
import subprocess

import numpy as np
import pytest

import gen
import oracle_lib as ol
from conftest import golden_sets, ROOT

pytestmark = pytest.mark.gpu


def build_storm(sb, sets):
    s = sb.Storm()
    for v in sets:
        s.add(np.asarray(v, dtype=np.uint32))
    return s


def storm_cases(z):
    return sorted({k.split("/")[1] for k in z.files if k.startswith("storm/")})


def test_golden_storm_sums_and_matrices(sb, golden):
    for name in storm_cases(golden):
        sets = golden_sets(golden, f"storm/{name}/")
        s = build_storm(sb, sets)
        want = int(golden[f"storm/{name}/sum"][0])
        assert s.pairw_intersect_cardinality() == want, name
        assert s.pairw_intersect_cardinality(blocked=5) == want, name
        mat, ssum = s.matrix()
        assert ssum == want
        n = len(sets)
        iu = np.triu_indices(n)
        strict = iu[0] != iu[1]
        np.testing.assert_array_equal(mat[strict], golden[f"storm/{name}/matrix"][strict], err_msg=name)
        diag = mat[~strict]
        np.testing.assert_array_equal(diag, [len(x) for x in sets], err_msg=name)


def test_golden_square(sb, golden):
    a = build_storm(sb, golden_sets(golden, "square/a_"))
    b = build_storm(sb, golden_sets(golden, "square/b_"))
    assert a.square(b) == int(golden["square/sum"][0])


@pytest.mark.parametrize("case", ["zipf", "runs", "haplo", "dense", "sweep"])
def test_config_shaped_sets_match_oracle(sb, case):
    if case == "zipf":
        sets = gen.zipf_sets(90, 1 << 24, 1.1, 16, 1 << 17, 5)
    elif case == "runs":
        sets = gen.run_sets(70, 1 << 26, 40, 256, 6)
    elif case == "haplo":
        sets = gen.haplotype_sets(200, 20000, 32, 7)
    elif case == "dense":
        sets = [gen.uniform_set(gen.rng(8 + i), 20000 + 3000 * i, 1 << 17) for i in range(20)]
    else:
        sets = []
        for d in (1e-5, 1e-4, 1e-3, 1e-2):
            sets += gen.bernoulli_sets(12, 1 << 22, d, int(d * 1e6))
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    mat, ssum = s.matrix()
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)


def test_empty_rows_clear_and_tiles(sb):
    sets = [np.zeros(0, np.uint32), np.arange(0, 70000, 3, dtype=np.uint32), np.zeros(0, np.uint32),
            np.arange(5, 200000, 11, dtype=np.uint32)]
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    assert s.pairw_intersect_cardinality() == ws
    col = s.tiles(3)
    iu = np.triu_indices(4)
    strict = iu[0] != iu[1]
    np.testing.assert_array_equal(col.out[strict], want[strict])
    s.clear()
    assert s.pairw_intersect_cardinality() == 0
    s.add(np.array([1, 2, 3], np.uint32))
    s.add(np.array([2, 3, 4], np.uint32))
    assert s.pairw_intersect_cardinality() == 2


def test_lowlevel_kernels_match_reference(sb, golden):
    for a, b, want in zip(golden_sets(golden, "vec16/a_"), golden_sets(golden, "vec16/b_"), golden["vec16/result"]):
        assert sb.intersect_vector16(a.astype(np.uint16), b.astype(np.uint16)) == want
    for a, b, o in zip(golden_sets(golden, "vec32/a_"), golden_sets(golden, "vec32/b_"),
                       golden_sets(golden, "vec32/out_")):
        got = sb.intersect_vector32(a, b)
        np.testing.assert_array_equal(got.ravel(), o)
    for a, b, want in zip(golden_sets(golden, "bsl/a_"), golden_sets(golden, "bsl/b_"), golden["bsl/result"]):
        ba = gen.sets_to_rows([a], 4096)[0]
        bb = gen.sets_to_rows([b], 4096)[0]
        assert sb.intersect_bitmaps_scalar_list(ba, bb, a, b) == want
        assert sb.intersect_bitmaps_scalar_list(bb, ba, b, a) == want


def test_single_bit_probe_cases(sb):
    # tests/test_storm.c:125-132 shape: one shared bit in word 1, every bit position.
    for bit in range(64):
        bm = np.array([0, 1 << bit], dtype=np.uint64)
        assert sb.intersect_bitmaps_scalar_list(bm, bm, [64 + bit], [64 + bit]) == 1


def test_reference_test_program_against_this_library():
    """The reference's own tests/test_storm.c, compiled unmodified against the
    reference header and linked against libstorm_b200.so (oracle/Makefile,
    target `dropin`), must report 0 failures."""
    exe = os.path.join(ROOT, "oracle", "_ref", "test_storm_b200")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/test_storm_b200 not built (needs the reference sources)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert " 0 failures" in r.stdout, r.stdout[-2000:]


def _dense_corpus(n_dense, n_sparse, universe, lo, hi, seed):
    g = gen.rng(seed)
    sets = [gen.uniform_set(g, int(g.integers(lo, hi)), universe) for _ in range(n_dense)]
    sets += [gen.uniform_set(g, int(g.integers(1, 40)), universe) for _ in range(n_sparse)]
    return [sets[k] for k in g.permutation(len(sets))]


def test_tensor_dense_block_matches_chunk_kernel_and_oracle(sb):
    """Plain dense rows are expanded into contiguous bitmaps and compared on
    the tensor cores; sparse rows stay on the chunk kernel. Counts are the
    oracle's, and identical with the block switched off."""
    sets = _dense_corpus(300, 150, 1 << 20, 1000, 8000, 91)
    s = build_storm(sb, sets)
    s.set_sparse_postings(0)                # the dense block alone (postings tested below)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    s.set_dense_block(1.0 / 16384)          # by value count: the 300 dense rows
    mat, ssum = s.matrix()
    rows, panels = s.last_dense()
    assert rows == 300 and panels == 1
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)
    assert s.pairw_intersect_cardinality() == ws
    s.set_dense_block(-1.0)                 # by predicted cost (the default)
    mat, ssum = s.matrix()
    assert s.last_dense()[0] >= 300 and ssum == ws
    np.testing.assert_array_equal(mat, want)
    s.set_dense_block(0.0)
    mat0, s0 = s.matrix()
    assert s.last_dense() == (0, 0) and s0 == ws
    np.testing.assert_array_equal(mat0, want)


def test_tensor_dense_block_in_panels(sb):
    """A budget of two 256-row panels forces three panels (full, full, ragged):
    triangle launches per panel, rectangle launches per panel pair, and the
    split-K path on the ragged panel's few tiles."""
    universe = 1 << 20
    sets = _dense_corpus(700, 60, universe, 500, 4000, 92)
    s = build_storm(sb, sets)
    s.set_sparse_postings(0)                # the dense block alone (postings tested below)
    row_bytes = universe // 65536 * 8256          # an expanded row: its 8 KiB chunk slots 64 bytes apart
    s.set_dense_block(1.0 / 16384, 2 * 256 * row_bytes + 4096)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    mat, ssum = s.matrix()
    assert s.last_dense() == (700, 3)
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)
    assert s.pairw_intersect_cardinality() == ws


def test_tensor_dense_block_rows_with_repeats_stay_on_chunks(sb):
    """Rows whose list chunks hold a repeated value (STORM_add does not
    deduplicate lists) keep the chunk kernel's k-th-copy count; the block
    takes only the plain rows and the totals match the block-off run."""
    sets = _dense_corpus(280, 20, 1 << 18, 300, 3000, 93)
    dup_rows = [3, 50, 120]
    s = sb.Storm()
    s.set_sparse_postings(0)
    for k, v in enumerate(sets):
        if k in dup_rows:
            v = np.sort(np.concatenate([v, v[:7]]))
        s.add(np.asarray(v, dtype=np.uint32))
    mat, ssum = s.matrix()
    rows, _ = s.last_dense()
    assert 256 <= rows <= len(sets) - len(dup_rows)
    s.set_dense_block(0.0)
    mat0, s0 = s.matrix()
    assert s0 == ssum
    np.testing.assert_array_equal(mat, mat0)
    # and both are the reference's chunk-by-chunk counts (repeats included)
    added = [np.sort(np.concatenate([v, v[:7]])) if k in dup_rows else v for k, v in enumerate(sets)]
    vals, offs = gen.to_csr(added)
    want, ws = ol.storm_matrix(vals, offs)
    assert ssum == ws
    iu = np.triu_indices(len(added))
    strict = iu[0] != iu[1]
    np.testing.assert_array_equal(mat[strict], want[strict])


def test_tensor_dense_block_long_universe(sb):
    """A 2^24-value universe (256 chunks per row, rows past 2^23 bits take the
    4-byte weight cycle) with Bernoulli(1e-3) rows."""
    sets = gen.bernoulli_sets(260, 1 << 24, 1e-3, 94)
    s = build_storm(sb, sets)
    s.set_sparse_postings(0)                # the dense block alone (postings tested below)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    mat, ssum = s.matrix()
    assert s.last_dense()[0] == 260
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)


def test_postings_sparse_rows_match_oracle(sb):
    """Sparse plain rows through the postings (value histogram, one increment
    per pair and shared value): forced (row sweep in shared memory, and list
    by list into the output), automatic and off agree with the oracle, for
    the per-pair matrix and the sum."""
    sets = gen.bernoulli_sets(400, 1 << 20, 2e-4, 95) + gen.bernoulli_sets(100, 1 << 20, 3e-5, 96)
    s = build_storm(sb, sets)
    s.set_dense_block(0.0)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    for mode in (1, 2, 3, -1, 0):           # 2 / 3: list-by-list / row-sweep form
        s.set_sparse_postings(mode)
        mat, ssum = s.matrix()
        if mode in (1, 2, 3):
            assert s.last_postings_rows() == len(sets)
        if mode == 0:
            assert s.last_postings_rows() == 0
        assert ssum == ws, mode
        np.testing.assert_array_equal(mat, want, err_msg=str(mode))
        assert s.pairw_intersect_cardinality() == ws


def test_postings_with_dense_block_and_chunk_rows(sb):
    """All three row classes at once -- tensor-core dense block, postings
    rows, and rows that must stay on the chunk kernel (repeated list values)
    -- give the same counts as the chunk kernel alone."""
    g = gen.rng(97)
    # dense rows with bitmap chunks (>= 4096 values per 65536-bit chunk)
    sets = [gen.uniform_set(g, int(g.integers(70000, 200000)), 1 << 20) for _ in range(280)]
    sets += [gen.uniform_set(g, int(g.integers(1, 40)), 1 << 20) for _ in range(150)]
    dup = [np.sort(np.concatenate([v, v[:3]])) for v in
           (gen.uniform_set(g, int(g.integers(20, 60)), 1 << 20) for _ in range(4))]
    sets += dup
    sets = [sets[k] for k in g.permutation(len(sets))]
    s = build_storm(sb, sets)
    s.set_dense_block(1.0 / 16384)
    s.set_sparse_postings(1)
    mat, ssum = s.matrix()
    assert s.last_dense()[0] == 280 and s.last_postings_rows() == 150
    s.set_dense_block(0.0)
    s.set_sparse_postings(0)
    mat0, s0 = s.matrix()
    assert s.last_dense()[0] == 0 and s.last_postings_rows() == 0
    assert ssum == s0
    np.testing.assert_array_equal(mat, mat0)
    s.set_dense_block(1.0 / 16384)
    s.set_sparse_postings(1)
    assert s.pairw_intersect_cardinality() == s0
    # the reference's chunk-by-chunk counts (the repeated-value rows included)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.storm_matrix(vals, offs)
    assert s0 == ws
    iu = np.triu_indices(len(sets))
    strict = iu[0] != iu[1]
    np.testing.assert_array_equal(mat[strict], want[strict])


def test_tensor_rows_with_postings_in_panels(sb):
    """Heavy rows on the tensor cores for all their pairs (heavy x heavy and
    heavy x light, the light rows expanded too), light x light pairs by the
    postings; a budget of two 256-row panels makes the expanded order
    [heavy | padding | light] span four panels."""
    universe = 1 << 20
    g = gen.rng(98)
    sets = [gen.uniform_set(g, int(g.integers(2000, 6000)), universe) for _ in range(300)]
    sets += [gen.uniform_set(g, int(g.integers(5, 50)), universe) for _ in range(300)]
    sets = [sets[k] for k in g.permutation(len(sets))]
    s = build_storm(sb, sets)
    s.set_dense_block(1.0 / 1024, 2 * 256 * (universe // 65536 * 8256) + 4096)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    for mode in (2, 3):
        s.set_sparse_postings(mode)
        mat, ssum = s.matrix()
        assert s.last_dense() == (300, 4) and s.last_postings_rows() == 300
        assert ssum == ws
        np.testing.assert_array_equal(mat, want)
    assert s.pairw_intersect_cardinality() == ws


def test_default_plan_on_mixed_rows_matches_oracle(sb):
    """The default plan (cost-chosen cut between tensor rows and postings
    rows) on Zipf-distributed rows."""
    sets = gen.zipf_sets(600, 1 << 20, 1.1, 16, 1 << 15, 99)
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    mat, ssum = s.matrix()
    assert s.last_dense()[0] + s.last_postings_rows() > 0
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)
    assert s.pairw_intersect_cardinality() == ws


def test_threshold_storm_t_matches_oracle(sb):
    """Thresholded form over STORM_t rows (triangle compaction on the device),
    on a mix of heavy, light and very sparse rows."""
    g = gen.rng(101)
    sets = [gen.uniform_set(g, int(g.integers(2000, 6000)), 1 << 18) for _ in range(150)]
    sets += [gen.uniform_set(g, int(g.integers(1, 80)), 1 << 18) for _ in range(250)]
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    want, _ = ol.sets_matrix(vals, offs)
    for t in (0.0, 0.01, 0.05, 0.5):
        wi, wj, wc = ol.threshold_pairs(want, len(sets), t)
        gi, gj, gc, found = s.threshold(t, cap=len(sets) ** 2)
        assert found == len(wi), t
        np.testing.assert_array_equal(gi, wi)
        np.testing.assert_array_equal(gj, wj)
        np.testing.assert_array_equal(gc, wc)


def test_square_of_plain_rows_by_histograms(sb):
    """STORM_intersect_cardinality_square on plain rows (list and bitmap
    chunks): the rectangle sum from two value histograms equals the oracle's."""
    g = gen.rng(102)
    xa = [gen.uniform_set(g, int(g.integers(1, 9000)), 1 << 19) for _ in range(60)]
    xa += [gen.uniform_set(g, int(g.integers(70000, 120000)), 1 << 19) for _ in range(10)]   # bitmap chunks
    yb = [gen.uniform_set(g, int(g.integers(1, 3000)), 1 << 19) for _ in range(50)]
    a, b = build_storm(sb, xa), build_storm(sb, yb)
    xv, xo = gen.to_csr(xa)
    yv, yo = gen.to_csr(yb)
    want = ol.oracle().oracle_sets_square(xv.ctypes.data_as(ol.u32p), xo.ctypes.data_as(ol.u64p), len(xa),
                                          yv.ctypes.data_as(ol.u32p), yo.ctypes.data_as(ol.u64p), len(yb))
    assert a.square(b) == want
    assert b.square(a) == want


def test_planner_at_the_largest_universe(sb):
    """Values up to 2^27 - 1 (2048 chunks, the largest universe of the tensor
    rows and the postings): forced tensor rows, forced postings and the
    chunk kernel agree with the oracle."""
    g = gen.rng(103)
    top = (1 << 27) - 1
    sets = []
    for k in range(300):
        v = gen.uniform_set(g, int(g.integers(1, 300)), 1 << 27)
        if k % 7 == 0:
            v = np.unique(np.concatenate([v, [top]])).astype(np.uint32)
        sets.append(v)
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    for dense, post in ((1e-9, 0), (0.0, 1), (0.0, 3), (0.0, 0), (-1.0, -1)):
        s.set_dense_block(dense)
        s.set_sparse_postings(post)
        mat, ssum = s.matrix()
        if dense > 0:
            assert s.last_dense()[0] == len(sets)
        if post > 0:
            assert s.last_postings_rows() == len(sets)
        assert ssum == ws, (dense, post)
        np.testing.assert_array_equal(mat, want, err_msg=f"{dense}/{post}")


def test_autotune_storm_t(sb):
    """The STORM_t autotuner times the planner with tensor rows and postings on
    or off, keeps the fastest, and later calls stay exact."""
    g = gen.rng(905)
    sets = [gen.uniform_set(g, int(g.integers(1000, 6000)), 1 << 20) for _ in range(260)]
    sets += gen.bernoulli_sets(300, 1 << 20, 2e-5, 906)
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    dens, post, times = s.autotune()
    assert all(t > 0 for t in times)
    k = int(np.argmin(times))
    assert (dens, post) == ((-1.0, -1), (-1.0, 0), (0.0, -1), (0.0, 0))[k]
    mat, ssum = s.matrix()
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)


def test_row_changed_through_public_struct_is_repacked(sb):
    """The STORM_t layout is public, so a caller may append to one of its rows
    with STORM_bitmap_cont_add on s->conts[r] instead of STORM_add; the next
    all-pairs call must see the new values (the device copy is re-packed).

    Values appended into a chunk the row already holds become a second chunk
    with the same id (storm.cpp:737-803), which the reference's chunk-id merge
    matches once: that case is checked against the reference library itself
    when it is built, the new-chunk case against the set oracle."""
    import ctypes as C

    class Cont(C.Structure):
        _fields_ = [("bitmaps", C.c_void_p), ("block_ids", C.c_void_p), ("n_bitmaps", C.c_uint32),
                    ("m_bitmaps", C.c_uint32), ("prev", C.c_uint32)]

    class StormT(C.Structure):
        _fields_ = [("conts", C.POINTER(Cont)), ("n_conts", C.c_uint32), ("m_conts", C.c_uint32)]

    def append(lib, h, r, extra):
        st = C.cast(h, C.POINTER(StormT)).contents
        cont = C.addressof(st.conts[r])
        return lib.STORM_bitmap_cont_add(C.c_void_p(cont), extra.ctypes.data_as(sb.u32p), C.c_uint32(extra.size))

    g = gen.rng(931)
    u = 1 << 20
    sets = [gen.uniform_set(g, int(g.integers(50, 5000)), u // 2) for _ in range(40)]
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    assert s.pairw_intersect_cardinality() == ol.sets_matrix(vals, offs)[1]
    # new chunks only (every row lies below u / 2): the set oracle applies;
    # rows 3 and 17 share the appended values, so their count must move
    L = sb.lib()
    extra = np.unique(g.integers(u // 2, u, 500)).astype(np.uint32)
    for r in (3, 17):
        assert append(L, s.h, r, extra) == 1
        sets[r] = np.concatenate([sets[r], extra])
    vals, offs = gen.to_csr(sets)
    want_mat, want_sum = ol.sets_matrix(vals, offs)
    assert s.pairw_intersect_cardinality() == want_sum
    mat, ssum = s.matrix()
    assert ssum == want_sum
    n = len(sets)
    iu = np.triu_indices(n)
    strict = iu[0] != iu[1]
    np.testing.assert_array_equal(mat[strict], want_mat[strict])
    # into the row's last chunk: against the reference's own containers
    if ol.reference() is None:
        return
    R = ol.reference()
    R.STORM_new.restype = C.c_void_p
    R.STORM_add.argtypes = [C.c_void_p, sb.u32p, C.c_uint32]
    R.STORM_pairw_intersect_cardinality.restype = C.c_uint64
    R.STORM_pairw_intersect_cardinality.argtypes = [C.c_void_p]
    R.STORM_free.argtypes = [C.c_void_p]
    hr = R.STORM_new()
    try:
        for v in sets:
            v = np.ascontiguousarray(v, dtype=np.uint32)
            R.STORM_add(hr, v.ctypes.data_as(sb.u32p), v.size)
        for r in (5, 29):
            top = int(sets[r][-1])
            extra = np.unique(g.integers(top + 1, top + 3000, 200)).astype(np.uint32)
            assert append(L, s.h, r, extra) == 1 and append(R, hr, r, extra) == 1
        assert s.pairw_intersect_cardinality() == R.STORM_pairw_intersect_cardinality(hr)
    finally:
        R.STORM_free(hr)


def test_repeated_and_unordered_list_values_match_reference(sb):
    """List chunks that are not strictly increasing are counted as the
    reference counts them (its SSE4.2 list x list kernel, storm.cpp:15-88,
    whose answer then differs from the set size): per-pair counts and the sum
    against the oracle's chunk-by-chunk restatement (itself checked against
    the reference's own STORM_t, oracle/_ref, when that is built). The
    single-pair STORM_intersect_vector16_cardinality is checked on the same
    lists."""
    import ctypes as C
    for seed in (941, 942):
        sets = gen.repeat_corpus(seed)
        n = len(sets)
        vals, offs = gen.to_csr(sets)
        want, ws = ol.storm_matrix(vals, offs)
        # the corpus does reach the cases where the reference's count is not the set size
        assert ol.sets_matrix(vals, offs)[1] != ws
        R = ol.reference()
        if R is not None:   # the oracle is pinned to the reference here too
            ref = np.zeros(n * (n + 1) // 2, dtype=np.uint32)
            u32p, u64p = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
            assert R.ref_storm_matrix(vals.ctypes.data_as(u32p), offs.ctypes.data_as(u64p), n,
                                      ref.ctypes.data_as(u32p)) == ws
            np.testing.assert_array_equal(ref, want)
        s = build_storm(sb, sets)
        assert s.pairw_intersect_cardinality() == ws
        mat, ssum = s.matrix()
        assert ssum == ws
        iu = np.triu_indices(n)
        strict = iu[0] != iu[1]
        np.testing.assert_array_equal(mat[strict], want[strict], err_msg=str(seed))
        # single pair, lists as given (the reference's first argument is v1)
        for a, b in ((0, 2), (2, 0), (3, 7), (4, 8), (6, 10), (11, 3)):
            la = np.ascontiguousarray(sets[a][sets[a] < 65536], dtype=np.uint16)
            lb = np.ascontiguousarray(sets[b][sets[b] < 65536], dtype=np.uint16)
            if la.size and lb.size:
                want1 = ol.oracle().oracle_list16_blocked(la.ctypes.data_as(C.POINTER(C.c_uint16)),
                                                          lb.ctypes.data_as(C.POINTER(C.c_uint16)), la.size, lb.size)
                assert sb.intersect_vector16(la, lb) == want1, (seed, a, b)



def test_list_longer_than_a_staging_buffer(sb):
    """A list chunk can be longer than one upload worker's pinned buffer (the
    public layout sets no limit: STORM_bitmap_add_scalar_only appends to a
    chunk's list without one, repeats included); such a list goes to the
    device straight from its own memory. Every pair against the reference's
    per-chunk rules (storm.cpp:652-690) computed here from the rows' lists:
    list x list by the oracle's restatement of the blocked SSE4.2 count
    (pinned to the reference by test_list16_cpu.py), bitmap x list one probe
    per list entry, bitmap x bitmap AND + POPC."""
    import ctypes as C
    from test_ingest_cpu import StormT
    L = sb.lib()
    L.STORM_bitmap_add_scalar_only.argtypes = [C.c_void_p, sb.u32p, C.c_uint32]
    g = np.random.default_rng(77)
    rows = [np.array([5, 10, 20, 70000], np.uint32),                               # list chunks 0 and 1
            np.sort(g.choice(65536, 3000, replace=False)).astype(np.uint32),       # list
            np.sort(g.choice(65536, 5000, replace=False)).astype(np.uint32),       # bitmap
            np.sort(g.choice(np.arange(65536, 131072), 2000, replace=False)).astype(np.uint32),
            np.array([1, 2, 3], np.uint32)]
    # (row, chunk index) -> values STORM_bitmap_add_scalar_only appends
    longs = {(0, 0): g.integers(0, 65536, 9_000_000).astype(np.uint32),   # 18 MB: longer than a lane buffer (>= 4 host threads)
             (0, 1): g.integers(65536, 131072, 700_000).astype(np.uint32),
             (4, 0): np.sort(g.integers(0, 65536, 1_200_000)).astype(np.uint32)}
    st = sb.Storm()
    for v in rows:
        st.add(v)
    s = C.cast(st.h, C.POINTER(StormT)).contents
    for (r, k), v in longs.items():
        assert L.STORM_bitmap_add_scalar_only(C.addressof(s.conts[r].bitmaps[k]), v.ctypes.data_as(sb.u32p),
                                              v.size) == v.size
    # the rows' chunks as the reference sees them: id -> ("list", u16 entries) or ("bitmap", words)
    chunks = []
    for r, v in enumerate(rows):
        ids = np.unique(v >> 16)
        row = {}
        for k, cid in enumerate(ids):
            part = (v[(v >> 16) == cid] & 0xFFFF).astype(np.uint16)
            if (r, k) in longs:
                part = np.concatenate([part, (longs[(r, k)] & 0xFFFF).astype(np.uint16)])
            if part.size >= 4096 and (r, k) not in longs:
                row[int(cid)] = ("bitmap", gen.sets_to_rows([part.astype(np.uint32)], 65536)[0])
            else:
                row[int(cid)] = ("list", np.ascontiguousarray(part))
        chunks.append(row)
    O = ol.oracle()

    def pair(a, b):
        total = 0
        for cid in sorted(set(a) & set(b)):
            (ka, xa), (kb, xb) = a[cid], b[cid]
            if ka == "list" and kb == "list":
                total += O.oracle_list16_blocked(xa.ctypes.data_as(ol.u16p), xb.ctypes.data_as(ol.u16p),
                                                 xa.size, xb.size)
            elif ka == "bitmap" and kb == "bitmap":
                total += int(np.unpackbits((xa & xb).view(np.uint8)).sum())
            else:
                words, lst = (xa, xb) if ka == "bitmap" else (xb, xa)
                total += int(((words[lst >> 6] >> (lst & 63).astype(np.uint64)) & np.uint64(1)).sum())
        return total

    n = len(rows)
    want = {(i, j): pair(chunks[i], chunks[j]) for i in range(n) for j in range(i + 1, n)}
    assert st.pairw_intersect_cardinality() == sum(want.values())
    mat, ssum = st.matrix()
    assert ssum == sum(want.values())
    k = 0
    for i in range(n):
        for j in range(i, n):
            if j > i:
                assert mat[k] == want[(i, j)], (i, j, int(mat[k]), want[(i, j)])
            k += 1
    st.close()


def test_triangle_into_pageable_host_memory(sb):
    """A per-pair triangle of more than 32 MiB copied into pageable host
    memory goes through the handle's pinned lanes, one host worker per share
    of the output: equal, entry for entry, to the triangle the same call
    writes into device memory, for row counts that split unevenly."""
    import torch
    for n, seed in ((4100, 31), (5003, 32)):
        sets = gen.bernoulli_sets(n, 1 << 20, 1e-3, seed)
        vals, offs = gen.to_csr(sets)
        st = sb.Storm()
        st.add_rows(vals, offs)
        tri = n * (n + 1) // 2
        host = np.full(tri, 0xFFFFFFFF, np.uint32)   # pageable
        got, s1 = st.matrix(host)
        d = torch.empty(tri, dtype=torch.int32, device="cuda")
        s2 = st.matrix_device(d.data_ptr(), tri)
        assert s1 == s2
        assert np.array_equal(got, d.cpu().numpy().view(np.uint32)), n
        xf = st.last_transfer_ms()
        assert xf["copy_back_ms"] == 0.0   # the device form copies nothing back
        st.matrix(host)
        xf = st.last_transfer_ms()
        assert xf["upload_ms"] == 0.0 and xf["copy_back_bytes"] == tri * 4
        st.close()


@pytest.mark.parametrize("universe,mean_len", [(1 << 20, 64), (1 << 24, 256), (1 << 26, 700)])
def test_run_sweep_matches_oracle(sb, universe, mean_len):
    """The run form of the postings (pieces of runs per bin, overlaps summed
    in a row sweep), forced, on run-clustered rows plus rows that reach its
    edge cases -- empty rows, single values, runs across chunk and bin
    boundaries, scattered values, a row equal to another -- against the
    oracle, every pair and the sum."""
    sets = gen.run_sets(160, universe, 40, mean_len, universe % 1009)
    g = gen.rng(universe % 97)
    sets += [np.zeros(0, np.uint32), np.array([0], np.uint32), np.array([universe - 1], np.uint32),
             np.arange(65536 - 300, 65536 + 300, dtype=np.uint32),
             np.arange(0, min(universe, 1 << 18), 3, dtype=np.uint32),
             np.unique(g.integers(0, universe, 4000)).astype(np.uint32), sets[3].copy()]
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    st = sb.Storm()
    st.add_rows(vals, offs)
    st.set_dense_block(0.0)
    st.set_panel(0)
    st.set_sparse_postings(4)
    got, s = st.matrix()
    assert st.last_postings_form() == 2
    assert st.last_postings_rows() >= len(sets) // 2
    assert s == ws
    np.testing.assert_array_equal(got, want)
    assert st.pairw_intersect_cardinality() == ws
    st.close()


def test_default_plan_takes_the_run_sweep_on_run_clustered_rows(sb):
    """Config-4-shaped rows (Poisson runs of Geometric(256) length over 2^26):
    the planner's own choice indexes runs, and the counts match the value
    postings' forced on the same rows and the oracle on sampled rows."""
    sets = gen.run_sets(1200, 1 << 26, 120, 256, 4242)
    vals, offs = gen.to_csr(sets)
    st = sb.Storm()
    st.add_rows(vals, offs)
    got, s = st.matrix()
    assert st.last_postings_form() == 2
    st.set_sparse_postings(3)
    ref, s3 = st.matrix()
    assert st.last_postings_form() == 1
    assert s == s3
    np.testing.assert_array_equal(got, ref)
    n = len(sets)
    pick = [0, 1, 599, n - 1]
    sub_vals, sub_offs = gen.to_csr([sets[i] for i in pick])
    want, _ = ol.sets_matrix(sub_vals, sub_offs)
    iu = np.triu_indices(len(pick))
    for k, (a, b) in enumerate(zip(iu[0], iu[1])):
        i, j = pick[a], pick[b]
        assert got[i * n - i * (i - 1) // 2 + (j - i)] == want[k], (i, j)
    st.close()


@pytest.mark.parametrize("universe", [1 << 20, 1 << 24])
def test_run_sweep_with_bitmap_chunks(sb, universe):
    """The run form over rows that also hold bitmap chunks (runs of set bits
    cut at bin and word boundaries): long runs, half-dense chunks, a full
    chunk, runs ending on a chunk's last bit, beside list rows -- every plain
    row forced into the run sweep, against the oracle."""
    g = gen.rng(universe % 101)
    sets = gen.run_sets(90, universe, 30, 300, universe % 1013)
    extra = []
    for k in range(30):
        v = set()
        for _ in range(int(g.integers(1, 4))):
            s0 = int(g.integers(0, universe - 9000))
            v.update(range(s0, s0 + int(g.integers(4096, 9000))))          # a bitmap chunk or two
        if k % 3 == 0:
            c0 = int(g.integers(0, universe // 65536)) * 65536
            v.update((c0 + np.flatnonzero(g.random(65536) < 0.5)).tolist())   # half-dense chunk
        if k % 5 == 0:
            c0 = int(g.integers(0, universe // 65536)) * 65536
            v.update(range(c0, c0 + 65536))                                  # full chunk
        if k % 7 == 0:
            v.update(range(65536 - 5000, 65536 + 37))                         # ends past a chunk's last bit
        extra.append(np.array(sorted(v), np.uint32))
    sets += extra
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    st = sb.Storm()
    st.add_rows(vals, offs)
    st.set_sparse_postings(4)
    got, s = st.matrix()
    assert st.last_postings_form() == 2
    assert st.last_postings_rows() == len(sets)
    assert s == ws
    np.testing.assert_array_equal(got, want)
    st.close()


def test_row_sweeps_beyond_one_partner_block(sb):
    """More postings rows than the row sweeps' shared-memory counters hold
    (51200): partners are counted block by block. 60000 sparse rows (about
    168 values each over 2^24, plus empty rows) by the value row sweep, the
    run sweep and the list-by-list form -- three independent code paths --
    agree on every pair; the diagonal is the cardinalities and the sum the
    value-histogram identity."""
    import torch
    n, U = 60000, 1 << 24
    g = np.random.default_rng(60000)
    cards = g.binomial(U, 1e-5, size=n)
    cards[::997] = 0
    draws = g.integers(0, U, size=int(cards.sum()), dtype=np.uint64).astype(np.uint32)
    ends = np.cumsum(cards)
    sets = [np.unique(draws[e - c:e]) for c, e in zip(cards, ends)]
    vals, offs = gen.to_csr(sets)
    st = sb.Storm()
    st.add_rows(vals, offs)
    st.set_dense_block(0.0)
    st.set_panel(0)
    tri = n * (n + 1) // 2
    got = {}
    for mode, form in ((3, 1), (4, 2), (2, 0)):
        st.set_sparse_postings(mode)
        d = torch.full((tri,), -1, dtype=torch.int32, device="cuda")
        s = st.matrix_device(d.data_ptr(), tri)
        assert st.last_postings_form() == form
        assert st.last_postings_rows() == n
        got[mode] = (s, d)
    hist = np.bincount(vals, minlength=U).astype(np.int64)
    want_sum = int((hist * (hist - 1) // 2).sum())
    for mode in (3, 4, 2):
        assert got[mode][0] == want_sum, mode
    assert torch.equal(got[3][1], got[2][1])
    assert torch.equal(got[4][1], got[2][1])
    ii = torch.arange(n, device="cuda", dtype=torch.int64)
    diag = got[2][1][ii * n - ii * (ii - 1) // 2].cpu().numpy()
    np.testing.assert_array_equal(diag, [len(x) for x in sets])
    st.close()


def test_host_output_call_refuses_device_memory(sb):
    """The per-pair call that copies the triangle into host memory returns
    STORM_B200_EARG, without writing, when the buffer it is given is device
    memory (the device form is STORM_pairw_intersect_matrix_device)."""
    import ctypes as C
    import torch
    sets = gen.zipf_sets(300, 1 << 20, 1.1, 16, 1 << 15, 5)
    vals, offs = gen.to_csr(sets)
    st = sb.Storm()
    st.add_rows(vals, offs)
    tri = 300 * 301 // 2
    d = torch.zeros(tri, dtype=torch.int32, device="cuda")
    s = C.c_uint64(0)
    rc = sb.lib().STORM_pairw_intersect_matrix(st.h, C.cast(d.data_ptr(), sb.u32p), tri, C.byref(s))
    assert rc == sb.EARG
    assert int(d.abs().sum().item()) == 0
    got, _ = st.matrix()   # the container still works
    want, _ = ol.sets_matrix(vals, offs)
    np.testing.assert_array_equal(got, want)
    st.close()
