"""The CPU oracle (oracle/storm_oracle.c) pinned against the golden vectors
the reference itself produced (tests/golden/make_golden.py).  No GPU."""
import numpy as np
import pytest

import gen
import oracle_lib as ol
from conftest import golden_sets

P = ol._p


def contig_cases(z):
    return sorted({k.split("/")[1] for k in z.files if k.startswith("contig/")})


def storm_cases(z):
    return sorted({k.split("/")[1] for k in z.files if k.startswith("storm/")})


def test_oracle_contig_matches_reference(golden):
    for name in contig_cases(golden):
        words = golden[f"contig/{name}/words"]
        mat, s = ol.contig_matrix(words)
        assert s == int(golden[f"contig/{name}/sum"][0]), name
        np.testing.assert_array_equal(mat, golden[f"contig/{name}/matrix"], err_msg=name)


def test_oracle_sets_match_reference(golden):
    for name in storm_cases(golden):
        vals, offs = golden[f"storm/{name}/vals"], golden[f"storm/{name}/offs"]
        mat, s = ol.sets_matrix(vals, offs)
        assert s == int(golden[f"storm/{name}/sum"][0]), name
        # The reference's diagonal is not part of its output; compare i < j.
        n = len(offs) - 1
        iu = np.triu_indices(n)
        strict = iu[0] != iu[1]
        np.testing.assert_array_equal(mat[strict], golden[f"storm/{name}/matrix"][strict], err_msg=name)


def test_oracle_strips_match_reference(golden):
    """oracle_strip_* (whole rows of the matrix for a few query rows, rows
    streamed in batches on several threads) equals the reference's per-pair
    counts i < j on every golden set corpus, for query rows at the start, in
    the middle and at the end."""
    for name in storm_cases(golden):
        vals, offs = golden[f"storm/{name}/vals"], golden[f"storm/{name}/offs"]
        n = len(offs) - 1
        full = golden[f"storm/{name}/matrix"]
        sets = gen.from_csr(vals, offs)
        q = sorted({0, n // 2, n - 1})
        universe = int(vals.max()) + 1 if vals.size else 1
        st = ol.SetStrip([sets[i] for i in q], universe)
        got = np.concatenate([st.count(vals[int(offs[a]):], offs[a:b + 1] - offs[a], threads=3)
                              for a, b in ((0, n // 3), (n // 3, n))])
        st.close()
        for k, i in enumerate(q):
            for j in range(n):
                if i == j:
                    assert got[j, k] == len(sets[i])
                    continue
                a, b = min(i, j), max(i, j)
                assert got[j, k] == full[a * n - (a * (a - 1)) // 2 + (b - a)], (name, i, j)


def test_oracle_chunk_by_chunk_matches_reference(golden):
    """oracle_storm_matrix (STORM_t counted chunk by chunk, as the reference
    counts it) equals the golden matrices and sums, and -- on rows with
    repeated and out-of-order list entries, where that count is not the set
    size -- the reference's own STORM_t (oracle/_ref) when it is built; its
    list x list count equals the reference's STORM_intersect_vector16_
    cardinality on seeded lists."""
    import ctypes as C
    for name in storm_cases(golden):
        vals, offs = golden[f"storm/{name}/vals"], golden[f"storm/{name}/offs"]
        mat, s = ol.storm_matrix(vals, offs)
        assert s == int(golden[f"storm/{name}/sum"][0]), name
        n = len(offs) - 1
        iu = np.triu_indices(n)
        strict = iu[0] != iu[1]
        np.testing.assert_array_equal(mat[strict], golden[f"storm/{name}/matrix"][strict], err_msg=name)
    R = ol.reference()
    if R is None:
        pytest.skip("reference library not built (oracle/_ref)")
    u16p, u32p, u64p = C.POINTER(C.c_uint16), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
    for seed in range(941, 947):
        sets = gen.repeat_corpus(seed)
        vals, offs = gen.to_csr(sets)
        n = len(sets)
        mat, s = ol.storm_matrix(vals, offs)
        ref = np.zeros(n * (n + 1) // 2, dtype=np.uint32)
        assert R.ref_storm_matrix(vals.ctypes.data_as(u32p), offs.ctypes.data_as(u64p), n,
                                  ref.ctypes.data_as(u32p)) == s, seed
        np.testing.assert_array_equal(mat, ref, err_msg=str(seed))
        assert ol.sets_matrix(vals, offs)[1] != s     # the corpus reaches the non-set counts
    g = gen.rng(948)
    for _ in range(3000):
        a = np.sort(g.integers(0, int(g.integers(2, 400)), int(g.integers(1, 80)))).astype(np.uint16)
        b = g.integers(0, 400, int(g.integers(1, 80))).astype(np.uint16)
        if g.random() < 0.5:
            b = np.sort(b)
        want = R.ref_vector16(a.ctypes.data_as(u16p), b.ctypes.data_as(u16p), a.size, b.size)
        got = ol.oracle().oracle_list16_blocked(a.ctypes.data_as(u16p), b.ctypes.data_as(u16p), a.size, b.size)
        assert got == want, (a, b)


def test_oracle_chunk_split_matches_reference_layout(golden):
    O = ol.oracle()
    for name in storm_cases(golden):
        if f"storm/{name}/layout" not in golden.files:
            continue
        r = int(golden[f"storm/{name}/layout_row"][0])
        sets = golden_sets(golden, f"storm/{name}/")
        v = np.ascontiguousarray(sets[r], dtype=np.uint32)
        ids = np.zeros(v.size, np.uint32); kinds = np.zeros(v.size, np.uint8); cnt = np.zeros(v.size, np.uint32)
        k = O.oracle_chunk_split(P(v, ol.u32p), v.size, P(ids, ol.u32p), P(kinds, ol.u8p), P(cnt, ol.u32p))
        want = golden[f"storm/{name}/layout"]
        np.testing.assert_array_equal(ids[:k], want[0], err_msg=name)
        np.testing.assert_array_equal(kinds[:k], want[1], err_msg=name)
        np.testing.assert_array_equal(cnt[:k], want[2], err_msg=name)


def test_oracle_square_matches_reference(golden):
    O = ol.oracle()
    av, ao, bv, bo = (np.ascontiguousarray(golden[f"square/{k}"]) for k in ("a_vals", "a_offs", "b_vals", "b_offs"))
    s = O.oracle_sets_square(P(av, ol.u32p), P(ao, ol.u64p), len(ao) - 1, P(bv, ol.u32p), P(bo, ol.u64p), len(bo) - 1)
    assert s == int(golden["square/sum"][0])


def test_oracle_lowlevel_matches_reference(golden):
    O = ol.oracle()
    A = golden_sets(golden, "vec16/a_")
    B = golden_sets(golden, "vec16/b_")
    for a, b, want in zip(A, B, golden["vec16/result"]):
        a = np.ascontiguousarray(a, np.uint32); b = np.ascontiguousarray(b, np.uint32)
        assert O.oracle_list_intersect(P(a, ol.u32p), a.size, P(b, ol.u32p), b.size) == want
    A = golden_sets(golden, "bsl/a_")
    B = golden_sets(golden, "bsl/b_")
    for a, b, want in zip(A, B, golden["bsl/result"]):
        a = np.ascontiguousarray(a, np.uint32); b = np.ascontiguousarray(b, np.uint32)
        assert O.oracle_list_intersect(P(a, ol.u32p), a.size, P(b, ol.u32p), b.size) == want
    w = golden["wrapper_diag/words"]
    _, s = ol.contig_matrix(w)
    assert s == golden["wrapper_diag/sum"][0] == golden["wrapper_diag/sum"][1]


def test_oracle_kernel_layer_matches_reference(golden):
    names = sorted({k.split("/")[1] for k in golden.files if k.startswith("rows/")})
    assert names
    for name in names:
        vals, offs = golden[f"rows/{name}/vals"], golden[f"rows/{name}/offs"]
        mat, s = ol.sets_matrix(vals, offs)
        for pol, tile, ssum, pairs, skipped, dec in golden[f"rows/{name}/allpairs_sum"]:
            assert ssum == s, (name, pol, tile)
            n = len(offs) - 1
            assert pairs == n * (n - 1) // 2
        n = len(offs) - 1
        iu = np.triu_indices(n)
        strict = iu[0] != iu[1]
        np.testing.assert_array_equal(mat[strict], golden[f"rows/{name}/tiles_strict"][strict], err_msg=name)
    A = golden_sets(golden, "cells/a_")
    B = golden_sets(golden, "cells/b_")
    O = ol.oracle()
    for a, b, want in zip(A, B, golden["cells/result"]):
        a = np.ascontiguousarray(a, np.uint32); b = np.ascontiguousarray(b, np.uint32)
        assert O.oracle_list_intersect(P(a, ol.u32p), a.size, P(b, ol.u32p), b.size) == want


def _csr_item(z, key, i):
    offs = z[key + "_offs"]
    return z[key + "_vals"][int(offs[i]):int(offs[i + 1])]


def test_oracle_representations_match_reference(golden):
    O = ol.oracle()
    rows = golden_sets(golden, "repr/")
    for i, (v, u) in enumerate(zip(rows, golden["repr/universe"])):
        v = np.ascontiguousarray(v, np.uint32)
        u = int(u)
        nw = (u + 63) // 64
        rs = np.zeros(v.size + 1, np.uint32); re = np.zeros(v.size + 1, np.uint32)
        k = O.oracle_runs(P(v, ol.u32p), v.size, P(rs, ol.u32p), P(re, ol.u32p))
        np.testing.assert_array_equal(rs[:k], _csr_item(golden, "repr/runs", i))
        np.testing.assert_array_equal(re[:k], _csr_item(golden, "repr/run_end", i))
        bm = gen.sets_to_rows([v], u)[0]
        ew = np.zeros(2 * nw + 2, np.uint64)
        k = O.oracle_ewah(P(bm, ol.u64p), nw, P(ew, ol.u64p))
        np.testing.assert_array_equal(ew[:k], _csr_item(golden, "repr/ewah", i))
        dec = np.zeros(nw, np.uint64)
        O.oracle_ewah_decode(P(ew, ol.u64p), k, P(dec, ol.u64p))
        np.testing.assert_array_equal(dec, bm)
        meta = np.zeros(8, np.uint32)
        O.oracle_row_meta(P(v, ol.u32p), v.size, u, P(meta, ol.u32p))
        np.testing.assert_array_equal(meta, golden["repr/meta"][i])
        want_rank = _csr_item(golden, "repr/rank", i)
        if want_rank.size:   # built only where the reference gates it on (mean run >= 512)
            rk = np.zeros(2 * ((nw + 7) // 8 + 1), np.uint64)
            O.oracle_rank9(P(bm, ol.u64p), nw, P(rk, ol.u64p))
            np.testing.assert_array_equal(rk, want_rank)
        want_occ = _csr_item(golden, "repr/occ", i)
        if want_occ.size:
            oc = np.zeros(want_occ.size, np.uint64)
            O.oracle_occ(P(bm, ol.u64p), nw, 8, P(oc, ol.u64p))
            np.testing.assert_array_equal(oc, want_occ)
        want_comp = _csr_item(golden, "repr/comp", i)
        if want_comp.size:
            cp = np.zeros(u, np.uint32)
            k = O.oracle_complement(P(v, ol.u32p), v.size, u, P(cp, ol.u32p))
            np.testing.assert_array_equal(cp[:k], want_comp)


def test_oracle_catches_a_planted_mistake(golden):
    """A checker that cannot fail is worthless: flip one bit, expect a mismatch."""
    words = golden["contig/dense_1024/words"].copy()
    words[3, 5] ^= np.uint64(1 << 17)
    mat, _ = ol.contig_matrix(words)
    assert not np.array_equal(mat, golden["contig/dense_1024/matrix"])


@pytest.mark.parametrize("shape", ["runs_2^20", "runs_2^24_long", "runs_across_chunks", "zipf_2^20", "mixed"])
def test_oracle_sets_fuzzed_against_reference_build(shape):
    """Beyond the golden vectors: the oracle's per-pair set counts (the
    checker of every STORM_t engine, the run postings included) against the
    reference built here from its sources (oracle/_ref, STORM_t through its
    own STORM_add and STORM_pairw_intersect_cardinality per pair) on seeded
    run-clustered, Zipf and mixed corpora. Skipped without oracle/_ref."""
    R = ol.reference()
    if R is None:
        pytest.skip("reference library not built (oracle/_ref)")
    seed = sum(map(ord, shape))
    if shape == "runs_2^20":
        sets = gen.run_sets(60, 1 << 20, 20, 64, seed)
    elif shape == "runs_2^24_long":
        sets = gen.run_sets(40, 1 << 24, 30, 2000, seed)
    elif shape == "runs_across_chunks":
        g = gen.rng(seed)
        sets = [np.arange(65536 * k - int(g.integers(1, 5000)), 65536 * k + int(g.integers(1, 5000)),
                          dtype=np.uint32) for k in range(1, 30)]
    elif shape == "zipf_2^20":
        sets = gen.zipf_sets(60, 1 << 20, 1.1, 16, 1 << 18, seed)
    else:
        sets = (gen.run_sets(20, 1 << 22, 10, 500, seed) + gen.zipf_sets(20, 1 << 22, 1.1, 16, 1 << 16, seed) +
                [np.zeros(0, np.uint32), np.array([0], np.uint32)])
    vals, offs = gen.to_csr(sets)
    n = len(sets)
    want, ws = ol.sets_matrix(vals, offs)
    ref = np.zeros(n * (n + 1) // 2, np.uint32)
    assert R.ref_storm_matrix(P(vals, ol.u32p), P(offs, ol.u64p), n, P(ref, ol.u32p)) == ws
    iu = np.triu_indices(n)
    strict = iu[0] != iu[1]
    np.testing.assert_array_equal(want[strict], ref[strict])


@pytest.mark.parametrize("u", [64, 100, 4103, 65536, (1 << 20) + 13])
def test_oracle_representations_fuzzed_against_reference_build(u):
    """The oracle's builders (runs, EWAH-64, rank9, zone map, complement,
    RowMeta) -- the checker of the device-built representations -- against
    the reference's own storm::build_row (oracle/_ref) on rows that reach
    every EWAH segmentation case, beyond the golden rows. Skipped without
    oracle/_ref."""
    R = ol.reference()
    if R is None:
        pytest.skip("reference library not built (oracle/_ref)")
    O = ol.oracle()
    nw = (u + 63) // 64
    for v in gen.segmentation_rows(u, gen.rng(u + 7)):
        v = np.ascontiguousarray(v, np.uint32)
        rs = np.zeros(v.size + 1, np.uint32)
        re = np.zeros(v.size + 1, np.uint32)
        ew = np.zeros(2 * nw + 2, np.uint64)
        rk = np.zeros(2 * ((nw + 7) // 8 + 1) + 2, np.uint64)
        oc = np.zeros((((nw + 7) // 8) + 63) // 64 + 1, np.uint64)
        cp = np.zeros(max(u, 1), np.uint32)
        sizes = np.zeros(6, np.uint64)
        meta = np.zeros(8, np.uint32)
        R.ref_build_row(P(v, ol.u32p), v.size, u, P(rs, ol.u32p), P(re, ol.u32p), P(ew, ol.u64p), P(rk, ol.u64p),
                        P(oc, ol.u64p), P(cp, ol.u32p), P(sizes, ol.u64p), P(meta, ol.u32p))
        tag = f"u={u} card={v.size}"
        ors = np.zeros(v.size + 1, np.uint32)
        ore = np.zeros(v.size + 1, np.uint32)
        k = O.oracle_runs(P(v, ol.u32p), v.size, P(ors, ol.u32p), P(ore, ol.u32p))
        assert k == sizes[0], tag
        np.testing.assert_array_equal(ors[:k], rs[:k], err_msg=tag)
        np.testing.assert_array_equal(ore[:k], re[:k], err_msg=tag)
        bm = gen.sets_to_rows([v], u)[0][:nw].copy()
        oew = np.zeros(2 * nw + 2, np.uint64)
        kw = O.oracle_ewah(P(bm, ol.u64p), nw, P(oew, ol.u64p))
        assert kw == sizes[1], tag
        np.testing.assert_array_equal(oew[:kw], ew[:kw], err_msg=tag)
        om = np.zeros(8, np.uint32)
        O.oracle_row_meta(P(v, ol.u32p), v.size, u, P(om, ol.u32p))
        np.testing.assert_array_equal(om, meta, err_msg=tag)
        if sizes[2]:
            ork = np.zeros(2 * ((nw + 7) // 8 + 1), np.uint64)
            O.oracle_rank9(P(bm, ol.u64p), nw, P(ork, ol.u64p))
            np.testing.assert_array_equal(ork, rk[:int(sizes[2])], err_msg=tag)
        if sizes[3]:
            ooc = np.zeros(int(sizes[3]), np.uint64)
            O.oracle_occ(P(bm, ol.u64p), nw, 8, P(ooc, ol.u64p))
            np.testing.assert_array_equal(ooc, oc[:int(sizes[3])], err_msg=tag)
        if sizes[4]:
            ocp = np.zeros(max(u, 1), np.uint32)
            kc = O.oracle_complement(P(v, ol.u32p), v.size, u, P(ocp, ol.u32p))
            assert kc == sizes[4], tag
            np.testing.assert_array_equal(ocp[:kc], cp[:kc], err_msg=tag)
