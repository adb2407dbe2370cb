"""The kernel layer's row representations, built on the device from the
rows' sorted positions (csrc/rows_pack.cu), read back form by form through
STORM_rows_repr and compared with

  * the reference's own build_row outputs (storm_repr.cpp:25-207; golden
    vectors written by the reference, tests/golden/make_golden.py), and
  * the oracle's restatement of each builder (oracle_runs, oracle_ewah,
    oracle_rank9, oracle_occ, oracle_complement) on rows shaped to reach
    every EWAH segmentation case: empty and full rows, full words at the
    first and last word, full runs next to literals and zero gaps, partial
    last words, rows longer than one thread block's tile, and rows that get
    no bitmap under a small budget."""
import numpy as np
import pytest

import gen
import oracle_lib as ol
from conftest import golden_sets

pytestmark = pytest.mark.gpu
P = ol._p


def _csr_item(z, key, i):
    offs = z[key + "_offs"]
    return z[key + "_vals"][int(offs[i]):int(offs[i + 1])]


def _markers(stream):
    """(stream position, first decoded word) of every marker of an EWAH-64
    stream (fill length in bits 1..31, literal count in bits 32..63)."""
    out, pos, word = [], 0, 0
    while pos < len(stream):
        m = int(stream[pos])
        fl, ll = (m >> 1) & 0x7FFFFFFF, m >> 32
        out.append((pos, word))
        word += fl + ll
        pos += 1 + ll
    return np.array(out, np.uint32).reshape(-1, 2)


def _oracle_forms(v, u):
    O = ol.oracle()
    v = np.ascontiguousarray(v, np.uint32)
    nw = (u + 63) // 64
    rs = np.zeros(v.size + 1, np.uint32)
    re = np.zeros(v.size + 1, np.uint32)
    k = O.oracle_runs(P(v, ol.u32p), v.size, P(rs, ol.u32p), P(re, ol.u32p))
    bm = gen.sets_to_rows([v], u)[0][:nw].copy() if nw else np.zeros(0, np.uint64)
    ew = np.zeros(2 * nw + 2, np.uint64)
    kw = O.oracle_ewah(P(bm, ol.u64p), nw, P(ew, ol.u64p))
    rk = np.zeros(2 * ((nw + 7) // 8 + 1), np.uint64)
    O.oracle_rank9(P(bm, ol.u64p), nw, P(rk, ol.u64p))
    oc = np.zeros((((nw + 7) // 8) + 63) // 64, np.uint64)
    O.oracle_occ(P(bm, ol.u64p), nw, 8, P(oc, ol.u64p))
    cp = np.zeros(max(u, 1), np.uint32)
    kc = O.oracle_complement(P(v, ol.u32p), v.size, u, P(cp, ol.u32p))
    return {"runs": rs[:k], "run_end": re[:k], "ewah": ew[:kw], "bitmap": bm, "rank": rk, "occ": oc,
            "comp": cp[:kc]}


def _check_row(sb, r, i, v, u, want=None):
    want = want or _oracle_forms(v, u)
    meta = r.meta(i)
    tag = f"u={u} row {i} card {len(v)}"
    np.testing.assert_array_equal(r.repr(i, sb.REPR_RUN_START), want["runs"], err_msg=tag)
    np.testing.assert_array_equal(r.repr(i, sb.REPR_RUN_END), want["run_end"], err_msg=tag)
    ew = r.repr(i, sb.REPR_EWAH)
    np.testing.assert_array_equal(ew, want["ewah"], err_msg=tag)
    np.testing.assert_array_equal(r.repr(i, sb.REPR_MARKERS), _markers(want["ewah"]), err_msg=tag)
    has_bm, has_comp = bool(meta[8] & 1), bool(meta[8] & 2)
    if has_bm:
        np.testing.assert_array_equal(r.repr(i, sb.REPR_BITMAP), want["bitmap"], err_msg=tag)
    else:
        assert r.repr(i, sb.REPR_BITMAP).size == 0
    if meta[6]:
        np.testing.assert_array_equal(r.repr(i, sb.REPR_RANK), want["rank"], err_msg=tag)
    if meta[7]:
        np.testing.assert_array_equal(r.repr(i, sb.REPR_OCC), want["occ"], err_msg=tag)
    if has_comp:
        np.testing.assert_array_equal(r.repr(i, sb.REPR_COMPLEMENT), want["comp"], err_msg=tag)
    else:
        assert r.repr(i, sb.REPR_COMPLEMENT).size == 0


def test_device_build_matches_reference_build_row(sb, golden):
    """Every golden row: the reference's runs, EWAH stream, rank9, zone map,
    complement and RowMeta, as the reference's own build_row wrote them."""
    rows = golden_sets(golden, "repr/")
    for k, (v, u) in enumerate(zip(rows, golden["repr/universe"])):
        u = int(u)
        r = sb.StormRows(u)
        r.add(np.asarray(v, np.uint32))
        sizes = golden["repr/sizes"][k]
        meta = r.meta(0)
        np.testing.assert_array_equal(meta[:8], golden["repr/meta"][k], err_msg=f"row {k}")
        np.testing.assert_array_equal(r.repr(0, sb.REPR_RUN_START), _csr_item(golden, "repr/runs", k))
        np.testing.assert_array_equal(r.repr(0, sb.REPR_RUN_END), _csr_item(golden, "repr/run_end", k))
        np.testing.assert_array_equal(r.repr(0, sb.REPR_EWAH), _csr_item(golden, "repr/ewah", k))
        if sizes[2]:
            np.testing.assert_array_equal(r.repr(0, sb.REPR_RANK), _csr_item(golden, "repr/rank", k))
        if sizes[3]:
            np.testing.assert_array_equal(r.repr(0, sb.REPR_OCC), _csr_item(golden, "repr/occ", k))
        assert r.repr(0, sb.REPR_COMPLEMENT).size == sizes[4]
        if sizes[4]:
            np.testing.assert_array_equal(r.repr(0, sb.REPR_COMPLEMENT), _csr_item(golden, "repr/comp", k))
        r.close()


@pytest.mark.parametrize("u", [64, 100, 4103, 65536, (1 << 20) + 13])
def test_device_build_matches_oracle(sb, u):
    g = gen.rng(u + 7)
    rows = gen.segmentation_rows(u, g)
    r = sb.StormRows(u)
    for v in rows:
        r.add(v)
    for i, v in enumerate(rows):
        _check_row(sb, r, i, v, u)
    # the same rows again after a clear: the build starts from nothing
    r.clear()
    for v in rows[::-1]:
        r.add(v)
    for i, v in enumerate(rows[::-1]):
        _check_row(sb, r, i, v, u)
    r.close()


def test_rows_without_bitmap_under_budget(sb):
    """A budget for a few bitmaps: the densest rows get B (and rank, zone
    map, complement under their gates); the others keep S, R and W only."""
    u = 1 << 18
    g = gen.rng(91)
    rows = [np.flatnonzero(g.random(u) < d).astype(np.uint32) for d in (0.001, 0.7, 0.01, 0.2, 0.0001, 0.6)]
    r = sb.StormRows(u)
    r.set_bitmap_budget(2 * (u // 8) + 64)
    for v in rows:
        r.add(v)
    have = [bool(r.meta(i)[8] & 1) for i in range(len(rows))]
    assert have == [False, True, False, False, False, True]
    for i, v in enumerate(rows):
        _check_row(sb, r, i, v, u)
    r.close()
