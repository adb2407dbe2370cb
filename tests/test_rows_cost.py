"""The cost-model port (select_pairing / predict, host build of the same code
the GPU tile driver runs) against the reference's own decisions and
predictions (golden vectors from kernels/storm_cost.cpp).  No GPU."""
import numpy as np


def test_select_pairing_and_predict_match_reference(sb, golden):
    A, B = golden["select/meta_a"], golden["select/meta_b"]
    want_sel, want_pred = golden["select/pairing"], golden["select/predict"]
    assert len(A) > 20
    for a, b, ws, wp in zip(A, B, want_sel, want_pred):
        got, pred = sb.select_pairing(a, b)
        assert got == ws, (a, b, got, ws)
        for p in range(11):
            np.testing.assert_allclose(sb.predict(p, a, b), wp[p], rtol=1e-12, atol=1e-9, err_msg=f"pairing {p}")


def test_span_test_settles_disjoint_pairs(sb):
    a = np.array([10, 2, 2048, 2, 100, 200, 0, 0], np.uint32)   # card, runs, nw, nnz, first, last, rank, occ
    b = np.array([10, 2, 2048, 2, 300, 400, 0, 0], np.uint32)
    assert sb.select_pairing(a, b)[0] == sb.P_EMPTY
    e = np.array([0, 0, 2048, 0, 0xFFFFFFFF, 0, 0, 0], np.uint32)
    assert sb.select_pairing(a, e)[0] == sb.P_EMPTY


def test_select_pairing_fuzzed_against_reference_library(sb):
    """2000 seeded RowMeta pairs across densities, run counts, spans and the
    rank / zone-map flags, decided by the port and by the reference's own
    select_pairing / predict (oracle/_ref); skipped when it is not built."""
    import ctypes as C

    import oracle_lib as ol
    R = ol.reference()
    if R is None:
        import pytest
        pytest.skip("reference library not built (oracle/_ref)")
    g = np.random.default_rng(20261204)
    u32p, dblp = C.POINTER(C.c_uint32), C.POINTER(C.c_double)

    def meta(universe):
        card = int(min(universe, 2 ** g.uniform(0, np.log2(universe) + 0.01)))
        runs = int(max(1, min(card, card / 2 ** g.uniform(0, 12)))) if card else 0
        nw = (universe + 63) // 64
        nnz = int(min(nw, card, max(1 if card else 0, card / 2 ** g.uniform(0, 6))))
        if not card:
            return np.array([0, 0, nw, 0, 0xFFFFFFFF, 0, 0, 0], dtype=np.uint32)
        first = int(g.integers(0, max(1, (universe - card) // 8 + 1)))    # spans mostly overlap
        last = int(min(universe - 1, max(first + card - 1, universe - 1 - g.integers(0, universe // 8 + 1))))
        return np.array([card, runs, nw, nnz, first, last, g.integers(0, 2), g.integers(0, 2)], dtype=np.uint32)

    seen = set()
    for _ in range(2000):
        universe = int(2 ** g.integers(10, 27))
        a, b = meta(universe), meta(universe)
        if g.random() < 0.15 and a[0] and b[0] and a[0] + b[0] < universe // 2:   # disjoint spans
            a[4], a[5] = 0, a[0] - 1
            b[4], b[5] = universe - b[0], universe - 1
        pred = np.zeros(11, dtype=np.float64)
        want = R.ref_select_pairing(a.ctypes.data_as(u32p), b.ctypes.data_as(u32p), pred.ctypes.data_as(dblp))
        got, _ = sb.select_pairing(a, b)
        assert got == want, (a, b, got, want)
        seen.add(int(got))
        for p in range(11):
            np.testing.assert_allclose(sb.predict(p, a, b), pred[p], rtol=1e-12, atol=1e-9, err_msg=f"{a} {b} {p}")
    assert len(seen) >= 5, seen   # the draws reach several different cells
