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
