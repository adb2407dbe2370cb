"""The learned cell selector: the device forward/backward kernels against a
CPU reference of the same network (numpy, analytic gradients checked by
finite differences), training on this GPU's own cell timings, and what the
trained network gains over the cost model it replaces."""
import numpy as np
import pytest

import gen
import oracle_lib as ol

pytestmark = pytest.mark.gpu


def np_mlp(params, F, H, C, x, y):
    """CPU reference: logits, mean cross-entropy, gradients (same layout)."""
    W1 = params[:H * F].reshape(H, F).astype(np.float64)
    b1 = params[H * F:H * F + H].astype(np.float64)
    W2 = params[H * F + H:H * F + H + C * H].reshape(C, H).astype(np.float64)
    b2 = params[H * F + H + C * H:].astype(np.float64)
    x = x.astype(np.float64)
    pre = x @ W1.T + b1
    h = np.maximum(pre, 0)
    lg = h @ W2.T + b2
    m = lg.max(axis=1, keepdims=True)
    p = np.exp(lg - m)
    p /= p.sum(axis=1, keepdims=True)
    B = len(y)
    loss = float(np.mean(-np.log(p[np.arange(B), y])))
    d = p.copy()
    d[np.arange(B), y] -= 1
    d /= B
    gW2 = d.T @ h
    gb2 = d.sum(0)
    dh = (d @ W2) * (pre > 0)
    gW1 = dh.T @ x
    gb1 = dh.sum(0)
    return lg, loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2])


def test_forward_backward_kernels_match_cpu_reference(sb):
    F, H, C, B = 16, 32, 10, 300
    g = gen.rng(5)
    params = (g.standard_normal(H * F + H + C * H + C) * 0.3).astype(np.float32)
    x = g.random((B, F)).astype(np.float32)
    y = g.integers(0, C, size=B).astype(np.int32)
    lg, loss, grads = sb.mlp_forward_backward(params, F, H, C, x, y)
    lg_ref, loss_ref, g_ref = np_mlp(params, F, H, C, x, y)
    np.testing.assert_allclose(lg, lg_ref, rtol=1e-4, atol=1e-4)
    assert abs(loss - loss_ref) < 1e-4 * max(1, loss_ref)
    np.testing.assert_allclose(grads, g_ref, rtol=2e-3, atol=2e-5)
    # the CPU reference's gradient is itself checked by central differences
    eps = 1e-4
    for k in g.choice(params.size, size=25, replace=False):
        pp, pm = params.astype(np.float64).copy(), params.astype(np.float64).copy()
        pp[k] += eps
        pm[k] -= eps
        fd = (np_mlp(pp, F, H, C, x, y)[1] - np_mlp(pm, F, H, C, x, y)[1]) / (2 * eps)
        assert abs(fd - g_ref[k]) < 1e-5 + 1e-3 * abs(fd), k


def mixed_corpus():
    """Mixed density and structure over one universe: the regime where one
    cell per corpus is wrong and selection matters."""
    u = 1 << 18
    sets = []
    sets += gen.bernoulli_sets(96, u, 0.002, 61)
    sets += gen.run_sets(96, u, 30, 300, 62)
    sets += gen.bernoulli_sets(64, u, 0.2, 63)
    sets += gen.zipf_sets(96, u, 1.1, 16, 1 << 14, 64)
    return sets, u


def test_training_learns_and_beats_the_cost_model(sb):
    sets, u = mixed_corpus()
    r = sb.StormRows(u)
    for s in sets:
        r.add(s)
    st = r.train_selector(tile=32, samples=0, epochs=400, seed=3)
    lt = r.last_training()
    assert st["samples"] > 50
    assert st["train_accuracy"] > 0.5, st
    # Regret against the measured-best cell on held-out tiles: the network
    # beats the reference's default model (its constants are another
    # machine's), and it is no worse than the cost model calibrated on this
    # GPU's timings of the same training tiles.
    assert lt["regret_mlp"] < lt["regret_default_model"], lt
    assert lt["regret_mlp"] <= lt["regret_calibrated_model"] + 0.02, lt
    assert st["regret_cost_model"] == pytest.approx(lt["regret_calibrated_model"])
    # The kept model is the fitted one or the reference's default, whichever
    # picked better cells on the training tiles.
    model, calibrated = r.cost_model()
    assert calibrated == (lt["kept_calibrated_model"] == 1.0) and all(x >= 0 for x in model)
    # Counts stay exact under the learned policy in both execution forms.
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    for ex in (sb.EXEC_BATCHED, sb.EXEC_PER_TILE):
        mat, s2 = r.allpairs_matrix(sb.POLICY_LEARNED, 32, exec_=ex)
        np.testing.assert_array_equal(mat, want)
    # Parameters round-trip.
    p = r.selector_params()
    r.reset_selector()
    r.selector_params(load=p)
    assert np.array_equal(r.selector_params(), p)


def test_gpu_calibration_of_the_cost_model(sb):
    """STORM_rows_calibrate fits the cost model to this GPU's cell timings on
    the container's own tiles; the calibrated model prices the cells (counts
    unchanged), can be read back, replaced, and reset to the reference's."""
    sets, u = mixed_corpus()
    r = sb.StormRows(u)
    for s in sets:
        r.add(s)
    model, rms = r.calibrate(tile=32, samples=0, seed=5)
    assert len(model) == 26 and all(x >= 0 for x in model)
    assert 0.0 <= rms < 10.0
    got, cal = r.cost_model()
    assert cal and np.allclose(got, model)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    for pol in (sb.POLICY_PERTILE, sb.POLICY_PERPAIR, sb.POLICY_REFINE):
        mat, st = r.allpairs_matrix(pol, 32)
        np.testing.assert_array_equal(mat, want)
    r.cost_model(reset=True)
    got, cal = r.cost_model()
    assert not cal
    mat, st = r.allpairs_matrix(sb.POLICY_PERTILE, 32)
    np.testing.assert_array_equal(mat, want)


def test_complement_cell_as_a_candidate(sb):
    """C x B (|A & B| = |B| - |A' & B|, kernels/cell_comp.cpp) is a candidate
    of a calibrated cost model: with a model that prices it cheaply, pairs of
    rows denser than one half with rows that have bitmaps run on it, and the
    counts stay the oracle's; the reference's default model never picks it."""
    u = 1 << 16
    sets = gen.bernoulli_sets(60, u, 0.9, 71) + gen.bernoulli_sets(60, u, 0.05, 72)
    r = sb.StormRows(u)
    for s in sets:
        r.add(s)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    mat, st = r.allpairs_matrix(sb.POLICY_PERPAIR, 32)
    np.testing.assert_array_equal(mat, want)
    assert st["cell_pairs"].get("CB", 0) == 0
    model, _ = r.cost_model()
    model[13] = 1e-6                     # C x B nearly free
    r.cost_model(set_to=model)
    for pol in (sb.POLICY_PERPAIR, sb.POLICY_PERTILE):
        mat, st = r.allpairs_matrix(pol, 32)
        np.testing.assert_array_equal(mat, want)
        assert st["cell_pairs"].get("CB", 0) > 0, (pol, st["cell_pairs"])
    model, rms = r.calibrate(tile=32, samples=0, seed=9)
    mat, st = r.allpairs_matrix(sb.POLICY_PERPAIR, 32)
    np.testing.assert_array_equal(mat, want)
