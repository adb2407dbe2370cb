"""The transposed-panel engine of the STORM_t per-pair calls (csrc/panel.cuh)
against the oracle: every plain row in the panel (two 2048-row blocks,
queries with list and bitmap chunks), the cost-chosen three-way split with
the panel forced on and left to the planner, and rows that must stay on the
chunk kernel beside it."""
import numpy as np
import pytest

import gen
import oracle_lib as ol

pytestmark = pytest.mark.gpu


def build_storm(sb, sets):
    s = sb.Storm()
    for v in sets:
        s.add(np.asarray(v, dtype=np.uint32))
    return s


def _corpus_two_blocks(seed):
    """2600 rows over 2^18: 40 with bitmap chunks (>= 4096 values in each of
    the 4 chunks), the rest 0 .. 3000 values; shuffled."""
    g = gen.rng(seed)
    sets = [gen.uniform_set(g, int(g.integers(17000, 30000)), 1 << 18) for _ in range(40)]
    sets += [gen.uniform_set(g, int(g.integers(0, 3000)), 1 << 18) for _ in range(2560)]
    return [sets[k] for k in g.permutation(len(sets))]


def test_every_plain_row_in_the_panel(sb):
    sets = _corpus_two_blocks(301)
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    s.set_panel(2)
    mat, ssum = s.matrix()
    assert s.last_panel_rows() == len(sets)
    assert s.last_dense()[0] == 0 and s.last_postings_rows() == 0
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)
    assert s.pairw_intersect_cardinality() == ws


@pytest.mark.parametrize("mode", [1, -1])
def test_three_way_split_with_panel(sb, mode):
    """Zipf-sized rows over 2^20 (the mixed-density shape): tensor rows,
    panel rows and postings rows at once (mode 1 forces some rows into the
    panel; -1 leaves the choice to the cost model)."""
    sets = gen.zipf_sets(900, 1 << 20, 1.1, 16, 1 << 17, 302)
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    s.set_panel(mode)
    mat, ssum = s.matrix()
    if mode == 1:
        assert s.last_panel_rows() > 0
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)
    s.set_panel(0)
    mat0, s0 = s.matrix()
    assert s.last_panel_rows() == 0 and s0 == ws
    np.testing.assert_array_equal(mat0, want)


def test_panel_beside_chunk_rows(sb):
    """Rows with repeated list values stay on the chunk kernel (the
    reference's chunk-by-chunk count); every plain row goes to the panel."""
    g = gen.rng(303)
    sets = [gen.uniform_set(g, int(g.integers(1, 5000)), 3 << 16) for _ in range(300)]
    sets += [gen.uniform_set(g, int(g.integers(13000, 40000)), 3 << 16) for _ in range(20)]
    dup = [np.sort(np.concatenate([v, v[:5]])) for v in
           (gen.uniform_set(g, int(g.integers(20, 200)), 3 << 16) for _ in range(6))]
    sets += dup
    sets = [sets[k] for k in g.permutation(len(sets))]
    s = build_storm(sb, sets)
    s.set_panel(2)
    mat, ssum = s.matrix()
    assert s.last_panel_rows() == len(sets) - len(dup)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.storm_matrix(vals, offs)
    assert ssum == ws
    iu = np.triu_indices(len(sets))
    strict = iu[0] != iu[1]
    np.testing.assert_array_equal(mat[strict], want[strict])
    assert s.pairw_intersect_cardinality() == ws


def test_planner_calibration_keeps_counts(sb):
    """STORM_calibrate scales the planner's constants by the measured /
    predicted device time of each engine on a strided row sample; the plans
    it leads to give the oracle's counts, and every engine's time of the
    last call is reported beside its prediction."""
    sets = gen.zipf_sets(700, 1 << 20, 1.1, 16, 1 << 17, 304)
    s = build_storm(sb, sets)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    scales = s.calibrate(256)
    assert scales[3] == 256
    assert all(x > 0 for x in scales[:3]), scales
    mat, ssum = s.matrix()
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)
    eng = s.last_engine_ms()
    assert all(v[0] >= 0 for v in eng.values())
    assert sum(v[0] for v in eng.values()) > 0
    s.reset_cost_model()
    mat, ssum = s.matrix()
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)
