"""The kernel layer on the GPU (STORM_rows_t): every cell on every ordered
pair of the reference's edge rows, every policy and both execution forms
against the reference's golden all-pairs outputs and the oracle."""
import numpy as np
import pytest

import gen
import oracle_lib as ol
from conftest import golden_sets

pytestmark = pytest.mark.gpu


def rows_of(sb, sets, universe, budget=None):
    r = sb.StormRows(universe)
    if budget is not None:
        r.set_bitmap_budget(budget)
    for s in sets:
        r.add(np.asarray(s, dtype=np.uint32))
    return r


def edge_rows(u):
    cand = [[], [0], [u - 1], [63, 64], [511, 512], list(range(u)), list(range(0, u, 64)), list(range(0, u, 2)),
            list(range(u // 2, min(u // 2 + 300, u))), list(range(1, min(200, u)))]
    return [np.array(sorted(set(p for p in c if p < u)), dtype=np.uint32) for c in cand]


CELLS = ["BB", "BS", "BR", "BW", "SS", "SR", "SW", "RR", "RW", "WW", "CB"]


@pytest.mark.parametrize("u", [64, 128, 1024, 1025, 4033, 5000, 8192, 65536, 70001])
def test_every_cell_on_edge_rows_both_orders(sb, u):
    """tests/test_cells.cpp:195-230 shapes at the same universes, every cell,
    both argument orders, against the oracle."""
    rows = edge_rows(u) + gen.run_sets(3, u, 6, 40, u) + [gen.uniform_set(gen.rng(u), u // 3, u)]
    r = rows_of(sb, rows, u)
    n = len(rows)
    for i in range(n):
        for j in range(n):
            want = ol.oracle().oracle_list_intersect(ol._p(rows[i], ol.u32p), rows[i].size,
                                                     ol._p(rows[j], ol.u32p), rows[j].size)
            meta_i = r.meta(i)
            for name in CELLS:
                p = CELLS.index(name) if name != "CB" else sb.P_CB
                if name == "CB" and not (meta_i[8] & 2):
                    continue   # complement exists only above density 1/2
                got = r.cell(p, i, j)
                assert got == want, (u, name, i, j, got, want)


def test_representation_metadata_matches_reference(sb, golden):
    rows = golden_sets(golden, "repr/")
    for k, (v, u) in enumerate(zip(rows, golden["repr/universe"])):
        r = rows_of(sb, [v], int(u))
        m = r.meta(0)
        np.testing.assert_array_equal(m[:8], golden["repr/meta"][k], err_msg=f"row {k}")
        assert bool(m[8] & 2) == (golden["repr/sizes"][k][4] > 0)   # complement built iff reference builds it


POLICIES = ["ALLBITMAP", "PERPAIR", "PERTILE", "ORACLE", "PROBE", "REFINE", "LEARNED"]


@pytest.mark.parametrize("exec_", ["batched", "per_tile"])
def test_golden_allpairs_every_policy(sb, golden, exec_):
    ex = sb.EXEC_BATCHED if exec_ == "batched" else sb.EXEC_PER_TILE
    names = sorted({k.split("/")[1] for k in golden.files if k.startswith("rows/")})
    for name in names:
        sets = golden_sets(golden, f"rows/{name}/")
        u = int(golden[f"rows/{name}/universe"][0])
        r = rows_of(sb, sets, u)
        want = int(golden[f"rows/{name}/allpairs_sum"][0][2])
        n = len(sets)
        strict_want = golden[f"rows/{name}/tiles_strict"]
        iu = np.triu_indices(n)
        strict = iu[0] != iu[1]
        for pol in POLICIES:
            for tile in (8, 16, 64):
                s, st = r.allpairs_sum(getattr(sb, "POLICY_" + pol), tile, exec_=ex)
                assert s == want, (name, pol, tile)
                assert st["pairs"] == n * (n - 1) // 2, (name, pol, tile, st)
            mat, st = r.allpairs_matrix(getattr(sb, "POLICY_" + pol), 16, exec_=ex)
            np.testing.assert_array_equal(mat[strict], strict_want[strict], err_msg=f"{name}/{pol}")
            np.testing.assert_array_equal(mat[~strict], [len(x) for x in sets])


def test_fixed_cell_policy_every_cell(sb, golden):
    sets = golden_sets(golden, "rows/runs_u4033/")
    r = rows_of(sb, sets, 4033)
    want = int(golden["rows/runs_u4033/allpairs_sum"][0][2])
    for p in range(10):
        s, st = r.allpairs_sum(sb.POLICY_FIXED, 16, fixed_cell=p)
        assert s == want, sb.PAIRINGS[p]
        live = {k: v for k, v in st["cell_pairs"].items() if k != "EMPTY"}
        assert set(live) <= {sb.PAIRINGS[p]}, st


def test_tiles_visitor_original_order(sb, golden):
    sets = golden_sets(golden, "rows/inverse_u16384/")
    r = rows_of(sb, sets, 16384)
    col, st = r.allpairs_tiles(sb.POLICY_PERTILE, 64)
    n = len(sets)
    iu = np.triu_indices(n)
    strict = iu[0] != iu[1]
    np.testing.assert_array_equal(col.out[strict], golden["rows/inverse_u16384/tiles_strict"][strict])


@pytest.mark.parametrize("case", ["zipf", "runs", "haplo", "sweep"])
def test_config_shaped_corpora_all_policies(sb, case):
    if case == "zipf":
        sets, u = gen.zipf_sets(120, 1 << 24, 1.1, 16, 1 << 16, 41), 1 << 24
    elif case == "runs":
        sets, u = gen.run_sets(100, 1 << 26, 30, 256, 42), 1 << 26
    elif case == "haplo":
        sets, u = gen.haplotype_sets(240, 20000, 32, 43), 20000
    else:
        sets, u = [], 1 << 22
        for d in (1e-5, 1e-4, 1e-3, 1e-2, 0.17):
            sets += gen.bernoulli_sets(20, u, d, int(d * 1e6) + 44)
    r = rows_of(sb, sets, u)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    for pol in ("PERPAIR", "PERTILE", "PROBE", "REFINE", "LEARNED"):
        for ex in (sb.EXEC_BATCHED, sb.EXEC_PER_TILE):
            mat, st = r.allpairs_matrix(getattr(sb, "POLICY_" + pol), 32, exec_=ex)
            assert st["sum"] == ws, (case, pol)
            np.testing.assert_array_equal(mat, want, err_msg=f"{case}/{pol}/{ex}")


@pytest.mark.parametrize("universe", [4096 + 64, 1 << 17])
def test_tensor_core_dense_block(sb, universe):
    """The densest rows of the density order are compared by the tcgen05
    kernel and scattered back through the row map; counts stay exact for
    every policy and both execution forms, with and without the block."""
    g = gen.rng(universe)
    sets = [gen.uniform_set(g, int(universe * g.uniform(0.05, 0.5)), universe) for _ in range(300)]
    sets += gen.bernoulli_sets(200, universe, 0.002, 71)
    order = g.permutation(len(sets))
    sets = [sets[k] for k in order]
    r = rows_of(sb, sets, universe)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    for thr in (1.0 / 64, 0.0):
        r.set_dense_block(thr)
        for pol in ("PERTILE", "LEARNED", "REFINE", "PROBE"):
            for ex in (sb.EXEC_BATCHED, sb.EXEC_PER_TILE):
                mat, st = r.allpairs_matrix(getattr(sb, "POLICY_" + pol), 64, exec_=ex)
                np.testing.assert_array_equal(mat, want, err_msg=f"{pol}/{ex}/{thr}")
                assert st["sum"] == ws and st["pairs"] == len(sets) * (len(sets) - 1) // 2
                if thr > 0:
                    assert st["cell_pairs"].get("BB", 0) >= 300 * 299 // 2


def test_rows_without_bitmaps_stay_exact(sb):
    """A bitmap budget too small for every row leaves the sparse rows without
    B (the reference's sparse_only rows): B cells are skipped for them and
    all-bitmap is refused, every other policy stays exact."""
    sets = gen.zipf_sets(80, 1 << 20, 1.1, 16, 1 << 15, 51)
    r = rows_of(sb, sets, 1 << 20, budget=10 * (1 << 20) // 8)   # room for ~10 bitmaps
    metas = [r.meta(i) for i in range(len(sets))]
    assert 0 < sum(int(m[8] & 1) for m in metas) < len(sets)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    with pytest.raises(sb.StormError):
        r.allpairs_sum(sb.POLICY_ALLBITMAP)
    for pol in ("PERPAIR", "PERTILE", "PROBE", "REFINE"):
        mat, st = r.allpairs_matrix(getattr(sb, "POLICY_" + pol), 16)
        np.testing.assert_array_equal(mat, want, err_msg=pol)


def test_autotune_tile_and_dense_block(sb):
    """The kernel-layer autotuner times tile x dense-block candidates on the
    corpus, keeps the fastest (tile used when calls pass tile 0), and a
    trained learned selector keeps its training tile."""
    g = gen.rng(903)
    sets = gen.zipf_sets(400, 1 << 18, 1.1, 16, 1 << 15, 904)
    r = rows_of(sb, sets, 1 << 18)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    tile, dens, times = r.autotune(sb.POLICY_PERTILE)
    assert all(t > 0 for t in times)
    k = int(np.argmin(times))
    assert tile == (32, 64, 128, 256)[k // 4] and dens == (0.0, 1 / 65536, 1 / 16384, 1 / 4096)[k % 4]
    mat, st = r.allpairs_matrix(sb.POLICY_PERTILE, 0)
    assert st["sum"] == ws
    np.testing.assert_array_equal(mat, want)
    r.train_selector(tile=64, samples=256, epochs=50, seed=3)
    tile, dens, times = r.autotune(sb.POLICY_LEARNED)
    assert tile == 64 and all(t < 0 for k, t in enumerate(times) if k // 4 != 1)
    mat, st = r.allpairs_matrix(sb.POLICY_LEARNED, 0)
    np.testing.assert_array_equal(mat, want)


def test_autotune_times_each_dense_block_candidate(sb):
    """The batched form's CUDA graph is re-captured when the dense block
    changes: on rows where the tensor block is many times faster than the
    B x B cells, the autotuner's density-0 candidate (no block) must time
    slower than the candidates that put every row in the block, and counts
    stay equal to the oracle's."""
    u, n = 1 << 18, 1024
    words = gen.bernoulli_rows(n, u, 0.3, 913)
    sets = gen.rows_to_sets(words, u)
    r = rows_of(sb, sets, u)
    _, want = ol.contig_matrix(words, want_matrix=False)
    tile, dens, times = r.autotune(sb.POLICY_PERTILE)
    for a in range(4):
        t = times[4 * a: 4 * a + 4]
        assert t[0] > 1.5 * min(t[1:]), (a, t)
    assert dens > 0.0
    for d in (0.0, 1 / 16384, 0.0):
        r.set_dense_block(d)
        s, st = r.allpairs_sum(sb.POLICY_PERTILE, 64, exec_=sb.EXEC_BATCHED)
        assert s == want
        if d > 0.0:   # every row is in the block: all pairs on the tensor cores
            assert st["cell_pairs"] == {"BB": n * (n - 1) // 2}


def test_batched_graph_after_buffers_grow(sb):
    """A batched call, a per-tile call at a smaller tile (which grows the
    per-call device buffers), then the first call again: the replayed graph
    must not address the buffers freed in between."""
    sets = gen.zipf_sets(700, 1 << 16, 1.1, 8, 1 << 12, 918)
    r = rows_of(sb, sets, 1 << 16)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    for tile, ex in ((64, sb.EXEC_BATCHED), (32, sb.EXEC_PER_TILE), (64, sb.EXEC_BATCHED), (16, sb.EXEC_PER_TILE),
                     (64, sb.EXEC_BATCHED)):
        mat, st = r.allpairs_matrix(sb.POLICY_PERTILE, tile, exec_=ex)
        assert st["sum"] == ws
        np.testing.assert_array_equal(mat, want)


def clustered_sets(n, universe, width, seed):
    """Position-clustered rows: each row's values lie in a window of `width`
    positions at a uniform start -- most row blocks then share no zone bin."""
    g = gen.rng(seed)
    out = []
    for _ in range(n):
        start = int(g.integers(0, universe - width))
        k = int(g.integers(1, width // 4))
        out.append(np.sort(g.choice(width, size=k, replace=False)).astype(np.uint32) + np.uint32(start))
    return out


@pytest.mark.parametrize("universe,width", [(1 << 20, 2000), (1 << 16, 300), (1 << 24, 50000)])
def test_zone_rejected_tiles_stay_exact(sb, universe, width):
    """Tiles whose two row blocks' zone maps share no bin are skipped whole
    (bench/bench_tile.cpp's zone-map filter at tile granularity): on
    position-clustered rows the per-pair counts equal the oracle's under
    every policy and both execution forms, and the skipped pairs are
    reported."""
    sets = clustered_sets(700, universe, width, universe + width)
    r = rows_of(sb, sets, universe)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    for pol in (sb.POLICY_PERTILE, sb.POLICY_PERPAIR, sb.POLICY_PROBE, sb.POLICY_REFINE):
        for ex in (sb.EXEC_BATCHED, sb.EXEC_PER_TILE):
            mat, st = r.allpairs_matrix(pol, 64, exec_=ex)
            assert st["sum"] == ws, (pol, ex)
            np.testing.assert_array_equal(mat, want, err_msg=f"{pol}/{ex}")
    s, st = r.allpairs_sum(sb.POLICY_PERTILE, 64)
    assert s == ws and st["skipped"] > 0
