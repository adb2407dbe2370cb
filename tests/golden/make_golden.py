"""Generate the golden vectors in tests/golden/ from the REFERENCE itself.

    make -C oracle reflib        # compiles the reference from its own sources
    python tests/golden/make_golden.py

Every expected value below comes out of oracle/_ref/libstorm_ref.so, i.e. the
StormBitmaps reference code (storm.cpp, kernels/*.cpp) compiled unmodified;
see oracle/ref_harness.cpp for which reference function produces which
number.  Inputs are seeded (tests/gen.py) and stored next to the outputs, so
the fixtures do not depend on the generator staying the same.

Output: tests/golden/golden.npz (a flat dict of arrays; see `keys` below).
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import gen  # noqa: E402
import oracle_lib as ol  # noqa: E402

R = ol.reference()
if R is None:
    sys.exit("oracle/_ref/libstorm_ref.so missing: run `make -C oracle reflib` first")

P = ol._p
out: dict[str, np.ndarray] = {}


def tri(n):
    return n * (n + 1) // 2


# ---------------------------------------------------------------- contiguous
CONTIG = {
    "dense_1024": (40, 1024, 0.4, 11),
    "sparse_4096": (40, 4096, 0.0008, 12),
    "mixed_8192": (60, 8192, (0.0, 0.05), 13),
    "odd_4033": (37, 4033, 0.3, 14),
    "cfg1_slice": (130, 65536, 0.5, 15),
    "cfg2_slice": (20, 262144, (0.05, 0.5), 16),
    "tiny_1": (1, 640, 0.5, 17),
    "pair_2": (2, 64, 0.5, 18),
}
for name, (n, m, p, seed) in CONTIG.items():
    w = gen.bernoulli_rows(n, m, p, seed)
    words = np.ascontiguousarray(w)
    nw = words.shape[1]
    s0 = R.ref_contig_sum(P(words, ol.u64p), n, nw, m, 0)
    s8 = R.ref_contig_sum(P(words, ol.u64p), n, nw, m, 8)
    mat = np.zeros(max(1, tri(n)), dtype=np.uint32)
    s_mt = R.ref_contig_matrix_mt(P(words, ol.u64p), n, nw, 0, n, P(mat, ol.u32p), 4)
    assert s0 == s8 == s_mt, (name, s0, s8, s_mt)
    out[f"contig/{name}/words"] = words
    out[f"contig/{name}/m"] = np.array([m], dtype=np.uint64)
    out[f"contig/{name}/sum"] = np.array([s0], dtype=np.uint64)
    out[f"contig/{name}/matrix"] = mat[: tri(n)]

# ------------------------------------------------------------------ STORM_t
g = gen.rng(21)
STORM = {
    "multiblock_sparse": [gen.uniform_set(g, int(g.integers(1, 300)), 200000) for _ in range(30)],
    "very_sparse": [gen.uniform_set(g, int(g.integers(1, 3)), 100000) for _ in range(30)],
    "mixed_rep": [gen.uniform_set(g, 9000 if i % 2 == 0 else 50, 65536) for i in range(12)],
    "dense_multichunk": [gen.uniform_set(g, int(g.integers(1, 30000)), 1 << 18) for _ in range(10)],
    "zipf_small": gen.zipf_sets(48, 1 << 24, 1.1, 16, 1 << 16, 22),
    "runs_small": gen.run_sets(40, 1 << 26, 20, 256, 23),
    "haplo_small": gen.haplotype_sets(96, 20000, 32, 24),
    "sweep_1e-3": gen.bernoulli_sets(24, 1 << 20, 1e-3, 25),
    "sweep_0.17": gen.bernoulli_sets(6, 1 << 18, 0.17, 26),
    "with_empty": [np.zeros(0, np.uint32), gen.uniform_set(g, 100, 70000), np.zeros(0, np.uint32),
                   np.arange(0, 65536 * 2, 7, dtype=np.uint32)],
}
for name, sets in STORM.items():
    vals, offs = gen.to_csr(sets)
    n = len(sets)
    s0 = R.ref_storm_sum(P(vals, ol.u32p), P(offs, ol.u64p), n, 0)
    s5 = R.ref_storm_sum(P(vals, ol.u32p), P(offs, ol.u64p), n, 5)
    mat = np.zeros(max(1, tri(n)), dtype=np.uint32)
    s_m = R.ref_storm_matrix(P(vals, ol.u32p), P(offs, ol.u64p), n, P(mat, ol.u32p))
    assert s0 == s5 == s_m, (name, s0, s5, s_m)
    out[f"storm/{name}/vals"] = vals
    out[f"storm/{name}/offs"] = offs
    out[f"storm/{name}/sum"] = np.array([s0], dtype=np.uint64)
    out[f"storm/{name}/matrix"] = mat[: tri(n)]
    # Chunk layout of the first non-empty row.
    for r in range(n):
        v = np.ascontiguousarray(sets[r], dtype=np.uint32)
        if v.size:
            ids = np.zeros(v.size, np.uint32)
            kinds = np.zeros(v.size, np.uint8)
            cards = np.zeros(v.size, np.uint32)
            k = R.ref_storm_layout(P(v, ol.u32p), v.size, P(ids, ol.u32p), P(kinds, ol.u8p), P(cards, ol.u32p))
            out[f"storm/{name}/layout_row"] = np.array([r], dtype=np.uint64)
            out[f"storm/{name}/layout"] = np.stack([ids[:k], kinds[:k].astype(np.uint32), cards[:k]])
            break

a_sets = STORM["multiblock_sparse"][:10]
b_sets = STORM["dense_multichunk"][:7]
av, ao = gen.to_csr(a_sets)
bv, bo = gen.to_csr(b_sets)
out["square/a_vals"], out["square/a_offs"], out["square/b_vals"], out["square/b_offs"] = av, ao, bv, bo
out["square/sum"] = np.array([R.ref_storm_square(P(av, ol.u32p), P(ao, ol.u64p), 10, P(bv, ol.u32p),
                                                 P(bo, ol.u64p), 7)], dtype=np.uint64)

# ---------------------------------------------------------------- low level
g = gen.rng(31)
v16a, v16b, v16r = [], [], []
for t in range(60):
    a = np.unique(g.integers(0, 65535, size=int(g.integers(1, 300)))).astype(np.uint16)
    b = np.unique(g.integers(0, 65535, size=int(g.integers(1, 300)))).astype(np.uint16)
    if t % 5 == 0:
        b = np.unique(np.concatenate([b, a[::3]])).astype(np.uint16)
    v16a.append(a); v16b.append(b)
    v16r.append(R.ref_vector16(P(a, ol.u16p), P(b, ol.u16p), a.size, b.size))
for key, lst in (("a", v16a), ("b", v16b)):
    vv, oo = gen.to_csr([x.astype(np.uint32) for x in lst])
    out[f"vec16/{key}_vals"], out[f"vec16/{key}_offs"] = vv, oo
out["vec16/result"] = np.array(v16r, dtype=np.uint64)

v32a, v32b, v32o = [], [], []
for t in range(20):
    a = np.unique(g.integers(0, 5000, size=int(g.integers(1, 400)))).astype(np.uint32)
    b = np.unique(g.integers(0, 5000, size=int(g.integers(1, 400)))).astype(np.uint32)
    o = np.zeros(2 * min(a.size, b.size) + 2, dtype=np.uint32)
    k = R.ref_vector32(P(a, ol.u32p), P(b, ol.u32p), a.size, b.size, P(o, ol.u32p))
    v32a.append(a); v32b.append(b); v32o.append(o[:k])
for key, lst in (("a", v32a), ("b", v32b), ("out", v32o)):
    vv, oo = gen.to_csr(lst)
    out[f"vec32/{key}_vals"], out[f"vec32/{key}_offs"] = vv, oo

bsl = []
for t in range(40):
    la = gen.uniform_set(g, int(g.integers(1, 64)), 4096)
    lb = gen.uniform_set(g, int(g.integers(1, 256)), 4096)
    ba = gen.sets_to_rows([la], 4096)[0]
    bb = gen.sets_to_rows([lb], 4096)[0]
    bsl.append((la, lb, R.ref_bitmaps_scalar_list(P(ba, ol.u64p), P(bb, ol.u64p), P(la, ol.u32p),
                                                   P(lb, ol.u32p), la.size, lb.size)))
for key, idx in (("a", 0), ("b", 1)):
    vv, oo = gen.to_csr([x[idx] for x in bsl])
    out[f"bsl/{key}_vals"], out[f"bsl/{key}_offs"] = vv, oo
out["bsl/result"] = np.array([x[2] for x in bsl], dtype=np.uint64)

wd = gen.bernoulli_rows(33, 640, 0.3, 32)
out["wrapper_diag/words"] = wd
out["wrapper_diag/sum"] = np.array([R.ref_wrapper_diag(33, P(wd, ol.u64p), wd.shape[1], 0),
                                    R.ref_wrapper_diag(33, P(wd, ol.u64p), wd.shape[1], 4)], dtype=np.uint64)

# ------------------------------------------------------------- kernel layer
POLICIES = {"AllBitmap": 0, "PerPair": 1, "PerTile": 2, "Probe": 5}
corp = {}
for u in (1024, 4033, 16384):
    corp[f"uniform_u{u}"] = gen.bernoulli_sets(40, u, 0.02, 0x9911 + u)
    corp[f"runs_u{u}"] = gen.run_sets(40, u, max(1, u * 0.02 / 32), 32, 0x9911 + u)
    corp[f"inverse_u{u}"] = [gen.uniform_set(g, int(np.exp(g.random() * np.log(u * 0.05))), u) for _ in range(40)]
for name, sets in corp.items():
    u = int(name.split("_u")[1])
    vals, offs = gen.to_csr(sets)
    n = len(sets)
    out[f"rows/{name}/vals"], out[f"rows/{name}/offs"] = vals, offs
    out[f"rows/{name}/universe"] = np.array([u], dtype=np.uint64)
    stats = []
    for pol, pv in POLICIES.items():
        for tile in (8, 16, 64):
            st = np.zeros(4, dtype=np.uint64)
            R.ref_allpairs_sum(P(vals, ol.u32p), P(offs, ol.u64p), n, u, pv, tile, P(st, ol.u64p))
            stats.append([pv, tile, st[0], st[1], st[2], st[3]])
    out[f"rows/{name}/allpairs_sum"] = np.array(stats, dtype=np.uint64)
    mat = np.zeros(tri(n), dtype=np.uint32)
    R.ref_allpairs_tiles(P(vals, ol.u32p), P(offs, ol.u64p), n, u, 64, P(mat, ol.u32p))
    out[f"rows/{name}/tiles_strict"] = mat

# build_row on edge rows (tests/test_cells.cpp:195-230 shapes).
edge_rows, edge_u = [], []
for u in (64, 128, 1024, 1025, 4033, 5000, 8192, 65536, 70001):
    cand = [[], [0], [u - 1], [63, 64], [511, 512], list(range(u)), list(range(0, u, 64)),
            list(range(0, u, 2)), list(range(u // 2, min(u // 2 + 300, u))), list(range(1, min(200, u)))]
    for c in cand:
        v = np.array(sorted(set(p for p in c if p < u)), dtype=np.uint32)
        edge_rows.append(v)
        edge_u.append(u)
# plus a few random rows with long runs (rank index) and dense rows (zone map).
for u, (k, L) in ((65536, (20, 900)), (70001, (40, 64)), (1 << 20, (50, 2000))):
    edge_rows.append(gen.run_sets(1, u, k, L, u)[0])
    edge_u.append(u)
repr_out = {"runs": [], "run_end": [], "ewah": [], "rank": [], "occ": [], "comp": [], "meta": [], "sizes": []}
for v, u in zip(edge_rows, edge_u):
    nw = (u + 63) // 64
    rs = np.zeros(v.size + 1, np.uint32); re = np.zeros(v.size + 1, np.uint32)
    ew = np.zeros(2 * nw + 2, np.uint64)
    rk = np.zeros(2 * ((nw + 7) // 8 + 1) + 2, np.uint64)
    oc = np.zeros((nw + 7) // 8 // 64 + 2, np.uint64)
    cp = np.zeros(u + 1, np.uint32)
    sz = np.zeros(6, np.uint64); me = np.zeros(8, np.uint32)
    R.ref_build_row(P(v, ol.u32p), v.size, u, P(rs, ol.u32p), P(re, ol.u32p), P(ew, ol.u64p), P(rk, ol.u64p),
                    P(oc, ol.u64p), P(cp, ol.u32p), P(sz, ol.u64p), P(me, ol.u32p))
    repr_out["runs"].append(rs[: sz[0]]); repr_out["run_end"].append(re[: sz[0]])
    repr_out["ewah"].append(ew[: sz[1]]); repr_out["rank"].append(rk[: sz[2]])
    repr_out["occ"].append(oc[: sz[3]]); repr_out["comp"].append(cp[: sz[4]])
    repr_out["meta"].append(me); repr_out["sizes"].append(sz)
vv, oo = gen.to_csr(edge_rows)
out["repr/vals"], out["repr/offs"] = vv, oo
out["repr/universe"] = np.array(edge_u, dtype=np.uint64)
for k in ("runs", "run_end", "comp"):
    out[f"repr/{k}_vals"], out[f"repr/{k}_offs"] = gen.to_csr(repr_out[k])
for k in ("ewah", "rank", "occ"):
    lst = repr_out[k]
    offs = np.zeros(len(lst) + 1, np.uint64)
    for i, x in enumerate(lst):
        offs[i + 1] = offs[i] + x.size
    out[f"repr/{k}_vals"] = np.concatenate(lst).astype(np.uint64) if lst else np.zeros(0, np.uint64)
    out[f"repr/{k}_offs"] = offs
out["repr/meta"] = np.stack(repr_out["meta"])
out["repr/sizes"] = np.stack(repr_out["sizes"])

# select_pairing / predict on metadata of row pairs from the corpora above.
metas = []
for name in ("uniform_u4033", "runs_u16384", "inverse_u1024", "runs_u1024"):
    sets = corp[name]
    u = int(name.split("_u")[1])
    for k in range(0, 36, 3):
        a, b = sets[k], sets[k + 1]
        ma = np.zeros(8, np.uint32); mb = np.zeros(8, np.uint32)
        ol.oracle().oracle_row_meta(P(a, ol.u32p), a.size, u, P(ma, ol.u32p))
        ol.oracle().oracle_row_meta(P(b, ol.u32p), b.size, u, P(mb, ol.u32p))
        pred = np.zeros(11, np.float64)
        sel = R.ref_select_pairing(P(ma, ol.u32p), P(mb, ol.u32p), pred.ctypes.data_as(ol.dblp))
        metas.append((ma, mb, sel, pred))
out["select/meta_a"] = np.stack([m[0] for m in metas])
out["select/meta_b"] = np.stack([m[1] for m in metas])
out["select/pairing"] = np.array([m[2] for m in metas], dtype=np.uint32)
out["select/predict"] = np.stack([m[3] for m in metas])

# Every cell variant of the reference on a few ordered pairs: all must agree.
cells = []
for name in ("uniform_u1024", "runs_u4033", "inverse_u16384"):
    sets = corp[name]
    u = int(name.split("_u")[1])
    for k in range(0, 12, 4):
        a, b = sets[k], sets[k + 1]
        res = np.zeros(256, np.uint64)
        nres = R.ref_all_cells(P(a, ol.u32p), a.size, P(b, ol.u32p), b.size, u, P(res, ol.u64p))
        want = R.ref_oracle_intersect(P(a, ol.u32p), a.size, P(b, ol.u32p), b.size, u)
        assert np.all(res[:nres] == want), (name, k)
        cells.append((u, a, b, want))
vv, oo = gen.to_csr([c[1] for c in cells])
out["cells/a_vals"], out["cells/a_offs"] = vv, oo
vv, oo = gen.to_csr([c[2] for c in cells])
out["cells/b_vals"], out["cells/b_offs"] = vv, oo
out["cells/universe"] = np.array([c[0] for c in cells], dtype=np.uint64)
out["cells/result"] = np.array([c[3] for c in cells], dtype=np.uint64)

path = os.path.join(HERE, "golden.npz")
np.savez_compressed(path, **out)
print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path) / 1e6:.2f} MB")
