"""STORMBIN corpus files (the reference's on-disk format, written by its
tools/*2bin.py and read by bench/bench_allpairs.cpp:44-72) loaded into
STORM_t and STORM_rows_t. Loading is host work: these run without a GPU,
except the last one, which also compares the loaded corpus's all-pairs
counts with the oracle."""
import struct

import numpy as np
import pytest

import gen
import oracle_lib as ol


def write_stormbin(path, rows, n_bits, header_rows=None):
    with open(path, "wb") as f:
        f.write(b"STORMBIN" + struct.pack("<IIII", 1, len(rows) if header_rows is None else header_rows, n_bits, 0))
        for r in rows:
            r = np.asarray(r, dtype="<u4")
            f.write(struct.pack("<I", len(r)) + r.tobytes())


def corpus():
    g = gen.rng(7)
    rows = [gen.uniform_set(g, int(g.integers(0, 400)), 1 << 18) for _ in range(40)]
    rows[5] = np.zeros(0, np.uint32)
    return rows


def test_load_into_storm_t_and_rows(sb, tmp_path):
    rows = corpus()
    p = str(tmp_path / "c.bin")
    write_stormbin(p, rows, 1 << 18, header_rows=0)      # writers patch n_rows late; readers do not need it
    kept = [r for r in rows if len(r)]
    s = sb.Storm()
    n, nb = s.load_stormbin(p)
    assert (n, nb) == (len(kept), 1 << 18) and len(s) == len(kept)
    r = sb.StormRows.from_stormbin(p)
    assert r.universe == 1 << 18 and len(r) == len(kept)
    # stride counts every row of the file, empty ones too; max_rows caps the kept rows
    s2 = sb.Storm()
    n2, _ = s2.load_stormbin(p, max_rows=7, stride=3)
    want = [x for k, x in enumerate(rows) if k % 3 == 0 and len(x)][:7]
    assert n2 == len(want)


def test_rejects_bad_files(sb, tmp_path):
    s = sb.Storm()
    with pytest.raises(sb.StormError):
        s.load_stormbin(str(tmp_path / "missing.bin"))
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"NOTSTORM" + b"\0" * 16)
    with pytest.raises(sb.StormError):
        s.load_stormbin(str(bad))
    p = str(tmp_path / "range.bin")
    write_stormbin(p, [[1, 2, 70000]], 65536)            # position >= n_bits
    with pytest.raises(sb.StormError):
        sb.StormRows.from_stormbin(p)
    p = str(tmp_path / "order.bin")
    write_stormbin(p, [[5, 3]], 65536)                   # not ascending
    with pytest.raises(sb.StormError):
        s.load_stormbin(p)
    p = str(tmp_path / "trunc.bin")
    write_stormbin(p, [[1, 2, 3]], 65536)
    with open(p, "r+b") as f:
        f.truncate(24 + 4 + 8)
    with pytest.raises(sb.StormError):
        s.load_stormbin(p)


@pytest.mark.gpu
def test_loaded_corpus_all_pairs_match_oracle(sb, tmp_path):
    rows = corpus()
    p = str(tmp_path / "c.bin")
    write_stormbin(p, rows, 1 << 18)
    kept = [r for r in rows if len(r)]
    vals, offs = gen.to_csr(kept)
    want, ws = ol.sets_matrix(vals, offs)
    s = sb.Storm()
    s.load_stormbin(p)
    mat, ssum = s.matrix()
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)
    r = sb.StormRows.from_stormbin(p)
    mat, st = r.allpairs_matrix(sb.POLICY_PERTILE, 64)
    np.testing.assert_array_equal(mat, want)


def write_stormpack(path, rows, n_bits):
    """The reference's STORMPACK layout (tools/pack.cpp:100-145), with every
    stored representation: bitmap, u16 array, u16 runs, full, empty."""
    nw = (n_bits + 63) // 64
    blob, offs, lens, tags = bytearray(), [], [], []
    for k, r in enumerate(rows):
        r = np.asarray(r, dtype=np.int64)
        while len(blob) % 8:
            blob.append(0)
        start = len(blob)
        if len(r) == 0:
            t = 4
        elif len(r) == n_bits:
            t = 3
        elif k % 3 == 0:
            t = 0
            bm = np.zeros(nw, np.uint64)
            np.bitwise_or.at(bm, r >> 6, (np.uint64(1) << (r & 63).astype(np.uint64)))
            blob += bm.astype("<u8").tobytes()
        elif k % 3 == 1:
            t = 1
            blob += r.astype("<u2").tobytes()
        else:
            t = 2
            cuts = np.flatnonzero(np.diff(r) != 1) + 1
            for seg in np.split(r, cuts):
                blob += struct.pack("<HH", int(seg[0]), len(seg))
        offs.append(start)
        lens.append(len(blob) - start)
        tags.append(t)
    head = b"STRMPACK" + struct.pack("<IIII", 1, len(rows), n_bits, 0)
    head += np.asarray(offs, "<u4").tobytes() + np.asarray(lens, "<u4").tobytes() + bytes(tags)
    head += b"\0" * (-len(head) % 8)
    with open(path, "wb") as f:
        f.write(head + bytes(blob))


def pack_corpus():
    g = gen.rng(8)
    rows = [gen.uniform_set(g, int(g.integers(0, 3000)), 5008) for _ in range(30)]
    rows += [np.arange(100, 400, dtype=np.uint32), np.zeros(0, np.uint32), np.arange(5008, dtype=np.uint32)]
    return rows


def test_load_stormpack(sb, tmp_path):
    rows = pack_corpus()
    p = str(tmp_path / "c.pack")
    write_stormpack(p, rows, 5008)
    s = sb.Storm()
    assert s.load_stormpack(p) == (len(rows), 5008)
    r = sb.StormRows.from_stormpack(p)
    assert r.universe == 5008 and len(r) == len(rows)
    bad = tmp_path / "bad.pack"
    bad.write_bytes(open(p, "rb").read()[:40])
    with pytest.raises(sb.StormError):
        sb.Storm().load_stormpack(str(bad))


@pytest.mark.gpu
def test_loaded_stormpack_all_pairs_match_oracle(sb, tmp_path):
    rows = pack_corpus()
    p = str(tmp_path / "c.pack")
    write_stormpack(p, rows, 5008)
    vals, offs = gen.to_csr(rows)
    want, ws = ol.sets_matrix(vals, offs)
    s = sb.Storm()
    s.load_stormpack(p)
    mat, ssum = s.matrix()
    assert ssum == ws
    np.testing.assert_array_equal(mat, want)
    r = sb.StormRows.from_stormpack(p)
    mat, st = r.allpairs_matrix(sb.POLICY_PERTILE, 64)
    np.testing.assert_array_equal(mat, want)


def _fixture_sets():
    import importlib.util
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "make_corpus_fixtures.py")
    spec = importlib.util.spec_from_file_location("make_corpus_fixtures", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.corpus_sets()


def _fixture(name):
    import os
    return os.path.join(os.path.dirname(__file__), "golden", name)


def test_reference_written_fixtures_load(sb):
    """Files written by the reference's own tools (tools/sets2bin.py and
    tools/pack.cpp, tests/golden/make_corpus_fixtures.py) load with their row
    counts and universe."""
    rows = _fixture_sets()
    s = sb.Storm()
    assert s.load_stormbin(_fixture("corpus.stormbin")) == (len(rows), 5008)
    s = sb.Storm()
    assert s.load_stormpack(_fixture("corpus.stormpack")) == (len(rows), 5008)
    r = sb.StormRows.from_stormpack(_fixture("corpus.stormpack"))
    assert (len(r), r.universe) == (len(rows), 5008)


@pytest.mark.gpu
def test_reference_written_fixtures_match_oracle(sb):
    """All-pairs counts of the reference-written STORMBIN and STORMPACK files
    equal the oracle's on the sets they were written from."""
    rows = _fixture_sets()
    vals, offs = gen.to_csr(rows)
    want, ws = ol.sets_matrix(vals, offs)
    for loader in ("stormbin", "stormpack"):
        s = sb.Storm()
        getattr(s, "load_" + loader)(_fixture("corpus." + loader))
        mat, ssum = s.matrix()
        assert ssum == ws, loader
        np.testing.assert_array_equal(mat, want, err_msg=loader)
        r = (sb.StormRows.from_stormbin if loader == "stormbin" else sb.StormRows.from_stormpack)(
            _fixture("corpus." + loader))
        mat, st = r.allpairs_matrix(sb.POLICY_PERTILE, 64)
        np.testing.assert_array_equal(mat, want, err_msg=loader)


def _threshold_golden():
    import json
    with open(_fixture("threshold_hits.json")) as f:
        return {float(k): v for k, v in json.load(f).items()}


def test_oracle_threshold_pinned_to_reference():
    """The oracle's thresholded set on the fixture corpus has exactly the hit
    counts the reference's bench/bench_threshold.cpp reports for it."""
    rows = _fixture_sets()
    vals, offs = gen.to_csr(rows)
    tri, _ = ol.sets_matrix(vals, offs)
    for t, hits in _threshold_golden().items():
        assert len(ol.threshold_pairs(tri, len(rows), t)[0]) == hits, t


@pytest.mark.gpu
def test_threshold_forms_match_reference_counts(sb):
    """STORM_t (loaded from the reference-written STORMBIN file) and
    STORM_contiguous_t thresholded forms: the reference's hit counts, and the
    oracle's pairs and counts."""
    rows = _fixture_sets()
    vals, offs = gen.to_csr(rows)
    tri, _ = ol.sets_matrix(vals, offs)
    s = sb.Storm()
    s.load_stormbin(_fixture("corpus.stormbin"))
    words = gen.sets_to_rows(rows, 5008)
    c = sb.StormContig(5008)
    c.add_bitmaps(words)
    for t, hits in _threshold_golden().items():
        wi, wj, wc = ol.threshold_pairs(tri, len(rows), t)
        for h in (s, c):
            gi, gj, gc, found = h.threshold(t, cap=4096)
            assert found == hits, (type(h).__name__, t)
            np.testing.assert_array_equal(gi, wi)
            np.testing.assert_array_equal(gj, wj)
            np.testing.assert_array_equal(gc, wc)
