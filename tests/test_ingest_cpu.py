"""STORM_t ingest (STORM_add) against the reference's own STORM_add, field by
field on the public structs -- chunk ids, bitmap/list choice, n_bits_set,
list entries, bitmap words, capacities, last inserted value -- on seeded
sorted, unsorted and repeated-value rows. Host only; needs the reference
library built from its sources (oracle/_ref), skipped without it."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as ol


class Bitmap(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_uint64)), ("_pad0", C.c_char * 56), ("scalar", C.POINTER(C.c_uint16)),
                ("bits", C.c_uint32), ("n_bits_set", C.c_uint32), ("n_scalar_word", C.c_uint32),
                ("n_missing", C.c_uint32), ("m_scalar", C.c_uint32), ("id", C.c_uint32), ("_pad1", C.c_char * 32)]


class Cont(C.Structure):
    _fields_ = [("bitmaps", C.POINTER(Bitmap)), ("block_ids", C.POINTER(C.c_uint32)),
                ("n_bitmaps", C.c_uint32), ("m_bitmaps", C.c_uint32), ("prev", C.c_uint32)]


class StormT(C.Structure):
    _fields_ = [("conts", C.POINTER(Cont)), ("n_conts", C.c_uint32), ("m_conts", C.c_uint32)]


def _dump(h):
    s = C.cast(h, C.POINTER(StormT)).contents
    rows = []
    for r in range(s.n_conts):
        c = s.conts[r]
        row = [c.n_bitmaps, c.m_bitmaps, c.prev]
        for k in range(c.n_bitmaps):
            b = c.bitmaps[k]
            nb, ns = b.bits & 0x3FFFFFFF, b.n_scalar_word & 0x7FFFFFFF
            row.append((c.block_ids[k], b.id, nb, b.n_bits_set, ns,
                        C.string_at(b.data, nb * 8) if nb and b.data else None,
                        C.string_at(b.scalar, ns * 2) if ns and b.scalar else None))
        rows.append(row)
    return rows


def test_storm_add_matches_reference_structs(sb):
    R = ol.reference()
    if R is None:
        pytest.skip("reference library not built (oracle/_ref)")
    L = sb.lib()
    for lib in (R, L):
        lib.STORM_new.restype = C.c_void_p
        lib.STORM_add.argtypes = [C.c_void_p, sb.u32p, C.c_uint32]
        lib.STORM_free.argtypes = [C.c_void_p]
    g = np.random.default_rng(20261204)
    for trial in range(16):
        hr, hl = R.STORM_new(), L.STORM_new()
        try:
            for r in range(20):
                kind, n = int(g.integers(0, 4)), int(g.integers(1, 30000))
                if kind == 0:
                    v = np.sort(g.integers(0, 1 << 20, n))                              # sorted, repeats possible
                elif kind == 1:
                    v = np.sort(g.choice(1 << 18, size=min(n, 1 << 17), replace=False))  # dense chunks
                elif kind == 2:
                    v = g.integers(0, 1 << 20, n)                                        # unsorted
                else:
                    v = np.sort(np.repeat(g.integers(0, 1 << 19, n // 3 + 1), 3))       # every value 3 times
                v = np.ascontiguousarray(v, dtype=np.uint32)
                assert R.STORM_add(hr, v.ctypes.data_as(sb.u32p), v.size) == L.STORM_add(hl, v.ctypes.data_as(sb.u32p),
                                                                                          v.size)
            assert _dump(hl) == _dump(hr), trial
        finally:
            R.STORM_free(hr)
            L.STORM_free(hl)


def test_add_rows_builds_what_add_builds(sb):
    """STORM_add_rows (rows split on several host threads) leaves exactly the
    public structs that one STORM_add per row leaves -- empty rows, sorted,
    unsorted and repeated values included -- appended after existing rows."""
    L = sb.lib()
    L.STORM_new.restype = C.c_void_p
    L.STORM_add.argtypes = [C.c_void_p, sb.u32p, C.c_uint32]
    L.STORM_free.argtypes = [C.c_void_p]
    g = np.random.default_rng(77)
    rows = []
    for r in range(3000):
        kind, n = int(g.integers(0, 5)), int(g.integers(0, 9000))
        if kind == 0:
            v = np.sort(g.integers(0, 1 << 20, n))
        elif kind == 1:
            v = np.sort(g.choice(1 << 18, size=min(n * 8, 1 << 17), replace=False))
        elif kind == 2:
            v = g.integers(0, 1 << 20, n)
        elif kind == 3:
            v = np.sort(np.repeat(g.integers(0, 1 << 19, n // 3 + 1), 3))
        else:
            v = np.zeros(0)
        rows.append(np.ascontiguousarray(v, dtype=np.uint32))
    one, bulk = L.STORM_new(), L.STORM_new()
    try:
        head = rows[:7]
        for v in rows:
            assert L.STORM_add(one, v.ctypes.data_as(sb.u32p), v.size) == 1
        for v in head:   # rows already present before the bulk call
            L.STORM_add(bulk, v.ctypes.data_as(sb.u32p), v.size)
        rest = rows[7:]
        vals = np.ascontiguousarray(np.concatenate(rest), dtype=np.uint32)
        offs = np.zeros(len(rest) + 1, np.uint64)
        offs[1:] = np.cumsum([len(v) for v in rest])
        assert L.STORM_add_rows(bulk, vals.ctypes.data_as(sb.u32p), offs.ctypes.data_as(sb.u64p), len(rest)) == len(rest)
        assert _dump(bulk) == _dump(one)
        bad = np.array([0, 5, 3], np.uint64)
        assert L.STORM_add_rows(bulk, vals.ctypes.data_as(sb.u32p), bad.ctypes.data_as(sb.u64p), 2) == sb.EARG
        assert L.STORM_add_rows(None, vals.ctypes.data_as(sb.u32p), offs.ctypes.data_as(sb.u64p), 1) == sb.ENULL
    finally:
        L.STORM_free(one)
        L.STORM_free(bulk)


def test_add_bitmap_rows_builds_what_add_builds(sb):
    """STORM_add_bitmap_rows leaves the public structs that STORM_add of each
    row's set positions leaves: empty rows, list chunks, bitmap chunks and a
    partial last chunk."""
    import gen
    L = sb.lib()
    L.STORM_new.restype = C.c_void_p
    L.STORM_add.argtypes = [C.c_void_p, sb.u32p, C.c_uint32]
    L.STORM_free.argtypes = [C.c_void_p]
    g = np.random.default_rng(5)
    m = 3 * 65536 + 4096 + 64 * 7        # three whole chunks and a partial one
    nw = (m + 63) // 64
    words = np.zeros((40, nw), np.uint64)
    for r in range(40):
        p = [0.0, 1e-4, 0.03, 0.3][r % 4]
        bits = g.random(m) < p
        words[r] = gen.pack_bool_rows(bits[None, :])[0]
    one, bulk = L.STORM_new(), L.STORM_new()
    try:
        for v in gen.rows_to_sets(words, m):
            v = np.ascontiguousarray(v, dtype=np.uint32)
            L.STORM_add(one, v.ctypes.data_as(sb.u32p), v.size)
        assert L.STORM_add_bitmap_rows(bulk, words.ctypes.data_as(sb.u64p), 40, nw) == 40
        assert _dump(bulk) == _dump(one)
    finally:
        L.STORM_free(one)
        L.STORM_free(bulk)
