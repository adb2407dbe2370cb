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
