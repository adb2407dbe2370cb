"""ctypes view of the CPU checkers (test infrastructure only).

    oracle()     oracle/liboracle.so -- this repo's C restatement (always present)
    reference()  oracle/_ref/libstorm_ref.so -- the reference compiled from its
                 own sources, when it was built (None otherwise)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libstorm_ref.so")

u8p, u16p, u32p, u64p = (C.POINTER(t) for t in (C.c_uint8, C.c_uint16, C.c_uint32, C.c_uint64))
dblp = C.POINTER(C.c_double)
_cache = {}


def _p(a, t):
    return a.ctypes.data_as(t)


def oracle():
    if "o" in _cache:
        return _cache["o"]
    src = os.path.join(ROOT, "oracle", "storm_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)
    L = C.CDLL(ORACLE_SO)
    sigs = {
        "oracle_and_popcount": (C.c_uint64, [u64p, u64p, C.c_uint64]),
        "oracle_contig_matrix": (C.c_uint64, [u64p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, u32p]),
        "oracle_list_intersect": (C.c_uint64, [u32p, C.c_uint64, u32p, C.c_uint64]),
        "oracle_sets_matrix": (C.c_uint64, [u32p, u64p, C.c_uint64, C.c_uint64, C.c_uint64, u32p]),
        "oracle_sets_square": (C.c_uint64, [u32p, u64p, C.c_uint64, u32p, u64p, C.c_uint64]),
        "oracle_chunk_split": (C.c_uint64, [u32p, C.c_uint64, u32p, u8p, u32p]),
        "oracle_storm_matrix": (C.c_uint64, [u32p, u64p, C.c_uint64, u32p]),
        "oracle_list16_blocked": (C.c_uint64, [u16p, u16p, C.c_uint32, C.c_uint32]),
        "oracle_runs": (C.c_uint64, [u32p, C.c_uint64, u32p, u32p]),
        "oracle_ewah": (C.c_uint64, [u64p, C.c_uint64, u64p]),
        "oracle_ewah_decode": (None, [u64p, C.c_uint64, u64p]),
        "oracle_rank9": (None, [u64p, C.c_uint64, u64p]),
        "oracle_occ": (None, [u64p, C.c_uint64, C.c_uint64, u64p]),
        "oracle_row_meta": (None, [u32p, C.c_uint64, C.c_uint32, u32p]),
        "oracle_complement": (C.c_uint64, [u32p, C.c_uint64, C.c_uint32, u32p]),
        "oracle_contig_row": (C.c_uint64, [u64p, C.c_uint64, C.c_uint64, C.c_uint64, u32p]),
        "oracle_row_popcounts": (None, [u64p, C.c_uint64, C.c_uint64, u32p]),
        "oracle_strip_new": (C.c_void_p, [u32p, u64p, C.c_uint32, C.c_uint64]),
        "oracle_strip_count": (None, [C.c_void_p, u32p, u64p, C.c_uint64, u32p]),
        "oracle_strip_free": (None, [C.c_void_p]),
        "oracle_contig_strip": (None, [u64p, C.c_uint32, u64p, C.c_uint64, C.c_uint64, u32p]),
    }
    for k, (r, a) in sigs.items():
        f = getattr(L, k)
        f.restype, f.argtypes = r, a
    _cache["o"] = L
    return L


def reference():
    if "r" in _cache:
        return _cache["r"]
    if not os.path.exists(REF_SO):
        _cache["r"] = None
        return None
    L = C.CDLL(REF_SO)
    sigs = {
        "ref_contig_sum": (C.c_uint64, [u64p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32]),
        "ref_contig_matrix_mt": (C.c_uint64, [u64p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, u32p, C.c_uint32]),
        "ref_storm_sum": (C.c_uint64, [u32p, u64p, C.c_uint64, C.c_uint32]),
        "ref_storm_sum_timed": (C.c_uint64, [u32p, u64p, C.c_uint64, C.POINTER(C.c_double)]),
        "ref_storm_sum_mt": (C.c_uint64, [u32p, u64p, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)]),
        "ref_storm_square": (C.c_uint64, [u32p, u64p, C.c_uint64, u32p, u64p, C.c_uint64]),
        "ref_storm_matrix": (C.c_uint64, [u32p, u64p, C.c_uint64, u32p]),
        "ref_storm_layout": (C.c_uint32, [u32p, C.c_uint32, u32p, u8p, u32p]),
        "ref_vector16": (C.c_uint64, [u16p, u16p, C.c_uint32, C.c_uint32]),
        "ref_vector32": (C.c_uint64, [u32p, u32p, C.c_uint32, C.c_uint32, u32p]),
        "ref_bitmaps_scalar_list": (C.c_uint64, [u64p, u64p, u32p, u32p, C.c_uint32, C.c_uint32]),
        "ref_wrapper_diag": (C.c_uint64, [C.c_uint32, u64p, C.c_uint32, C.c_uint32]),
        "ref_allpairs_sum": (None, [u32p, u64p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, u64p]),
        "ref_allpairs_tiles": (C.c_uint64, [u32p, u64p, C.c_uint64, C.c_uint32, C.c_uint32, u32p]),
        "ref_oracle_intersect": (C.c_uint64, [u32p, C.c_uint64, u32p, C.c_uint64, C.c_uint32]),
        "ref_build_row": (None, [u32p, C.c_uint64, C.c_uint32, u32p, u32p, u64p, u64p, u64p, u32p, u64p, u32p]),
        "ref_select_pairing": (C.c_uint32, [u32p, u32p, dblp]),
        "ref_all_cells": (C.c_uint32, [u32p, C.c_uint64, u32p, C.c_uint64, C.c_uint32, u64p]),
    }
    for k, (r, a) in sigs.items():
        f = getattr(L, k)
        f.restype, f.argtypes = r, a
    _cache["r"] = L
    return L


# --- convenience wrappers over the oracle ---------------------------------
def contig_matrix(words: np.ndarray, r0: int = 0, r1: int | None = None, want_matrix: bool = True):
    words = np.ascontiguousarray(words, dtype=np.uint64)
    n, w = words.shape
    r1 = n if r1 is None else r1
    out = np.zeros(max(1, n * (n + 1) // 2), dtype=np.uint32) if want_matrix else None
    s = oracle().oracle_contig_matrix(_p(words, u64p), n, w, r0, r1, _p(out, u32p) if out is not None else None)
    return (out[: n * (n + 1) // 2] if out is not None else None), int(s)


def sets_matrix(vals: np.ndarray, offs: np.ndarray):
    vals = np.ascontiguousarray(vals, dtype=np.uint32)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    n = len(offs) - 1
    out = np.zeros(max(1, n * (n + 1) // 2), dtype=np.uint32)
    s = oracle().oracle_sets_matrix(_p(vals, u32p), _p(offs, u64p), n, 0, n, _p(out, u32p))
    return out[: n * (n + 1) // 2], int(s)


def storm_matrix(vals: np.ndarray, offs: np.ndarray):
    """STORM_t counts chunk by chunk as the reference counts them (rows as
    handed to STORM_add): packed triangle incl. the diagonal, sum over i < j."""
    vals = np.ascontiguousarray(vals, dtype=np.uint32)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    n = len(offs) - 1
    out = np.zeros(max(1, n * (n + 1) // 2), dtype=np.uint32)
    s = oracle().oracle_storm_matrix(_p(vals, u32p), _p(offs, u64p), n, _p(out, u32p))
    return out[: n * (n + 1) // 2], int(s)


def and_popcount(a: np.ndarray, b: np.ndarray) -> int:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    return int(oracle().oracle_and_popcount(_p(a, u64p), _p(b, u64p), a.size))


def contig_row(words: np.ndarray, i: int) -> np.ndarray:
    """|Xi & Xj| for j in [i, n) (one strip of the packed triangle)."""
    words = np.ascontiguousarray(words, dtype=np.uint64)
    n, w = words.shape
    out = np.zeros(n - i, dtype=np.uint32)
    oracle().oracle_contig_row(_p(words, u64p), n, w, i, _p(out, u32p))
    return out


def row_popcounts(words: np.ndarray) -> np.ndarray:
    words = np.ascontiguousarray(words, dtype=np.uint64)
    n, w = words.shape
    out = np.zeros(n, dtype=np.uint32)
    oracle().oracle_row_popcounts(_p(words, u64p), n, w, _p(out, u32p))
    return out


def threshold_pairs(tri: np.ndarray, n: int, t: float):
    """The thresholded contract on a packed triangle (i <= j, diagonal = |Xi|):
    pairs i < j with v > 0 and v / (|Xi| + |Xj| - v) >= t in double precision
    (bench/bench_threshold.cpp:129-132). Returns (i, j, v) sorted by (i, j)."""
    iu = np.triu_indices(n)
    v = tri.astype(np.float64)
    diag = v[iu[0] == iu[1]]
    off = iu[0] != iu[1]
    i, j, c = iu[0][off], iu[1][off], v[off]
    u = diag[i] + diag[j] - c
    with np.errstate(divide="ignore", invalid="ignore"):
        ok = (c > 0) & (u > 0) & (c / np.where(u > 0, u, 1.0) >= t)
    return i[ok].astype(np.uint32), j[ok].astype(np.uint32), c[ok].astype(np.uint32)


class SetStrip:
    """Whole rows of the per-pair matrix for up to 8 query rows, counted
    against row batches streamed through count() (several host threads at
    once, one batch each): oracle_strip_* of oracle/storm_oracle.c."""

    def __init__(self, queries, universe: int):
        L = oracle()
        qv = np.ascontiguousarray(np.concatenate(queries) if len(queries) else np.zeros(0), dtype=np.uint32)
        qo = np.zeros(len(queries) + 1, np.uint64)
        qo[1:] = np.cumsum([len(q) for q in queries])
        self.nq = len(queries)
        self.h = L.oracle_strip_new(_p(qv, u32p), _p(qo, u64p), self.nq, universe)
        if not self.h:
            raise ValueError("oracle_strip_new: 1..8 query rows")

    def count(self, vals: np.ndarray, offs: np.ndarray, threads: int = 1) -> np.ndarray:
        """[n_rows, nq] counts for the CSR batch (vals u32, offs u64 from 0)."""
        import concurrent.futures as cf
        vals = np.ascontiguousarray(vals, dtype=np.uint32)
        offs = np.ascontiguousarray(offs, dtype=np.uint64)
        n = len(offs) - 1
        out = np.zeros((n, self.nq), np.uint32)
        L = oracle()
        cuts = np.linspace(0, n, max(1, min(threads, n)) + 1).astype(np.int64)

        def part(a, b):
            if b > a:
                L.oracle_strip_count(self.h, _p(vals, u32p), offs[a:].ctypes.data_as(u64p), b - a,
                                     out[a:].ctypes.data_as(u32p))

        with cf.ThreadPoolExecutor(max_workers=len(cuts) - 1) as ex:
            list(ex.map(lambda k: part(int(cuts[k]), int(cuts[k + 1])), range(len(cuts) - 1)))
        return out

    def close(self):
        if self.h:
            oracle().oracle_strip_free(self.h)
            self.h = None


class BitmapStrip:
    """Whole rows of the per-pair matrix for query rows given as packed
    bitmaps, counted against bitmap row batches (oracle_contig_strip)."""

    def __init__(self, qwords: np.ndarray):
        self.q = np.ascontiguousarray(qwords, dtype=np.uint64)
        self.nq = self.q.shape[0]

    def count(self, words: np.ndarray, offs=None, threads: int = 1) -> np.ndarray:
        import concurrent.futures as cf
        words = np.ascontiguousarray(words, dtype=np.uint64)
        n, nw = words.shape
        out = np.zeros((n, self.nq), np.uint32)
        L = oracle()
        cuts = np.linspace(0, n, max(1, min(threads, n)) + 1).astype(np.int64)

        def part(a, b):
            if b > a:
                L.oracle_contig_strip(_p(self.q, u64p), self.nq, words[a:].ctypes.data_as(u64p), b - a, nw,
                                      out[a:].ctypes.data_as(u32p))

        with cf.ThreadPoolExecutor(max_workers=len(cuts) - 1) as ex:
            list(ex.map(lambda k: part(int(cuts[k]), int(cuts[k + 1])), range(len(cuts) - 1)))
        return out

    def close(self):
        pass
