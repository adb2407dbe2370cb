"""Python mirror of the storm.h interface, over libstorm_b200.so (ctypes).

The shipped product is the C-ABI library; this module is the host-side view
that tests and bench.py use.  Class and method names follow the reference's
C entry points (storm.h:214-231):

    StormContig(vector_length)      STORM_contig_new / add / pairw_* / clear
    Storm()                         STORM_new / add / pairw_* / clear / square

Every all-pairs method runs on the GPU through the library.  There is no
host fallback: if libstorm_b200.so is missing this module fails to import,
and on a machine without an sm_100 device the calls raise StormError
(STORM_B200_ECUDA).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libstorm_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is not built; run `python stormbitmaps-internal_b200/build.py` "
        "(or __graft_entry__.build())"
    )

_lib = C.CDLL(LIB_PATH)

u8p = C.POINTER(C.c_uint8)
u16p = C.POINTER(C.c_uint16)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
TILE_CB = C.CFUNCTYPE(None, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, u32p, C.c_void_p)

KERNEL_AUTO, KERNEL_POPC, KERNEL_MMA, KERNEL_MMA_SS, KERNEL_MMA_DB, KERNEL_MMA_2CTA = 0, 1, 2, 3, 4, 5
SCHED_AUTO, SCHED_TILES, SCHED_STREAM_K = 0, 1, 2
OK, ENULL, EVALUES, EARG, ENOMEM, ECUDA, ETIMEOUT, ESIZE, ELIMIT = 0, -1, -2, -3, -4, -5, -6, -7, -8


def _sig(name, res, args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args
    return f


# --- declarations (include/storm.h, include/storm_b200.h) ----------------
_sig("STORM_b200_strerror", C.c_char_p, [C.c_int])
_sig("STORM_b200_last_status", C.c_int, [])
_sig("STORM_b200_wait_selftest", C.c_int, [C.c_uint32])
_sig("STORM_intersect_vector16_cardinality", C.c_uint64, [u16p, u16p, C.c_uint32, C.c_uint32])
_sig("STORM_intersect_vector32_unsafe", C.c_uint64, [u32p, u32p, C.c_uint32, C.c_uint32, u32p])
_sig("STORM_intersect_bitmaps_scalar_list", C.c_uint64, [u64p, u64p, u32p, u32p, C.c_uint32, C.c_uint32])
_sig("STORM_wrapper_diag", C.c_uint64, [C.c_uint32, u64p, C.c_uint32, C.c_void_p])
_sig("STORM_wrapper_diag_blocked", C.c_uint64, [C.c_uint32, u64p, C.c_uint32, C.c_void_p, C.c_uint32])
_sig("STORM_wrapper_square", C.c_uint64, [C.c_uint32, u64p, C.c_uint32, u64p, C.c_uint32, C.c_void_p])
_sig("STORM_contig_new", C.c_void_p, [C.c_size_t])
_sig("STORM_contig_free", None, [C.c_void_p])
_sig("STORM_contig_add", C.c_int, [C.c_void_p, u32p, C.c_uint32])
_sig("STORM_contig_clear", C.c_int, [C.c_void_p])
_sig("STORM_contig_pairw_intersect_cardinality", C.c_uint64, [C.c_void_p])
_sig("STORM_contig_pairw_intersect_cardinality_blocked", C.c_uint64, [C.c_void_p, C.c_uint32])
_sig("STORM_contig_pairw_intersect_cardinality_list", C.c_uint64, [C.c_void_p])
_sig("STORM_contig_pairw_intersect_cardinality_blocked_list", C.c_uint64, [C.c_void_p, C.c_uint32])
_sig("STORM_contig_add_bitmaps", C.c_int, [C.c_void_p, u64p, C.c_uint32, C.c_uint32])
_sig("STORM_contig_size", C.c_uint64, [C.c_void_p])
_sig("STORM_contig_set_kernel", C.c_int, [C.c_void_p, C.c_int])
_sig("STORM_contig_set_schedule", C.c_int, [C.c_void_p, C.c_int])
_sig("STORM_contig_autotune", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)])
_sig("STORM_autotune", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_double)])
_sig("STORM_rows_autotune", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)])
_sig("STORM_contig_pairw_threshold", C.c_int, [C.c_void_p, C.c_double, u32p, u32p, u32p, C.c_uint64,
                                               C.POINTER(C.c_uint64)])
_sig("STORM_load_stormbin", C.c_int64, [C.c_void_p, C.c_char_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32)])
_sig("STORM_rows_universe", C.c_uint32, [C.c_void_p])
_sig("STORM_load_stormpack", C.c_int64, [C.c_void_p, C.c_char_p, C.POINTER(C.c_uint32)])
_sig("STORM_rows_load_stormpack", C.c_int64, [C.c_char_p, C.POINTER(C.c_void_p)])
_sig("STORM_rows_load_stormbin", C.c_int64, [C.c_char_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p)])
_sig("STORM_pairw_threshold", C.c_int, [C.c_void_p, C.c_double, u32p, u32p, u32p, C.c_uint64,
                                        C.POINTER(C.c_uint64)])
_sig("STORM_contig_upload", C.c_int, [C.c_void_p])
_sig("STORM_contig_pairw_intersect_matrix", C.c_int, [C.c_void_p, u32p, C.c_uint64, u64p])
_sig("STORM_contig_pairw_intersect_matrix_from_host", C.c_int,
     [C.c_void_p, u64p, C.c_uint32, C.c_uint32, u32p, C.c_uint64, u64p])
_sig("STORM_contig_pairw_intersect_matrix_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, u64p])
_sig("STORM_contig_pairw_intersect_tiles", C.c_int, [C.c_void_p, C.c_uint32, TILE_CB, C.c_void_p])
_sig("STORM_contig_stream", C.c_void_p, [C.c_void_p])
_sig("STORM_contig_last_kernel_ms", C.c_float, [C.c_void_p])
_sig("STORM_contig_last_launches", C.c_uint32, [C.c_void_p])
_sig("STORM_contig_last_kernel", C.c_int, [C.c_void_p])
_sig("STORM_new", C.c_void_p, [])
_sig("STORM_free", None, [C.c_void_p])
_sig("STORM_add", C.c_int, [C.c_void_p, u32p, C.c_uint32])
_sig("STORM_clear", C.c_int, [C.c_void_p])
_sig("STORM_add_rows", C.c_int64, [C.c_void_p, u32p, u64p, C.c_uint64])
_sig("STORM_add_bitmap_rows", C.c_int64, [C.c_void_p, u64p, C.c_uint64, C.c_uint64])
_sig("STORM_pairw_intersect_matrix_device", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, u64p])
_sig("STORM_pairw_intersect_cardinality", C.c_uint64, [C.c_void_p])
_sig("STORM_pairw_intersect_cardinality_blocked", C.c_uint64, [C.c_void_p, C.c_uint32])
_sig("STORM_intersect_cardinality_square", C.c_uint64, [C.c_void_p, C.c_void_p])
_sig("STORM_serialized_size", C.c_uint64, [C.c_void_p])
_sig("STORM_upload", C.c_int, [C.c_void_p])
_sig("STORM_pairw_intersect_matrix", C.c_int, [C.c_void_p, u32p, C.c_uint64, u64p])
_sig("STORM_pairw_intersect_tiles", C.c_int, [C.c_void_p, C.c_uint32, TILE_CB, C.c_void_p])
_sig("STORM_last_kernel_ms", C.c_float, [C.c_void_p])
_sig("STORM_set_dense_block", C.c_int, [C.c_void_p, C.c_double, C.c_uint64])
_sig("STORM_last_dense_rows", C.c_uint64, [C.c_void_p])
_sig("STORM_last_dense_panels", C.c_uint64, [C.c_void_p])
_sig("STORM_set_sparse_postings", C.c_int, [C.c_void_p, C.c_int])
_sig("STORM_last_postings_rows", C.c_uint64, [C.c_void_p])
_sig("STORM_set_panel", C.c_int, [C.c_void_p, C.c_int])
_sig("STORM_last_engine_ms", C.c_int, [C.c_void_p, C.POINTER(C.c_double)])
_sig("STORM_last_plan_ms", C.c_double, [C.c_void_p])
_sig("STORM_last_postings_form", C.c_int, [C.c_void_p])
_sig("STORM_last_transfer_ms", C.c_int, [C.c_void_p, C.POINTER(C.c_double)])
_sig("STORM_calibrate", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)])
_sig("STORM_reset_cost_model", C.c_int, [C.c_void_p])
_sig("STORM_last_panel_rows", C.c_uint64, [C.c_void_p])


class StormError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        msg = _lib.STORM_b200_strerror(code).decode()
        super().__init__(f"{where}: {msg} ({code})" if where else f"{msg} ({code})")


def lib():
    """The loaded ctypes library (for calling entry points directly)."""
    return _lib


def _check(rc: int, where: str) -> int:
    if rc < 0:
        raise StormError(rc, where)
    return rc


def _check_status(where: str):
    s = _lib.STORM_b200_last_status()
    if s < 0:
        raise StormError(s, where)


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _threshold(fn, h, jaccard_min, cap):
    """(i, j, counts, found) of a thresholded call; raises on errors other
    than a full output (STORM_B200_ESIZE, when found > cap)."""
    oi = np.zeros(max(1, cap), np.uint32)
    oj = np.zeros(max(1, cap), np.uint32)
    oc = np.zeros(max(1, cap), np.uint32)
    found = C.c_uint64(0)
    rc = fn(h, float(jaccard_min), _p(oi, u32p), _p(oj, u32p), _p(oc, u32p), cap, C.byref(found))
    if rc < 0 and rc != ESIZE:
        raise StormError(rc, "thresholded all-pairs")
    m = min(int(found.value), cap)
    return oi[:m], oj[:m], oc[:m], int(found.value)


def tri_size(n: int) -> int:
    return n * (n + 1) // 2


def tri_index(n: int, i, j):
    """Packed upper-triangle index of (i, j), i <= j (storm_b200.h)."""
    i = np.asarray(i, dtype=np.uint64)
    j = np.asarray(j, dtype=np.uint64)
    n = np.uint64(n)
    return i * n - (i * (i - np.uint64(1))) // np.uint64(2) * (i > 0) + (j - i)


def unpack_triangle(tri: np.ndarray, n: int) -> np.ndarray:
    """Dense symmetric n x n matrix from a packed upper triangle."""
    m = np.zeros((n, n), dtype=tri.dtype)
    iu = np.triu_indices(n)
    m[iu] = tri
    m.T[iu] = tri
    return m


def _u32(values) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.uint32))


# --- single-pair kernels (storm.h:56-61) ---------------------------------
def intersect_vector16(a, b) -> int:
    a = np.ascontiguousarray(a, dtype=np.uint16)
    b = np.ascontiguousarray(b, dtype=np.uint16)
    r = _lib.STORM_intersect_vector16_cardinality(_p(a, u16p), _p(b, u16p), len(a), len(b))
    _check_status("STORM_intersect_vector16_cardinality")
    return int(r)


def intersect_vector32(a, b):
    """Matched index pairs of two sorted u32 arrays (STORM_intersect_vector32_unsafe)."""
    a, b = _u32(a), _u32(b)
    out = np.zeros(2 * max(1, min(len(a), len(b))), dtype=np.uint32)
    k = _lib.STORM_intersect_vector32_unsafe(_p(a, u32p), _p(b, u32p), len(a), len(b), _p(out, u32p))
    _check_status("STORM_intersect_vector32_unsafe")
    return out[: int(k)].reshape(-1, 2)


def intersect_bitmaps_scalar_list(b1, b2, l1, l2) -> int:
    b1 = np.ascontiguousarray(b1, dtype=np.uint64)
    b2 = np.ascontiguousarray(b2, dtype=np.uint64)
    l1, l2 = _u32(l1), _u32(l2)
    r = _lib.STORM_intersect_bitmaps_scalar_list(_p(b1, u64p), _p(b2, u64p), _p(l1, u32p), _p(l2, u32p),
                                                 len(l1), len(l2))
    _check_status("STORM_intersect_bitmaps_scalar_list")
    return int(r)


def wrapper_diag(vals: np.ndarray, blocked: int = 0) -> int:
    vals = np.ascontiguousarray(vals, dtype=np.uint64)
    n, w = vals.shape
    if blocked:
        r = _lib.STORM_wrapper_diag_blocked(n, _p(vals, u64p), w, None, blocked)
    else:
        r = _lib.STORM_wrapper_diag(n, _p(vals, u64p), w, None)
    _check_status("STORM_wrapper_diag")
    return int(r)


def wrapper_square(v1: np.ndarray, v2: np.ndarray) -> int:
    v1 = np.ascontiguousarray(v1, dtype=np.uint64)
    v2 = np.ascontiguousarray(v2, dtype=np.uint64)
    r = _lib.STORM_wrapper_square(v1.shape[0], _p(v1, u64p), v2.shape[0], _p(v2, u64p), v1.shape[1], None)
    _check_status("STORM_wrapper_square")
    return int(r)


class _TileCollector:
    def __init__(self, n: int, tile: int):
        self.n, self.tile = n, tile
        self.out = np.zeros(tri_size(n), dtype=np.uint32)
        self.calls = []

    def __call__(self, i0, j0, nr, nc, counts, ctx):
        buf = np.ctypeslib.as_array(counts, shape=(self.tile * self.tile,)).reshape(self.tile, self.tile)
        self.calls.append((i0, j0, nr, nc, int(buf[:nr, :nc].astype(np.uint64).sum())))
        for a in range(nr):
            i = i0 + a
            js = np.arange(j0, j0 + nc, dtype=np.uint64)
            keep = js > i
            if keep.any():
                self.out[tri_index(self.n, i, js[keep])] = buf[a, :nc][keep]


class StormContig:
    """STORM_contiguous_t (storm.h:224-231)."""

    def __init__(self, vector_length: int):
        self.h = _lib.STORM_contig_new(vector_length)
        if not self.h:
            raise StormError(ENOMEM, "STORM_contig_new")
        self.vector_length = vector_length
        self.n_words = (vector_length + 63) // 64

    def close(self):
        if self.h:
            _lib.STORM_contig_free(self.h)
            self.h = None

    __del__ = close

    def add(self, values) -> int:
        v = _u32(values)
        return _check(_lib.STORM_contig_add(self.h, _p(v, u32p), len(v)), "STORM_contig_add")

    def add_bitmaps(self, words: np.ndarray) -> int:
        words = np.ascontiguousarray(words, dtype=np.uint64)
        return _check(_lib.STORM_contig_add_bitmaps(self.h, _p(words, u64p), words.shape[0], words.shape[1]),
                      "STORM_contig_add_bitmaps")

    def clear(self):
        return _lib.STORM_contig_clear(self.h)

    def __len__(self):
        return int(_lib.STORM_contig_size(self.h))

    def set_kernel(self, kernel: int):
        _check(_lib.STORM_contig_set_kernel(self.h, kernel), "STORM_contig_set_kernel")

    def threshold(self, jaccard_min: float, cap: int = 1 << 20):
        return _threshold(_lib.STORM_contig_pairw_threshold, self.h, jaccard_min, cap)

    def autotune(self):
        """Time every exact kernel/schedule on these rows and keep the fastest:
        (kernel, schedule, times_ms[7])."""
        k, sc, t = C.c_int(0), C.c_int(0), (C.c_double * 7)()
        _check(_lib.STORM_contig_autotune(self.h, C.byref(k), C.byref(sc), t), "STORM_contig_autotune")
        return k.value, sc.value, list(t)

    def set_schedule(self, schedule: int):
        _check(_lib.STORM_contig_set_schedule(self.h, schedule), "STORM_contig_set_schedule")

    def upload(self):
        _check(_lib.STORM_contig_upload(self.h), "STORM_contig_upload")

    def pairw_intersect_cardinality(self, blocked: int = 0) -> int:
        if blocked:
            r = _lib.STORM_contig_pairw_intersect_cardinality_blocked(self.h, blocked)
        else:
            r = _lib.STORM_contig_pairw_intersect_cardinality(self.h)
        _check_status("STORM_contig_pairw_intersect_cardinality")
        return int(r)

    def matrix(self, out: np.ndarray | None = None):
        n = len(self)
        if out is None:
            out = np.zeros(max(1, tri_size(n)), dtype=np.uint32)
        s = C.c_uint64(0)
        _check(_lib.STORM_contig_pairw_intersect_matrix(self.h, _p(out, u32p), out.size, C.byref(s)),
               "STORM_contig_pairw_intersect_matrix")
        return out[: tri_size(n)], int(s.value)

    def matrix_from_host(self, words: np.ndarray, out: np.ndarray | None = None):
        """Replace the rows with `words` (n x ceil(len/64) u64, host) and return
        (packed triangle, sum) in one overlapped call."""
        words = np.ascontiguousarray(words, dtype=np.uint64)
        n = words.shape[0]
        if out is None:
            out = np.zeros(max(1, tri_size(n)), dtype=np.uint32)
        s = C.c_uint64(0)
        _check(_lib.STORM_contig_pairw_intersect_matrix_from_host(self.h, _p(words, u64p), n, words.shape[1],
                                                                  _p(out, u32p), out.size, C.byref(s)),
               "STORM_contig_pairw_intersect_matrix_from_host")
        return out[: tri_size(n)], int(s.value)

    def matrix_device(self, d_out_ptr: int, out_len: int) -> int:
        s = C.c_uint64(0)
        _check(_lib.STORM_contig_pairw_intersect_matrix_device(self.h, C.c_void_p(d_out_ptr), out_len, C.byref(s)),
               "STORM_contig_pairw_intersect_matrix_device")
        return int(s.value)

    def tiles(self, tile: int = 64):
        col = _TileCollector(len(self), tile)
        cb = TILE_CB(col)
        _check(_lib.STORM_contig_pairw_intersect_tiles(self.h, tile, cb, None), "STORM_contig_pairw_intersect_tiles")
        return col

    def stream(self) -> int:
        return _lib.STORM_contig_stream(self.h) or 0

    def last_kernel_ms(self) -> float:
        return float(_lib.STORM_contig_last_kernel_ms(self.h))

    def last_launches(self) -> int:
        return int(_lib.STORM_contig_last_launches(self.h))

    def last_kernel(self) -> int:
        return int(_lib.STORM_contig_last_kernel(self.h))


class Storm:
    """STORM_t (storm.h:214-221): rows split into 65536-bit chunks."""

    def __init__(self):
        self.h = _lib.STORM_new()
        if not self.h:
            raise StormError(ENOMEM, "STORM_new")
        self.n = 0

    def close(self):
        if self.h:
            _lib.STORM_free(self.h)
            self.h = None

    __del__ = close

    def add(self, values) -> int:
        v = _u32(values)
        rc = _lib.STORM_add(self.h, _p(v, u32p), len(v))
        _check(rc, "STORM_add")
        self.n += 1
        return rc

    def add_rows(self, vals, offs) -> int:
        """Rows in CSR form (u32 values, u64 offsets of n + 1 entries) through
        STORM_add_rows: the same rows as one add() per row."""
        v = np.ascontiguousarray(vals, dtype=np.uint32)
        o = np.ascontiguousarray(offs, dtype=np.uint64)
        rc = int(_lib.STORM_add_rows(self.h, _p(v, u32p), _p(o, u64p), len(o) - 1))
        _check(rc, "STORM_add_rows")
        self.n += rc
        return rc

    def add_bitmap_rows(self, words: np.ndarray) -> int:
        """Rows as packed bitmaps ([n, words_per_row] u64, host memory) through
        STORM_add_bitmap_rows: the same rows as add() of each row's positions."""
        w = np.ascontiguousarray(words, dtype=np.uint64)
        rc = int(_lib.STORM_add_bitmap_rows(self.h, _p(w, u64p), w.shape[0], w.shape[1]))
        _check(rc, "STORM_add_bitmap_rows")
        self.n += rc
        return rc

    def matrix_device(self, d_out_ptr: int, out_len: int) -> int:
        """Per-pair counts into a device buffer (0 = sum only); returns the sum."""
        s = C.c_uint64(0)
        _check(_lib.STORM_pairw_intersect_matrix_device(self.h, C.c_void_p(d_out_ptr or None), out_len,
                                                        C.byref(s)), "STORM_pairw_intersect_matrix_device")
        return int(s.value)

    def clear(self):
        self.n = 0
        return _lib.STORM_clear(self.h)

    def __len__(self):
        return self.n

    def upload(self):
        _check(_lib.STORM_upload(self.h), "STORM_upload")

    def pairw_intersect_cardinality(self, blocked: int = 0) -> int:
        if blocked:
            r = _lib.STORM_pairw_intersect_cardinality_blocked(self.h, blocked)
        else:
            r = _lib.STORM_pairw_intersect_cardinality(self.h)
        _check_status("STORM_pairw_intersect_cardinality")
        return int(r)

    def square(self, other: "Storm") -> int:
        r = _lib.STORM_intersect_cardinality_square(self.h, other.h)
        _check_status("STORM_intersect_cardinality_square")
        return int(r)

    def serialized_size(self) -> int:
        return int(_lib.STORM_serialized_size(self.h))

    def matrix(self, out: np.ndarray | None = None):
        if out is None:
            out = np.zeros(max(1, tri_size(self.n)), dtype=np.uint32)
        s = C.c_uint64(0)
        _check(_lib.STORM_pairw_intersect_matrix(self.h, _p(out, u32p), out.size, C.byref(s)),
               "STORM_pairw_intersect_matrix")
        return out[: tri_size(self.n)], int(s.value)

    def tiles(self, tile: int = 64):
        col = _TileCollector(self.n, tile)
        cb = TILE_CB(col)
        _check(_lib.STORM_pairw_intersect_tiles(self.h, tile, cb, None), "STORM_pairw_intersect_tiles")
        return col

    def last_kernel_ms(self) -> float:
        return float(_lib.STORM_last_kernel_ms(self.h))

    def set_dense_block(self, min_density: float, budget_bytes: int = 0):
        _check(_lib.STORM_set_dense_block(self.h, float(min_density), int(budget_bytes)), "STORM_set_dense_block")

    def threshold(self, jaccard_min: float, cap: int = 1 << 20):
        return _threshold(_lib.STORM_pairw_threshold, self.h, jaccard_min, cap)

    def load_stormbin(self, path: str, max_rows: int = 0, stride: int = 1):
        """Append a STORMBIN corpus file's rows; returns (rows added, n_bits)."""
        nb = C.c_uint32(0)
        r = _lib.STORM_load_stormbin(self.h, os.fsencode(path), max_rows, stride, C.byref(nb))
        _check(int(r), "STORM_load_stormbin")
        self.n += int(r)
        return int(r), int(nb.value)

    def load_stormpack(self, path: str):
        """Append a STORMPACK file's rows; returns (rows added, n_bits)."""
        nb = C.c_uint32(0)
        r = _lib.STORM_load_stormpack(self.h, os.fsencode(path), C.byref(nb))
        _check(int(r), "STORM_load_stormpack")
        self.n += int(r)
        return int(r), int(nb.value)

    def autotune(self):
        """(min_density, postings_mode, times_ms[4]) kept for later calls."""
        dm, pm, t = C.c_double(0), C.c_int(0), (C.c_double * 4)()
        _check(_lib.STORM_autotune(self.h, C.byref(dm), C.byref(pm), t), "STORM_autotune")
        return dm.value, pm.value, list(t)

    def set_sparse_postings(self, mode: int):
        _check(_lib.STORM_set_sparse_postings(self.h, int(mode)), "STORM_set_sparse_postings")

    def last_postings_rows(self) -> int:
        return int(_lib.STORM_last_postings_rows(self.h))

    def last_engine_ms(self):
        """{engine: (device ms, predicted ms, work)} of the last per-pair call
        (work: int8 ops for the tensor cores, pairs for the chunk kernel,
        bytes for the panel and the postings)."""
        o = (C.c_double * 12)()
        _check(_lib.STORM_last_engine_ms(self.h, o), "STORM_last_engine_ms")
        return {k: (o[i], o[4 + i], o[8 + i]) for i, k in enumerate(("tensor", "chunk", "panel", "postings"))}

    def last_postings_form(self) -> int:
        """Per-pair form of the last call's postings: 0 list by list, 1 row
        sweep, 2 run sweep, -1 none."""
        return int(_lib.STORM_last_postings_form(self.h))

    def last_transfer_ms(self) -> dict:
        """Host-side transfers of the last all-pairs call: packing and upload
        of the rows (ms, payload bytes; 0 when they were on the device), and
        the copy of the triangle into host memory (ms, bytes)."""
        o = (C.c_double * 4)()
        _check(_lib.STORM_last_transfer_ms(self.h, o), "STORM_last_transfer_ms")
        return {"upload_ms": o[0], "upload_bytes": o[1], "copy_back_ms": o[2], "copy_back_bytes": o[3]}

    def last_plan_ms(self) -> float:
        """Device time of the last per-pair call spent before its engines on
        planning (host), the row order's upload and clearing the output."""
        return float(_lib.STORM_last_plan_ms(self.h))

    def calibrate(self, sample_rows: int = 0):
        """GPU calibration of the planner: (tensor, panel, postings) scales and sample rows."""
        o = (C.c_double * 4)()
        _check(_lib.STORM_calibrate(self.h, sample_rows, o), "STORM_calibrate")
        return list(o)

    def reset_cost_model(self):
        _check(_lib.STORM_reset_cost_model(self.h), "STORM_reset_cost_model")

    def set_panel(self, mode: int):
        _check(_lib.STORM_set_panel(self.h, int(mode)), "STORM_set_panel")

    def last_panel_rows(self) -> int:
        return int(_lib.STORM_last_panel_rows(self.h))

    def last_dense(self):
        """(rows, panels) the last all-pairs call gave to the tensor-core block."""
        return int(_lib.STORM_last_dense_rows(self.h)), int(_lib.STORM_last_dense_panels(self.h))


# --- kernel layer (include/storm_rows.h) ---------------------------------
POLICY_ALLBITMAP, POLICY_PERPAIR, POLICY_PERTILE, POLICY_ORACLE, POLICY_FIXED, POLICY_PROBE, POLICY_REFINE, \
    POLICY_LEARNED = range(8)
REPR_RUN_START, REPR_RUN_END, REPR_EWAH, REPR_MARKERS, REPR_BITMAP, REPR_RANK, REPR_OCC, REPR_COMPLEMENT = range(8)
POLICY_NAMES = ["all-bitmap", "per-pair", "per-tile", "oracle", "fixed-cell", "probe", "refine", "learned"]
PAIRINGS = ["BB", "BS", "BR", "BW", "SS", "SR", "SW", "RR", "RW", "WW", "EMPTY", "CB"]
(P_BB, P_BS, P_BR, P_BW, P_SS, P_SR, P_SW, P_RR, P_RW, P_WW, P_EMPTY, P_CB) = range(12)
EXEC_PER_TILE, EXEC_BATCHED = 0, 1


class AllPairsStats(C.Structure):
    _fields_ = [("sum", C.c_uint64), ("pairs", C.c_uint64), ("decisions", C.c_uint64), ("skipped", C.c_uint64),
                ("ns_total", C.c_double), ("ns_selection", C.c_double), ("cell_pairs", C.c_uint64 * 12),
                ("launches", C.c_uint32)]

    def as_dict(self):
        return {"sum": self.sum, "pairs": self.pairs, "decisions": self.decisions, "skipped": self.skipped,
                "ns_total": self.ns_total, "ns_selection": self.ns_selection,
                "cell_pairs": {PAIRINGS[k]: int(self.cell_pairs[k]) for k in range(12) if self.cell_pairs[k]},
                "launches": self.launches}


_sig("STORM_rows_new", C.c_void_p, [C.c_uint32])
_sig("STORM_rows_free", None, [C.c_void_p])
_sig("STORM_rows_add", C.c_int, [C.c_void_p, u32p, C.c_uint32])
_sig("STORM_rows_clear", C.c_int, [C.c_void_p])
_sig("STORM_rows_size", C.c_uint64, [C.c_void_p])
_sig("STORM_rows_set_bitmap_budget", C.c_int, [C.c_void_p, C.c_uint64])
_sig("STORM_rows_upload", C.c_int, [C.c_void_p])
_sig("STORM_rows_set_dense_block", C.c_int, [C.c_void_p, C.c_double])
_sig("STORM_rows_meta", C.c_int, [C.c_void_p, C.c_uint64, u32p])
_sig("STORM_rows_repr", C.c_int64, [C.c_void_p, C.c_uint64, C.c_int, C.c_void_p, C.c_uint64])
_sig("STORM_rows_allpairs_sum", C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_int, C.c_int, C.POINTER(AllPairsStats)])
_sig("STORM_rows_allpairs_matrix", C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_int, C.c_int, u32p, C.c_uint64,
                                             C.POINTER(AllPairsStats)])
_sig("STORM_rows_allpairs_tiles", C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_int, TILE_CB, C.c_void_p,
                                            C.POINTER(AllPairsStats)])
_sig("STORM_select_pairing", C.c_int, [u32p, u32p, C.POINTER(C.c_double)])
_sig("STORM_predict", C.c_double, [C.c_int, u32p, u32p])
_sig("STORM_rows_cell", C.c_int64, [C.c_void_p, C.c_int, C.c_uint64, C.c_uint64])
_sig("STORM_rows_train_selector", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                            C.POINTER(C.c_double)])
_sig("STORM_rows_reset_selector", C.c_int, [C.c_void_p])
_sig("STORM_rows_last_training", C.c_int, [C.c_void_p, C.POINTER(C.c_double)])
_sig("STORM_rows_calibrate", C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(C.c_double)])
_sig("STORM_rows_cost_model", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int])
_sig("STORM_rows_selector_params", C.c_int64, [C.c_void_p, C.POINTER(C.c_float), C.c_uint64, C.c_int])
_sig("STORM_mlp_forward_backward", C.c_int, [C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_uint32,
                                             C.POINTER(C.c_float), C.POINTER(C.c_int32), C.c_uint32,
                                             C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)])


def select_pairing(meta_a, meta_b):
    a = np.ascontiguousarray(meta_a[:8], dtype=np.uint32)
    b = np.ascontiguousarray(meta_b[:8], dtype=np.uint32)
    pred = C.c_double(0)
    return int(_lib.STORM_select_pairing(_p(a, u32p), _p(b, u32p), C.byref(pred))), float(pred.value)


def predict(pairing, meta_a, meta_b):
    a = np.ascontiguousarray(meta_a[:8], dtype=np.uint32)
    b = np.ascontiguousarray(meta_b[:8], dtype=np.uint32)
    return float(_lib.STORM_predict(pairing, _p(a, u32p), _p(b, u32p)))


def mlp_forward_backward(params, F, H, Cn, x, labels):
    params = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    B = labels.size
    logits = np.zeros((B, Cn), np.float32)
    loss = C.c_float(0)
    grads = np.zeros_like(params)
    fp = C.POINTER(C.c_float)
    _check(_lib.STORM_mlp_forward_backward(params.ctypes.data_as(fp), F, H, Cn, x.ctypes.data_as(fp),
                                           labels.ctypes.data_as(C.POINTER(C.c_int32)), B,
                                           logits.ctypes.data_as(fp), C.byref(loss), grads.ctypes.data_as(fp)),
           "STORM_mlp_forward_backward")
    return logits, float(loss.value), grads


class StormRows:
    """STORM_rows_t: the reference's kernel layer (kernels/storm_allpairs.h) on the GPU."""

    @classmethod
    def from_stormpack(cls, path: str) -> "StormRows":
        h = C.c_void_p(None)
        r = _lib.STORM_rows_load_stormpack(os.fsencode(path), C.byref(h))
        _check(int(r), "STORM_rows_load_stormpack")
        obj = cls.__new__(cls)
        obj.h = h.value
        obj.universe = int(_lib.STORM_rows_universe(obj.h))
        return obj

    @classmethod
    def from_stormbin(cls, path: str, max_rows: int = 0, stride: int = 1) -> "StormRows":
        h = C.c_void_p(None)
        r = _lib.STORM_rows_load_stormbin(os.fsencode(path), max_rows, stride, C.byref(h))
        _check(int(r), "STORM_rows_load_stormbin")
        obj = cls.__new__(cls)
        obj.h = h.value
        obj.universe = int(_lib.STORM_rows_universe(obj.h))
        return obj

    def __init__(self, universe: int):
        self.h = _lib.STORM_rows_new(universe)
        if not self.h:
            raise StormError(ENOMEM, "STORM_rows_new")
        self.universe = universe

    def close(self):
        if self.h:
            _lib.STORM_rows_free(self.h)
            self.h = None

    __del__ = close

    def add(self, positions) -> int:
        v = _u32(positions)
        return _check(_lib.STORM_rows_add(self.h, _p(v, u32p), len(v)), "STORM_rows_add")

    def clear(self):
        return _lib.STORM_rows_clear(self.h)

    def __len__(self):
        return int(_lib.STORM_rows_size(self.h))

    def set_bitmap_budget(self, nbytes: int):
        _check(_lib.STORM_rows_set_bitmap_budget(self.h, nbytes), "STORM_rows_set_bitmap_budget")

    def upload(self):
        _check(_lib.STORM_rows_upload(self.h), "STORM_rows_upload")

    def set_dense_block(self, min_density: float):
        _check(_lib.STORM_rows_set_dense_block(self.h, float(min_density)), "STORM_rows_set_dense_block")

    def autotune(self, policy, exec_=EXEC_BATCHED):
        """(tile, min_density, times_ms[16]) kept for later calls with tile 0."""
        bt, bd, t = C.c_uint32(0), C.c_double(0), (C.c_double * 16)()
        _check(_lib.STORM_rows_autotune(self.h, policy, exec_, C.byref(bt), C.byref(bd), t), "STORM_rows_autotune")
        return bt.value, bd.value, list(t)

    def meta(self, row: int) -> np.ndarray:
        m = np.zeros(9, dtype=np.uint32)
        _check(_lib.STORM_rows_meta(self.h, row, _p(m, u32p)), "STORM_rows_meta")
        return m

    def repr(self, row: int, kind: int) -> np.ndarray:
        """One stored form of one row (REPR_*), copied from the device;
        markers come as an (m, 2) array of (stream position, first word)."""
        n = _check(_lib.STORM_rows_repr(self.h, row, kind, None, 0), "STORM_rows_repr")
        dt = np.uint32 if kind in (REPR_RUN_START, REPR_RUN_END, REPR_COMPLEMENT) else \
            np.uint64 if kind != REPR_MARKERS else np.uint32
        out = np.zeros(n * (2 if kind == REPR_MARKERS else 1), dt)
        if n:
            _check(_lib.STORM_rows_repr(self.h, row, kind, out.ctypes.data, n), "STORM_rows_repr")
        return out.reshape(-1, 2) if kind == REPR_MARKERS else out

    def allpairs_sum(self, policy, tile=64, fixed_cell=P_BS, exec_=EXEC_BATCHED):
        st = AllPairsStats()
        _check(_lib.STORM_rows_allpairs_sum(self.h, policy, tile, fixed_cell, exec_, C.byref(st)),
               "STORM_rows_allpairs_sum")
        return int(st.sum), st.as_dict()

    def allpairs_matrix(self, policy, tile=64, fixed_cell=P_BS, exec_=EXEC_BATCHED):
        n = len(self)
        out = np.zeros(max(1, tri_size(n)), dtype=np.uint32)
        st = AllPairsStats()
        _check(_lib.STORM_rows_allpairs_matrix(self.h, policy, tile, fixed_cell, exec_, _p(out, u32p), out.size,
                                               C.byref(st)), "STORM_rows_allpairs_matrix")
        return out[: tri_size(n)], st.as_dict()

    def allpairs_tiles(self, policy, tile=64, exec_=EXEC_BATCHED):
        col = _TileCollector(len(self), tile)
        cb = TILE_CB(col)
        st = AllPairsStats()
        _check(_lib.STORM_rows_allpairs_tiles(self.h, policy, tile, exec_, cb, None, C.byref(st)),
               "STORM_rows_allpairs_tiles")
        return col, st.as_dict()

    def cell(self, pairing, a, b) -> int:
        return int(_lib.STORM_rows_cell(self.h, pairing, a, b))

    def train_selector(self, tile=64, samples=0, epochs=400, seed=1):
        stats = (C.c_double * 6)()
        _check(_lib.STORM_rows_train_selector(self.h, tile, samples, epochs, seed, stats), "STORM_rows_train_selector")
        keys = ["samples", "epochs", "loss", "train_accuracy", "regret_mlp", "regret_cost_model"]
        return dict(zip(keys, list(stats)))

    def last_training(self):
        out = (C.c_double * 9)()
        _check(_lib.STORM_rows_last_training(self.h, out), "STORM_rows_last_training")
        keys = ["regret_mlp", "regret_calibrated_model", "regret_default_model", "test_tiles", "train_tiles",
                "calibration_rms", "calibrated_fixed_cycles", "sampled_tiles", "kept_calibrated_model"]
        return dict(zip(keys, list(out)))

    def calibrate(self, tile=64, samples=0, seed=1):
        """GPU calibration of the cost model on these rows; returns the model
        (ns_per_unit[11], fixed, zone-map word, C x B per complement position,
        fixed cost per pair of each pairing [12], in SM cycles) and the fit's
        relative RMS error."""
        out = (C.c_double * 27)()
        _check(_lib.STORM_rows_calibrate(self.h, tile, samples, seed, out), "STORM_rows_calibrate")
        return list(out)[:26], float(out[26])

    def cost_model(self, set_to=None, reset=False):
        """Read the cost model ((model[26], calibrated)) or install one / the default."""
        if reset:
            _check(_lib.STORM_rows_cost_model(self.h, None, 1), "STORM_rows_cost_model")
            return None
        if set_to is not None:
            m = (C.c_double * 26)(*[float(x) for x in set_to])
            _check(_lib.STORM_rows_cost_model(self.h, m, 1), "STORM_rows_cost_model")
            return None
        m = (C.c_double * 26)()
        rc = _check(_lib.STORM_rows_cost_model(self.h, m, 0), "STORM_rows_cost_model")
        return list(m), bool(rc)

    def reset_selector(self):
        _check(_lib.STORM_rows_reset_selector(self.h), "STORM_rows_reset_selector")

    def selector_params(self, load: np.ndarray | None = None):
        n = int(_lib.STORM_rows_selector_params(self.h, None, 0, 0))
        fp = C.POINTER(C.c_float)
        if load is not None:
            p = np.ascontiguousarray(load, dtype=np.float32)
            _check(_lib.STORM_rows_selector_params(self.h, p.ctypes.data_as(fp), p.size, 1), "selector_params")
            return p
        p = np.zeros(n, dtype=np.float32)
        _check(_lib.STORM_rows_selector_params(self.h, p.ctypes.data_as(fp), n, 0), "selector_params")
        return p
