"""The C-ABI boundary without a GPU: the library loads, exports every entry
point include/*.h declares, keeps the reference's public struct layouts, and
its host-side argument checks return the reference's codes."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "stormbitmaps-internal_b200", "libstorm_b200.so")


def declared_functions():
    names = set()
    for h in os.listdir(INCLUDE):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"static inline[^{]*\{[^}]*\}", "", text)
        text = re.sub(r"^\s*#.*$", "", text, flags=re.M)
        for m in re.finditer(r"\b(STORM_[A-Za-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    # typedef'd function-pointer types and macros are not symbols
    return {n for n in names if n not in ("STORM_ALIGN",)}


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_entry_point():
    decl = declared_functions()
    assert len(decl) > 50
    missing = decl - exported_symbols()
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_library_loads_and_symbols_resolve(sb):
    L = sb.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def _layout_probe(include_dir, extra=""):
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "storm.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(STORM_bitmap_t), offsetof(STORM_bitmap_t, scalar),
         offsetof(STORM_bitmap_t, n_bits_set), offsetof(STORM_bitmap_t, m_scalar), offsetof(STORM_bitmap_t, id),
         sizeof(STORM_bitmap_cont_t), sizeof(STORM_t));
  return 0;
}
"""
    d = os.path.join(ROOT, "_build", "layout_probe")
    os.makedirs(d, exist_ok=True)
    cfile = os.path.join(d, "probe.c")
    exe = os.path.join(d, "probe" + extra)
    open(cfile, "w").write(src)
    subprocess.run(["gcc", "-std=c11", "-msse4.2", "-I", include_dir, cfile, "-o", exe], check=True,
                   capture_output=True)
    return subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()


def test_public_struct_layout_matches_reference():
    ours = _layout_probe(INCLUDE)
    assert ours[:2] == ["128", "64"]   # 64-byte aligned members: scalar at 64, struct 128 bytes
    ref = os.environ.get("STORM_REFERENCE", "/root/reference")
    if os.path.exists(os.path.join(ref, "storm.h")):
        assert _layout_probe(ref, "_ref") == ours


def test_host_argument_checks_follow_reference_codes(sb):
    L = sb.lib()
    # NULL handles (storm.cpp:1177-1179, 928, 1233).
    assert L.STORM_contig_add(None, None, 0) == -1
    assert L.STORM_contig_pairw_intersect_cardinality(None) == 0
    assert L.STORM_pairw_intersect_cardinality(None) == (1 << 64) - 1
    assert L.STORM_add(None, None, 0) == -1
    assert L.STORM_clear(None) == -1
    assert L.STORM_contig_clear(None) == -1
    c = L.STORM_contig_new(1000)
    try:
        assert L.STORM_contig_add(c, None, 3) == -2
        v = np.array([1, 2, 3], dtype=np.uint32)
        assert L.STORM_contig_add(c, v.ctypes.data_as(sb.u32p), 0) == 0   # n == 0: no row
        assert L.STORM_contig_size(c) == 0
        bad = np.array([5, 1000], dtype=np.uint32)                          # 1000 >= vector_length
        assert L.STORM_contig_add(c, bad.ctypes.data_as(sb.u32p), 2) == sb.EARG
        assert L.STORM_contig_add(c, v.ctypes.data_as(sb.u32p), 3) == 3
        assert L.STORM_contig_size(c) == 1
        # the one-call host form checks its arguments before any device work
        F = L.STORM_contig_pairw_intersect_matrix_from_host
        rows = np.zeros((4, 16), dtype=np.uint64)                           # ceil(1000 / 64) = 16 words
        out = np.zeros(10, dtype=np.uint32)
        u64 = rows.ctypes.data_as(sb.u64p)
        assert F(None, u64, 4, 16, out.ctypes.data_as(sb.u32p), 10, None) == sb.ENULL
        assert F(c, None, 4, 16, out.ctypes.data_as(sb.u32p), 10, None) == sb.EVALUES
        assert F(c, u64, 4, 16, None, 10, None) == sb.EVALUES
        assert F(c, u64, 4, 15, out.ctypes.data_as(sb.u32p), 10, None) == sb.EARG    # words per row
        assert F(c, u64, 4, 16, out.ctypes.data_as(sb.u32p), 9, None) == sb.ESIZE    # 4 rows: 10 counts
        rows[2, 15] = 1 << 40                                                         # bit 1000 >= length
        assert F(c, u64, 4, 16, out.ctypes.data_as(sb.u32p), 10, None) == sb.EARG
        assert L.STORM_contig_size(c) == 1                                            # untouched on a refusal
    finally:
        L.STORM_contig_free(c)


def test_storm_t_ingest_builds_reference_layout(sb, golden):
    """STORM_add fills the public structs exactly as the reference does
    (storm.cpp:737-803): chunk ids, list-vs-bitmap, n_bits_set."""
    import gen

    class Bitmap(C.Structure):
        _fields_ = [("data", C.c_void_p), ("_pad0", C.c_char * 56), ("scalar", C.c_void_p),
                    ("bits", C.c_uint32), ("n_bits_set", C.c_uint32), ("n_scalar_word", C.c_uint32),
                    ("n_missing", C.c_uint32), ("m_scalar", C.c_uint32), ("id", C.c_uint32),
                    ("_pad1", C.c_char * 32)]

    class Cont(C.Structure):
        _fields_ = [("bitmaps", C.POINTER(Bitmap)), ("block_ids", C.POINTER(C.c_uint32)),
                    ("n_bitmaps", C.c_uint32), ("m_bitmaps", C.c_uint32), ("prev", C.c_uint32)]

    class StormT(C.Structure):
        _fields_ = [("conts", C.POINTER(Cont)), ("n_conts", C.c_uint32), ("m_conts", C.c_uint32)]

    assert C.sizeof(Bitmap) == 128
    L = sb.lib()
    names = sorted({k.split("/")[1] for k in golden.files if k.startswith("storm/") and k.endswith("/layout")})
    for name in names:
        r = int(golden[f"storm/{name}/layout_row"][0])
        sets = gen.from_csr(golden[f"storm/{name}/vals"], golden[f"storm/{name}/offs"])
        v = np.ascontiguousarray(sets[r], dtype=np.uint32)
        h = L.STORM_new()
        try:
            assert L.STORM_add(h, v.ctypes.data_as(sb.u32p), v.size) == 1
            s = C.cast(h, C.POINTER(StormT)).contents
            assert s.n_conts == 1
            cont = s.conts[0]
            want = golden[f"storm/{name}/layout"]
            assert cont.n_bitmaps == want.shape[1], name
            for k in range(cont.n_bitmaps):
                b = cont.bitmaps[k]
                assert cont.block_ids[k] == want[0, k] and b.id == want[0, k]
                assert ((b.bits & 0x3FFFFFFF) != 0) == bool(want[1, k])
                assert b.n_bits_set == want[2, k]
        finally:
            L.STORM_free(h)
