"""The allocation-free entry point (STORM_contig_pairw_intersect_matrix_noalloc)
for callers that cannot allocate device memory when they need the counts:
through the C ABI, it must give exactly what the allocating entry point
gives, on two calls in a row, and leave free device memory unchanged.

Collected last on purpose, so that a run stopping at the first failure has
already run every other test.  It passes alone in a fresh process too."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry(sb):
    f = sb.lib().STORM_contig_pairw_intersect_matrix_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint64, C.c_void_p, C.c_uint64,
                  C.POINTER(C.c_uint64), C.c_void_p]
    return f


# (rows, bits, calls): short and long rows (rows over 2^17 bits take the
# epilogue without the shared-memory staging), and the largest row count the
# 32768-tile list holds (46080 rows, tiles at large block-row offsets).
@pytest.mark.parametrize("n,m,calls", [(300, 4096 + 64, 3), (1000, 65536, 3), (300, (1 << 17) + 512, 2),
                                       (46080, 512, 2)])
def test_noalloc_matches_allocating_entry_point_twice(sb, n, m, calls):
    import torch
    import bench
    dev = torch.device("cuda")
    w = (m + 63) // 64
    pitch = (w + 7) // 8 * 8
    n_pad = (n + 255) // 256 * 256
    rows = bench.bernoulli_rows_gpu(n, m, (0.05, 0.5), 1234 + n, dev)
    padded = torch.zeros((n_pad, pitch), dtype=torch.int64, device=dev)
    padded[:n, :w] = rows
    tri = n * (n + 1) // 2

    # the existing, allocating entry point
    c = sb.StormContig(m)
    c.set_kernel(sb.KERNEL_MMA)
    c.add_bitmaps(rows.cpu().numpy().view(np.uint64))
    want = torch.empty(tri, dtype=torch.int32, device=dev)
    want_sum = c.matrix_device(want.data_ptr(), tri)

    f = _entry(sb)
    outs = [torch.full((tri,), -1, dtype=torch.int32, device=dev) for _ in range(calls)]
    torch.cuda.synchronize()
    sums, free = [], []
    for out in outs:
        s = C.c_uint64(0)
        rc = f(padded.data_ptr(), n, pitch, m, out.data_ptr(), tri, C.byref(s), None)
        assert rc == 0, sb.StormError(rc)
        sums.append(int(s.value))
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    # The first call on a device may load kernel code (lazy module loading);
    # the calls after it must not change free device memory at all.
    assert all(fr == free[0] for fr in free[1:]), free
    for out, s in zip(outs, sums):   # every call, the last two in a row included
        assert torch.equal(out, want)
        assert s == want_sum


def test_noalloc_rejects_what_it_cannot_do(sb):
    import torch
    f = _entry(sb)
    d = torch.zeros((256, 8), dtype=torch.int64, device="cuda")
    s = C.c_uint64(0)
    assert f(None, 10, 8, 512, None, 0, C.byref(s), None) == sb.EVALUES
    assert f(d.data_ptr(), 10, 7, 448, None, 0, C.byref(s), None) == sb.EARG       # pitch not a multiple of 8
    assert f(d.data_ptr() + 16, 10, 8, 512, None, 0, C.byref(s), None) == sb.EARG  # rows not 32-byte aligned
    big = (1 << 23) + 64                                                           # rows too long to stay exact
    assert f(d.data_ptr(), 10, (big // 64 + 7) // 8 * 8, big, None, 0, C.byref(s), None) == sb.ELIMIT
    assert f(d.data_ptr(), 46081, 8, 512, None, 0, C.byref(s), None) == sb.ELIMIT  # tile list over its maximum
    assert f(d.data_ptr(), 10, 8, 512, d.data_ptr(), 3, C.byref(s), None) == sb.ESIZE
