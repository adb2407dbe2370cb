"""Failure detection on the GPU without a fault: the bounded mbarrier wait of
the tensor-core kernels, run on a barrier nothing arrives on with a short
limit, gives up, frees its tensor memory and returns; the call reports
STORM_B200_ETIMEOUT and the context stays usable (the next all-pairs calls
are exact)."""
import time

import numpy as np
import pytest

import gen
import oracle_lib as ol

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("limit_us", [2000, 50000])
def test_bounded_wait_gives_up_and_context_survives(sb, limit_us):
    L = sb.lib()
    t0 = time.perf_counter()
    assert L.STORM_b200_wait_selftest(limit_us) == sb.ETIMEOUT
    dt = time.perf_counter() - t0
    assert dt >= limit_us * 1e-6
    assert dt < 30.0
    assert L.STORM_b200_wait_selftest(0) == sb.EARG
    # the context is intact: tensor-core and chunked all-pairs calls stay exact
    words = gen.bernoulli_rows(300, 4096 + 64, (0.05, 0.5), 44)
    want, ws = ol.contig_matrix(words)
    c = sb.StormContig(4096 + 64)
    c.set_kernel(sb.KERNEL_MMA)
    c.add_bitmaps(words)
    got, s = c.matrix()
    assert s == ws and np.array_equal(got, want)
    c.close()
    sets = gen.zipf_sets(60, 1 << 18, 1.1, 16, 1 << 12, 45)
    st = sb.Storm()
    for v in sets:
        st.add(v)
    vals, offs = gen.to_csr(sets)
    want, ws = ol.sets_matrix(vals, offs)
    got, s = st.matrix()
    assert s == ws and np.array_equal(got, want)
    st.close()
