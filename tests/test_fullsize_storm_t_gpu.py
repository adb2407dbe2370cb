"""STORM_t all-pairs at the full size of the sparse and mixed-density
configurations, through the reference's own container (rows appended with
STORM_add_rows / STORM_add_bitmap_rows, exactly the chunks STORM_add builds),
per-pair counts into HBM:

    config3        100,000 rows over 2^24, card ~ Zipf(1.1) on [16, 2^22]
    config4        50,000 rows over 2^26, Poisson(200) runs of mean 256
    config5b_0.01  20,000 rows over 2^24, Bernoulli(0.01)
    config5b_0.17  20,000 rows over 2^24, Bernoulli(0.17)

Each triangle is checked three ways:
  * eight whole rows -- the heaviest and the lightest by drawn size, the
    first, the last and four at random -- against the CPU oracle, every
    partner j of each (strips counted while the rows stream in);
  * every row of the full symmetric matrix sums to sum over the row's
    values v of (rows holding v), from the value histogram, and the diagonal
    equals the cardinalities -- an identity over the whole triangle;
  * the sum over i < j equals sum_v C(rows holding v, 2), from both the
    per-pair call and the reference's sum-only call
    (STORM_pairw_intersect_cardinality).
The inputs are seeded and generated on the GPU (bench.py FullCorpus)."""
import os

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu


def _sample_rows(corpus, n):
    if corpus.cards is not None:
        size = np.asarray(corpus.cards, np.int64)
    elif corpus.kind == "runs":
        size = np.zeros(n, np.int64)
        nz = corpus.nrun > 0
        size[nz] = np.add.reduceat(corpus.lens, corpus.run0[:-1][nz])
    else:
        size = None
    g = np.random.default_rng(corpus.seed)
    rows = [0, n - 1] + [int(x) for x in g.integers(1, n - 1, size=4)]
    if size is not None:
        rows += [int(np.argmax(size)), int(np.argmin(size))]
    else:
        rows += [int(x) for x in g.integers(1, n - 1, size=2)]
    out = []
    for r in rows:
        if r not in out:
            out.append(r)
    return out[:8]


def _query_rows(corpus, rows):
    """Values (or bitmap words) of the sample rows, from their batches."""
    got = {}
    for b in sorted({corpus.batch_of(r) for r in rows}):
        r0, r1, x, offs = corpus.batch(b)
        host = x.cpu().numpy()
        for r in rows:
            if r0 <= r < r1:
                if offs is None:
                    got[r] = host[r - r0].view(np.uint64).copy()
                else:
                    got[r] = host.view(np.uint32)[int(offs[r - r0]):int(offs[r - r0 + 1])].copy()
        del x
    return [got[r] for r in rows]


@pytest.mark.timeout(3600)
@pytest.mark.parametrize("name", ["config4", "config5b_0.01", "config5b_0.17", "config3"])
def test_full_size_configuration(sb, name):
    import torch
    import bench
    dev = torch.device("cuda")
    torch.cuda.empty_cache()
    corpus = bench.full_corpus(name, dev)
    n = corpus.n
    rows = _sample_rows(corpus, n)
    q = _query_rows(corpus, rows)
    strip = ol.BitmapStrip(np.stack(q)) if corpus.kind == "bits" else ol.SetStrip(q, corpus.universe)
    strips = np.zeros((n, len(rows)), np.uint32)
    threads = os.cpu_count() or 1

    def on_batch(r0, r1, host, offs):
        strips[r0:r1] = strip.count(host, offs, threads=threads)

    res = bench.load_full_corpus(sb, corpus, on_batch=on_batch)
    strip.close()
    st, hist, cards, want_row = res["storm"], res["hist"], res["cards"], res["want_row"]
    assert len(st) == n
    tri = n * (n + 1) // 2
    d_tri = torch.full((tri,), -1, dtype=torch.int32, device=dev)
    s = st.matrix_device(d_tri.data_ptr(), tri)

    want_sum = int((hist * (hist - 1) // 2).sum().item())
    assert s == want_sum
    # eight whole rows against the oracle strips
    for k, i in enumerate(rows):
        j = np.arange(n, dtype=np.int64)
        a, b = np.minimum(i, j), np.maximum(i, j)
        idx = torch.as_tensor(a * n - (a * (a - 1)) // 2 + (b - a), device=dev)
        got = d_tri[idx].cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, strips[:, k], err_msg=f"{name}: row {i}")
    del strips
    # whole triangle: symmetric row sums and the diagonal
    got_row, diag = bench.triangle_row_sums(d_tri, n)
    assert torch.equal(diag.cpu(), torch.as_tensor(cards)), name
    bad = int((got_row != want_row).sum().item())
    assert bad == 0, f"{name}: {bad} rows whose sums differ from the histogram identity"
    assert (int(got_row.sum().item()) - int(cards.sum())) // 2 == want_sum
    del d_tri, got_row
    torch.cuda.empty_cache()
    # the reference's own sum-only call
    assert st.pairw_intersect_cardinality() == want_sum
    st.close()
