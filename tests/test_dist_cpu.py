"""The N > 1 bench plumbing on CPU: two gloo ranks exercise the reductions
bench.py uses for multi-GPU timing (max over ranks for the step time, sum
for the aggregate), the same calls in the same order on every rank."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import torch
    import bench
    r, w, l = bench.dist_env()
    dist = bench.init_dist(w, "gloo")
    dev = torch.device("cpu")
    step_ms = 100.0 + 50.0 * r                     # rank 1 is the slow one
    mx = bench.max_over_ranks(step_ms, dist, dev)
    total = bench.sum_over_ranks(float(bench.pairs_of(1000 + r)), dist, dev)
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, mx, total))


@pytest.mark.timeout(120)
def test_two_rank_timing_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    want_total = 1000 * 1001 / 2 + 1001 * 1002 / 2
    for r, w, mx, total in out:
        assert w == 2 and mx == 150.0 and total == want_total
