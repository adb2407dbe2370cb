"""The N > 1 bench plumbing on CPU: two gloo ranks exercise the reductions
bench.py uses for multi-GPU timing (max over ranks for the step time, sum
for the aggregate), the same calls in the same order on every rank; and a
rank that leaves between steps makes the other's next collective fail
within the process group's timeout instead of hanging."""
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


def _rank_leaves(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import time
    import torch
    import bench
    r, w, _ = bench.dist_env()
    dist = bench.init_dist(w, "gloo", timeout_s=5.0)
    dev = torch.device("cpu")
    bench.max_over_ranks(1.0, dist, dev)           # step 1: both ranks
    if r == 1:
        q.put((r, "left"))
        q.close()
        q.join_thread()                            # the message is out before the process goes
        os._exit(0)                                # leaves between steps, nothing in flight
    t0 = time.time()
    try:
        bench.max_over_ranks(2.0, dist, dev)       # step 2: the peer never arrives
        q.put((r, "no error"))
    except Exception as e:                         # gloo: peer closed / timeout
        q.put((r, f"error after {time.time() - t0:.1f}s: {type(e).__name__}"))
    q.close()
    q.join_thread()
    os._exit(0)


@pytest.mark.timeout(120)
def test_rank_leaving_fails_the_next_collective():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_leaves, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
    assert out[1] == "left"
    assert out[0].startswith("error after"), out[0]
    assert float(out[0].split()[2].rstrip("s:")) < 30.0
