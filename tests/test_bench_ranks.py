"""bench.py's multi-rank plumbing on CPU: two gloo ranks (spawned processes)
agree on the max time and the summed work, which is how the N-GPU replica
run reports whole-job throughput."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, loc = bench.dist_env()
    assert (w, r, loc) == (ws, rank, rank)
    dist = bench.dist_init(w, loc)
    bench.barrier(dist, loc)
    tmax, usum = bench.reduce_max_sum(dist, loc, 1.0 + rank, 10.0 * (rank + 1))
    out.put((rank, tmax, usum))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in ps)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [(t, u) for _, t, u in res] == [(2.0, 30.0), (2.0, 30.0)]


def test_single_rank_has_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.dist_init(1, 0) is None
    assert bench.reduce_max_sum(None, 0, 3.0, 4.0) == (3.0, 4.0)
