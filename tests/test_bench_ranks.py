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


def _shard_rank(rank, ws, port, out):
    """One rank of a query-sharded batch: it 'solves' its queries (a fake
    solver writes query q's words as q * 1000 + i) and the results meet on
    rank 0 through gather_to_root."""
    import numpy as np
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.dist_init(ws, rank)
    mine = bench.shard_queries(11, ws, rank)
    lens = [3 + (q % 4) for q in mine]
    words = np.concatenate([np.arange(n, dtype=np.uint32) + 1000 * q for q, n in zip(mine, lens)]) \
        if mine else np.zeros(0, dtype=np.uint32)
    parts = bench.gather_to_root(dist, rank, words)
    out.put((rank, mine, None if parts is None else [p.tolist() for p in parts]))
    dist.destroy_process_group()


def test_query_sharding_and_host_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in ps)
    res = {r: (m, parts) for r, m, parts in (q.get(timeout=5) for _ in range(2))}
    m0, m1 = res[0][0], res[1][0]
    assert sorted(m0 + m1) == list(range(11)) and not set(m0) & set(m1)
    assert res[1][1] is None  # only rank 0 receives
    got = res[0][1]
    for rank, mine in ((0, m0), (1, m1)):
        want = [w for qq in mine for w in range(1000 * qq, 1000 * qq + 3 + qq % 4)]
        assert got[rank] == want


def test_single_rank_has_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.dist_init(1, 0) is None
    assert bench.reduce_max_sum(None, 0, 3.0, 4.0) == (3.0, 4.0)
