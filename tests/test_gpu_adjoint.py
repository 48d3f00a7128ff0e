"""GPU adjoint (dL/dw of distances) against the CPU reference gradient.

The engine's backward pass builds the same tie-broken predecessor tree as
oracle/oracle.c (smallest-index strict tight in-edge, zero-gap ties in
breadth-first rounds) and sums lambda in the same orders, so the gradient
must match the oracle bit for bit.  It is also checked against float64
central finite differences on edges whose tie margin exceeds 10*eps.
"""
import numpy as np
import pytest

import adds_b200 as A
from adds_b200 import graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
FMAX = np.float32(3.4028234663852886e38)


def softplus_grid(sx, sy, seed):
    rng = np.random.default_rng(seed)
    g = G.grid(sx, sy, 0.0, 8, wtype=G.F32, seed=seed)
    theta = rng.standard_normal(g.m).astype(np.float32)
    w = torch.nn.functional.softplus(torch.from_numpy(theta)).numpy().astype(np.float32)
    return G.CSR(g.n, g.row, g.dst, w.view(np.uint32), G.F32), theta


def seeds_for(g, ns, nt, rng):
    s = np.zeros((ns, g.n), dtype=np.float32)
    for i in range(ns):
        t = rng.choice(g.n, size=nt, replace=False)
        s[i, t] = rng.uniform(0, 1, size=nt).astype(np.float32)
    return s


def test_single_graph_backward_bit_exact():
    g, _ = softplus_grid(40, 30, 1)
    rng = np.random.default_rng(2)
    srcs = [0, 15 * 40 + 20, 1199, 333]
    dg = A.Graph.from_csr(g)
    dist = np.stack([dg.sssp(s, A.default_opts(timeout_ms=10000))[0] for s in srcs])
    for i, s in enumerate(srcs):
        assert np.array_equal(dist[i], O.dijkstra(g, s)[0])
    seeds = seeds_for(g, len(srcs), 25, rng)
    want, _ = O.adjoint(g, srcs, dist.view(np.float32), seeds)
    dd = torch.from_numpy(dist.view(np.float32)).cuda().contiguous()
    sd = torch.from_numpy(seeds).cuda().contiguous()
    gw = torch.full((g.m,), 7.0, device="cuda")  # overwritten
    dg.backward(srcs, dd.data_ptr(), sd.data_ptr(), gw.data_ptr())
    got = gw.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    dg.close()


def test_batch_backward_bit_exact_accumulates_per_graph():
    rng = np.random.default_rng(5)
    gs = [softplus_grid(24 + 8 * i, 20 + 4 * i, 10 + i)[0] for i in range(3)]
    dgs = [A.Graph.from_csr(g) for g in gs]
    qg, srcs, qc = [], [], []
    for i, (g, dg) in enumerate(zip(gs, dgs)):
        for s in rng.choice(g.n, size=4, replace=False):
            qg.append(dg)
            qc.append(g)
            srcs.append(int(s))
    b = A.Batch(qg, srcs, A.default_opts(timeout_ms=10000))
    b.run()
    dists = [b.dist(q) for q in range(len(qg))]
    for q in range(len(qg)):
        assert np.array_equal(dists[q], O.dijkstra(qc[q], srcs[q])[0])
    seeds = [seeds_for(qc[q], 1, 10, rng)[0] for q in range(len(qg))]
    sd = [torch.from_numpy(x).cuda() for x in seeds]
    gw = [torch.zeros(g.m, device="cuda") for g in gs]
    b.backward([t.data_ptr() for t in sd], [t.data_ptr() for t in gw])
    for i, g in enumerate(gs):
        qs = [q for q in range(len(qg)) if qc[q] is g]
        want, _ = O.adjoint(g, [srcs[q] for q in qs],
                            np.stack([dists[q].view(np.float32) for q in qs]),
                            np.stack([seeds[q] for q in qs]))
        assert np.array_equal(gw[i].cpu().numpy().view(np.uint32), want.view(np.uint32)), i
    # backward accumulates into grad_w
    b.backward([t.data_ptr() for t in sd], [t.data_ptr() for t in gw])
    g0 = gw[0].cpu().numpy()
    qs = [q for q in range(len(qg)) if qc[q] is gs[0]]
    w0, _ = O.adjoint(gs[0], [srcs[q] for q in qs],
                      np.stack([dists[q].view(np.float32) for q in qs]), np.stack([seeds[q] for q in qs]))
    assert np.array_equal(g0, (w0 + w0).astype(np.float32))
    b.close()
    for dg in dgs:
        dg.close()


def test_zero_gap_ties():
    g = G.from_edges(5, [0, 1, 2, 2, 3], [1, 2, 1, 3, 4], [1.0, 0.0, 0.0, 0.0, 2.0], wtype=G.F32)
    dg = A.Graph.from_csr(g)
    d, _ = dg.sssp(0, A.default_opts(timeout_ms=10000))
    seeds = np.array([[0, 1, 10, 100, 1000]], dtype=np.float32)
    want, _ = O.adjoint(g, [0], d.view(np.float32)[None], seeds)
    dd = torch.from_numpy(d.view(np.float32)).cuda()
    sd = torch.from_numpy(seeds).cuda()
    gw = torch.zeros(g.m, device="cuda")
    dg.backward([0], dd.data_ptr(), sd.data_ptr(), gw.data_ptr())
    assert gw.cpu().numpy().tolist() == want.tolist() == [1111.0, 1110.0, 0.0, 1100.0, 1000.0]
    dg.close()


def test_autograd_matches_finite_differences():
    rng = np.random.default_rng(7)
    g, theta = softplus_grid(20, 16, 21)
    dg = A.Graph.from_csr(g)
    srcs = [0, 170]
    b = A.Batch([dg, dg], srcs, A.default_opts(timeout_ms=10000))
    th = torch.from_numpy(theta).cuda().requires_grad_(True)
    from adds_b200.autograd import batched_sssp, query_offsets
    c = [torch.zeros(g.n, device="cuda") for _ in srcs]
    for x in c:
        t = rng.choice(g.n, size=20, replace=False)
        x[torch.from_numpy(t).cuda()] = torch.from_numpy(rng.uniform(0, 1, 20).astype(np.float32)).cuda()
    flat = batched_sssp(b, [dg], [torch.nn.functional.softplus(th)])
    off = query_offsets(b)
    d = [flat[int(o):int(o) + g.n] for o in off]
    loss = sum((ci * di).sum() for ci, di in zip(c, d))
    loss.backward()
    grad = th.grad.cpu().numpy().astype(np.float64)
    w64 = np.log1p(np.exp(theta.astype(np.float64)))
    cs = [x.cpu().numpy().astype(np.float64) for x in c]

    def L(th64):
        w = np.log1p(np.exp(th64))
        return sum(float((ci * O.dijkstra_f64(g, w, s)).sum()) for ci, s in zip(cs, srcs))

    def tree(th64, s):
        w = np.log1p(np.exp(th64))
        d = O.dijkstra_f64(g, w, s)
        src = np.repeat(np.arange(g.n), np.diff(g.row).astype(np.int64))
        tight = (d[src] + w == d[g.dst]) & (d[src] < d[g.dst])
        return np.flatnonzero(tight)
    eps = 1e-3
    checked = 0
    for e in rng.choice(g.m, size=60, replace=False):
        base = theta.astype(np.float64)
        up, dn = base.copy(), base.copy()
        up[e] += 10 * eps
        dn[e] -= 10 * eps
        if not all(np.array_equal(tree(up, s), tree(base, s)) and np.array_equal(tree(dn, s), tree(base, s))
                   for s in srcs):
            continue
        up[e] = base[e] + eps
        dn[e] = base[e] - eps
        fd = (L(up) - L(dn)) / (2 * eps)
        assert abs(fd - grad[e]) <= 2e-3 * max(1.0, abs(fd)), (e, fd, grad[e])
        checked += 1
    assert checked >= 20
    b.close()
    dg.close()
