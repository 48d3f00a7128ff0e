"""GPU parity at the sizes the benchmark configurations name, against the CPU
oracle (serial Dijkstra, oracle/oracle.c), bit for bit.

The other GPU tests use graphs small enough for the oracle to run in a
blink.  These take the benchmark shapes at the largest size a test can
afford: R-MAT 20 with eight sources (the R-MAT 24 headline shape, 1/16 of
its size), a 1024 x 1024 float grid with 2 % shortcuts (the 4096^2 shape,
1/16), a 64-query slice of the batched configuration that includes an
Erdos-Renyi graph of 10^6 vertices, and the differentiable configuration's
full batch of 128 grids x 16 sources (forward and backward).  The oracle
runs in a thread pool (its calls release the GIL).
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

import adds_b200 as A
from adds_b200 import graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ASYNC, PHASE = 1, 2
OPTS = dict(timeout_ms=30000)


def _pool():
    O.lib()  # load once before the threads use it
    return cf.ThreadPoolExecutor(max_workers=max(2, min(32, os.cpu_count() or 2)))


def _oracle_many(jobs):
    """[(csr, src)] -> [distance words] from serial Dijkstra, in parallel."""
    with _pool() as ex:
        return list(ex.map(lambda j: O.dijkstra(j[0], j[1])[0], jobs))


def _sources(csr, k, seed):
    deg = np.diff(csr.row.astype(np.int64))
    return [int(x) for x in np.random.default_rng(seed).choice(np.flatnonzero(deg > 0), k,
                                                              replace=False)]


@pytest.mark.parametrize("engine", [0, ASYNC, PHASE])
def test_rmat20_int_eight_sources(engine):
    spec = A.gen_spec("rmat", scale=20, edge_factor=16, wtype=0, w_lo=1, w_hi=10000, seed=20)
    g = A.Graph.generate(spec, 0)
    try:
        csr = g.download()
        srcs = _sources(csr, 8, 2024)
        want = _oracle_many([(csr, s) for s in srcs])
        o = A.default_opts(engine=engine, **OPTS)
        for s, ref in zip(srcs, want):
            d, _ = g.sssp(s, o)
            bad = np.flatnonzero(d != ref)
            assert bad.size == 0, f"source {s}: {bad.size} mismatches, first {bad[:5]}"
    finally:
        g.close()


@pytest.mark.parametrize("engine", [ASYNC, PHASE])
def test_grid1024_float_with_shortcuts(engine):
    spec = A.gen_spec("grid", side=1024, shortcut_frac=0.02, radius=8, wtype=1, w_lo=1.0,
                      w_hi=100.0, seed=1024)
    g = A.Graph.generate(spec, 0)
    try:
        csr = g.download()
        srcs = [512 * 1024 + 512, 7, 1024 * 1024 - 1]
        want = _oracle_many([(csr, s) for s in srcs])
        o = A.default_opts(engine=engine, **OPTS)
        for s, ref in zip(srcs, want):
            d, _ = g.sssp(s, o)
            bad = np.flatnonzero(d != ref)
            assert bad.size == 0, f"source {s}: {bad.size} mismatches, first {bad[:5]}"
    finally:
        g.close()


def test_batched_slice_with_million_vertex_er():
    """64 queries of the batched configuration's kinds: 56 Erdos-Renyi graphs
    (n log-uniform in [1e3, 1e6], one of exactly 1e6 vertices; 8 draws per
    vertex, U[1,1000]) and 8 sources on one R-MAT 20 graph, one launch,
    replayed."""
    rng = np.random.default_rng(64)
    ns = np.exp(rng.uniform(np.log(1e3), np.log(1e6), size=56)).round().astype(int)
    ns[0] = 1_000_000
    graphs, csrs, srcs = [], [], []
    try:
        for i, n in enumerate(ns):
            g = A.Graph.generate(A.gen_spec("er", n=int(n), edge_factor=8, wtype=0, w_lo=1,
                                            w_hi=1000, seed=10_000 + i), 0)
            graphs.append(g)
            csrs.append(g.download())
            srcs.append(int(rng.integers(0, g.n)))
        r20 = A.Graph.generate(A.gen_spec("rmat", scale=20, wtype=0, w_lo=1, w_hi=1000, seed=20),
                               0)
        graphs.append(r20)
        rc = r20.download()
        rs = _sources(rc, 8, 65)
        qg = graphs[:-1] + [r20] * 8
        qc = csrs + [rc] * 8
        qs = srcs + rs
        want = _oracle_many(list(zip(qc, qs)))
        b = A.Batch(qg, qs, A.default_opts(**OPTS))
        try:
            for rep in range(2):  # the second run replays the captured launch
                b.run()
                for q in range(len(qs)):
                    d = b.dist(q)
                    assert np.array_equal(d, want[q]), f"run {rep} query {q} (n={qc[q].n})"
        finally:
            b.close()
    finally:
        for g in graphs:
            g.close()


def test_diff_configuration_batch_forward_and_backward_bit_exact():
    """The differentiable configuration at full size: 128 grids (side
    log-uniform in [64, 512], w = softplus(theta), theta ~ N(0,1)), 16
    sources and 64 targets each, L = sum c_t d(s, t).  Every query's
    distances equal serial Dijkstra's and every graph's dL/dw equals the
    oracle adjoint's, bit for bit."""
    import torch
    rng = np.random.default_rng(128)
    sides = np.exp(rng.uniform(np.log(64), np.log(512), size=128)).round().astype(int)
    graphs, csrs = [], []
    qg, qs, qi, seeds = [], [], [], []
    try:
        for i, sd in enumerate(sides):
            g = A.Graph.generate(A.gen_spec("plain_grid", side=int(sd), wtype=1, w_lo=1.0,
                                            w_hi=2.0, seed=500 + i), 0)
            theta = rng.standard_normal(g.m).astype(np.float32)
            w = torch.nn.functional.softplus(torch.from_numpy(theta)).numpy().astype(np.float32)
            g.set_weights(np.ascontiguousarray(w.view(np.uint32)))
            graphs.append(g)
            csrs.append(g.download())
            t = rng.choice(g.n, size=64, replace=False)
            c = rng.uniform(0, 1, size=64).astype(np.float32)
            for s in rng.choice(g.n, size=16, replace=False):
                qg.append(g)
                qs.append(int(s))
                qi.append(i)
                sv = np.zeros(g.n, dtype=np.float32)
                sv[t] = c
                seeds.append(sv)
        b = A.Batch(qg, qs, A.default_opts(**OPTS))
        try:
            b.run()
            dists = [b.dist(q) for q in range(len(qg))]
            want = _oracle_many([(csrs[qi[q]], qs[q]) for q in range(len(qg))])
            for q in range(len(qg)):
                assert np.array_equal(dists[q], want[q]), f"query {q}"
            sd = [torch.from_numpy(x).cuda() for x in seeds]
            gw = [torch.zeros(g.m, device="cuda") for g in graphs]
            b.backward([t.data_ptr() for t in sd], [t.data_ptr() for t in gw])
            torch.cuda.synchronize()

            def adj(i):
                qq = [q for q in range(len(qg)) if qi[q] == i]
                return O.adjoint(csrs[i], [qs[q] for q in qq],
                                 np.stack([dists[q].view(np.float32) for q in qq]),
                                 np.stack([seeds[q] for q in qq]))[0]
            with _pool() as ex:
                grads = list(ex.map(adj, range(len(graphs))))
            for i, want_g in enumerate(grads):
                got = gw[i].cpu().numpy()
                assert np.array_equal(got.view(np.uint32), want_g.view(np.uint32)), f"graph {i}"
        finally:
            b.close()
    finally:
        for g in graphs:
            g.close()


def test_diff_finite_differences_256_edges():
    """Central finite differences (eps = 1e-3 on theta, float64 Dijkstra) on
    256 random edges of four grids whose sides come from the differentiable
    configuration's distribution (log-uniform in [64, 512]), 16 sources x
    64 targets each; an edge is used when no source's shortest-path tree
    changes within +-10 eps of theta (its tie margin exceeds 10 eps)."""
    import torch
    from adds_b200.autograd import batched_sssp, query_offsets
    rng = np.random.default_rng(256)
    sides = np.exp(rng.uniform(np.log(64), np.log(512), size=4)).round().astype(int)
    eps = 1e-3
    total = 0
    for gi, sd in enumerate(sides):
        g0 = G.grid(int(sd), int(sd), 0.0, 8, wtype=G.F32, seed=700 + gi)
        theta = rng.standard_normal(g0.m).astype(np.float32)
        w32 = torch.nn.functional.softplus(torch.from_numpy(theta)).numpy().astype(np.float32)
        g = G.CSR(g0.n, g0.row, g0.dst, w32.view(np.uint32), G.F32)
        srcs = [int(s) for s in rng.choice(g.n, size=16, replace=False)]
        coef = []
        for _ in srcs:
            c = np.zeros(g.n, dtype=np.float64)
            t = rng.choice(g.n, size=64, replace=False)
            c[t] = rng.uniform(0, 1, size=64)
            coef.append(c)
        dg = A.Graph.from_csr(g)
        b = A.Batch([dg] * len(srcs), srcs, A.default_opts(**OPTS))
        try:
            th = torch.from_numpy(theta).cuda().requires_grad_(True)
            flat = batched_sssp(b, [dg], [torch.nn.functional.softplus(th)])
            off = query_offsets(b)
            cs = [torch.from_numpy(c.astype(np.float32)).cuda() for c in coef]
            loss = sum((ci * flat[int(o):int(o) + g.n]).sum() for ci, o in zip(cs, off))
            loss.backward()
            grad = th.grad.cpu().numpy().astype(np.float64)
        finally:
            b.close()
            dg.close()
        base = theta.astype(np.float64)
        wb = np.log1p(np.exp(base))
        esrc = np.repeat(np.arange(g.n), np.diff(g.row).astype(np.int64))
        O.lib()
        with _pool() as ex:
            d0 = list(ex.map(lambda s: O.dijkstra_f64(g, wb, s), srcs))

        def trees(th64, idx):
            w = np.log1p(np.exp(th64))
            out = []
            for k in idx:
                d = O.dijkstra_f64(g, w, srcs[k])
                out.append(np.flatnonzero((d[esrc] + w == d[g.dst]) & (d[esrc] < d[g.dst])))
            return out

        def check_edge(e):
            """(used, fd, grad) for edge e"""
            u, v = esrc[e], g.dst[e]
            # sources whose tree may react to a +-10 eps change of w_e
            slack = np.array([d[u] + wb[e] - d[v] for d in d0])
            near = np.flatnonzero(slack <= 10 * eps)
            b0 = trees(base, near)
            up, dn = base.copy(), base.copy()
            up[e] += 10 * eps
            dn[e] -= 10 * eps
            if not all(np.array_equal(x, y) for x, y in zip(trees(up, near), b0)) or \
               not all(np.array_equal(x, y) for x, y in zip(trees(dn, near), b0)):
                return False, 0.0, 0.0
            up[e], dn[e] = base[e] + eps, base[e] - eps
            wu, wd = np.log1p(np.exp(up)), np.log1p(np.exp(dn))
            fd = 0.0
            for k in near:  # the other sources' distances do not move
                fd += float((coef[k] * (O.dijkstra_f64(g, wu, srcs[k]) -
                                        O.dijkstra_f64(g, wd, srcs[k]))).sum())
            return True, fd / (2 * eps), float(grad[e])

        edges = rng.choice(g.m, size=64, replace=False)
        with _pool() as ex:
            res = list(ex.map(check_edge, edges))
        for e, (used, fd, gr) in zip(edges, res):
            if used:
                assert abs(fd - gr) <= 2e-3 * max(1.0, abs(fd)), (gi, int(e), fd, gr)
                total += 1
    assert total >= 128, f"only {total} of 256 edges had a tie margin above 10 eps"
