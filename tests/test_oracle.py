"""CPU oracle: known answers, cross-checks, and the adjoint reference.

The reference ships no golden vectors or known-answer tests for its path
(its only check is a text diff against Galois Dijkstra output, verify.py).
The oracle is pinned here by the reference's own output (the ADDS binaries
built from the reference sources and run on a B200, fixtures ref_*.npz), by
hand-computed answers, by scipy's float64 Dijkstra on integer graphs, and by
frozen oracle outputs (oracle_golden.npz).
"""
import os

import numpy as np
import pytest

from adds_b200 import graphs as G
from oracle import oracle as O

INF_I = 0x7FFFFFFF
INF_F = 0x7F7FFFFF
HERE = os.path.dirname(os.path.abspath(__file__))


def f32(x):
    return np.float32(x).view(np.uint32)


def test_known_answers_int():
    # 0->1 (4), 0->2 (1), 2->1 (2), 1->3 (5), 2->3 (8), 3->3 self loop, 4 isolated,
    # duplicate 0->2 with a larger weight, zero-weight edge 3->5
    src = [0, 0, 2, 1, 2, 3, 0, 3]
    dst = [1, 2, 1, 3, 3, 3, 2, 5]
    w = [4, 1, 2, 5, 8, 7, 9, 0]
    g = G.from_edges(6, src, dst, w)
    d, work = O.dijkstra(g, 0)
    assert d.tolist() == [0, 3, 1, 8, INF_I, 8]
    assert work == 5  # vertices settled: all reached ones


def test_known_answer_float_rounding():
    # the fold is fl(fl(0 + a) + b): 1e8 + 1 + 1 stays 1e8 in float32,
    # while the direct edge of weight 1e8 + 4 wins
    a = np.float32(1.0e8)
    g = G.from_edges(3, [0, 1, 0], [1, 2, 2], [a, 1.0, np.float32(100000004.0)], wtype=G.F32)
    d, _ = O.dijkstra(g, 0)
    assert d[1] == f32(a)
    assert d[2] == f32(np.float32(a + np.float32(1.0)))  # == 1e8 after rounding
    assert d[2] == f32(1.0e8)


def test_unreachable_and_single_vertex():
    g = G.from_edges(3, [1], [2], [5])
    d, work = O.dijkstra(g, 0)
    assert d.tolist() == [0, INF_I, INF_I] and work == 1
    g1 = G.from_edges(1, [], [], [])
    d, _ = O.dijkstra(g1, 0)
    assert d.tolist() == [0]


def test_int_overflow_rule():
    # sums >= INT32_MAX are never accepted (reported INF)
    g = G.from_edges(3, [0, 1], [1, 2], [0x7FFFFFF0, 0x20])
    d, _ = O.dijkstra(g, 0)
    assert d.tolist() == [0, 0x7FFFFFF0, INF_I]


@pytest.mark.parametrize("gen", ["rmat", "er", "grid"])
def test_dijkstra_matches_scipy_on_int_graphs(gen):
    import scipy.sparse as sp
    import scipy.sparse.csgraph as cg
    if gen == "rmat":
        g = G.rmat(12, 16, seed=3, w_hi=1000)
    elif gen == "er":
        g = G.erdos_renyi(3000, 8, seed=4)
    else:
        g = G.grid(40, 30, 0.02, 8, wtype=G.I32, w_lo=1, w_hi=99, seed=5)
    src = int(np.argmax(np.diff(g.row)))
    d, _ = O.dijkstra(g, src)
    A = sp.csr_matrix((g.w.astype(np.float64) + 0.0, g.dst.astype(np.int64), g.row.astype(np.int64)),
                      shape=(g.n, g.n))
    ref = cg.dijkstra(A, indices=src)
    ref = np.where(np.isinf(ref), INF_I, ref).astype(np.int64)
    assert np.array_equal(d.astype(np.int64), ref)


@pytest.mark.parametrize("shift", [0, 3, 8, 12])
def test_delta_stepping_equals_dijkstra_int(shift):
    g = G.rmat(11, 16, seed=7, w_hi=5000)
    d, _ = O.dijkstra(g, 1)
    d2, work, ms = O.delta_step(g, 1, shift=shift, threads=4)
    assert np.array_equal(d, d2) and work >= 1


@pytest.mark.parametrize("div", [0.5, 10.0, 1000.0])
def test_delta_stepping_equals_dijkstra_float(div):
    g = G.grid(50, 40, 0.02, 8, wtype=G.F32, seed=9)
    d, _ = O.dijkstra(g, 20 * 50 + 25)
    d2, _, _ = O.delta_step(g, 20 * 50 + 25, div=div, threads=3)
    assert np.array_equal(d, d2)


def test_golden_fixtures():
    """Oracle outputs committed by tests/golden/make_golden.py."""
    z = np.load(os.path.join(HERE, "golden", "oracle_golden.npz"))
    for name in sorted({k.split("__")[0] for k in z.files}):
        g = G.CSR(int(z[name + "__n"]), z[name + "__row"], z[name + "__dst"], z[name + "__w"],
                  int(z[name + "__wtype"]))
        d, _ = O.dijkstra(g, int(z[name + "__src"]))
        assert np.array_equal(d, z[name + "__dist"]), name


def _fd_tree_check(g, srcs, seeds):
    """dL/dw from the oracle adjoint equals float64 finite differences of
    L = sum_s sum_v seed[s,v] * d_s(v) on tie-free edges."""
    w64 = g.weights().astype(np.float64)
    dist = np.stack([O.dijkstra(g, s)[0].view(np.float32) for s in srcs])
    grad, pred = O.adjoint(g, srcs, dist, seeds)

    def L(w):
        tot = 0.0
        for i, s in enumerate(srcs):
            d = O.dijkstra_f64(g, w, s)
            m = d < 1e299
            tot += float((seeds[i][m] * d[m]).sum())
        return tot
    eps = 1e-3
    rng = np.random.default_rng(0)
    checked = 0
    for e in rng.choice(g.m, size=min(40, g.m), replace=False):
        wp, wm = w64.copy(), w64.copy()
        wp[e] += 10 * eps
        wm[e] -= 10 * eps
        # tie margin > 10 eps: the float64 trees at +-10 eps agree with the tree at w
        same = all(np.array_equal(_tree64(g, wp, s), _tree64(g, w64, s)) and
                   np.array_equal(_tree64(g, wm, s), _tree64(g, w64, s)) for s in srcs)
        if not same:
            continue
        wp[e] = w64[e] + eps
        wm[e] = w64[e] - eps
        fd = (L(wp) - L(wm)) / (2 * eps)
        assert abs(fd - grad[e]) <= 1e-3 * max(1.0, abs(fd)), (e, fd, grad[e])
        checked += 1
    assert checked >= 10


def _tree64(g, w64, s):
    d = O.dijkstra_f64(g, w64, s)
    src = np.repeat(np.arange(g.n), np.diff(g.row).astype(np.int64))
    tight = (d[src] + w64 == d[g.dst]) & (d[src] < d[g.dst]) & (d[g.dst] < 1e299)
    pred = np.full(g.n, -1, dtype=np.int64)
    idx = np.flatnonzero(tight)
    # smallest edge index per head
    for e in idx[::-1]:
        pred[g.dst[e]] = e
    return pred


def test_adjoint_oracle_matches_finite_differences():
    rng = np.random.default_rng(3)
    g = G.grid(12, 10, 0.0, 8, wtype=G.F32, seed=2)
    theta = rng.standard_normal(g.m).astype(np.float32)
    w = np.log1p(np.exp(theta)).astype(np.float32)
    g = G.CSR(g.n, g.row, g.dst, w.view(np.uint32), G.F32)
    srcs = [0, 57]
    seeds = np.zeros((2, g.n), dtype=np.float32)
    for i in range(2):
        t = rng.choice(g.n, size=12, replace=False)
        seeds[i, t] = rng.uniform(0, 1, size=12).astype(np.float32)
    _fd_tree_check(g, srcs, seeds)


def test_adjoint_zero_gap_ties_form_a_tree():
    # 0 -(1)-> 1, 1 -(0)-> 2, 2 -(0)-> 1, 2 -(0)-> 3: vertices 1, 2, 3 share d=1;
    # 2 and 3 are reached only through zero-gap edges
    g = G.from_edges(4, [0, 1, 2, 2], [1, 2, 1, 3], [1.0, 0.0, 0.0, 0.0], wtype=G.F32)
    d, _ = O.dijkstra(g, 0)
    dist = d.view(np.float32)[None, :]
    seeds = np.array([[0, 1, 10, 100]], dtype=np.float32)
    grad, pred = O.adjoint(g, [0], dist, seeds)
    e = pred[0] >> np.uint64(32)
    # tree edges: 1 <- e0 (strict), 2 <- e1 (round 1), 3 <- e3 (round 2)
    assert [int(x) for x in e[1:]] == [0, 1, 3]
    # lambda: 3 -> 100, 2 -> 10 + 100, 1 -> 1 + 110
    assert grad.tolist() == [111.0, 110.0, 0.0, 100.0]


def _ref_cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_ref_golden", os.path.join(HERE, "golden", "make_ref_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("name", ["ref_rmat16_int", "ref_rmat12_int", "ref_grid96_float"])
def test_oracle_pinned_to_reference_output(name):
    """The fixtures hold what the reference ADDS binaries (built for sm_100a
    by oracle/build_ref.sh, run on a B200 by tests/golden/make_ref_golden.py)
    printed for these seeded graphs; the oracle must reproduce them exactly
    (int: every distance; float: the reference's %f text)."""
    import gzip
    m = _ref_cases()
    build, rule, binary = m.CASES[name]
    g = build()
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    src = int(z["src"])
    assert src == m.source_of(g, rule)
    d, _ = O.dijkstra(g, src)
    if binary == "ads_int_sssp":
        assert np.array_equal(d, z["dist"])
    else:
        text = gzip.decompress(z["text_gz"].tobytes()).decode()
        assert G.dist_text(d, G.F32) == text


@pytest.mark.parametrize("kind", ["rmat_int", "rmat_float", "grid_float", "plain_grid"])
def test_host_generator_matches_numpy_twin(kind):
    """oracle/gen.c (the reference arm's graph builder) produces the CSR of
    adds_b200/graphs.py (and so of the GPU generator) bit for bit."""
    if kind == "rmat_int":
        a = O.gen_rmat(13, 16, wtype=0, w_lo=1, w_hi=10000, seed=24, threads=3)
        b = G.rmat(13, 16, wtype=0, w_lo=1, w_hi=10000, seed=24)
    elif kind == "rmat_float":
        a = O.gen_rmat(11, 16, wtype=1, w_lo=0.0, w_hi=1.0, seed=26, threads=4)
        b = G.rmat(11, 16, wtype=1, w_lo=0.0, w_hi=1.0, seed=26)
    elif kind == "grid_float":
        a = O.gen_grid(131, 77, 0.02, 8, wtype=1, w_lo=1.0, w_hi=100.0, seed=4096, threads=5)
        b = G.grid(131, 77, 0.02, 8, wtype=1, w_lo=1.0, w_hi=100.0, seed=4096)
    else:
        a = O.gen_grid(40, 33, 0.0, 8, wtype=1, w_lo=1.0, w_hi=2.0, seed=9, threads=2)
        b = G.grid(40, 33, 0.0, 8, wtype=1, w_lo=1.0, w_hi=2.0, seed=9)
    assert a.n == b.n and a.m == b.m
    assert np.array_equal(a.row, b.row)
    assert np.array_equal(a.dst, b.dst)
    assert np.array_equal(a.w, b.w)
