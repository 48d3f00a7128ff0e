"""The no-allocation entry point (adds_sssp_noalloc) against adds_sssp.

adds_sssp_noalloc exists for callers that must not have a library allocate
device memory (an application that owns all device memory through its own
allocator or arena, or a loop that cannot absorb cudaMalloc/cudaFree
synchronisations).  It takes device arrays the caller owns and works in a
fixed device array inside the library.  This test calls it through the C
ABI, twice in a row per graph (the second call must not depend on what the
first left in the shared array), and requires distances bit-identical to
the allocating entry point's and to the CPU oracle's, the same tolerance as
every other distance test here.  Arrays with a defect are refused before
the solver reads them.  It lives in its own file so that it is collected
last.
"""
import ctypes as C

import numpy as np
import pytest

import adds_b200 as A
from adds_b200 import _lib as L
from adds_b200 import graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _device_csr(g):
    import torch
    row = torch.from_numpy(g.row.astype(np.uint32).view(np.int32)).cuda()
    inter = np.empty(2 * g.m, dtype=np.uint32)
    inter[0::2] = g.dst
    inter[1::2] = g.w
    edges = torch.from_numpy(inter.view(np.int32)).cuda()
    return row, edges


def _noalloc(g, row, edges, src):
    import torch
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = L.lib().adds_sssp_noalloc(g.n, g.m, row.data_ptr(), edges.data_ptr(), g.wtype, src,
                                   out.data_ptr(), None)
    L.check(rc, "adds_sssp_noalloc")
    return out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("kind", ["rmat_int", "grid_float"])
def test_noalloc_matches_allocating_entry_point(kind):
    if kind == "rmat_int":
        g = G.rmat(14, 16, seed=31, w_hi=10000)
        srcs = [G.max_degree_vertex(g), 17]
    else:
        g = G.grid(128, 96, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=32)
        srcs = [48 * 128 + 64, 5]
    row, edges = _device_csr(g)
    dg = A.Graph.from_csr(g)
    try:
        for s in srcs:  # two calls in a row on the shared scratch array
            want, _ = dg.sssp(s, A.default_opts(timeout_ms=10000))
            got = _noalloc(g, row, edges, s)
            assert np.array_equal(got, want), f"source {s}"
            ref, _ = O.dijkstra(g, s)  # and the CPU oracle directly
            assert np.array_equal(got, ref), f"source {s} vs oracle"
    finally:
        dg.close()


def _corrupt(kind):
    """A small graph with one defect made on the host."""
    g = G.rmat(10, 8, seed=33, w_hi=1000)
    row, dst, w = g.row.copy(), g.dst.copy(), g.w.copy()
    if kind == "dst":
        dst[g.m // 2] = g.n + 5
    elif kind == "rows":
        row[g.n // 2] = row[g.n // 2 + 1] + 1  # offsets decrease
    elif kind == "int_weight":
        w[7] = np.uint32(0x80000001)  # negative as int32
    return G.CSR(g.n, row, dst, w, g.wtype)


@pytest.mark.parametrize("kind", ["dst", "rows", "int_weight"])
def test_noalloc_rejects_invalid_arrays(kind):
    """Arrays that would send the solver outside the caller's buffers are
    refused before it reads them, and the output is left untouched."""
    import torch
    g = _corrupt(kind)
    row, edges = _device_csr(g)
    out = torch.full((g.n,), 12345, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = L.lib().adds_sssp_noalloc(g.n, g.m, row.data_ptr(), edges.data_ptr(), g.wtype, 0,
                                   out.data_ptr(), None)
    assert rc == -3  # ADDS_ERR_FORMAT
    assert b"invalid graph arrays" in L.lib().adds_last_cuda_error()
    assert bool((out == 12345).all())
    # the shared array is usable again at once
    good = G.rmat(10, 8, seed=34, w_hi=1000)
    r2, e2 = _device_csr(good)
    ref, _ = O.dijkstra(good, 3)
    assert np.array_equal(_noalloc(good, r2, e2, 3), ref)


def test_noalloc_rejects_graphs_over_the_limit():
    lib = L.lib()
    p = C.c_void_p(16)  # never dereferenced: the size check comes first
    assert lib.adds_sssp_noalloc((1 << 20) + 1, 10, p, p, 0, 0, p, None) == -9
    assert b"no-allocation limits" in lib.adds_last_cuda_error()
    assert lib.adds_sssp_noalloc(10, (1 << 24) + 1, p, p, 0, 0, p, None) == -9
