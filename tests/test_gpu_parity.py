"""GPU parity: the engine's distances, through the C ABI, must equal the
CPU oracle's bit for bit (int32 and float32 folds)."""
import numpy as np
import pytest

import adds_b200 as A
from adds_b200 import graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu
OPTS = dict(timeout_ms=10000)


def _check(g, src, **kw):
    dg = A.Graph.from_csr(g)
    try:
        d, st = dg.sssp(src, A.default_opts(**{**OPTS, **kw}))
    finally:
        dg.close()
    ref, _ = O.dijkstra(g, src)
    mism = np.flatnonzero(d != ref)
    assert mism.size == 0, f"{mism.size} mismatches, first {mism[:5]} got {d[mism[:5]]} want {ref[mism[:5]]}"
    return st


def test_rmat16_int_max_degree_source():
    g = G.rmat(16, 16, seed=1)
    st = _check(g, G.max_degree_vertex(g))
    assert st["items_popped"] > 0


def test_grid_float_with_shortcuts():
    g = G.grid(256, 256, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=3)
    _check(g, 128 * 256 + 128)


def test_erdos_renyi_int():
    g = G.erdos_renyi(20000, 8, seed=11)
    _check(g, 5)


@pytest.mark.parametrize("shift", [0, 4, 9, 14, 20])
def test_any_delta_gives_same_distances(shift):
    g = G.rmat(13, 16, seed=2)
    _check(g, G.max_degree_vertex(g), delta_shift=shift)
