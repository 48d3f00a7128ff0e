"""Failure detection without a GPU fault.

The reference traps with a device assert when its worklist runs out
(ads_int/wl.h:614-619) and has no watchdog.  Here every device wait is
bounded: a wait that runs out records an error word and wait site and the
kernel returns, so the host gets an error code and the GPU context stays
usable.  The test makes a wait run out on purpose (a flag that nothing
sets, through the engine's own barrier wait), then solves a graph in the
same process.
"""
import ctypes as C
import time

import numpy as np
import pytest

import adds_b200 as A
from adds_b200 import _lib as L
from adds_b200 import graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ADDS_ERR_DEVICE_TIMEOUT = -6


def test_bounded_wait_times_out_and_context_survives():
    lib = L.lib()
    waited = C.c_double()
    t0 = time.perf_counter()
    rc = lib.adds_diag_wait_timeout(0, 50, C.byref(waited))
    wall = time.perf_counter() - t0
    assert rc == ADDS_ERR_DEVICE_TIMEOUT, rc
    assert b"wait site" in lib.adds_last_cuda_error()
    assert 45.0 <= waited.value < 5000.0 and wall < 10.0
    # the same process keeps solving on the same GPU
    g = G.rmat(12, 16, seed=3)
    src = G.max_degree_vertex(g)
    dg = A.Graph.from_csr(g)
    try:
        d, _ = dg.sssp(src, A.default_opts(timeout_ms=10000))
    finally:
        dg.close()
    ref, _ = O.dijkstra(g, src)
    assert np.array_equal(d, ref)
