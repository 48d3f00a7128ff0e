"""GPU parity: the engine's distances, through the C ABI, must equal the
CPU oracle's bit for bit (int32 and float32 folds)."""
import numpy as np
import pytest

import adds_b200 as A
from adds_b200 import graphs as G
from oracle import oracle as O

pytestmark = pytest.mark.gpu
OPTS = dict(timeout_ms=10000)
ASYNC, PHASE = 1, 2
# phase-engine kernel variants: (threads per CTA, CTAs per SM)
VARIANTS = [(256, 4), (512, 2), (1024, 1), (256, 2), (512, 1), (128, 8)]


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


@pytest.mark.parametrize("engine", [ASYNC, PHASE])
def test_rmat16_int_max_degree_source(engine):
    g = G.rmat(16, 16, seed=1)
    st = _check(g, G.max_degree_vertex(g), engine=engine)
    assert st["items_popped"] > 0 and st["engine"] == engine


@pytest.mark.parametrize("engine", [ASYNC, PHASE])
def test_grid_float_with_shortcuts(engine):
    g = G.grid(256, 256, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=3)
    _check(g, 128 * 256 + 128, engine=engine)


@pytest.mark.parametrize("engine", [ASYNC, PHASE])
def test_erdos_renyi_int(engine):
    g = G.erdos_renyi(20000, 8, seed=11)
    _check(g, 5, engine=engine)


@pytest.mark.parametrize("engine", [ASYNC, PHASE])
def test_sources_overlapped_copy_out(engine):
    """adds_sssp_sources: results of several sources into pageable, pinned
    and device buffers, one buffer reused (the later result wins), each equal
    to the oracle's distances for its source."""
    import torch
    g = G.rmat(14, 16, seed=5, w_hi=5000)
    deg = np.diff(g.row.astype(np.int64))
    srcs = [int(x) for x in np.random.default_rng(3).choice(np.flatnonzero(deg > 0), 6,
                                                             replace=False)]
    dg = A.Graph.from_csr(g)
    try:
        pageable = [np.full(g.n, 7, dtype=np.uint32) for _ in range(2)]
        pinned = torch.full((g.n,), 7, dtype=torch.int32).pin_memory()
        dev = torch.full((g.n,), 7, dtype=torch.int32, device="cuda")
        reuse = np.full(g.n, 7, dtype=np.uint32)
        outs = [pageable[0], pinned, dev, reuse, pageable[1], reuse]
        st = dg.sssp_sources(srcs, outs, A.default_opts(engine=engine, **OPTS))
        assert st["engine"] == engine and st["kernel_ms"] > 0
        got = [pageable[0], pinned.numpy().view(np.uint32), dev.cpu().numpy().view(np.uint32),
               None, pageable[1], reuse]
        for s, d in zip(srcs, got):
            if d is None:
                continue
            ref, _ = O.dijkstra(g, s)
            assert np.array_equal(d, ref), s
        # the last solve's distances also stay in the graph
        assert np.array_equal(dg.last_dist(), reuse)
    finally:
        dg.close()


@pytest.mark.parametrize("engine", [ASYNC, PHASE])
@pytest.mark.parametrize("shift", [0, 4, 9, 14, 20])
@pytest.mark.parametrize("lh", [0, 1])
def test_any_delta_gives_same_distances(engine, shift, lh):
    g = G.rmat(13, 16, seed=2)
    _check(g, G.max_degree_vertex(g), delta_shift=shift, light_heavy=lh, engine=engine)


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("solo", [0, 64, 100000])
@pytest.mark.parametrize("lh", [0, 1, 2])
def test_phase_schedules_int_rmat(variant, solo, lh):
    """Kernel variants, solo-CTA thresholds (0: never, 100000: whole solve on
    one CTA) and split rows (hub threshold 64 edges) all give the oracle's
    distances; shift 1 overflows the bucket ring into the far slot."""
    g = G.rmat(12, 16, seed=5, w_hi=10000)
    for shift in (1, 6, 9, 12):
        _check(g, 3, engine=PHASE, delta_shift=shift, light_heavy=lh, solo_max=solo,
               block_threads=variant[0], ctas_per_sm=variant[1], hub_threshold=64)


@pytest.mark.parametrize("wt", [G.I32, G.F32])
def test_tuner_then_auto_solves(wt):
    """adds_tune picks an engine and knobs on sample sources; later solves
    with default options use them and still match the oracle."""
    if wt == G.I32:
        g = G.rmat(15, 16, seed=21, w_hi=10000)
    else:
        g = G.grid(128, 96, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=22)
    deg = np.diff(g.row.astype(np.int64))
    srcs = [int(x) for x in np.random.default_rng(5).choice(np.flatnonzero(deg > 0), 3,
                                                             replace=False)]
    dg = A.Graph.from_csr(g)
    try:
        best, ms = dg.tune(srcs[:2])
        assert best.engine in (ASYNC, PHASE) and ms > 0 and best.delta_shift >= 0
        for s in srcs:
            d, st = dg.sssp(s, A.default_opts(**OPTS))
            assert st["engine"] == best.engine
            ref, _ = O.dijkstra(g, s)
            assert np.array_equal(d, ref), s
    finally:
        dg.close()


@pytest.mark.parametrize("lh", [0, 1, 2])
@pytest.mark.parametrize("solo", [0, 64])
@pytest.mark.parametrize("shift", [6, 10])
def test_near_far_schedule_int_rmat(lh, solo, shift):
    """The near-far comparator schedule (one far pile split against a moving
    threshold) reaches the oracle's distances, re-pushing what stays far."""
    g = G.rmat(14, 16, seed=9, w_hi=5000)
    st = _check(g, G.max_degree_vertex(g), engine=PHASE, near_far=1, light_heavy=lh,
                solo_max=solo, delta_shift=shift)
    assert st["engine"] == PHASE and st["repushes"] > 0


@pytest.mark.parametrize("lh", [0, 2])
def test_near_far_schedule_float_grid(lh):
    g = G.grid(96, 80, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=12)
    _check(g, 40 * 96 + 48, engine=PHASE, near_far=1, light_heavy=lh)


def test_near_far_batch():
    gs = [G.erdos_renyi(3000 + 500 * i, 8, seed=40 + i) for i in range(5)]
    dgs = [A.Graph.from_csr(g) for g in gs]
    try:
        b = A.Batch(dgs, [1, 2, 3, 4, 5], A.default_opts(engine=PHASE, near_far=1, **OPTS))
        b.run()
        for q, g in enumerate(gs):
            ref, _ = O.dijkstra(g, q + 1)
            assert np.array_equal(b.dist(q), ref), q
        b.close()
    finally:
        for d in dgs:
            d.close()


@pytest.mark.parametrize("engine", [ASYNC, PHASE])
@pytest.mark.parametrize("wt", [G.I32, G.F32])
def test_frontier_bellman_ford(engine, wt):
    """delta_shift 31 with light/heavy off is frontier Bellman-Ford (every
    distance in one bucket): the comparator the reference ran through nf/nv
    (nf_int.patch, nv_int/kernel.cu), here as a schedule of the same engine."""
    g = (G.rmat(13, 16, seed=14, w_hi=10000) if wt == G.I32 else
         G.grid(120, 90, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=15))
    _check(g, 0 if wt == G.F32 else G.max_degree_vertex(g), engine=engine, delta_shift=31,
           light_heavy=0)


def test_phase_trace_and_stats():
    """The phase trace records every decided phase in time order and the
    statistics account for the work (pops = stale + expanded)."""
    g = G.rmat(14, 16, seed=16, w_hi=10000)
    src = G.max_degree_vertex(g)
    dg = A.Graph.from_csr(g)
    try:
        dg.trace(4096)
        d, st = dg.sssp(src, A.default_opts(**OPTS, engine=PHASE, delta_shift=8, solo_max=64))
        tr, n = dg.trace_read(4096)
        dg.trace(0)
    finally:
        dg.close()
    ref, _ = O.dijkstra(g, src)
    assert np.array_equal(d, ref)
    assert n == len(tr) and n == st["phases"]  # one record per decision, exit included
    assert (np.diff(tr["t_ns"].astype(np.int64)) >= 0).all()
    modes = tr["mode"] & 0xFF
    assert modes[0] == 0 and modes[-1] == 4  # init first, exit last
    assert ((tr["mode"] & 0x100) != 0).sum() == st["solo_phases"]
    # per-phase work adds up to the solve's counters
    assert int(tr["edges"].astype(np.int64).sum()) == st["edges_scanned"]
    assert int(tr["pushes"].astype(np.int64).sum()) <= st["pushes"]
    assert (tr["tail_ns"][(tr["mode"] & 0x100) != 0] == 0).all()
    assert st["items_popped"] >= st["items_stale"] and st["edges_scanned"] > 0
    assert st["engine"] == PHASE and st["ctas"] > 0


@pytest.mark.parametrize("dense", [-1, 6, 20])
@pytest.mark.parametrize("lh", [0, 1, 2])
@pytest.mark.parametrize("adapt", [0, 1])
def test_dense_bucket_scan(dense, lh, adapt):
    """Dense bucket slots (dense_scan > 0): a slot that received more than
    max(n >> dense_scan, 4096) pushes stops storing them and its bucket is
    collected by a scan of the distances when it opens.  Distances stay the
    oracle's (int R-MAT, float grid); with the scan on, the trace shows scan
    phases (mode 6) on the R-MAT, whose big buckets pass the threshold."""
    g = G.rmat(15, 16, seed=24, w_hi=10000)
    src = G.max_degree_vertex(g)
    dg = A.Graph.from_csr(g)
    try:
        dg.trace(1 << 16)
        d, st = dg.sssp(src, A.default_opts(**OPTS, engine=PHASE, delta_shift=10, light_heavy=lh,
                                            adapt=adapt, dense_scan=dense))
        tr, n = dg.trace_read(1 << 16)
        dg.trace(0)
    finally:
        dg.close()
    ref, _ = O.dijkstra(g, src)
    assert np.array_equal(d, ref)
    scans = int(((tr["mode"] & 0xFF) == 6).sum())
    if dense < 0:
        assert scans == 0
    else:
        assert scans > 0
    f = G.grid(128, 96, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=25)
    _check(f, 48 * 128 + 64, engine=PHASE, delta_shift=14, light_heavy=lh, adapt=adapt,
           dense_scan=dense)


@pytest.mark.parametrize("ctas", [1, 16, 64])
def test_plain_solve_with_few_ctas(ctas):
    """group_ctas on a plain solve launches that many CTAs (a cheaper group
    barrier for small graphs); the distances stay the oracle's."""
    g = G.rmat(14, 16, seed=26, w_hi=1000)
    st = _check(g, G.max_degree_vertex(g), engine=PHASE, group_ctas=ctas)
    assert st["ctas"] == ctas
    f = G.grid(64, 48, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=27)
    _check(f, 24 * 64 + 32, engine=PHASE, group_ctas=ctas)


def test_dense_bucket_scan_batch():
    """Dense slots per query inside one batched launch (each query's scan
    reads its own distances)."""
    gs = [G.rmat(13, 16, seed=30 + i, w_hi=10000) for i in range(3)]
    dgs = [A.Graph.from_csr(g) for g in gs]
    try:
        srcs = [G.max_degree_vertex(g) for g in gs]
        b = A.Batch(dgs + dgs, srcs + [1, 2, 3],
                    A.default_opts(engine=PHASE, delta_shift=7, dense_scan=20, **OPTS))
        for _ in range(2):
            b.run()
            for q, (g, s) in enumerate(zip(gs + gs, srcs + [1, 2, 3])):
                ref, _ = O.dijkstra(g, s)
                assert np.array_equal(b.dist(q), ref), q
        b.close()
    finally:
        for x in dgs:
            x.close()


@pytest.mark.parametrize("variant", VARIANTS[:3])
@pytest.mark.parametrize("lh", [0, 1, 2])
def test_phase_schedules_float_grid(variant, lh):
    g = G.grid(96, 80, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=8)
    for shift in (6, 12, 16, 20):
        _check(g, 40 * 96 + 48, engine=PHASE, delta_shift=shift, light_heavy=lh,
               block_threads=variant[0], ctas_per_sm=variant[1], solo_max=256)


@pytest.mark.parametrize("adapt", [0, 1])
@pytest.mark.parametrize("solo", [0, 64])
@pytest.mark.parametrize("lh", [0, 1, 2])
def test_phase_bucket_widening(adapt, solo, lh):
    """The leader widens a bucket over up to four thin consecutive slots
    (adapt 1): the distances stay the oracle's, int32 and float32, with the
    far slot in use (shift 2 on the R-MAT, shift 8 on the grid)."""
    g = G.rmat(12, 16, seed=21, w_hi=10000)
    for shift in (2, 7, 11):
        _check(g, G.max_degree_vertex(g), engine=PHASE, delta_shift=shift, light_heavy=lh,
               solo_max=solo, adapt=adapt, hub_threshold=64)
    g = G.grid(150, 100, 0.02, 8, wtype=G.F32, w_lo=0.0, w_hi=3.0, seed=22)
    for shift in (8, 14):
        _check(g, 75, engine=PHASE, delta_shift=shift, light_heavy=lh, solo_max=solo,
               adapt=adapt)


def test_phase_bucket_widening_merges_thin_slots():
    """On a high-diameter grid with a narrow bucket, widening takes fewer
    phases than one bucket slot per phase, and the trace shows the base
    advancing by more than one bucket in a single light phase."""
    g = G.grid(160, 120, 0.0, 8, wtype=G.F32, w_lo=1.0, w_hi=2.0, seed=23)
    dg = A.Graph.from_csr(g)
    try:
        res = {}
        for adapt in (0, 1):
            dg.trace(1 << 16)
            d, st = dg.sssp(0, A.default_opts(**OPTS, engine=PHASE, delta_shift=14,
                                              solo_max=4096, adapt=adapt))
            tr, n = dg.trace_read(1 << 16)
            dg.trace(0)
            res[adapt] = (d, st, tr)
    finally:
        dg.close()
    ref, _ = O.dijkstra(g, 0)
    for adapt in (0, 1):
        assert np.array_equal(res[adapt][0], ref)
    assert res[1][1]["phases"] < res[0][1]["phases"]
    tr = res[1][2]
    light = (tr["mode"] & 0xFF) == 1
    steps = np.diff(tr["base"].astype(np.int64))[light[1:]]
    assert (steps > 1).any()


def test_adaptive_light_heavy_saves_phases():
    """light_heavy 2 relaxes whole rows once buckets turn sparse: the same
    distances as the split schedule in fewer phases, with no more than a few
    percent more edges (vertices re-improved inside a sparse bucket relax
    their heavy edges twice)."""
    g = G.rmat(17, 16, seed=31, w_hi=10000)
    src = G.max_degree_vertex(g)
    st = {lh: _check(g, src, engine=PHASE, delta_shift=10, light_heavy=lh) for lh in (1, 2)}
    assert st[2]["phases"] < st[1]["phases"]
    assert st[2]["edges_scanned"] <= 1.05 * st[1]["edges_scanned"]


def _pull_phases(g, src, **kw):
    """Distances, statistics and the number of pull phases of one solve."""
    dg = A.Graph.from_csr(g)
    try:
        dg.trace(1 << 14)
        d, st = dg.sssp(src, A.default_opts(**{**OPTS, **kw}))
        tr, _ = dg.trace_read(1 << 14)
        dg.trace(0)
    finally:
        dg.close()
    ref, _ = O.dijkstra(g, src)
    mism = np.flatnonzero(d != ref)
    assert mism.size == 0, f"{mism.size} mismatches, first {mism[:5]} got {d[mism[:5]]} want {ref[mism[:5]]}"
    return st, int(((tr["mode"] & 0xFF) == 7).sum())


@pytest.mark.parametrize("variant", [(256, 4), (1024, 1), (128, 8)])
def test_pull_heavy_phase_int_rmat(variant):
    """A giant bucket's heavy edges taken as a pull over the in-edges of the
    vertices above it (R-MAT, int weights U[1, 10000), bucket 2^10): a pull
    phase runs, the distances equal the oracle's, and fewer edges are read
    than with pushes only (pull = -1)."""
    g = G.rmat(17, 16, seed=41, w_hi=10000)
    src = G.max_degree_vertex(g)
    kw = dict(engine=PHASE, delta_shift=10, light_heavy=1, block_threads=variant[0],
              ctas_per_sm=variant[1])
    st_pull, npull = _pull_phases(g, src, pull=1, **kw)
    st_push, npush = _pull_phases(g, src, pull=-1, **kw)
    assert npull >= 1 and npush == 0
    assert st_pull["edges_scanned"] < st_push["edges_scanned"]
    # the launch chain (phase, pull, phase, pull, phase) against one launch
    assert st_pull["launches"] == 5 and st_push["launches"] == 1


@pytest.mark.parametrize("solo", [0, 1024])
@pytest.mark.parametrize("adapt", [0, 1])
def test_pull_with_widened_buckets(adapt, solo):
    """Pull phases next to on-device bucket widening: a widened light phase
    leaves vertices of several buckets in the settled list, whose heavy
    edges a pull above the top bucket would miss -- those lists go to a
    push.  Eight sources of an R-MAT with narrow buckets, each equal to the
    oracle."""
    g = G.rmat(17, 16, seed=47, w_hi=10000)
    deg = np.diff(g.row.astype(np.int64))
    srcs = [int(x) for x in np.random.default_rng(47).choice(np.flatnonzero(deg > 0), 8,
                                                              replace=False)]
    dg = A.Graph.from_csr(g)
    try:
        o = A.default_opts(**OPTS, engine=PHASE, delta_shift=9, light_heavy=2, adapt=adapt,
                           solo_max=solo, pull=1)
        for s in srcs:
            d, _ = dg.sssp(s, o)
            ref, _ = O.dijkstra(g, s)
            mism = np.flatnonzero(d != ref)
            assert mism.size == 0, f"source {s}: {mism.size} mismatches"
    finally:
        dg.close()


@pytest.mark.parametrize("lh", [1, 2])
def test_pull_heavy_phase_float(lh):
    """Float keys (the rounded lower bound of a heavy candidate): R-MAT with
    float weights and a float grid, pull on and off, equal to the oracle."""
    g = G.rmat(16, 16, seed=43, wtype=G.F32, w_lo=0.0, w_hi=1.0)
    src = G.max_degree_vertex(g)
    for shift in (4, 8, 12):
        _pull_phases(g, src, engine=PHASE, delta_shift=shift, light_heavy=lh, pull=1)
    gg = G.grid(128, 128, 0.02, 8, wtype=G.F32, w_lo=0.0, w_hi=3.0, seed=44)
    for shift in (8, 14):
        _pull_phases(gg, 64 * 128 + 64, engine=PHASE, delta_shift=shift, light_heavy=lh, pull=1)


def test_pull_after_weight_update_and_in_batch():
    """The in-edge copy follows adds_graph_set_weights; a batch of one query
    replays the launch chain of a pulled solve from its CUDA graph (twice),
    and a batch of several stays on pushes; all equal the oracle."""
    g = G.rmat(15, 16, seed=45, w_hi=10000)
    src = G.max_degree_vertex(g)
    dg = A.Graph.from_csr(g)
    try:
        o = A.default_opts(**OPTS, engine=PHASE, delta_shift=10, pull=1)
        d0, _ = dg.sssp(src, o)
        assert np.array_equal(d0, O.dijkstra(g, src)[0])
        w2 = (np.random.default_rng(7).integers(1, 10000, size=g.w.size)).astype(np.uint32)
        dg.set_weights(w2)
        d1, _ = dg.sssp(src, o)
        assert np.array_equal(d1, O.dijkstra(G.CSR(g.n, g.row, g.dst, w2, g.wtype), src)[0])
    finally:
        dg.close()
    graphs = [G.rmat(15, 16, seed=46 + i, w_hi=10000) for i in range(3)]
    dgs = [A.Graph.from_csr(x) for x in graphs]
    srcs = [G.max_degree_vertex(x) for x in graphs]
    try:
        for k in (1, 3):
            b = A.Batch(dgs[:k], srcs[:k],
                        A.default_opts(**OPTS, engine=PHASE, delta_shift=10, pull=1))
            try:
                for _ in range(2):
                    b.run()
                    for q, (x, s) in enumerate(zip(graphs[:k], srcs[:k])):
                        assert np.array_equal(b.dist(q), O.dijkstra(x, s)[0])
            finally:
                b.close()
    finally:
        for x in dgs:
            x.close()


def test_phase_float_grid_large_keys():
    """A high-diameter float grid with a narrow bucket (many slots, far-slot
    re-pushes) and zero-weight edges mixed in."""
    g = G.grid(200, 150, 0.02, 8, wtype=G.F32, w_lo=0.0, w_hi=3.0, seed=12)
    for shift in (8, 14):
        _check(g, 0, engine=PHASE, delta_shift=shift, solo_max=128)


@pytest.mark.parametrize("window", [1, 2, 4])
@pytest.mark.parametrize("lh", [0, 1])
@pytest.mark.parametrize("local", [0, 512])
@pytest.mark.parametrize("block", [128, 256, 512])
def test_schedules_int_rmat(window, lh, local, block):
    g = G.rmat(12, 16, seed=5, w_hi=10000)
    for shift in (6, 9, 12):
        _check(g, 3, engine=ASYNC, delta_shift=shift, window=window, light_heavy=lh,
               local_max=local, block_threads=block, hub_threshold=256)


@pytest.mark.parametrize("window", [1, 2])
@pytest.mark.parametrize("lh", [0, 1])
@pytest.mark.parametrize("block", [128, 512])
def test_schedules_float_grid(window, lh, block):
    g = G.grid(96, 80, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=8)
    for shift in (12, 16, 20):
        _check(g, 40 * 96 + 48, engine=ASYNC, delta_shift=shift, window=window,
               light_heavy=lh, block_threads=block)


@pytest.mark.parametrize("window", [1, 2, 4])
def test_async_window_adapted_on_device(window):
    """The async engine's on-device window (adapt 1: wider while CTAs find
    nothing inside it but entries beyond, narrower as buckets retire with no
    CTA idle) changes the schedule, not the distances."""
    g = G.grid(128, 96, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=31)
    for shift in (12, 16, 20):
        _check(g, 48 * 128 + 64, engine=ASYNC, adapt=1, window=window, delta_shift=shift)
    r = G.rmat(13, 16, seed=32, w_hi=10000)
    for shift in (5, 9, 12):
        _check(r, G.max_degree_vertex(r), engine=ASYNC, adapt=1, window=window,
               delta_shift=shift, hub_threshold=256)


def test_non_strict_order():
    g = G.rmat(12, 16, seed=6, w_hi=10000)
    for lh in (0, 1):
        _check(g, 1, engine=ASYNC, strict_order=0, light_heavy=lh, delta_shift=8)


@pytest.mark.parametrize("engine,group", [(ASYNC, 0), (PHASE, 0), (PHASE, 1), (PHASE, 7),
                                          (PHASE, 1000)])
def test_batch_mixed_graphs_replayed_twice(engine, group):
    gs = [G.erdos_renyi(3000 + 997 * i, 8, seed=100 + i) for i in range(5)]
    r = G.rmat(12, 16, seed=9)
    graphs = [A.Graph.from_csr(g) for g in gs] + [A.Graph.from_csr(r)]
    qg = graphs + [graphs[-1]] * 3
    srcs = [0, 1, 2, 3, 4, G.max_degree_vertex(r), 1, 2, 3]
    b = A.Batch(qg, srcs, A.default_opts(**OPTS, engine=engine, group_ctas=group))
    csrs = gs + [r] * 4
    for _ in range(2):  # second run replays the captured CUDA graph
        st = b.run()
        for q, (c, s) in enumerate(zip(csrs, srcs)):
            ref, _ = O.dijkstra(c, s)
            assert np.array_equal(b.dist(q), ref), f"query {q}"
    new = [5, 6, 7, 8, 9, 10, 11, 12, 13]
    b.set_sources(new)
    b.run()
    for q, (c, s) in enumerate(zip(csrs, new)):
        ref, _ = O.dijkstra(c, s)
        assert np.array_equal(b.dist(q), ref), f"query {q} after set_sources"
    b.close()
    for g in graphs:
        g.close()


@pytest.mark.parametrize("forced", [0, ASYNC, PHASE])
def test_batch_engine_follows_average_degree(forced):
    """With the engine left on auto, a batch of grids (average degree about
    4) runs on the asynchronous engine and a batch of R-MAT graphs (16) on
    the phase engine; a named engine wins.  A graph's single-solve tuning
    does not decide it.  Distances equal the oracle's either way."""
    grids = [G.grid(64 + 16 * i, 40 + 8 * i, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0,
                    seed=60 + i) for i in range(3)]
    rmats = [G.rmat(11 + (i % 2), 16, seed=70 + i, w_hi=5000) for i in range(3)]
    for csrs, auto in ((grids, ASYNC), (rmats, PHASE)):
        graphs = [A.Graph.from_csr(c) for c in csrs]
        try:
            if csrs is rmats:  # tuned for plain solves: must not steer the batch
                graphs[-1].tune([1], A.default_opts(engine=ASYNC))
            srcs = [3, 7, 11]
            b = A.Batch(graphs, srcs, A.default_opts(**OPTS, engine=forced))
            st = b.run()
            assert st["engine"] == (forced or auto)
            for q, (c, s) in enumerate(zip(csrs, srcs)):
                ref, _ = O.dijkstra(c, s)
                assert np.array_equal(b.dist(q), ref), f"query {q}"
            b.close()
        finally:
            for g in graphs:
                g.close()


def test_cli_int_matches_reference_text(tmp_path):
    import os
    import subprocess
    g = G.rmat(12, 16, seed=4)
    p = str(tmp_path / "r12.gr")
    G.write_gr(p, g)
    out = str(tmp_path / "out.txt")
    rec = str(tmp_path / "fd3.txt")
    exe = os.path.join(os.path.dirname(A._lib.HERE), "adds_b200", "bin", "sssp_int")
    r = subprocess.run(["bash", "-c", f'"{exe}" -q -s 7 -r 2 -o "{out}" "{p}" 3>"{rec}"'],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    ref, _ = O.dijkstra(g, 7)
    assert open(out).read() == G.dist_text(ref, G.I32)
    name, ms, work = open(rec).read().split()
    assert name == "r12.gr" and float(ms) > 0 and int(work) > 0


def test_cli_float_text_and_raw_words_match_oracle(tmp_path):
    """sssp_float as run_all.sh runs it: the "%d %f" text equals the
    oracle's, the raw words (-b) equal the oracle's bit for bit, and the
    checker (python -m adds_b200.verify) agrees; the fd-3 record counts
    scanned edges, as the reference float build does."""
    import os
    import subprocess
    import sys
    g = G.grid(96, 80, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=44)
    src = 40 * 96 + 48
    d1, d2 = tmp_path / "ours", tmp_path / "oracle"
    d1.mkdir()
    d2.mkdir()
    p = str(tmp_path / "g96.gr")
    G.write_gr(p, g)
    rec = str(tmp_path / "fd3.txt")
    exe = os.path.join(os.path.dirname(A._lib.HERE), "adds_b200", "bin", "sssp_float")
    cmd = f'"{exe}" -q -s {src} -o "{d1}/g96.gr" -b "{d1}/g96.bin" "{p}" 3>"{rec}"'
    r = subprocess.run(["bash", "-c", cmd], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    ref, _ = O.dijkstra(g, src)
    assert open(f"{d1}/g96.gr").read() == G.dist_text(ref, G.F32)
    assert np.array_equal(np.fromfile(f"{d1}/g96.bin", dtype="<u4"), ref)
    name, ms, work = open(rec).read().split()
    assert name == "g96.gr" and float(ms) > 0 and int(work) >= g.m // 2
    (d2 / "g96.gr").write_text(G.dist_text(ref, G.F32))
    ref.astype("<u4").tofile(str(d2 / "g96.bin"))
    lst = tmp_path / "list"
    lst.write_text(f"g96.gr\t{src}\ng96.bin\t{src}\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    v = subprocess.run([sys.executable, "-m", "adds_b200.verify", f"{d1}/", f"{d2}/", str(lst),
                        "--float"], capture_output=True, text=True, cwd=root, timeout=120)
    assert v.returncode == 0 and "all results match!!!" in v.stdout, v.stdout


@pytest.mark.parametrize("name", ["ref_rmat16_int", "ref_rmat12_int", "ref_grid96_float"])
def test_engine_matches_reference_adds_output(name):
    """The engine against what the reference ADDS binary itself printed
    (tests/golden/ref_*.npz, see tests/golden/make_ref_golden.py)."""
    import gzip
    import importlib.util
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("mrg", os.path.join(here, "make_ref_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    build, rule, binary = m.CASES[name]
    g = build()
    z = np.load(os.path.join(here, name + ".npz"))
    dg = A.Graph.from_csr(g)
    d, _ = dg.sssp(int(z["src"]), A.default_opts(**OPTS))
    dg.close()
    if binary == "ads_int_sssp":
        assert np.array_equal(d, z["dist"])
    else:
        assert G.dist_text(d, G.F32) == gzip.decompress(z["text_gz"].tobytes()).decode()


def test_relax_ceiling_diagnostic():
    """adds_diag_relax_pass: four positive pass times; the pass with the
    gather is not faster than the pure stream."""
    g = G.rmat(15, 16, seed=17, w_hi=10000)
    dg = A.Graph.from_csr(g)
    try:
        ms = dg.relax_ceiling(G.max_degree_vertex(g))
    finally:
        dg.close()
    assert len(ms) == 4 and all(x > 0 for x in ms)
