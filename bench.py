#!/usr/bin/env python3
"""Benchmark of the asynchronous delta-stepping SSSP engine.

Headline workload (default): R-MAT scale 24 (16.8M vertices, 16 directed
draws per vertex, a/b/c/d = .57/.19/.19/.05, self-loops and duplicates
removed), int32 weights uniform in [1, 10000], 8 seeded sources with
out-degree > 0.  A step is one solve from the next source.  Metric: GTEPS =
out-edges of the reached vertices / solve time (the Graph500 convention).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload rmat24|rmat16|rmat21|rmat22|grid4096|rmat26|batched|diff]

--impl reference times the reference's CPU delta-stepping path (Galois
OBIM delta-stepping, restated in oracle/oracle.c because Galois is not
vendored) with all host threads on a bounded sample of the same workload.
Inputs are generated by seeded synthetic generators (the reference's
SuiteSparse/DIMACS/SNAP files are not available).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


# ---------------------------------------------------------------- utilities
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, device: int, path: str):
        self.path = path
        self.proc = None
        try:
            self.f = open(path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={device}", f"--query-gpu={SMI_FIELDS}", "--format=csv",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9 or not p[1].split()[0].isdigit():
                    continue
                sm.append(int(p[1].split()[0]))
                mx.append(int(p[2].split()[0]))
                for nm, val in zip(names[1:], p[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": int(statistics.median(loaded)), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def clock_dir():
    """Where the nvidia-smi clock samples of the timed region are written
    (ADDS_BENCH_OUT, else the temporary directory)."""
    import tempfile
    return os.environ.get("ADDS_BENCH_OUT") or tempfile.gettempdir()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name: str):
    """dram bytes per launch from a committed ncu summary (profiles/*.json)."""
    p = os.path.join(ROOT, "profiles", f"{name}.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


# ---------------------------------------------------------------- workloads
WORKLOADS = {
    "rmat24": dict(kind="rmat", scale=24, wtype=0, w_lo=1, w_hi=10000, nsrc=8, seed=24),
    "rmat26": dict(kind="rmat", scale=26, wtype=1, w_lo=0.0, w_hi=1.0, nsrc=8, seed=26),
    "rmat16": dict(kind="rmat", scale=16, wtype=0, w_lo=1, w_hi=1000, nsrc=1, seed=16,
                   src="maxdeg"),
    "rmat21": dict(kind="rmat", scale=21, wtype=0, w_lo=1, w_hi=10000, nsrc=8, seed=21),
    "rmat22": dict(kind="rmat", scale=22, wtype=0, w_lo=1, w_hi=10000, nsrc=8, seed=22),
    "rmat23": dict(kind="rmat", scale=23, wtype=0, w_lo=1, w_hi=10000, nsrc=8, seed=23),
    "grid4096": dict(kind="grid", side=4096, wtype=1, w_lo=1.0, w_hi=100.0, nsrc=1, seed=4096,
                     src="center"),
}


def make_graph(wl: dict, device: int):
    import adds_b200 as A
    if wl["kind"] == "rmat":
        spec = A.gen_spec("rmat", scale=wl["scale"], edge_factor=16, a=0.57, b=0.19, c=0.19,
                          wtype=wl["wtype"], w_lo=wl["w_lo"], w_hi=wl["w_hi"], seed=wl["seed"])
    else:
        spec = A.gen_spec("grid", side=wl["side"], shortcut_frac=0.02, radius=8,
                          wtype=wl["wtype"], w_lo=wl["w_lo"], w_hi=wl["w_hi"], seed=wl["seed"])
    return A.Graph.generate(spec, device)


def pick_sources(g, wl: dict, row: np.ndarray):
    deg = np.diff(row)
    if wl.get("src") == "maxdeg":
        return [int(np.argmax(deg))]
    if wl.get("src") == "center":
        s = wl["side"]
        return [(s // 2) * s + s // 2]
    rng = np.random.default_rng(wl["seed"])
    cand = np.flatnonzero(deg > 0)
    return [int(x) for x in rng.choice(cand, size=wl["nsrc"], replace=False)]


def describe(wl_name: str, wl: dict):
    if wl["kind"] == "rmat":
        w = (f"int32 U[{wl['w_lo']},{wl['w_hi']}]" if wl["wtype"] == 0
             else f"float32 U[{wl['w_lo']},{wl['w_hi']})")
        return {"workload": f"{wl_name}: R-MAT scale {wl['scale']}, edge factor 16, "
                            f"a/b/c/d=.57/.19/.19/.05, {w}, {wl['nsrc']} source(s)",
                "scale": wl["scale"], "edge_factor": 16, "sources": wl["nsrc"], "seed": wl["seed"]}
    return {"workload": f"{wl_name}: {wl['side']}x{wl['side']} 4-neighbour grid + 2% shortcuts "
                        f"(Manhattan radius 8), float32 U[{wl['w_lo']},{wl['w_hi']}), centre source",
            "side": wl["side"], "sources": 1, "seed": wl["seed"]}


# ---------------------------------------------------------------- distributed
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws, local):
    if ws <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def barrier(dist, local):
    if dist is None:
        return
    import torch
    if torch.cuda.is_available():
        t = torch.ones(1, device=f"cuda:{local}")
        dist.all_reduce(t)
        torch.cuda.synchronize(local)
    else:
        dist.barrier()


def reduce_max_sum(dist, local, tmax, usum):
    if dist is None:
        return tmax, usum
    import torch
    dev = f"cuda:{local}" if torch.cuda.is_available() else "cpu"
    a = torch.tensor([tmax], dtype=torch.float64, device=dev)
    b = torch.tensor([usum], dtype=torch.float64, device=dev)
    dist.all_reduce(a, op=dist.ReduceOp.MAX)
    dist.all_reduce(b, op=dist.ReduceOp.SUM)
    return float(a.item()), float(b.item())


def shard_queries(nq: int, ws: int, rank: int):
    """Queries of a batch this rank solves: every ws-th one from its rank
    (round-robin, so ranks get a similar mix of sizes).  No exchange is
    needed while solving: the queries are independent."""
    return list(range(rank, nq, ws))


def gather_to_root(dist, local, words: np.ndarray):
    """Host gather of each rank's flat result words (uint32, any length) to
    rank 0; returns the per-rank arrays in rank order on rank 0, None
    elsewhere.  One collective for the lengths, one for the padded data."""
    if dist is None:
        return [words]
    import torch
    ws, rank = dist.get_world_size(), dist.get_rank()
    dev = f"cuda:{local}" if torch.cuda.is_available() else "cpu"
    n = torch.tensor([words.size], dtype=torch.int64, device=dev)
    sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(ws)]
    dist.all_gather(sizes, n)
    cap = int(max(int(s.item()) for s in sizes))
    buf = torch.zeros(cap, dtype=torch.int32, device=dev)
    buf[:words.size] = torch.from_numpy(words.view(np.int32)).to(dev)
    parts = [torch.zeros(cap, dtype=torch.int32, device=dev) for _ in range(ws)] if rank == 0 \
        else None
    dist.gather(buf, parts, dst=0)
    if rank != 0:
        return None
    return [p[:int(s.item())].cpu().numpy().view(np.uint32) for p, s in zip(parts, sizes)]


# ---------------------------------------------------------------- CPU arm
CPU_NOTE = ("the CPU path is oracle/oracle.c's restatement of the Galois delta-stepping the "
            "reference compares against (cpu_sssp_int.patch): buckets keyed dist >> shift (float: "
            "dist / div), bulk-synchronous over pthreads; Galois runs it asynchronously with OBIM "
            "chunked buckets, and its source is not vendored, so the port's speed is not pinned "
            "to it")


def cpu_pick_bucket(csr, src, threads, budget_s=20.0):
    """Bucket width of the CPU delta-stepping: the fastest of a few
    candidates on one source (the timing of this choice is not reported)."""
    from oracle import oracle as O
    if csr.wtype == 0:
        cands = [dict(shift=s) for s in (8, 10, 12, 13)]
    else:
        aw = float(csr.weights().mean()) if csr.m else 1.0
        cands = [dict(div=aw * f) for f in (0.25, 1.0, 4.0)]
    best, best_t, t_used = None, 1e30, 0.0
    for c in cands:
        _, _, ms = O.delta_step(csr, src, threads=threads, **c)
        t_used += ms / 1e3
        if ms < best_t:
            best, best_t = c, ms
        if t_used > budget_s:
            break
    return best


def cpu_delta_step(csr, srcs, budget_s=20.0, threads=None):
    """Times the CPU delta-stepping restatement (Galois OBIM semantics) on
    sources until the time budget is spent; picks the bucket width first on
    the first source.  Returns GTEPS, a description and the distances of
    every source it solved (the oracle's fixed point, used as the parity
    check of the GPU solves)."""
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    deg = np.diff(csr.row.astype(np.int64))
    best = cpu_pick_bucket(csr, srcs[0], threads, budget_s)
    edges, secs, used, dists = 0, 0.0, [], {}
    for s in srcs:
        d, work, ms = O.delta_step(csr, s, threads=threads, **best)
        reached = d != (0x7FFFFFFF if csr.wtype == 0 else 0x7F7FFFFF)
        edges += int(deg[reached].sum())
        secs += ms / 1e3
        used.append(s)
        dists[s] = d
        if secs > budget_s:
            break
    return edges / secs / 1e9, dict(best=best, sources=used, threads=threads, secs=secs), dists


# ---------------------------------------------------------------- our arm
def run_ours(args, wl_name, wl, ws, rank, local, dist):
    import adds_b200 as A
    g = make_graph(wl, local)
    csr_row = g.download().row if wl["kind"] == "grid" else None
    if csr_row is None:
        csr_row = np.empty(g.n + 1, dtype=np.uint64)
        A.check(A.lib().adds_graph_download(g.handle, csr_row.ctypes.data, None, None))
    srcs = pick_sources(g, wl, csr_row)
    tuned, tune_ms = None, None
    extra_opts = json.loads(args.opts) if args.opts else {}
    if not args.no_tune:
        tuned, tune_ms = g.tune(srcs[:2], A.default_opts(engine=args.engine))
    opts = A.default_opts(timeout_ms=60000, engine=args.engine, **extra_opts)
    # per-source reached vertices / edges and distances (outside the timed
    # region; the distances are checked against the CPU oracle below)
    mr, nr, gpu_d = {}, {}, {}
    check_parity = rank == 0 and ws == 1 and not args.no_cpu
    for s in srcs:
        d, _ = g.sssp(s, opts)
        nr[s], mr[s] = g.reached()
        if check_parity:
            gpu_d[s] = d
    for i in range(args.warmup):
        g.sssp_async(srcs[i % len(srcs)], opts)
    g.sync()
    steps = [srcs[i % len(srcs)] for i in range(args.steps)]
    import torch
    torch.cuda.set_device(local)
    barrier(dist, local)
    torch.cuda.synchronize(local)
    smi = ClockSampler(local, os.path.join(clock_dir(), f"clocks_rank{rank}.csv"))
    t0 = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # solves run on the graph's own stream; bracket with host syncs + events
    ev0.record()
    torch.cuda.synchronize(local)
    t_host0 = time.perf_counter()
    for s in steps:
        g.sssp_async(s, opts)
    st = g.sync()
    t_host1 = time.perf_counter()
    ev1.record()
    torch.cuda.synchronize(local)
    clocks = smi.stop()
    barrier(dist, local)
    # the whole bracket on the device clock (includes any host enqueue gaps)
    elapsed = ev0.elapsed_time(ev1) / 1e3
    wall = t_host1 - t_host0
    units = sum(mr[s] for s in steps)
    tmax, usum = reduce_max_sum(dist, local, elapsed, units)
    value = usum / tmax / 1e9
    kernel_s = st["kernel_ms"] / 1e3
    balg = sum(12 * mr[s] + 24 * nr[s] for s in steps)
    peak, peak_kind = measured_peaks()
    achieved = balg / kernel_s / 1e9
    kname = "phase_kernel" if st["engine"] == 2 else "solve_kernel"
    prof = profile_traffic(f"{kname}_{wl_name}")
    traffic = None
    if prof and "dram_bytes_per_launch" in prof:
        traffic = prof["dram_bytes_per_launch"]
    # e2e: the C-ABI call with a pinned host output buffer, copies timed
    e2e_steps = steps[: max(1, min(len(steps), args.e2e_steps))]
    # every step's distances land in host memory: a ring of pinned buffers,
    # as a consumer that takes each result before the ring comes round
    ring = [torch.empty(g.n, dtype=torch.int32, pin_memory=True)
            for _ in range(min(4, len(e2e_steps)))]
    outs = [ring[i % len(ring)] for i in range(len(e2e_steps))]
    g.sssp_sources(e2e_steps[:2], outs[:2], opts)  # staging buffers made outside the timing
    barrier(dist, local)
    te0 = time.perf_counter()
    g.sssp_sources(e2e_steps, outs, opts)
    te1 = time.perf_counter()
    e2e_units = sum(mr[s] for s in e2e_steps)
    etmax, eusum = reduce_max_sum(dist, local, te1 - te0, e2e_units)
    e2e = {"value": eusum / etmax / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": 4,
           "d2h_bytes_per_step": 4 * g.n,
           "note": "adds_sssp_sources(graph, sources, a ring of 4 pinned host distance "
                   "arrays): each step's result is copied to host memory while the next step "
                   "solves; host wall clock; the 4-byte source id is the step input, the "
                   "distance array the result"}
    work_edges = st["edges_scanned"]
    # run-to-run spread: the timed steps again, one synchronous solve each
    # (outside the timed region; per-solve device time of the kernel)
    each = []
    for s_ in steps:
        _, st1 = g.sssp(s_, opts)
        each.append(st1["kernel_ms"])
    each_sorted = sorted(each)
    med = statistics.median(each_sorted)
    if args.trace:  # one more solve with the phase trace on (outside the timed region)
        g.trace(1 << 16)
        g.sssp(steps[0], opts)
        tr, ntr = g.trace_read(1 << 16)
        g.trace(0)
        np.save(args.trace, tr)
    out = {
        "metric": "sssp_gteps", "value": value, "unit": "GTEPS", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tmax / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32" if wl["wtype"] == 0 else "float32", "data": "synthetic",
        "config": {**describe(wl_name, wl), "parallelism": f"replicas{ws}",
                   "l2": "inputs larger than L2 (CSR > 126 MB), no flush"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind,
                     "kernel": ("adds_phase::phase_kernel (+ pull_kernel)" if st["engine"] == 2
                                else "adds::solve_kernel")
                               + f" (persistent, {st['launches']} launches per solve)",
                     "traffic_note": (prof or {}).get("scaled_by"),
                     "dram_gbs": (traffic / (kernel_s / args.steps) / 1e9) if traffic else None,
                     "l2_hit_rate_pct": (prof or {}).get("l2_hit_rate_pct"),
                     "bytes_model": "12*m_r + 24*n_r per solve"},
        "e2e": e2e,
        # phase engine: one persistent kernel per solve, or a chain of five
        # (phase, pull, phase, pull, phase) where pull phases are possible;
        # asynchronous engine: its init kernel and its persistent kernel
        "gpu_launches": st["launches"] * args.steps,
        "clocks": clocks,
        "extra": {
            "n": g.n, "m": g.m, "sources": srcs, "m_r": [mr[s] for s in srcs],
            "n_r": [nr[s] for s in srcs], "kernel_ms_per_step": st["kernel_ms"] / args.steps,
            "solve_ms_per_step": st["ms"] / args.steps, "host_wall_s": wall,
            "device_sum_of_solves_s": st["ms"] / 1e3,
            "work_gteps_last": None, "edges_scanned_last": work_edges,
            "items_last": st["items_popped"], "stale_last": st["items_stale"],
            "pushes_last": st["pushes"], "ctas": st["ctas"], "engine": st["engine"],
            "phases_last": st["phases"], "solo_phases_last": st["solo_phases"],
            "chunks_last": st["batches"],
            "phase_cycles_last": st["phase_cycles"] + [st["mid_flush_cycles"], st["mid_flushes"]],
            "tuned": ({k: getattr(tuned, k) for k in ("engine", "delta_shift", "block_threads",
                                                        "ctas_per_sm", "solo_max",
                                                        "hub_threshold", "light_heavy", "window",
                                                        "batch_max", "strict_order", "adapt",
                                                        "local_max", "greed", "group_ctas",
                                                        "dense_scan", "pull")}
                      if tuned else None),
            "lib": os.path.relpath(A._lib.LIB_PATH, ROOT),
            "tune_ms_per_solve": tune_ms,
            "solve_kernel_ms_each": each,
            "solve_kernel_ms_median": med,
            "solve_kernel_ms_spread_pct": 100.0 * (each_sorted[-1] - each_sorted[0]) / med,
        },
    }
    if check_parity:
        csr = g.download()
        gteps, info, cpu_d = cpu_delta_step(csr, srcs, budget_s=args.cpu_budget)
        out["cpu_baseline"] = {
            "value": gteps, "unit": "GTEPS", "cores": info["threads"], "kind": "port",
            "sample": (f"CPU delta-stepping (oracle/oracle.c) on the same graph, "
                       f"{len(info['sources'])} of the {len(srcs)} sources, "
                       f"{info['threads']} threads, bucket {info['best']}, {info['secs']:.1f} s"),
            "note": CPU_NOTE}
        # bit-exact parity: every source's GPU distances, and the distances
        # the last timed end-to-end steps delivered to host memory
        checked, bad = 0, 0
        for s, d in gpu_d.items():
            if s in cpu_d:
                checked += 1
                bad += int(not np.array_equal(d, cpu_d[s]))
        tail = list(range(max(0, len(e2e_steps) - len(ring)), len(e2e_steps)))
        e2e_checked, e2e_bad = 0, 0
        for i in tail:
            s = e2e_steps[i]
            if s in cpu_d:
                e2e_checked += 1
                e2e_bad += int(not np.array_equal(outs[i].numpy().view(np.uint32), cpu_d[s]))
        out["parity"] = {"sources_checked": checked, "mismatches": bad,
                         "timed_e2e_outputs_checked": e2e_checked, "timed_e2e_mismatches": e2e_bad,
                         "checker": "oracle delta-stepping (oracle/oracle.c) on the host, "
                                    "bit for bit"}
    g.close()
    return out


def make_host_graph(wl: dict, threads: int):
    """The workload's graph built on the host by the oracle's generator
    (oracle/gen.c, identical to the GPU generator's output); the reference
    arm uses it so that it loads no library of this package."""
    from oracle import oracle as O
    if wl["kind"] == "rmat":
        return O.gen_rmat(wl["scale"], 16, 0.57, 0.19, 0.19, wtype=wl["wtype"], w_lo=wl["w_lo"],
                          w_hi=wl["w_hi"], seed=wl["seed"], threads=threads)
    return O.gen_grid(wl["side"], wl["side"], 0.02, 8, wtype=wl["wtype"], w_lo=wl["w_lo"],
                      w_hi=wl["w_hi"], seed=wl["seed"], threads=threads)


def run_reference(args, wl_name, wl, ws, rank, local):
    """The reference's CPU path (Galois delta-stepping restated) on the same
    workload; each step is one CPU solve, bounded by the time budget.  The
    input graph comes from the host generator: nothing of the GPU product is
    loaded.  The bucket width is chosen as the CPU leg of our arm chooses it."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    csr = make_host_graph(wl, threads)  # input preparation only (not timed)
    srcs = pick_sources(None, wl, csr.row)
    kw = cpu_pick_bucket(csr, srcs[0], threads)
    deg = np.diff(csr.row.astype(np.int64))
    inf = 0x7FFFFFFF if csr.wtype == 0 else 0x7F7FFFFF
    total_edges, total_s = 0, 0.0
    for i in range(args.warmup + args.steps):
        s = srcs[i % len(srcs)]
        d, work, ms = O.delta_step(csr, s, threads=threads, **kw)
        if i >= args.warmup:
            total_edges += int(deg[d != inf].sum())
            total_s += ms / 1e3
        if i >= args.warmup and total_s > args.cpu_budget * 6:
            break
    v = total_edges / total_s / 1e9
    return {
        "impl": "reference", "metric": "sssp_gteps", "value": v, "unit": "GTEPS", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32" if wl["wtype"] == 0 else "float32",
        "data": "synthetic", "config": {**describe(wl_name, wl), "parallelism": "cpu"},
        "cpu_baseline": {"value": v, "unit": "GTEPS", "cores": threads, "kind": "port",
                         "sample": f"CPU delta-stepping restatement, bucket {kw} (the fastest "
                                   f"of the candidates on the first source), {threads} threads, "
                                   f"one solve per step",
                         "note": CPU_NOTE},
        "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_batched(args, ws, rank, local, dist):
    """256 solves of uneven size in one persistent, graph-captured launch:
    192 Erdos-Renyi graphs (n log-uniform in [1e3, 1e6], 8 draws per vertex,
    int weights U[1,1000]) and 64 distinct sources on one R-MAT 20 graph.
    Compared with a host loop of plain solves of the same queries.  With N
    ranks the batch is sharded by query (shard_queries: each GPU solves its
    queries in one launch of its own, no exchange while solving) and the
    end-to-end leg gathers every query's distances on rank 0's host
    (gather_to_root); the total work is fixed, so the scaling is strong."""
    import adds_b200 as A
    import torch
    rng = np.random.default_rng(4096)
    ns = np.exp(rng.uniform(np.log(1e3), np.log(1e6), size=192)).round().astype(int)
    er_src = [int(rng.integers(0, int(n))) for n in ns]  # an ER graph of n vertices has g.n == n
    mine = shard_queries(256, ws, rank)
    graphs, qg, qs = {}, [], []
    for i in (q for q in mine if q < 192):
        graphs[i] = A.Graph.generate(A.gen_spec("er", n=int(ns[i]), edge_factor=8, wtype=0,
                                                w_lo=1, w_hi=1000, seed=10_000 + i), local)
    r20 = A.Graph.generate(A.gen_spec("rmat", scale=20, wtype=0, w_lo=1, w_hi=1000, seed=20),
                           local)
    row = np.empty(r20.n + 1, dtype=np.uint64)
    A.check(A.lib().adds_graph_download(r20.handle, row.ctypes.data, None, None))
    cand = np.flatnonzero(np.diff(row) > 0)
    rsrc = [int(x) for x in rng.choice(cand, size=64, replace=False)]
    for q in mine:
        qg.append(graphs[q] if q < 192 else r20)
        qs.append(er_src[q] if q < 192 else rsrc[q - 192])
    opts = A.default_opts(timeout_ms=60000, engine=args.engine,
                          **(json.loads(args.opts) if args.opts else {}))
    # the autotuner picks per-graph knobs on a representative member
    if not args.no_tune:
        r20.tune(rsrc[:2])
        big = max(graphs, key=lambda i: ns[i]) if graphs else None
        if big is not None:
            graphs[big].tune([er_src[big]])
    b = A.Batch(qg, qs, opts)
    for _ in range(args.warmup):
        b.run()
    torch.cuda.set_device(local)
    barrier(dist, local)
    torch.cuda.synchronize(local)
    smi = ClockSampler(local, os.path.join(clock_dir(), f"clocks_batched_rank{rank}.csv"))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    torch.cuda.synchronize(local)
    kms = 0.0
    for _ in range(args.steps):
        b.launch()
        st = b.sync()
        kms += st["kernel_ms"]
    ev1.record()
    torch.cuda.synchronize(local)
    clocks = smi.stop()
    elapsed = ev0.elapsed_time(ev1) / 1e3
    tmax, usum = reduce_max_sum(dist, local, elapsed, float(len(qs) * args.steps))
    value = usum / tmax
    # the same queries as a host loop of plain solves
    uniq = list({id(g): g for g in qg}.values())
    for g, s in zip(qg, qs):
        g.sssp_async(s, opts)
    for g in uniq:
        g.sync()
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        for g, s in zip(qg, qs):
            g.sssp_async(s, opts)
        for g in uniq:
            g.sync()
    loop_s = (time.perf_counter() - t0) / max(1, args.steps // 2)
    loop_max, _ = reduce_max_sum(dist, local, loop_s, 0.0)
    loop_solves_per_s = 256 / loop_max
    # e2e: run through the C ABI, copy every distance array to pinned host
    # memory, and (N ranks) gather all of them on rank 0's host
    tot_n = int(b.layout()[1])
    host = torch.empty(tot_n, dtype=torch.int32, pin_memory=True)
    reps = max(1, args.steps // 2)
    barrier(dist, local)
    te0 = time.perf_counter()
    gathered = 0
    for _ in range(reps):
        b.run()
        b.dist_all(host.data_ptr())  # every query's distances, one copy
        parts = gather_to_root(dist, local, host.numpy().view(np.uint32))
        if parts is not None:
            gathered = sum(p.size for p in parts)
    e2e_s = (time.perf_counter() - te0) / reps
    e2e_max, _ = reduce_max_sum(dist, local, e2e_s, 0.0)
    out = {
        "metric": "batched_sssp_solves_per_s", "value": value, "unit": "solves/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tmax / args.steps * 1e3, "higher_is_better": True,
        "scaling": "strong" if ws > 1 else "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": "batched: 192 ER graphs (n log-uniform [1e3,1e6], 8 draws/vertex, "
                               "U[1,1000]) + 64 sources on R-MAT 20, one graph-captured launch "
                               "per GPU, queries sharded round-robin over the GPUs",
                   "queries": 256, "queries_this_rank": len(qs), "vertices_this_rank": tot_n,
                   "parallelism": f"query-sharded{ws}"},
        "loop_of_plain_solves_per_s": loop_solves_per_s,
        "speedup_vs_loop": value / loop_solves_per_s,
        "e2e": {"value": 256 / e2e_max, "unit": "solves/s",
                "h2d_bytes_per_step": 4 * len(qs), "d2h_bytes_per_step": 4 * tot_n,
                "gathered_words_on_rank0": gathered},
        "gpu_launches": st["launches"] * args.steps, "clocks": clocks,
        "extra": {"kernel_ms_per_launch": kms / args.steps},
    }
    b.close()
    for g in graphs.values():
        g.close()
    r20.close()
    return out


def run_diff(args, ws, rank, local, dist):
    """Differentiable batched SSSP: 128 grids (side log-uniform [64,512]),
    w = softplus(theta), theta ~ N(0,1); 16 sources and 64 targets per grid;
    L = sum c_t d(s,t), c_t ~ U(0,1).  A step is forward + backward."""
    import torch

    import adds_b200 as A
    from adds_b200.autograd import batched_sssp
    torch.cuda.set_device(local)
    rng = np.random.default_rng(128)
    sides = np.exp(rng.uniform(np.log(64), np.log(512), size=128)).round().astype(int)
    graphs, thetas, targets, coefs = [], [], [], []
    gen = torch.Generator(device="cuda").manual_seed(128)
    for i, sd in enumerate(sides):
        g = A.Graph.generate(A.gen_spec("plain_grid", side=int(sd), wtype=1, w_lo=1.0, w_hi=2.0,
                                        seed=500 + i), local)
        graphs.append(g)
        thetas.append(torch.randn(g.m, generator=gen, device="cuda"))
        t = torch.from_numpy(rng.choice(g.n, size=64, replace=False)).cuda()
        targets.append(t)
        coefs.append(torch.from_numpy(rng.uniform(0, 1, size=64).astype(np.float32)).cuda())
    qg, qs, qi = [], [], []
    for i, g in enumerate(graphs):
        for s in rng.choice(g.n, size=16, replace=False):
            qg.append(g)
            qs.append(int(s))
            qi.append(i)
    for g, th in zip(graphs, thetas):  # set weights once so the tuner sees them
        g.set_weights(torch.nn.functional.softplus(th).contiguous().data_ptr())
    if not args.no_tune:
        big = int(np.argmax(sides))
        graphs[big].tune([qs[qi.index(big)]])
    b = A.Batch(qg, qs, A.default_opts(timeout_ms=60000, engine=args.engine,
                                       **(json.loads(args.opts) if args.opts else {})))
    params = [th.clone().requires_grad_(True) for th in thetas]
    off = torch.from_numpy(b.layout()[0].astype(np.int64)).cuda()
    # flat indices of (query, target) pairs and their coefficients
    gidx = torch.cat([off[q] + targets[qi[q]] for q in range(len(qg))])
    gcoef = torch.cat([coefs[qi[q]] for q in range(len(qg))])

    def step(backward=True):
        w = [torch.nn.functional.softplus(p) for p in params]
        flat = batched_sssp(b, graphs, w)
        loss = (flat[gidx] * gcoef).sum()
        if backward:
            for p in params:
                p.grad = None
            loss.backward()
        return loss

    # where a step's time goes (outside the timed loops)
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    for g, p in zip(graphs, params):
        g.set_weights(torch.nn.functional.softplus(p.detach()).contiguous().data_ptr())
    t1 = time.perf_counter()
    st = b.run()
    t2 = time.perf_counter()
    parts = {"set_weights_ms": (t1 - t0) * 1e3, "batch_run_ms": (t2 - t1) * 1e3,
             "batch_kernel_ms": st["kernel_ms"], "items": st["items_popped"],
             "edges": st["edges_scanned"]}

    for _ in range(args.warmup):
        step(True)
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(False)
    torch.cuda.synchronize(local)
    fwd_s = (time.perf_counter() - t0) / args.steps
    barrier(dist, local)
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(True)
    torch.cuda.synchronize(local)
    fb_s = (time.perf_counter() - t0) / args.steps
    tmax, usum = reduce_max_sum(dist, local, fb_s, 1.0)
    out = {
        "metric": "diff_sssp_fwd_bwd_per_s", "value": usum / tmax, "unit": "fwd+bwd/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": tmax * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "float32",
        "data": "synthetic",
        "config": {"workload": "diff: 128 grids (side log-uniform [64,512]), w=softplus(theta), "
                               "16 sources x 64 targets per grid, L=sum c_t d(s,t)",
                   "queries": len(qg), "parallelism": f"replicas{ws}"},
        "fwd_ms": fwd_s * 1e3, "fwd_bwd_ms": fb_s * 1e3, "fwd_bwd_over_fwd": fb_s / fwd_s,
        "gpu_launches": None, "parts": parts,
    }
    b.close()
    for g in graphs:
        g.close()
    return out


def run_ceiling(args, ws, rank, local):
    """One pass over every R-MAT 24 edge with final distances resident, four
    ways (adds_diag_relax_pass): the memory-system bound of a relaxation."""
    wl = WORKLOADS["rmat24"]
    g = make_graph(wl, local)
    row = np.empty(g.n + 1, dtype=np.uint64)
    import adds_b200 as A
    A.check(A.lib().adds_graph_download(g.handle, row.ctypes.data, None, None))
    src = pick_sources(g, wl, row)[0]
    ms = g.relax_ceiling(src)
    m = g.m
    g.close()
    names = ["stream_12B_per_edge", "gather", "gather_and_min", "min_only"]
    return {"metric": "relax_pass_gedges_per_s", "unit": "Gedges/s", "higher_is_better": True,
            "n_gpus": ws, "config": {"workload": "relax ceiling: one pass over all R-MAT 24 "
                                                 "edges, final distances resident"},
            "value": m / ms[1] / 1e6,
            "passes": {k: {"ms": v, "gedges_per_s": m / v / 1e6, "gb_per_s_12B": 12 * m / v / 1e6}
                       for k, v in zip(names, ms)}}


def run_comparators(args, ws, rank, local):
    """The schedules of the reference's comparison set run in this engine on
    one R-MAT 22 graph (the Galois GPU nf and nvGraph nv binaries cannot be
    built here): delta-stepping, the reference's asynchronous bucket
    schedule, near-far (nf_int.patch: one far pile split against a moving
    threshold) and frontier Bellman-Ford (nv_int/kernel.cu's schedule), all
    at the same bucket width.  One synchronous solve per source after a
    warm-up; every schedule's distances must equal delta-stepping's."""
    import adds_b200 as A
    wl = WORKLOADS["rmat22"]
    g = make_graph(wl, local)
    row = np.empty(g.n + 1, dtype=np.uint64)
    A.check(A.lib().adds_graph_download(g.handle, row.ctypes.data, None, None))
    srcs = pick_sources(g, wl, row)
    shift = 10
    scheds = {
        "delta_stepping": A.default_opts(engine=2, delta_shift=shift),
        "async_buckets": A.default_opts(engine=1, delta_shift=shift),
        "near_far": A.default_opts(engine=2, near_far=1, delta_shift=shift, light_heavy=0),
        "bellman_ford": A.default_opts(engine=2, delta_shift=31, light_heavy=0),
    }
    ref, mr = {}, {}
    for s in srcs:
        d, _ = g.sssp(s, scheds["delta_stepping"])
        ref[s] = d
        mr[s] = g.reached()[1]
    res = {}
    for name, o in scheds.items():
        o.timeout_ms = 20000
        g.sssp(srcs[0], o)  # warm-up (engine set-up)
        kms, phases, same = 0.0, 0, True
        for s in srcs:
            d, st = g.sssp(s, o)
            kms += st["kernel_ms"]
            phases += st["phases"]
            same = same and bool(np.array_equal(d, ref[s]))
        res[name] = {"ms_per_solve": kms / len(srcs),
                     "gteps": sum(mr.values()) / (kms / 1e3) / 1e9,
                     "phases_per_solve": phases / len(srcs), "same_distances": same}
    g.close()
    return {"metric": "sssp_gteps", "unit": "GTEPS", "higher_is_better": True, "n_gpus": ws,
            "config": {"workload": "comparators: R-MAT 22 int32 U[1,10000], 8 sources, "
                                   "four schedules in one engine", "delta_shift": shift},
            "value": res["delta_stepping"]["gteps"], "schedules": res}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat24",
                    choices=sorted(WORKLOADS) + ["batched", "diff", "ceiling", "comparators"])
    ap.add_argument("--e2e-steps", type=int, default=16)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--engine", type=int, default=0, help="0 auto, 1 async, 2 phase")
    ap.add_argument("--opts", default="", help="JSON dict of adds_opts fields to override")
    ap.add_argument("--trace", default="", help="save the phase trace of one solve (.npy)")
    ap.add_argument("--lib", default="",
                    help="time another build of libadds.so (A/B of two builds of the engine)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.lib:
        import adds_b200._lib as L
        L.LIB_PATH = os.path.abspath(args.lib)
    ws, rank, local = dist_env()
    if args.workload in ("ceiling", "comparators"):
        if rank == 0:
            fn = run_ceiling if args.workload == "ceiling" else run_comparators
            print(json.dumps(fn(args, ws, rank, local)), flush=True)
        return
    if args.workload in ("batched", "diff"):
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the reference has no batched or differentiable path"}))
            return
        dist = dist_init(ws, local)
        fn = run_batched if args.workload == "batched" else run_diff
        out = fn(args, ws, rank, local, dist)
        if rank == 0:
            print(json.dumps(out), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, args.workload, wl, ws, rank, local)), flush=True)
        return
    dist = dist_init(ws, local)
    out = run_ours(args, args.workload, wl, ws, rank, local, dist)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
