"""adds_b200 — B200-native asynchronous delta-stepping SSSP (ctypes front end).

The engine is libadds.so (include/adds.h); this package only marshals
arguments to it.  Importing the package does not need a GPU; calling a
solver without the built library raises ImportError (no fallback).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (ADDS_F32, ADDS_I32, INF_F32_BITS, INF_I32, AddsError, GenSpec, GraphInfo,
                   Opts, Stats, check, default_opts, lib)
from .graphs import CSR

__all__ = ["Graph", "Batch", "AddsError", "Opts", "Stats", "default_opts", "ADDS_I32",
           "ADDS_F32", "INF_I32", "INF_F32_BITS", "gen_spec", "lib"]


def _ptr(x):
    """numpy array / torch tensor / int -> raw address (or None)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    raise TypeError(f"cannot take the address of {type(x)}")


def gen_spec(kind: str, **kw) -> GenSpec:
    """kind: 'rmat' | 'grid' (with shortcuts) | 'er' | 'plain_grid'."""
    s = GenSpec()
    s.kind = {"rmat": 0, "grid": 1, "er": 2, "plain_grid": 3}[kind]
    s.scale = kw.get("scale", 0)
    s.edge_factor = kw.get("edge_factor", 16)
    s.n = kw.get("n", 0)
    s.side_x = kw.get("side_x", kw.get("side", 0))
    s.side_y = kw.get("side_y", kw.get("side", 0))
    s.a, s.b, s.c = kw.get("a", 0.57), kw.get("b", 0.19), kw.get("c", 0.19)
    s.shortcut_frac = kw.get("shortcut_frac", 0.0)
    s.shortcut_radius = kw.get("radius", 8)
    s.wtype = kw.get("wtype", ADDS_I32)
    s.w_lo, s.w_hi = kw.get("w_lo", 1), kw.get("w_hi", 1000)
    s.seed = kw.get("seed", 1)
    return s


class Graph:
    """Device-resident CSR graph (adds_graph handle)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)
        info = GraphInfo()
        check(lib().adds_graph_info(self._h, C.byref(info)), "adds_graph_info")
        self.n, self.m, self.wtype = info.n, info.m, info.wtype
        self.device = info.device
        self.max_degree, self.avg_degree, self.avg_weight = (info.max_degree, info.avg_degree,
                                                             info.avg_weight)

    # -- construction
    @classmethod
    def from_csr(cls, g: CSR, device: int = 0) -> "Graph":
        h = C.c_void_p()
        row = np.ascontiguousarray(g.row, dtype=np.uint64)
        dst = np.ascontiguousarray(g.dst, dtype=np.uint32)
        w = np.ascontiguousarray(g.w, dtype=np.uint32)
        check(lib().adds_graph_from_csr(g.n, g.m, _ptr(row), _ptr(dst), _ptr(w), g.wtype, device,
                                        C.byref(h)), "adds_graph_from_csr")
        return cls(h.value)

    @classmethod
    def load_gr(cls, path: str, wtype: int = ADDS_I32, device: int = 0) -> "Graph":
        h = C.c_void_p()
        check(lib().adds_graph_load_gr(path.encode(), wtype, device, C.byref(h)),
              "adds_graph_load_gr")
        return cls(h.value)

    @classmethod
    def generate(cls, spec: GenSpec, device: int = 0) -> "Graph":
        h = C.c_void_p()
        check(lib().adds_graph_generate(C.byref(spec), device, C.byref(h)), "adds_graph_generate")
        return cls(h.value)

    def close(self):
        if self._h is not None and self._h.value:
            lib().adds_graph_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- data
    def download(self) -> CSR:
        row = np.empty(self.n + 1, dtype=np.uint64)
        dst = np.empty(self.m, dtype=np.uint32)
        w = np.empty(self.m, dtype=np.uint32)
        check(lib().adds_graph_download(self._h, _ptr(row), _ptr(dst), _ptr(w)),
              "adds_graph_download")
        return CSR(self.n, row, dst, w, self.wtype)

    def set_weights(self, w) -> None:
        if isinstance(w, np.ndarray):
            w = np.ascontiguousarray(w)
        check(lib().adds_graph_set_weights(self._h, _ptr(w)), "adds_graph_set_weights")
        info = GraphInfo()
        lib().adds_graph_info(self._h, C.byref(info))
        self.avg_weight = info.avg_weight

    def save_gr(self, path: str) -> None:
        check(lib().adds_graph_save_gr(self._h, path.encode()), "adds_graph_save_gr")

    # -- solves
    def sssp(self, src: int, opts: Opts | None = None, out=None):
        """One solve; returns (uint32 distance words, stats dict)."""
        st = Stats()
        if out is None:
            out = np.empty(self.n, dtype=np.uint32)
        check(lib().adds_sssp(self._h, src, _ptr(out), C.byref(opts) if opts else None,
                              C.byref(st)), "adds_sssp")
        return out, st.as_dict()

    def sssp_sources(self, srcs, outs, opts: Opts | None = None) -> dict:
        """One solve per source, result i copied into outs[i] (host or device
        buffers of n words; an address repeats to reuse a buffer) while solve
        i+1 runs; returns the stats."""
        st = Stats()
        ss = (C.c_uint32 * len(srcs))(*[int(s) for s in srcs])
        ps = (C.c_void_p * len(outs))(*[_ptr(o) for o in outs])
        if len(outs) != len(srcs):
            raise ValueError("one output buffer per source")
        check(lib().adds_sssp_sources(self._h, ss, len(srcs), ps, C.byref(opts) if opts else None,
                                      C.byref(st)), "adds_sssp_sources")
        return st.as_dict()

    def sssp_async(self, src: int, opts: Opts | None = None) -> None:
        check(lib().adds_sssp_async(self._h, src, C.byref(opts) if opts else None),
              "adds_sssp_async")

    def sync(self) -> dict:
        st = Stats()
        check(lib().adds_graph_sync(self._h, C.byref(st)), "adds_graph_sync")
        return st.as_dict()

    def last_dist(self, out=None):
        if out is None:
            out = np.empty(self.n, dtype=np.uint32)
        check(lib().adds_graph_last_dist(self._h, _ptr(out)), "adds_graph_last_dist")
        return out

    def reached(self):
        r, e = C.c_uint64(), C.c_uint64()
        check(lib().adds_graph_reached(self._h, C.byref(r), C.byref(e)), "adds_graph_reached")
        return r.value, e.value

    def relax_ceiling(self, src: int):
        """Times one pass over every edge with the final distances from src:
        stream only, gather, gather + reduction, reduction only (ms)."""
        out = (C.c_double * 4)()
        check(lib().adds_diag_relax_pass(self._h, src, out), "adds_diag_relax_pass")
        return list(out)

    def trace(self, cap: int) -> None:
        """Records up to cap phases of each later solve (0 turns it off)."""
        check(lib().adds_graph_trace(self._h, cap), "adds_graph_trace")

    def trace_read(self, cap: int = 1 << 16):
        """The last solve's phase records as a numpy structured array
        (t_ns, count, mode, base, edges, items, pushes, tail_ns) and the
        number the solve produced."""
        import numpy as np
        dt = np.dtype([("t_ns", "<u8"), ("count", "<u4"), ("mode", "<u2"), ("base", "<u2"),
                       ("edges", "<u4"), ("items", "<u4"), ("pushes", "<u4"),
                       ("tail_ns", "<u4")])
        buf = np.zeros(cap, dtype=dt)
        n = C.c_uint64()
        check(lib().adds_graph_trace_read(self._h, buf.ctypes.data, cap, C.byref(n)),
              "adds_graph_trace_read")
        return buf[: min(cap, n.value)], n.value

    def tune(self, srcs, base: Opts | None = None):
        arr = (C.c_uint32 * len(srcs))(*srcs)
        best = Opts()
        if base is not None:
            best.engine = base.engine
        ms = C.c_double()
        check(lib().adds_tune(self._h, arr, len(srcs), C.byref(best), C.byref(ms)), "adds_tune")
        return best, ms.value

    def backward(self, srcs, dist_dev: int, grad_dist_dev: int, grad_w_dev: int,
                 opts: Opts | None = None) -> None:
        """dL/dw for len(srcs) solves: dist / grad_dist are [ns][n] float32
        device buffers, grad_w an m-float device buffer (overwritten)."""
        arr = (C.c_uint32 * len(srcs))(*srcs)
        check(lib().adds_sssp_backward(self._h, len(srcs), arr, dist_dev, grad_dist_dev,
                                       grad_w_dev, C.byref(opts) if opts else None),
              "adds_sssp_backward")


class Batch:
    """Many solves (graph, source) in one persistent, graph-captured launch."""

    def __init__(self, graphs, srcs, opts: Opts | None = None):
        self.graphs = list(graphs)
        n = len(self.graphs)
        hs = (C.c_void_p * n)(*[g.handle.value for g in self.graphs])
        ss = (C.c_uint32 * n)(*[int(s) for s in srcs])
        h = C.c_void_p()
        check(lib().adds_batch_create(hs, ss, n, C.byref(opts) if opts else None, C.byref(h)),
              "adds_batch_create")
        self._h = h
        self.nq = n

    def run(self) -> dict:
        st = Stats()
        check(lib().adds_batch_run(self._h, C.byref(st)), "adds_batch_run")
        return st.as_dict()

    def launch(self) -> None:
        check(lib().adds_batch_launch(self._h), "adds_batch_launch")

    def sync(self) -> dict:
        st = Stats()
        check(lib().adds_batch_sync(self._h, C.byref(st)), "adds_batch_sync")
        return st.as_dict()

    def dist(self, q: int, out=None):
        if out is None:
            out = np.empty(self.graphs[q].n, dtype=np.uint32)
        check(lib().adds_batch_dist(self._h, q, _ptr(out)), "adds_batch_dist")
        return out

    def layout(self):
        """(offsets of each query in the flat distance array, total words)"""
        off = np.empty(self.nq, dtype=np.uint64)
        tot = C.c_uint64()
        check(lib().adds_batch_dist_all(self._h, None, off.ctypes.data, C.byref(tot)),
              "adds_batch_dist_all")
        return off, tot.value

    def dist_all(self, out) -> None:
        """Copies every query's distances (flat, see layout()) to out."""
        tot = C.c_uint64()
        check(lib().adds_batch_dist_all(self._h, _ptr(out), None, C.byref(tot)),
              "adds_batch_dist_all")

    def dist_ptr(self, q: int) -> int:
        p = C.c_void_p()
        check(lib().adds_batch_dist_ptr(self._h, q, C.byref(p)), "adds_batch_dist_ptr")
        return p.value

    def set_sources(self, srcs) -> None:
        ss = (C.c_uint32 * self.nq)(*[int(s) for s in srcs])
        check(lib().adds_batch_set_sources(self._h, ss), "adds_batch_set_sources")

    def backward(self, grad_dist_ptrs, grad_w_ptrs) -> None:
        gd = (C.c_void_p * len(grad_dist_ptrs))(*grad_dist_ptrs)
        gw = (C.c_void_p * len(grad_w_ptrs))(*grad_w_ptrs)
        check(lib().adds_batch_backward(self._h, gd, gw), "adds_batch_backward")

    def close(self):
        if self._h is not None and self._h.value:
            lib().adds_batch_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
