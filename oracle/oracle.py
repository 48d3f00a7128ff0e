"""ctypes wrapper of oracle/lib/liboracle.so — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline import this
module; the product never does.  See oracle.c for what it restates.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        L.oracle_dijkstra.argtypes = [u32, vp, vp, vp, u32, C.c_int, vp, C.POINTER(u64)]
        L.oracle_dijkstra.restype = C.c_int
        L.oracle_dijkstra_f64.argtypes = [u32, vp, vp, vp, u32, vp]
        L.oracle_dijkstra_f64.restype = C.c_int
        L.oracle_delta_step.argtypes = [u32, vp, vp, vp, u32, C.c_int, u32, C.c_float, C.c_int, vp,
                                        C.POINTER(u64), C.POINTER(C.c_double)]
        L.oracle_delta_step.restype = C.c_int
        L.oracle_adjoint.argtypes = [u32, u64, vp, vp, vp, u32, vp, vp, vp, vp, vp]
        L.oracle_adjoint.restype = C.c_int
        dbl = C.c_double
        L.oracle_gen_rmat.argtypes = [C.c_int, C.c_int, dbl, dbl, dbl, C.c_int, dbl, dbl, u64,
                                      C.c_int, vp, vp, vp, u64, C.POINTER(u64)]
        L.oracle_gen_rmat.restype = C.c_int
        L.oracle_gen_grid.argtypes = [u32, u32, dbl, C.c_int, C.c_int, dbl, dbl, u64, C.c_int, vp,
                                      vp, vp, u64, C.POINTER(u64)]
        L.oracle_gen_grid.restype = C.c_int
        _lib = L
    return _lib


@dataclasses.dataclass
class HostCSR:
    """CSR arrays on the host (row uint64[n+1], dst/w uint32[m], w holding
    int32 values or float32 bits per wtype); the layout of
    adds_b200.graphs.CSR, without importing the product package."""
    n: int
    row: np.ndarray
    dst: np.ndarray
    w: np.ndarray
    wtype: int

    @property
    def m(self) -> int:
        return int(self.dst.shape[0])

    def weights(self):
        return self.w.view(np.float32) if self.wtype == 1 else self.w.view(np.int32)


def gen_rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, wtype: int = 0,
             w_lo=1.0, w_hi=1000.0, seed: int = 1, threads: int | None = None) -> HostCSR:
    """The seeded R-MAT generator (gen.c), multithreaded on the host."""
    threads = threads or os.cpu_count() or 1
    n = 1 << scale
    cap = edge_factor * n
    row = np.empty(n + 1, dtype=np.uint64)
    dst = np.empty(cap, dtype=np.uint32)
    w = np.empty(cap, dtype=np.uint32)
    m = C.c_uint64()
    rc = lib().oracle_gen_rmat(scale, edge_factor, a, b, c, wtype, float(w_lo), float(w_hi), seed,
                               threads, row.ctypes.data, dst.ctypes.data, w.ctypes.data, cap,
                               C.byref(m))
    if rc:
        raise RuntimeError(f"oracle_gen_rmat failed ({rc})")
    return HostCSR(n, row, dst[:m.value], w[:m.value], wtype)


def gen_grid(side_x: int, side_y: int, shortcut_frac=0.0, radius=8, wtype: int = 1, w_lo=1.0,
             w_hi=100.0, seed: int = 1, threads: int | None = None) -> HostCSR:
    """The seeded grid-with-shortcuts generator (gen.c), on the host."""
    threads = threads or os.cpu_count() or 1
    n = side_x * side_y
    egrid = 2 * (side_x - 1) * side_y + 2 * side_x * (side_y - 1)
    cap = 4 * n + 2 * int(shortcut_frac * egrid + 0.5) + 2
    row = np.empty(n + 1, dtype=np.uint64)
    dst = np.empty(cap, dtype=np.uint32)
    w = np.empty(cap, dtype=np.uint32)
    m = C.c_uint64()
    rc = lib().oracle_gen_grid(side_x, side_y, float(shortcut_frac), radius, wtype, float(w_lo),
                               float(w_hi), seed, threads, row.ctypes.data, dst.ctypes.data,
                               w.ctypes.data, cap, C.byref(m))
    if rc:
        raise RuntimeError(f"oracle_gen_grid failed ({rc})")
    return HostCSR(n, row, dst[:m.value], w[:m.value], wtype)


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def dijkstra(g, src: int):
    """Serial Dijkstra with the engine's 32-bit fold; returns (dist words, work)."""
    row, dst, w = _arr(g.row, np.uint64), _arr(g.dst, np.uint32), _arr(g.w, np.uint32)
    out = np.empty(g.n, dtype=np.uint32)
    work = C.c_uint64()
    rc = lib().oracle_dijkstra(g.n, row.ctypes.data, dst.ctypes.data, w.ctypes.data, src,
                               int(g.wtype == 1), out.ctypes.data, C.byref(work))
    if rc:
        raise RuntimeError(f"oracle_dijkstra failed ({rc})")
    return out, work.value


def dijkstra_f64(g, w64: np.ndarray, src: int) -> np.ndarray:
    row, dst = _arr(g.row, np.uint64), _arr(g.dst, np.uint32)
    w64 = _arr(w64, np.float64)
    out = np.empty(g.n, dtype=np.float64)
    rc = lib().oracle_dijkstra_f64(g.n, row.ctypes.data, dst.ctypes.data, w64.ctypes.data, src,
                                   out.ctypes.data)
    if rc:
        raise RuntimeError(f"oracle_dijkstra_f64 failed ({rc})")
    return out


def delta_step(g, src: int, shift: int = 13, div: float = 1.0, threads: int | None = None):
    """Galois-style parallel delta-stepping; returns (dist, work, ms)."""
    threads = threads or os.cpu_count() or 1
    row, dst, w = _arr(g.row, np.uint64), _arr(g.dst, np.uint32), _arr(g.w, np.uint32)
    out = np.empty(g.n, dtype=np.uint32)
    work, ms = C.c_uint64(), C.c_double()
    rc = lib().oracle_delta_step(g.n, row.ctypes.data, dst.ctypes.data, w.ctypes.data, src,
                                 int(g.wtype == 1), shift, div, threads, out.ctypes.data,
                                 C.byref(work), C.byref(ms))
    if rc:
        raise RuntimeError(f"oracle_delta_step failed ({rc})")
    return out, work.value, ms.value


def adjoint(g, srcs, dist: np.ndarray, seed: np.ndarray | None):
    """Reference dL/dw (float graphs): dist/seed are [ns, n] float32."""
    row, dst = _arr(g.row, np.uint64), _arr(g.dst, np.uint32)
    w = _arr(g.w, np.uint32)
    srcs = _arr(srcs, np.uint32)
    dist = _arr(dist, np.float32)
    sp = None
    if seed is not None:
        seed = _arr(seed, np.float32)
        sp = seed.ctypes.data
    grad = np.empty(g.m, dtype=np.float32)
    pred = np.empty((len(srcs), g.n), dtype=np.uint64)
    rc = lib().oracle_adjoint(g.n, g.m, row.ctypes.data, dst.ctypes.data, w.ctypes.data,
                              len(srcs), srcs.ctypes.data, dist.ctypes.data, sp,
                              grad.ctypes.data, pred.ctypes.data)
    if rc:
        raise RuntimeError(f"oracle_adjoint failed ({rc})")
    return grad, pred
