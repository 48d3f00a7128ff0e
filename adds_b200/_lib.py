"""ctypes binding of include/adds.h (libadds.so).

This module is a thin loader: every call goes straight to the C ABI.  There
is no Python or CPU fallback; if the shared library is missing the import of
any solver entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libadds.so")

ADDS_I32 = 0
ADDS_F32 = 1

ERRORS = {
    0: "ADDS_OK",
    -1: "ADDS_ERR_INVALID",
    -2: "ADDS_ERR_IO",
    -3: "ADDS_ERR_FORMAT",
    -4: "ADDS_ERR_OOM",
    -5: "ADDS_ERR_CUDA",
    -6: "ADDS_ERR_DEVICE_TIMEOUT",
    -7: "ADDS_ERR_WL_OVERFLOW",
    -8: "ADDS_ERR_NO_DEVICE",
    -9: "ADDS_ERR_UNSUPPORTED",
}

INF_I32 = 0x7FFFFFFF
INF_F32_BITS = 0x7F7FFFFF


class AddsError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        name = ERRORS.get(code, str(code))
        super().__init__(f"{what}: {name}" if what else name)


class Opts(C.Structure):
    _fields_ = [
        ("stream", C.c_void_p),
        ("delta_shift", C.c_int32),
        ("delta_scale", C.c_float),
        ("window", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("batch_max", C.c_int32),
        ("hub_threshold", C.c_int32),
        ("timeout_ms", C.c_int32),
        ("adapt", C.c_int32),
        ("strict_order", C.c_int32),
        ("local_max", C.c_int32),
        ("light_heavy", C.c_int32),
        ("block_threads", C.c_int32),
        ("greed", C.c_int32),
        ("engine", C.c_int32),
        ("group_ctas", C.c_int32),
        ("solo_max", C.c_int32),
        ("near_far", C.c_int32),
        ("dense_scan", C.c_int32),
        ("pull", C.c_int32),
        ("reserved", C.c_int32 * 2),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("ms", C.c_double),
        ("kernel_ms", C.c_double),
        ("items_popped", C.c_uint64),
        ("items_stale", C.c_uint64),
        ("edges_scanned", C.c_uint64),
        ("pushes", C.c_uint64),
        ("batches", C.c_uint64),
        ("hub_chunks", C.c_uint64),
        ("hub_stale", C.c_uint64),
        ("local_batches", C.c_uint64),
        ("heavy_lists", C.c_uint64),
        ("phase_cycles", C.c_uint64 * 6),
        ("mid_flush_cycles", C.c_uint64),
        ("mid_flushes", C.c_uint64),
        ("reached", C.c_uint64),
        ("reached_edges", C.c_uint64),
        ("delta_shift", C.c_int32),
        ("retries", C.c_int32),
        ("ctas", C.c_int32),
        ("engine", C.c_int32),
        ("launches", C.c_int32),
        ("reserved", C.c_int32 * 3),
        ("phases", C.c_uint64),
        ("solo_phases", C.c_uint64),
        ("repushes", C.c_uint64),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("reserved", "phase_cycles")}
        d["phase_cycles"] = list(self.phase_cycles)
        return d


class GraphInfo(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("m", C.c_uint64),
        ("wtype", C.c_int),
        ("device", C.c_int),
        ("max_degree", C.c_uint32),
        ("avg_degree", C.c_double),
        ("avg_weight", C.c_double),
        ("device_bytes", C.c_uint64),
    ]


class GenSpec(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("scale", C.c_int32),
        ("edge_factor", C.c_int32),
        ("n", C.c_uint32),
        ("side_x", C.c_uint32),
        ("side_y", C.c_uint32),
        ("a", C.c_double),
        ("b", C.c_double),
        ("c", C.c_double),
        ("shortcut_frac", C.c_double),
        ("shortcut_radius", C.c_int32),
        ("wtype", C.c_int),
        ("w_lo", C.c_double),
        ("w_hi", C.c_double),
        ("seed", C.c_uint64),
    ]


# (name, restype, argtypes) of every exported symbol declared in adds.h
SIGNATURES = [
    ("adds_abi_version", C.c_int, []),
    ("adds_strerror", C.c_char_p, [C.c_int]),
    ("adds_opts_init", None, [C.POINTER(Opts)]),
    ("adds_last_cuda_error", C.c_char_p, []),
    ("adds_graph_load_gr", C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("adds_graph_from_csr", C.c_int, [C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("adds_graph_info", C.c_int, [C.c_void_p, C.POINTER(GraphInfo)]),
    ("adds_graph_download", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("adds_graph_set_weights", C.c_int, [C.c_void_p, C.c_void_p]),
    ("adds_graph_save_gr", C.c_int, [C.c_void_p, C.c_char_p]),
    ("adds_graph_free", None, [C.c_void_p]),
    ("adds_graph_generate", C.c_int, [C.POINTER(GenSpec), C.c_int, C.POINTER(C.c_void_p)]),
    ("adds_sssp", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(Opts), C.POINTER(Stats)]),
    ("adds_sssp_async", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(Opts)]),
    ("adds_sssp_sources", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.c_uint32,
                                     C.POINTER(C.c_void_p), C.POINTER(Opts), C.POINTER(Stats)]),
    ("adds_graph_sync", C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    ("adds_graph_last_dist", C.c_int, [C.c_void_p, C.c_void_p]),
    ("adds_graph_reached", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("adds_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_uint32), C.c_uint32,
                                    C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    ("adds_batch_run", C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    ("adds_batch_launch", C.c_int, [C.c_void_p]),
    ("adds_batch_sync", C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    ("adds_batch_dist", C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    ("adds_batch_dist_ptr", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("adds_batch_dist_all", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]),
    ("adds_batch_set_sources", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    ("adds_batch_free", None, [C.c_void_p]),
    ("adds_batch_backward", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    ("adds_sssp_backward", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.POINTER(Opts)]),
    ("adds_diag_relax_pass", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    ("adds_diag_wait_timeout", C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_double)]),
    ("adds_graph_trace", C.c_int, [C.c_void_p, C.c_uint32]),
    ("adds_graph_trace_read", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32,
                                        C.POINTER(C.c_uint64)]),
    ("adds_tune", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(Opts),
                            C.POINTER(C.c_double)]),
    ("adds_write_dist_text", C.c_int, [C.c_char_p, C.c_uint32, C.c_void_p, C.c_int]),
    ("adds_sssp_noalloc", C.c_int, [C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_uint32, C.c_void_p, C.c_void_p]),
]

_lib = None


def lib():
    """Loads libadds.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m adds_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc, what=""):
    if rc != 0:
        detail = lib().adds_last_cuda_error().decode(errors="replace")
        raise AddsError(rc, f"{what} ({detail})" if detail else what)
    return rc


def default_opts(**kw):
    o = Opts()
    lib().adds_opts_init(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o
