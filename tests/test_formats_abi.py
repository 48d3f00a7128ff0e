"""Host-side formats and the C ABI surface (no GPU needed).

- Galois .gr v1 files (csr_graph.cu:203-296 layout) round trip;
- the distance text format of support.cu:78-97 (int) and the Galois float
  writer (cpu_sssp_float.patch:241-247);
- libadds.so loads and exports every function include/adds.h declares, with
  struct layouts that agree between C and the ctypes mirror;
- argument errors are reported as return codes, never by exiting.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import adds_b200 as A
from adds_b200 import _lib as L
from adds_b200 import graphs as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "adds.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(adds_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_function_is_exported():
    lib = L.lib()
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    bound = {n for n, _, _ in L.SIGNATURES}
    assert set(names) <= bound, sorted(set(names) - bound)


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "adds.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", '
                   'sizeof(adds_opts), sizeof(adds_stats), sizeof(adds_graph_info_t), '
                   'sizeof(adds_gen_spec), offsetof(adds_stats, phase_cycles), '
                   'offsetof(adds_opts, solo_max), offsetof(adds_opts, near_far), '
                   'offsetof(adds_stats, repushes), offsetof(adds_opts, dense_scan), '
                   'offsetof(adds_opts, pull), offsetof(adds_stats, launches));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    want = [C.sizeof(L.Opts), C.sizeof(L.Stats), C.sizeof(L.GraphInfo), C.sizeof(L.GenSpec),
            L.Stats.phase_cycles.offset, L.Opts.solo_max.offset, L.Opts.near_far.offset,
            L.Stats.repushes.offset, L.Opts.dense_scan.offset, L.Opts.pull.offset,
            L.Stats.launches.offset]
    assert got == want


def test_strerror_and_defaults():
    lib = L.lib()
    assert lib.adds_abi_version() == 2
    assert lib.adds_strerror(-7) == b"worklist pool exhausted"
    assert lib.adds_strerror(0) == b"ok"
    o = A.default_opts()
    assert o.delta_shift == -1 and o.window == 0 and o.light_heavy == -1 and o.local_max == -1
    # pull phases: 0 = automatic (a field that was reserved, so callers that
    # zero the struct get the automatic choice)
    assert o.pull == 0 and list(o.reserved) == [0, 0]


def test_invalid_arguments_return_codes():
    lib = L.lib()
    h = C.c_void_p()
    assert lib.adds_graph_load_gr(None, 0, 0, C.byref(h)) == -1
    assert lib.adds_graph_load_gr(b"/x", 7, 0, C.byref(h)) == -1
    assert lib.adds_graph_from_csr(0, 0, None, None, None, 0, 0, C.byref(h)) == -1
    assert lib.adds_sssp(None, 0, None, None, None) == -1
    assert lib.adds_sssp_sources(None, None, 0, None, None, None) == -1
    assert lib.adds_diag_wait_timeout(0, 0, None) == -1
    assert lib.adds_diag_wait_timeout(0, 20000, None) == -1
    assert lib.adds_batch_create(None, None, 0, None, C.byref(h)) == -1
    assert lib.adds_tune(None, None, 0, None, None) == -1
    assert lib.adds_write_dist_text(None, 0, None, 0) == -1
    lib.adds_graph_free(None)
    lib.adds_batch_free(None)


def test_gr_round_trip(tmp_path):
    g = G.rmat(9, 16, seed=1, w_hi=77)
    p = str(tmp_path / "a.gr")
    G.write_gr(p, g)
    h = G.read_gr(p)
    assert h.n == g.n and np.array_equal(h.row, g.row) and np.array_equal(h.dst, g.dst)
    assert np.array_equal(h.w, g.w)
    # byte layout: header, u64 ends, u32 dst, pad to 8 when m is odd, u32 weights
    raw = open(p, "rb").read()
    assert len(raw) == 32 + 8 * g.n + 4 * g.m + (4 if g.m % 2 else 0) + 4 * g.m
    hdr = np.frombuffer(raw[:32], dtype="<u8")
    assert hdr.tolist() == [1, 4, g.n, g.m]


def test_gr_odd_edge_count_and_unweighted(tmp_path):
    g = G.from_edges(4, [0, 1, 2], [1, 2, 3], [5, 6, 7])
    p = str(tmp_path / "odd.gr")
    G.write_gr(p, g)
    assert G.read_gr(p).w.tolist() == [5, 6, 7]
    G.write_gr(p, g, edge_size=0)
    assert G.read_gr(p).w.tolist() == [0, 0, 0]  # the reference leaves weights zero


def test_gr_rejects_truncated(tmp_path):
    g = G.rmat(6, 8, seed=2)
    p = str(tmp_path / "t.gr")
    G.write_gr(p, g)
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-5])
    with pytest.raises(ValueError):
        G.read_gr(p)


def test_dist_text_formats(tmp_path):
    d = np.array([0, 17, 0x7FFFFFFF, 2147483646], dtype=np.uint32)
    assert G.dist_text(d, G.I32) == "0 0\n1 17\n2 INF\n3 2147483646\n"
    f = np.array([0.0, 1.5, 3.4028234663852886e38, 1e-7], dtype=np.float32).view(np.uint32)
    assert G.dist_text(f, G.F32) == "0 0.000000\n1 1.500000\n2 INF\n3 0.000000\n"
    # the C writer (threaded) produces the same bytes
    lib = L.lib()
    for arr, wt in ((d, 0), (f, 1)):
        p = str(tmp_path / f"o{wt}.txt")
        assert lib.adds_write_dist_text(p.encode(), arr.size, arr.ctypes.data, wt) == 0
        assert open(p).read() == G.dist_text(arr, wt)
    big = np.arange(3_000_000, dtype=np.uint32) % 1000
    p = str(tmp_path / "big.txt")
    assert lib.adds_write_dist_text(p.encode(), big.size, big.ctypes.data, 0) == 0
    lines = open(p).read().splitlines()
    assert len(lines) == big.size and lines[2_999_999] == "2999999 999"


def test_generators_are_deterministic_and_clean():
    a = G.rmat(10, 16, seed=5)
    b = G.rmat(10, 16, seed=5, chunk=1000)  # chunking must not matter
    assert np.array_equal(a.row, b.row) and np.array_equal(a.dst, b.dst) and np.array_equal(a.w, b.w)
    src = np.repeat(np.arange(a.n), np.diff(a.row).astype(np.int64))
    assert not np.any(src == a.dst)  # no self loops
    keys = src.astype(np.uint64) << np.uint64(32) | a.dst.astype(np.uint64)
    assert np.all(np.diff(keys.astype(np.int64)) > 0)  # sorted, no duplicates
    w = a.weights()
    assert w.min() >= 1 and w.max() <= 1000
    f = G.grid(30, 20, 0.02, 8, wtype=G.F32, seed=3)
    assert f.weights().min() >= 1.0 and f.weights().max() < 100.0
    e = G.erdos_renyi(500, 8, seed=1)
    assert e.m <= 4000 and e.m > 3900


def test_grid_structure():
    g = G.grid(5, 4, 0.0, 8, seed=1)
    assert g.m == 2 * 4 * 4 + 2 * 5 * 3  # 4-neighbour, both directions
    s = G.grid(64, 64, 0.02, 8, seed=1)
    egrid = 2 * 63 * 64 * 2
    extra = s.m - egrid
    assert 0 < extra <= 2 * round(0.02 * egrid)


def test_cli_argument_errors():
    exe = os.path.join(ROOT, "adds_b200", "bin", "sssp_int")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    r = subprocess.run([exe, "-g", "x1", "g.gr"], capture_output=True, text=True)
    assert r.returncode != 0 and "Invalid GPU device" in r.stderr
    r = subprocess.run([exe, "-s", "-4", "g.gr"], capture_output=True, text=True)
    assert r.returncode != 0
