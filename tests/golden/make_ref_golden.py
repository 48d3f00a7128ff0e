"""Runs the reference ADDS binaries (oracle/_ref/, built by
oracle/build_ref.sh) on seeded synthetic graphs and freezes their distance
output as fixtures in tests/golden/, so the oracle -- and through it the
engine -- is pinned to the reference's own results.  Needs a GPU; run once:

  python tests/golden/make_ref_golden.py [output_dir]   (default: tests/golden)

Graphs are regenerated from their seeds by the tests, so only distances (int)
or the reference's text output (float, compressed) are stored, together with
the fd-3 timing record the reference printed.
"""
import gzip
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from adds_b200 import graphs as G  # noqa: E402
from oracle import oracle as O  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
HERE = os.path.dirname(os.path.abspath(__file__))

# name: (builder, source rule, binary)
CASES = {
    "ref_rmat16_int": (lambda: G.rmat(16, 16, seed=16, w_lo=1, w_hi=1000), "maxdeg", "ads_int_sssp"),
    "ref_rmat12_int": (lambda: G.rmat(12, 16, seed=12, w_lo=1, w_hi=10000), "first", "ads_int_sssp"),
    "ref_grid96_float": (lambda: G.grid(96, 96, 0.02, 8, wtype=G.F32, w_lo=1.0, w_hi=100.0, seed=96),
                         "center", "ads_float_sssp"),
}


def source_of(g, rule):
    if rule == "maxdeg":
        return G.max_degree_vertex(g)
    if rule == "center":
        s = int(round(g.n ** 0.5))
        return (s // 2) * s + s // 2
    return int(np.flatnonzero(np.diff(g.row) > 0)[0])


def run_case(name, build, rule, binary, tmp, outdir):
    g = build()
    src = source_of(g, rule)
    gr = os.path.join(tmp, name + ".gr")
    G.write_gr(gr, g)
    out = os.path.join(tmp, name + ".txt")
    rec = os.path.join(tmp, name + ".fd3")
    cmd = f'timeout 120 "{os.path.join(REF, binary)}" -s {src} -o "{out}" "{gr}" 3>"{rec}"'
    r = subprocess.run(["bash", "-c", cmd], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{name}: reference exited {r.returncode}\n{r.stdout[-1500:]}\n{r.stderr[-1500:]}")
    text = open(out).read()
    fd3 = open(rec).read().strip()
    ref, _ = O.dijkstra(g, src)
    wt = G.I32 if binary == "ads_int_sssp" else G.F32
    mine = G.dist_text(ref, wt)
    print(f"{name}: n={g.n} m={g.m} src={src} fd3='{fd3}' oracle text == reference text: "
          f"{mine == text}", flush=True)
    rec_d = {"src": np.array(src), "fd3": np.frombuffer(fd3.encode(), dtype=np.uint8)}
    if wt == G.I32:
        rec_d["dist"] = G.read_dist_text(out, G.I32)
    else:
        rec_d["text_gz"] = np.frombuffer(gzip.compress(text.encode()), dtype=np.uint8)
    np.savez_compressed(os.path.join(outdir, name + ".npz"), **rec_d)
    return mine == text


def main():
    outdir = sys.argv[1] if len(sys.argv) > 1 else HERE
    os.makedirs(outdir, exist_ok=True)
    ok = True
    with tempfile.TemporaryDirectory() as tmp:
        for name, (build, rule, binary) in CASES.items():
            ok &= run_case(name, build, rule, binary, tmp, outdir)
    print("all equal" if ok else "MISMATCH")
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
