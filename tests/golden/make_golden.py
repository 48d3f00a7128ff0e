"""Generates tests/golden/oracle_golden.npz: small graphs (CSR) with their
oracle Dijkstra distances.  The fixture freezes the oracle's answers so a
change to the oracle or to the generators shows up as a test failure.

  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from adds_b200 import graphs as G  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    cases = {
        "rmat10_int": (G.rmat(10, 16, seed=11, w_hi=1000), None),
        "er800_int": (G.erdos_renyi(800, 8, seed=12), 3),
        "grid24x20_float": (G.grid(24, 20, 0.02, 8, wtype=G.F32, seed=13), 10 * 24 + 12),
        "rmat9_float01": (G.rmat(9, 16, seed=14, wtype=G.F32, w_lo=0.0, w_hi=1.0), None),
    }
    out = {}
    for name, (g, src) in cases.items():
        if src is None:
            src = G.max_degree_vertex(g)
        d, _ = O.dijkstra(g, src)
        out[name + "__n"] = np.array(g.n)
        out[name + "__row"] = g.row
        out[name + "__dst"] = g.dst
        out[name + "__w"] = g.w
        out[name + "__wtype"] = np.array(g.wtype)
        out[name + "__src"] = np.array(src)
        out[name + "__dist"] = d
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
