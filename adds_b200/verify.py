"""Distance-file checker for run_all.sh-style result directories.

    python -m adds_b200.verify DIR1/ DIR2/ GRAPH_LIST [--float] [--max-report N]

The reference's verify.py (verify.py:1-57) takes the same three arguments:
two result directories (DIR1 + graph name is one file) and the graph list
whose first tab-separated field on each line names a graph.  It has two
faults this tool does not have: it prints "match" after every graph, also
after a mismatch (verify.py:50), and it stops at the first differing line.
Here a graph is reported as "match" only when every line agrees, a
mismatch reports how many lines differ and the first few of them, a
missing or short file is a mismatch, and the exit status says the outcome
(0 all match, 1 a mismatch, 2 a usage error).

Files are the drop-in's output: one "<v> <dist>" or "<v> INF" line per
vertex (ads_int/support.cu:89-95; float "%d %f", cpu_sssp_float.patch).
Int distances compare as integers.  Float distances compare at the
granularity of the "%f" text the files hold (6 decimals, so two distances
whose bit patterns differ can print alike); where both sides are raw
32-bit distance dumps (files ending in .bin, as `sssp_float -b` writes),
they compare bit for bit.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np


def _parse_text(path: str, is_float: bool):
    """Vertex ids and distance tokens of a distance text file."""
    ids, vals = [], []
    with open(path) as f:
        for ln, line in enumerate(f, 1):
            parts = line.split()
            if len(parts) != 2:
                raise ValueError(f"{path}:{ln}: expected '<v> <dist>', got {line.rstrip()!r}")
            ids.append(int(parts[0]))
            tok = parts[1]
            if tok == "INF":
                vals.append(None)
            elif is_float:
                vals.append(f"{float(tok):f}")  # the %f text granularity
            else:
                vals.append(int(tok))
    return ids, vals


def compare_files(p1: str, p2: str, is_float: bool, max_report: int = 5):
    """Returns (ok, messages) for one pair of result files."""
    msgs = []
    for p in (p1, p2):
        if not os.path.exists(p):
            return False, [f"missing: {p}"]
    if p1.endswith(".bin") and p2.endswith(".bin"):
        a = np.fromfile(p1, dtype="<u4")
        b = np.fromfile(p2, dtype="<u4")
        if a.shape != b.shape:
            return False, [f"length differs: {a.size} vs {b.size} words"]
        bad = np.flatnonzero(a != b)
        for v in bad[:max_report]:
            msgs.append(f"vertex {v}: 0x{a[v]:08x} vs 0x{b[v]:08x}")
        if bad.size:
            msgs.insert(0, f"{bad.size} of {a.size} distances differ (bit patterns)")
        return bad.size == 0, msgs
    try:
        i1, v1 = _parse_text(p1, is_float)
        i2, v2 = _parse_text(p2, is_float)
    except ValueError as e:
        return False, [str(e)]
    ok = True
    if len(i1) != len(i2):
        ok = False
        msgs.append(f"length differs: {len(i1)} vs {len(i2)} lines")
    nbad = 0
    for k in range(min(len(i1), len(i2))):
        if i1[k] != i2[k] or v1[k] != v2[k]:
            nbad += 1
            if nbad <= max_report:
                a = "INF" if v1[k] is None else v1[k]
                b = "INF" if v2[k] is None else v2[k]
                msgs.append(f"line {k + 1}: '{i1[k]} {a}' vs '{i2[k]} {b}'")
    if nbad:
        ok = False
        msgs.insert(0, f"{nbad} of {min(len(i1), len(i2))} lines differ")
    return ok, msgs


def graph_names(list_path: str):
    with open(list_path) as f:
        return [line.split("\t", 1)[0].split()[0] for line in f.read().splitlines()
                if line.strip()]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("path1")
    ap.add_argument("path2")
    ap.add_argument("graph_list")
    ap.add_argument("--float", dest="is_float", action="store_true",
                    help="float distances (%%f text, or raw .bin words)")
    ap.add_argument("--max-report", type=int, default=5)
    try:
        a = ap.parse_args(argv)
    except SystemExit:
        return 2
    if not os.path.exists(a.graph_list):
        print(f"graph list not found: {a.graph_list}")
        return 2
    all_ok = True
    for g in graph_names(a.graph_list):
        f1, f2 = a.path1 + g, a.path2 + g
        ok, msgs = compare_files(f1, f2, a.is_float, a.max_report)
        print(f"{g}: {'match' if ok else 'MISMATCH'}")
        for m in msgs:
            print("  " + m)
        all_ok = all_ok and ok
    print("all results match!!!" if all_ok else "result mismatch!!!")
    return 0 if all_ok else 1


if __name__ == "__main__":
    sys.exit(main())
