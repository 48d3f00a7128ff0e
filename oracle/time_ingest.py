"""Times graph ingest (.gr file -> device CSR): the reference's reader and
upload (oracle/_ref/ref_ingest: CSRGraph::read + copy_to_gpu,
ads_int/csr_graph.cu:203-328) against adds_graph_load_gr, on the same file.
MEASUREMENT INFRASTRUCTURE ONLY.  Needs a GPU.

  python oracle/time_ingest.py [scale] [out.json]

The file is an R-MAT graph (int32 weights U[1,10000]; scale 23 gives about
1.1 GB) written by adds_graph_save_gr to a temporary directory.  Each side
reads it twice and reports the second (page-cached) time too; both sides
end with the CSR on the GPU (the reference keeps the host copy as well).
"""
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import adds_b200 as A  # noqa: E402


def main():
    scale = int(sys.argv[1]) if len(sys.argv) > 1 else 23
    out_json = sys.argv[2] if len(sys.argv) > 2 else None
    g = A.Graph.generate(A.gen_spec("rmat", scale=scale, wtype=0, w_lo=1, w_hi=10000, seed=scale),
                         0)
    n, m = g.n, g.m
    res = {"graph": f"R-MAT {scale} int32", "n": n, "m": m}
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_ingest")
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, f"rmat{scale}.gr")
        g.save_gr(p)
        g.close()
        res["file_bytes"] = os.path.getsize(p)
        if os.path.exists(ref):
            runs = []
            for _ in range(2):
                r = subprocess.run([ref, p], capture_output=True, text=True, timeout=900)
                if r.returncode != 0:
                    runs.append({"error": r.stderr[-400:]})
                    break
                runs.append(json.loads(r.stdout.strip().splitlines()[-1]))
            res["reference"] = runs
        else:
            res["reference"] = "oracle/_ref/ref_ingest not built (oracle/build_ref.sh)"
        ours = []
        for _ in range(2):
            t0 = time.perf_counter()
            h = A.Graph.load_gr(p, A.ADDS_I32, 0)
            t1 = time.perf_counter()
            ours.append({"load_s": t1 - t0})
            assert h.n == n and h.m == m
            h.close()
        res["ours"] = ours
    for k in ("reference", "ours"):
        runs = res.get(k)
        if isinstance(runs, list) and runs and "error" not in runs[-1]:
            last = runs[-1]
            tot = last.get("load_s", last.get("read_s", 0) + last.get("upload_s", 0))
            res[f"{k}_warm_s"] = tot
            res[f"{k}_warm_gb_per_s"] = res["file_bytes"] / tot / 1e9
    if "reference_warm_s" in res and "ours_warm_s" in res:
        res["speedup_warm"] = res["reference_warm_s"] / res["ours_warm_s"]
    txt = json.dumps(res, indent=1)
    print(txt)
    if out_json:
        with open(out_json, "w") as f:
            f.write(txt)


if __name__ == "__main__":
    main()
