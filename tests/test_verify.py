"""The distance-file checker (python -m adds_b200.verify), on the CPU.

It takes the reference verify.py's arguments (two result directories and a
graph list) but reports a mismatch as a mismatch: the reference prints
"match" after every graph, also after a difference (verify.py:50).
"""
import os

import numpy as np

from adds_b200 import graphs as G
from adds_b200 import verify as V


def _write(d, name, words, wtype):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, name), "w") as f:
        f.write(G.dist_text(np.asarray(words, dtype=np.uint32), wtype))


def _f(x):
    return int(np.float32(x).view(np.uint32))


def test_int_match_and_mismatch(tmp_path, capsys):
    a, b = str(tmp_path / "a") + "/", str(tmp_path / "b") + "/"
    lst = tmp_path / "list"
    lst.write_text("g1\t0\ng2\t5\n")
    _write(a, "g1", [0, 3, 0x7FFFFFFF], G.I32)
    _write(b, "g1", [0, 3, 0x7FFFFFFF], G.I32)
    _write(a, "g2", [0, 7, 9, 11], G.I32)
    _write(b, "g2", [0, 7, 8, 12], G.I32)
    assert V.main([a, b, str(lst)]) == 1
    out = capsys.readouterr().out
    assert "g1: match" in out
    assert "g2: MISMATCH" in out and "2 of 4 lines differ" in out
    assert "line 3: '2 9' vs '2 8'" in out
    assert "result mismatch!!!" in out and "all results match" not in out


def test_all_match_and_missing_file(tmp_path, capsys):
    a, b = str(tmp_path / "a") + "/", str(tmp_path / "b") + "/"
    lst = tmp_path / "list"
    lst.write_text("g1\t0\n")
    _write(a, "g1", [0, 1], G.I32)
    _write(b, "g1", [0, 1], G.I32)
    assert V.main([a, b, str(lst)]) == 0
    assert "all results match!!!" in capsys.readouterr().out
    lst.write_text("g1\t0\ngone\t0\n")
    assert V.main([a, b, str(lst)]) == 1
    assert "missing" in capsys.readouterr().out


def test_length_difference_is_a_mismatch(tmp_path, capsys):
    a, b = str(tmp_path / "a") + "/", str(tmp_path / "b") + "/"
    lst = tmp_path / "list"
    lst.write_text("g\t0\n")
    _write(a, "g", [0, 1, 2], G.I32)
    _write(b, "g", [0, 1], G.I32)
    assert V.main([a, b, str(lst)]) == 1
    assert "length differs" in capsys.readouterr().out


def test_float_text_granularity_and_bits(tmp_path, capsys):
    # 1.0 and its float32 successor print alike with %f: equal as text,
    # different as bit patterns
    x, y = _f(1.0), _f(1.0) + 1
    a, b = str(tmp_path / "a") + "/", str(tmp_path / "b") + "/"
    lst = tmp_path / "list"
    lst.write_text("g\t0\n")
    _write(a, "g", [0, x, 0x7F7FFFFF], G.F32)
    _write(b, "g", [0, y, 0x7F7FFFFF], G.F32)
    assert V.main([a, b, str(lst), "--float"]) == 0
    capsys.readouterr()
    np.array([0, x], dtype="<u4").tofile(a + "h.bin")
    np.array([0, y], dtype="<u4").tofile(b + "h.bin")
    lst.write_text("h.bin\t0\n")
    assert V.main([a, b, str(lst), "--float"]) == 1
    out = capsys.readouterr().out
    assert "1 of 2 distances differ (bit patterns)" in out


def test_usage_error():
    assert V.main(["only-one"]) == 2
