"""Host-side graph data: CSR container, Galois .gr v1 files, seeded generators.

The generators are the numpy twins of adds_b200/csrc/gen.cu: every random
draw is H(seed, stream, index) through the same splitmix64-style mixer, so
for the same spec both produce the identical CSR (checked by a GPU test).
They stand in for the reference's SuiteSparse / DIMACS / SNAP graphs
(graph_list_int / graph_list_float), which are not available.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

U64 = np.uint64
_M64 = (1 << 64) - 1
I32 = 0
F32 = 1


# ---------------------------------------------------------------- hashing
def _mix64(z):
    with np.errstate(over="ignore"):
        z = (z ^ (z >> U64(30))) * U64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> U64(27))) * U64(0x94D049BB133111EB)
        return z ^ (z >> U64(31))


def hash3(seed: int, stream: int, i):
    """H(seed, stream, i) of gen.cu for an array (or scalar) of indices i."""
    s = _mix64(np.array([(seed + 0x9E3779B97F4A7C15 * (stream + 1)) & _M64], dtype=U64))[0]
    i = np.asarray(i, dtype=U64)
    with np.errstate(over="ignore"):
        return _mix64(s ^ (i * U64(0xD1B54A32D192ED03) + U64(0x8CB92BA72F3D8DD7)))


def mulshift(r, n: int):
    return ((r >> U64(32)) * U64(n)) >> U64(32)


S_WEIGHT, S_SC_U, S_SC_OFF, S_ER_S, S_ER_D = 1000, 2000, 2001, 3000, 3001


# ---------------------------------------------------------------- CSR
@dataclasses.dataclass
class CSR:
    """row: uint64[n+1]; dst: uint32[m]; w: uint32[m] (int32 values or
    float32 bit patterns, per wtype)."""
    n: int
    row: np.ndarray
    dst: np.ndarray
    w: np.ndarray
    wtype: int

    @property
    def m(self) -> int:
        return int(self.dst.shape[0])

    def weights(self):
        return self.w.view(np.float32) if self.wtype == F32 else self.w.view(np.int32)

    def degrees(self):
        return np.diff(self.row).astype(np.int64)


def csr_from_keys(keys: np.ndarray, n: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Sorted unique (src<<32|dst) keys of valid edges -> row, dst, keys."""
    keys = np.unique(keys)
    keys = keys[keys != U64(_M64)]
    src = (keys >> U64(32)).astype(np.int64)
    dst = (keys & U64(0xFFFFFFFF)).astype(np.uint32)
    row = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(np.bincount(src, minlength=n), out=row[1:])
    return row, dst, keys


def hashed_weights(keys: np.ndarray, wtype: int, lo: float, hi: float, seed: int) -> np.ndarray:
    r = hash3(seed, S_WEIGHT, keys)
    if wtype == F32:
        u = (r >> U64(40)).astype(np.float32) * np.float32(2.0 ** -24)
        w = np.float32(lo) + np.float32(hi - lo) * u  # two float32 roundings, as __fadd_rn(__fmul_rn)
        return w.astype(np.float32).view(np.uint32)
    span = U64(int(hi) - int(lo) + 1)
    return (U64(int(lo)) + (((r >> U64(32)) * span) >> U64(32))).astype(np.uint32)


# ---------------------------------------------------------------- generators
def rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, wtype=I32, w_lo=1, w_hi=1000,
         seed=1, chunk=1 << 22) -> CSR:
    """R-MAT: edge_factor * 2^scale draws, self-loops and duplicates removed."""
    n = 1 << scale
    ndraw = edge_factor * n
    ab, abc = a + b, a + b + c
    parts = []
    for lo in range(0, ndraw, chunk):
        i = np.arange(lo, min(ndraw, lo + chunk), dtype=U64)
        s = np.zeros(i.shape, dtype=U64)
        d = np.zeros(i.shape, dtype=U64)
        for lvl in range(scale):
            r = hash3(seed, 1 + lvl, i)
            u = (r >> U64(11)).astype(np.float64) * (2.0 ** -53)
            q = np.where(u < a, 0, np.where(u < ab, 1, np.where(u < abc, 2, 3))).astype(U64)
            bit = U64(scale - 1 - lvl)
            s |= (q >> U64(1)) << bit
            d |= (q & U64(1)) << bit
        k = (s << U64(32)) | d
        k[s == d] = U64(_M64)
        parts.append(np.unique(k))
    row, dst, keys = csr_from_keys(np.concatenate(parts), n)
    return CSR(n, row, dst, hashed_weights(keys, wtype, w_lo, w_hi, seed), wtype)


def shortcut_offsets(radius: int):
    R = max(2, min(int(radius), 63))
    offs = [(dx, dy) for dy in range(-R, R + 1) for dx in range(-R, R + 1)
            if 2 <= abs(dx) + abs(dy) <= R]
    return np.array(offs, dtype=np.int64)


def grid(side_x: int, side_y: int, shortcut_frac=0.0, radius=8, wtype=F32, w_lo=1.0, w_hi=100.0,
         seed=1) -> CSR:
    """4-neighbour bidirectional grid plus shortcut pairs (both directions)
    to a vertex at Manhattan distance 2..radius; out-of-range draws are
    dropped, duplicates merged."""
    n = side_x * side_y
    v = np.arange(n, dtype=np.int64)
    x, y = v % side_x, v // side_x
    keys = []
    for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        nx, ny = x + dx, y + dy
        ok = (nx >= 0) & (ny >= 0) & (nx < side_x) & (ny < side_y)
        keys.append(((v[ok].astype(U64)) << U64(32)) | (ny[ok] * side_x + nx[ok]).astype(U64))
    if shortcut_frac > 0:
        egrid = 2 * (side_x - 1) * side_y + 2 * side_x * (side_y - 1)
        npairs = int(np.floor(shortcut_frac * egrid + 0.5))
        offs = shortcut_offsets(radius)
        j = np.arange(npairs, dtype=U64)
        u = mulshift(hash3(seed, S_SC_U, j), n).astype(np.int64)
        o = offs[mulshift(hash3(seed, S_SC_OFF, j), len(offs)).astype(np.int64)]
        tx, ty = u % side_x + o[:, 0], u // side_x + o[:, 1]
        ok = (tx >= 0) & (ty >= 0) & (tx < side_x) & (ty < side_y)
        uu = u[ok].astype(U64)
        tt = (ty[ok] * side_x + tx[ok]).astype(U64)
        keys.append((uu << U64(32)) | tt)
        keys.append((tt << U64(32)) | uu)
    row, dst, k = csr_from_keys(np.concatenate(keys), n)
    return CSR(n, row, dst, hashed_weights(k, wtype, w_lo, w_hi, seed), wtype)


def erdos_renyi(n: int, edge_factor=8, wtype=I32, w_lo=1, w_hi=1000, seed=1) -> CSR:
    """edge_factor * n uniform directed draws, self-loops/duplicates removed."""
    i = np.arange(edge_factor * n, dtype=U64)
    s = mulshift(hash3(seed, S_ER_S, i), n)
    d = mulshift(hash3(seed, S_ER_D, i), n)
    k = (s << U64(32)) | d
    k[s == d] = U64(_M64)
    row, dst, keys = csr_from_keys(k, n)
    return CSR(n, row, dst, hashed_weights(keys, wtype, w_lo, w_hi, seed), wtype)


def from_edges(n: int, src, dst, w, wtype=I32) -> CSR:
    """CSR from an edge list (kept in (src, input) order within a row;
    duplicates and self-loops are kept, as a .gr file may contain them)."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.uint32)
    order = np.argsort(src, kind="stable")
    row = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(np.bincount(src, minlength=n), out=row[1:])
    if wtype == F32:
        wb = np.asarray(w, dtype=np.float32).view(np.uint32)
    else:
        wb = np.asarray(w, dtype=np.int64).astype(np.uint32)
    return CSR(n, row, dst[order], wb[order], wtype)


# ---------------------------------------------------------------- .gr files
def write_gr(path: str, g: CSR, edge_size: int = 4) -> None:
    """Galois .gr v1 (csr_graph.cu:236-277 reads it): header, u64 end
    offsets, u32 dst, pad to 8 bytes, u32/f32 weights."""
    with open(path, "wb") as f:
        np.array([1, edge_size, g.n, g.m], dtype="<u8").tofile(f)
        g.row[1:].astype("<u8").tofile(f)
        g.dst.astype("<u4").tofile(f)
        if g.m % 2:
            np.zeros(1, dtype="<u4").tofile(f)
        if edge_size:
            g.w.astype("<u4").tofile(f)


def read_gr(path: str, wtype: int = I32) -> CSR:
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size < 32:
        raise ValueError("truncated .gr header")
    version, esz, n, m = (int(x) for x in raw[:32].view("<u8"))
    if version != 1 or esz not in (0, 4):
        raise ValueError("unsupported .gr version/edge size")
    need = 32 + 8 * n + 4 * m + (4 if m % 2 else 0) + (4 * m if esz else 0)
    if raw.size < need:
        raise ValueError("truncated .gr body")
    off = 32
    ends = raw[off:off + 8 * n].view("<u8")
    off += 8 * n
    dst = raw[off:off + 4 * m].view("<u4").copy()
    off += 4 * m + (4 if m % 2 else 0)
    w = raw[off:off + 4 * m].view("<u4").copy() if esz else np.zeros(m, dtype=np.uint32)
    row = np.zeros(n + 1, dtype=np.uint64)
    row[1:] = ends
    return CSR(n, row, dst, w, wtype)


def max_degree_vertex(g: CSR) -> int:
    """Source rule of the R-MAT 16 config: argmax out-degree, lowest id."""
    return int(np.argmax(g.degrees()))


def read_dist_text(path: str, wtype: int):
    """Parses a '<v> <d>' / '<v> INF' distance file into 32-bit words."""
    out = []
    inf = 0x7FFFFFFF if wtype == I32 else 0x7F7FFFFF
    with open(path) as f:
        for line in f:
            v, d = line.split()
            if d == "INF":
                out.append(inf)
            elif wtype == I32:
                out.append(int(d))
            else:
                out.append(int(np.float32(float(d)).view(np.uint32)))
    return np.array(out, dtype=np.uint32)


def dist_text(d: np.ndarray, wtype: int) -> str:
    """Reference text format of a distance array (verify.py compares this)."""
    lines = []
    for v, x in enumerate(d.tolist()):
        if wtype == I32:
            lines.append(f"{v} INF" if x == 0x7FFFFFFF else f"{v} {x}")
        else:
            lines.append(f"{v} INF" if x == 0x7F7FFFFF
                         else f"{v} {float(np.uint32(x).view(np.float32)):f}")
    return "\n".join(lines) + ("\n" if lines else "")


def ensure_dir(p):
    os.makedirs(p, exist_ok=True)
    return p
