"""The pull floor of float keys (phase.cu, pull_floor): a lower bound of
every heavy-edge candidate fl(d[u] + w) out of bucket `base`.

The device computes, with bw = 2^shift / scale * (1 - 1e-6),
    T = fadd_rd(double2float_rd(base * bw), double2float_rd(bw)).
A vertex at or below T is not visited by a pull phase, so T must not exceed
any candidate: for every float32 d with floor(fl(d * scale)) >> shift ==
base (the bucket) and every float32 weight w at or above the light
threshold fl(2^shift / scale) (a heavy edge), fl(d + w) >= T.  The test
restates the device arithmetic exactly (round-down conversions through
fractions) and checks the bound at the low edge of each bucket, where it
is tightest, for seeded bases, shifts and scales.
"""
from fractions import Fraction

import numpy as np

F32 = np.float32


def f32_rd(x: Fraction) -> np.float32:
    """Largest float32 not above the exact value x (x >= 0)."""
    f = F32(float(x))
    while Fraction(float(f)) > x:
        f = np.nextafter(f, F32(0))
    return f


def f32_rn_sum(a: np.float32, b: np.float32) -> np.float32:
    return F32(a) + F32(b)  # IEEE float32 addition, round to nearest


def pull_floor(base: int, shift: int, scale: float) -> np.float32:
    bw = Fraction(2.0 ** shift / float(scale) * (1.0 - 1e-6))  # the device's double
    lo = f32_rd(Fraction(float(base * float(bw))))
    dw = f32_rd(bw)
    return f32_rd(Fraction(float(lo)) + Fraction(float(dw)))


def key(d: np.float32, scale: np.float32) -> int:
    return int(np.floor(F32(d) * F32(scale)))  # __float2uint_rz(__fmul_rn(d, scale))


def bucket_low_edge(base: int, shift: int, scale: np.float32) -> np.float32:
    """Smallest float32 whose bucket is `base` (or above)."""
    target = base << shift
    d = F32(target / float(scale))
    step = 0
    while key(d, scale) >= target and d > 0 and step < 10000:
        d = np.nextafter(d, F32(0))
        step += 1
    while key(d, scale) < target:
        d = np.nextafter(d, F32(np.inf))
    return d


def light_threshold(shift: int, scale: float) -> np.float32:
    return F32(2.0 ** shift / float(scale))  # api.cu light_threshold: double, then nearest float


def test_pull_floor_bounds_every_heavy_candidate():
    rng = np.random.default_rng(5)
    checked = 0
    for _ in range(400):
        shift = int(rng.integers(0, 24))
        scale = F32(np.exp(rng.uniform(np.log(1e-3), np.log(1e7))))
        base = int(rng.integers(0, 1 << 12))
        if (base + 1) << shift >= 1 << 31:
            continue
        T = pull_floor(base, shift, float(scale))
        d = bucket_low_edge(base, shift, scale)
        assert (key(d, scale) >> shift) == base
        w0 = light_threshold(shift, float(scale))
        # the lightest heavy edges and a few heavier ones, from the bucket's
        # low edge and a little above it
        for dd in (d, np.nextafter(d, F32(np.inf)), F32(d * F32(1.0001))):
            if key(dd, scale) >> shift != base:
                continue
            for w in (w0, np.nextafter(w0, F32(np.inf)), F32(w0 * F32(1.5))):
                cand = f32_rn_sum(dd, w)
                assert cand >= T, (base, shift, float(scale), float(dd), float(w), float(cand), float(T))
                checked += 1
        # and the floor is close to the next bucket's first key, so a pull
        # still skips the settled buckets
        top = Fraction(((base + 1) << shift)) / Fraction(float(scale))
        assert Fraction(float(T)) >= top * Fraction(999, 1000) - Fraction(1, 10 ** 30)
    assert checked > 1000


def test_pull_floor_int_keys():
    """Integer keys: the floor is the next bucket's first key minus one,
    clamped at 2^32 - 1 (the device formula, restated)."""
    def floor_int(base, shift):
        t = (base + 1) << shift
        return 0xFFFFFFFF if t > 0xFFFFFFFF else t - 1
    for base, shift in ((0, 0), (0, 10), (7, 10), (1 << 20, 11), ((1 << 21) - 1, 11), (5, 31)):
        T = floor_int(base, shift)
        # the smallest heavy candidate: d = base << shift, w = 2^shift
        smallest = (base << shift) + (1 << shift)
        assert smallest > T or T == 0xFFFFFFFF
        assert T + 1 == smallest or T == 0xFFFFFFFF
