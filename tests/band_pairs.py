"""Particle pairs placed on the FP32 band around the squared linking length.

The FP32 + FP64-recheck form tests a pair with the FP32 value
d2_32 = fma(dz, dz, fma(dy, dy, dx * dx)) and re-tests it with the
reference's double expression ((dx*dx + dy*dy) + dz*dz) <= l^2
(FOF.c:351-357) only when d2_32 lies within `band` ulp of fl32(l^2)
(4 ulp for float positions, 8 for double ones).  These pairs put d2_32
exactly k ulp from fl32(l^2), for k in -K..K, on both sides of the double
threshold wherever the arithmetic allows, so that:

* pairs with |k| <= band must be re-checked (and counted as such),
* some of them are decided the other way by the FP32 value alone (d2_32 <=
  fl32(l^2) says linked while the double says not, or the reverse): a band
  that were too narrow, or a re-check that were skipped, gives a different
  catalog,
* pairs with |k| > band are decided by the FP32 value, which the band's
  proof says is then always the double's answer.

Every value is computed exactly with rationals: the coordinate differences,
the double expression (each operation rounded to 53 bits) and the FP32 chain
(each fused operation rounded once to 24 bits).  The pairs sit on a grid
far enough apart that no particle links to another pair.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np

from cm_halofinder_b200 import synth


def _round_bits(x: Fraction, bits: int) -> Fraction:
    """x rounded to `bits` significant bits, ties to even (normal range)."""
    if x == 0:
        return Fraction(0)
    sign = -1 if x < 0 else 1
    x = abs(x)
    e = x.numerator.bit_length() - x.denominator.bit_length()
    if Fraction(2) ** e > x:
        e -= 1
    # x in [2^e, 2^(e+1)): scale so that the kept bits are the integer part
    scaled = x / Fraction(2) ** (e - bits + 1)
    q, r = divmod(scaled.numerator, scaled.denominator)
    twice = 2 * r
    if twice > scaled.denominator or (twice == scaled.denominator and q % 2 == 1):
        q += 1
    return sign * Fraction(q) * Fraction(2) ** (e - bits + 1)


def f32(x: Fraction) -> Fraction:
    return _round_bits(x, 24)


def f64(x: Fraction) -> Fraction:
    return _round_bits(x, 53)


def d2_double(d):
    """The reference's ((dx*dx + dy*dy) + dz*dz) in double."""
    dx, dy, dz = d
    return f64(f64(f64(dx * dx) + f64(dy * dy)) + f64(dz * dz))


def d2_fp32(d):
    """fma(dz, dz, fma(dy, dy, dx * dx)) in FP32 on the FP32 differences."""
    fx, fy, fz = (f32(v) for v in d)
    return f32(fz * fz + f32(fy * fy + f32(fx * fx)))


def ulp32(x: Fraction) -> Fraction:
    e = x.numerator.bit_length() - x.denominator.bit_length()
    if Fraction(2) ** e > x:
        e -= 1
    return Fraction(2) ** (e - 23)


def make_band_workload(pos_dtype=np.float32, linklength=0.7, kmax=6, per_case=3, seed=5,
                       max_tries=40000):
    """Returns (workload, cases): a non-periodic box of isolated pairs and,
    per pair, (k, linked_by_double, linked_by_fp32_alone).  Up to per_case
    pairs of each (k, double outcome) combination that the arithmetic allows
    are searched for among max_tries random draws."""
    rng = np.random.default_rng(seed)
    dbl = np.dtype(pos_dtype) == np.float64
    l2 = Fraction(float(linklength)) * Fraction(float(linklength))
    l2d = f64(l2)                       # Linklength^2 in double (FOF.c:60)
    l2f = f32(l2d)                      # fl32(l^2)
    u = ulp32(l2f)
    # coordinate spacing of the pairs' home cell [32, 64): differences are
    # whole multiples of it, subtracted exactly (Sterbenz)
    step = Fraction(1, 2 ** 18) if not dbl else Fraction(1, 2 ** 40)
    want = {(k, side): per_case for k in range(-kmax, kmax + 1) for side in (True, False)}
    found = []
    target_s = {k: (l2f + k * u) / (step * step) for k in range(-kmax, kmax + 1)}
    # the small components tune the FP32 sum in steps well below one ulp
    bc_max = 3000 if not dbl else 1 << 30
    tries = 0
    while any(v > 0 for v in want.values()) and tries < max_tries:
        tries += 1
        k = int(rng.integers(-kmax, kmax + 1))
        b = int(rng.integers(0, bc_max))
        c = int(rng.integers(0, bc_max))
        rest = target_s[k] - b * b - c * c
        if rest <= 0:
            continue
        a = int(float(rest) ** 0.5) + int(rng.integers(-1, 2))
        d = (a * step, b * step, c * step)
        g32 = d2_fp32(d)
        kk = (g32 - l2f) / u
        if kk.denominator != 1 or abs(int(kk)) > kmax:
            continue
        kk = int(kk)
        lk64 = not (d2_double(d) > l2d)
        if want.get((kk, lk64), 0) <= 0:
            continue
        want[(kk, lk64)] -= 1
        found.append((kk, lk64, not (g32 > l2f), d))
    # place the pairs: p on a grid in [32, 64) with 2.5 between neighbours,
    # q = p + d (exact in the position type)
    n = len(found)
    side = int(np.ceil(n ** (1.0 / 3.0)))
    pos, cases = [], []
    for i, (kk, lk64, lk32, d) in enumerate(found):
        g = (i % side, (i // side) % side, i // (side * side))
        p = [Fraction(32) + Fraction(5, 2) * gi + Fraction(1, 4) for gi in g]
        q = [p[a] + d[a] for a in range(3)]
        if not dbl:
            assert all(f32(v) == v for v in p + q)
        else:
            assert all(f64(v) == v for v in p + q)
        pos.append([float(v) for v in p])
        pos.append([float(v) for v in q])
        cases.append((kk, lk64, lk32))
    pos = np.array(pos, np.float64).astype(pos_dtype)
    assert float(pos.max()) < 64.0
    vel = rng.normal(0, 300, pos.shape).astype(np.float32)
    w = synth.Workload(name=f"band_{'f64' if dbl else 'f32'}", pos=pos, vel=vel,
                       ids=np.arange(pos.shape[0], dtype=np.uint64), lo=(30.0,) * 3,
                       hi=(66.0,) * 3, linklength=float(linklength), boundary=1.0,
                       nphalomin=2.0, periodic=False, cells=12,
                       meta={"seed": seed, "pairs": n})
    return w, cases
