"""The FP32 band of the FP32 + FP64-recheck form, checked in exact arithmetic
on the CPU (the GPU side is in test_gpu_parity.py).

The kernel tests a pair with d2_32 = fma(dz, dz, fma(dy, dy, dx * dx)) and
decides it without the double expression of FOF.c:351-357 only outside the
band [t_lo, t_hi] = fl32(l^2) -+ 4 ulp (8 ulp for FP64 positions, whose FP32
differences carry one more rounding).  The claim: d2_32 < t_lo implies the
double test links, d2_32 > t_hi implies it does not."""
from fractions import Fraction

import numpy as np
import pytest

from oracle import cpu, reference
from tests.band_pairs import d2_double, d2_fp32, f32, f64, make_band_workload, ulp32


def band(l2d, ulps):
    """The kernel's thresholds (band_thresholds in fof_kernels.cuh): fl32(l2)
    -+ ulps * ulp, rounded outwards to float."""
    l2f = f32(l2d)
    u = ulp32(l2f)
    lo, hi = l2f - ulps * u, l2f + ulps * u
    flo, fhi = f32(lo), f32(hi)
    if flo > lo:
        flo -= ulp32(flo)
    if fhi < hi:
        fhi += ulp32(fhi)
    return flo, fhi


@pytest.mark.parametrize("fp64", [False, True])
def test_band_proof_holds_in_exact_arithmetic(fp64):
    """Random pairs at distance l (1 +- 1e-6) over linking lengths 1e-3..50
    and coordinates up to 4000: outside the band the FP32 decision is always
    the double one, and the sweep does put pairs inside the band."""
    rng = np.random.default_rng(41 if fp64 else 40)
    inside = outside = 0
    for _ in range(6000):
        ll = float(10 ** rng.uniform(-3, np.log10(50)))
        l2d = f64(Fraction(ll) * Fraction(ll))
        t_lo, t_hi = band(l2d, 8 if fp64 else 4)
        mag = float(10 ** rng.uniform(-1, np.log10(4000)))
        p = rng.uniform(-mag, mag, 3)
        v = rng.normal(size=3)
        q = p + ll * (1 + rng.normal() * 1e-6) * v / np.linalg.norm(v)
        if fp64:
            P = [Fraction(float(x)) for x in p]
            Q = [Fraction(float(x)) for x in q]
            d = [f64(Q[a] - P[a]) for a in range(3)]        # double differences
        else:
            P = [Fraction(float(np.float32(x))) for x in p]
            Q = [Fraction(float(np.float32(x))) for x in q]
            d = [f32(Q[a] - P[a]) for a in range(3)]        # float differences
        g32 = d2_fp32(d)
        linked = not (d2_double(d) > l2d)
        if g32 < t_lo:
            assert linked, (ll, p, q)
            outside += 1
        elif g32 > t_hi:
            assert not linked, (ll, p, q)
            outside += 1
        else:
            inside += 1
    assert inside > 100 and outside > 1000, (inside, outside)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_band_pairs_cover_the_band(dtype):
    """The constructed pairs reach every offset the GPU test needs, on both
    sides of the double threshold, including pairs that the FP32 value
    alone decides wrongly -- all of them inside the band."""
    w, cases = make_band_workload(dtype)
    width = 8 if dtype == np.float64 else 4
    ks = {k for k, _, _ in cases}
    assert {0, 1, -1, 3, -3, 4, -4, 5, -5} <= ks
    assert any(l64 for _, l64, _ in cases) and any(not l64 for _, l64, _ in cases)
    wrong = [(k, l64) for k, l64, l32 in cases if l64 != l32]
    assert len(wrong) >= 4, wrong
    assert all(abs(k) <= width for k, _ in wrong), wrong
    assert sum(abs(k) <= width for k, _, _ in cases) >= 20


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_oracle_links_exactly_the_double_pairs(dtype):
    w, cases = make_band_workload(dtype)
    o = cpu.run(w)
    g = o["group"]
    got = [bool(g[2 * i] == g[2 * i + 1]) for i in range(len(cases))]
    assert got == [l64 for _, l64, _ in cases]
    # pairs never link to one another
    assert np.unique(g).shape[0] == w.n - sum(got)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reference_binary_links_the_same_pairs(dtype):
    fp64 = dtype == np.float64
    if not reference.available("cmh_ref_f64" if fp64 else "cmh_ref_f32"):
        pytest.skip("reference binaries not built")
    w, cases = make_band_workload(dtype)
    src, ppos, _ = cpu.build_proc(w)
    halos, _ = reference.run_proc(w, ppos, w.vel[src].astype(ppos.dtype), w.ids[src], timeout=120)
    linked_pairs = sorted(int(h["ids"].min()) // 2 for h in halos)
    assert all(h["ids"].shape[0] == 2 for h in halos)
    assert linked_pairs == [i for i, (_, l64, _) in enumerate(cases) if l64]


def vl_band(lsq, ulps):
    """The kernels' band for a variable l^2 (vl_band in fof_kernels.cuh):
    from 2 ulps float steps below fl32(l^2) to ulps steps above."""
    b = int(np.array([lsq], np.float32).view(np.uint32)[0])
    lo = np.array([b - 2 * ulps], np.uint32).view(np.float32)[0]
    hi = np.array([b + ulps], np.uint32).view(np.float32)[0]
    return Fraction(float(lo)), Fraction(float(hi))


@pytest.mark.parametrize("ulps", [4, 8])
def test_variable_length_band_contains_the_proven_band(ulps):
    """Whatever fl32(l^2) is -- inside a binade or just above a power of two,
    where the steps below are half as wide -- the band derived from its bits
    contains band_thresholds()'s, so the proof covers it."""
    rng = np.random.default_rng(7 + ulps)
    vals = list(10 ** rng.uniform(-6, 4, 3000))
    for e in range(-20, 14):  # at and just around powers of two
        for d in (-3, -1, 0, 1, 2, 5, 9):
            vals.append(float(np.nextafter(np.float32(2.0 ** e), np.float32(np.inf)) * 1.0)
                        + d * 2.0 ** (e - 23))
    for v in vals:
        if v <= 0:
            continue
        l2d = f64(Fraction(v))
        lo, hi = vl_band(float(l2d), ulps)
        rlo, rhi = band(l2d, ulps)
        assert lo <= rlo and hi >= rhi, (v, lo, rlo, hi, rhi)
