"""The variable-linking-length rule of the oracle against an independent
brute-force restatement (every pair tested, numpy, no cell lists).

Rule (FOF.c:45-153 with link.c's per-cell length): the fixed grid has
`cells` cells per axis of side (hi - lo + 2 b) / cells from lo - b; a cell's
l is the table l(r) at the distance of its centre from the observer (linear
interpolation on r = 0, dr, ..., rmax; the last value beyond); a pair is
tested only when its cells are equal or neighbours, with the l of the lower
cell in (z, y, x) order, and links when ((dx dx + dy dy) + dz dz) <= l^2 in
double, dx the float difference for float positions.
"""
import numpy as np

from cm_halofinder_b200 import synth
from oracle import cpu


def _cell_linksq(w, ic):
    lo = np.array(w.lo, np.float64)
    hi = np.array(w.hi, np.float64)
    b = w.boundary
    rmin = lo - b
    lcell = (hi - lo + 2.0 * b) / w.cells
    org = np.array(w.varlink["origin"], np.float64)
    c = (rmin - org) + (ic.astype(np.float64) + 0.5) * lcell
    q = (c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1]) + c[:, 2] * c[:, 2]
    tab = np.asarray(w.varlink["table"], np.float64)
    dr = w.varlink["rmax"] / float(len(tab) - 1)
    t = np.sqrt(q) / dr
    i = np.minimum(t.astype(np.int64), len(tab) - 2)
    f = t - i
    lin = tab[i] * (1.0 - f) + tab[i + 1] * f
    lv = np.where(t >= len(tab) - 1, tab[-1], lin)
    return lv * lv


def _brute_groups(w, ppos):
    lo = np.array(w.lo, np.float64)
    hi = np.array(w.hi, np.float64)
    b = w.boundary
    rmin = lo - b
    lcell = (hi - lo + 2.0 * b) / w.cells
    ic = np.floor((ppos.astype(np.float64) - rmin) / lcell).astype(np.int64)
    lsq = _cell_linksq(w, ic)
    order_key = (ic[:, 2] << 42) | (ic[:, 1] << 21) | ic[:, 0]
    m = ppos.shape[0]
    parent = np.arange(m)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for i in range(m - 1):
        j = np.arange(i + 1, m)
        d = (ppos[i][None, :] - ppos[j]).astype(np.float64)   # float differences
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        nb = np.all(np.abs(ic[j] - ic[i]) <= 1, axis=1)
        lower = np.where(order_key[j] < order_key[i], j, i)
        ok = nb & ~(d2 > lsq[lower])
        for jj in j[ok]:
            a, c = find(i), find(int(jj))
            if a != c:
                parent[max(a, c)] = min(a, c)
    return np.array([find(x) for x in range(m)])


def test_varlink_oracle_matches_brute_force():
    n = 3000
    w = synth.make_lightcone(n, 1400.0 * (n / 50_000_000) ** (1 / 3), 60, 31)
    src, ppos, _ = cpu.build_proc(w)
    out = cpu.fof_proc(w, src, ppos, w.vel[src], n_src=w.n)
    want = _brute_groups(w, ppos)
    np.testing.assert_array_equal(out["group"], want)
    # the table actually varies over the sample: lengths differ across cells
    lo = np.array(w.lo) - w.boundary
    lcell = (np.array(w.hi) - np.array(w.lo) + 2 * w.boundary) / w.cells
    ic = np.floor((ppos.astype(np.float64) - lo) / lcell).astype(np.int64)
    ls = _cell_linksq(w, ic)
    assert ls.max() / ls.min() > 1.3
    assert (np.bincount(want) > 1).sum() > 10   # groups formed


def test_varlink_lower_cell_rule_is_asymmetric():
    """Two particles 1.5 apart straddling a cell face link with the lower
    cell's l, whichever of the two cells has the longer one."""
    tab = np.array([1.0, 1.0, 2.0, 2.0])         # l(r): 1 below r = 10, 2 from r = 20
    L = 60.0
    pos = np.array([[14.5, 0.5, 0.5], [16.0, 0.5, 0.5]], np.float32)
    w = synth.Workload(name="pair", pos=pos, vel=np.zeros_like(pos),
                       ids=np.arange(2, dtype=np.uint64), lo=(0.0,) * 3, hi=(L,) * 3,
                       linklength=2.0, boundary=0.0, nphalomin=2, periodic=False, cells=20,
                       varlink={"origin": (0.0, 0.0, 0.0), "rmax": 30.0, "table": tab})
    # cells of side 3: the pair sits in x-cells 4 and 5 (centres 13.5 and
    # 16.5); observer at 0: l = 1.37 (lower cell) and 1.66 -> not linked
    out = cpu.run(w)
    assert out["group"][0] != out["group"][1]
    # observer at x = 30: the lower cell now has l = 1.66 (upper 1.37) -> linked
    w.varlink["origin"] = (30.0, 0.0, 0.0)
    out = cpu.run(w)
    assert out["group"][0] == out["group"][1]
