"""A seeded sweep pinning the CPU oracle to the reference binary itself
(oracle/_ref, src_v2 built unmodified), beyond the committed golden
fixtures: small boxes over the run parameters -- periodic and isolated
(with particles in and beyond the shell), FP32 and FP64 positions, linking
lengths 0.12-0.3 of the mean separation, Nphalomin 2-20, shells of 2-8
linking lengths, sparse and crowded boxes.  Each case runs the reference on
the processing array and the oracle on the input; the halos must agree:
member ID sets in catalog order, heads, n, centres and mean velocities
within 1e-6.  Skipped where the reference is not built."""
import numpy as np
import pytest

from cm_halofinder_b200 import synth
from oracle import cpu, reference
from tests.helpers import PROP_RTOL, prop_errors

CASES = [
    # seed, n, L, clumps, linkb, nphalomin, boundary (in linking lengths), periodic, fp64
    (2001, 4000, 40.0, 40, 0.2, 5, 4.0, True, False),
    (2002, 3000, 30.0, 30, 0.3, 2, 2.0, True, False),
    (2003, 5000, 60.0, 60, 0.12, 10, 8.0, True, True),
    (2004, 4000, 50.0, 25, 0.2, 20, 5.0, False, False),
    (2005, 3500, 35.0, 50, 0.25, 3, 3.0, False, True),
    (2006, 6000, 80.0, 120, 0.2, 5, 6.0, True, False),
    (2007, 2500, 20.0, 10, 0.18, 8, 4.0, False, False),
    (2008, 4500, 45.0, 45, 0.22, 4, 2.5, True, True),
]
# and sixteen drawn from a seeded generator over the same ranges
_rng = np.random.default_rng(2100)
CASES += [(2100 + i, int(_rng.integers(2000, 6000)), float(_rng.uniform(20, 70)),
           int(_rng.integers(8, 90)), float(_rng.uniform(0.12, 0.3)), int(_rng.integers(2, 21)),
           float(_rng.uniform(2.0, 8.0)), bool(_rng.integers(0, 2)), bool(_rng.integers(0, 2)))
          for i in range(16)]


def _case(seed, n, L, clumps, linkb, nmin, bmul, periodic, fp64):
    sep = L / n ** (1.0 / 3.0)
    w = synth.make_box(n, L, clumps, seed, pos_dtype=np.float64 if fp64 else np.float32,
                       linkb=linkb, nphalomin=nmin, boundary=bmul * linkb * sep)
    w.cells = max(int((L + 2 * w.boundary) / (1.5 * w.linklength)), 1)
    if not periodic:
        w.periodic = False
        rng = np.random.default_rng(seed + 1)
        pos = w.pos.astype(np.float64)
        k = rng.choice(n, n // 20, replace=False)
        pos[k] -= rng.uniform(0.0, 1.6 * w.boundary, (k.size, 3))  # into and past the shell
        w.pos = pos.astype(w.pos.dtype)
    return w


@pytest.mark.parametrize("case", CASES, ids=[str(c[0]) for c in CASES])
def test_oracle_matches_the_reference_binary(case):
    fp64 = case[-1]
    if not reference.available("cmh_ref_f64" if fp64 else "cmh_ref_f32"):
        pytest.skip("reference binaries not built")
    w = _case(*case)
    src, ppos, _ = cpu.build_proc(w)
    halos, _ = reference.run_proc(w, ppos, w.vel[src].astype(ppos.dtype), w.ids[src],
                                  timeout=300)
    o = cpu.run(w, props=3)
    nh = o["stats"]["nhalos"]
    assert nh == len(halos)
    for h in range(nh):
        proc = np.nonzero(o["group"] == o["halo_head"][h])[0]
        np.testing.assert_array_equal(np.unique(w.ids[o["proc_src"][proc]]),
                                      np.unique(halos[h]["ids"]))
    if nh:
        np.testing.assert_array_equal(w.ids[o["proc_src"][o["halo_head"]]],
                                      np.array([int(h["ids"][0]) for h in halos], np.uint64))
        ref = np.stack([h["props"] for h in halos])
        err = prop_errors(o["halo_props"][:, :7], ref[:, :7])
        assert err[0] == 0 and np.all(err[1:] <= PROP_RTOL), err


def test_sweep_finds_halos():
    """The sweep is not vacuous: most cases hold several halos."""
    counts = [cpu.run(_case(*c))["stats"]["nhalos"] for c in CASES]
    assert sum(c >= 3 for c in counts) >= len(CASES) // 2, counts
