"""Edge cases of the GPU path against the oracle: empty and one-particle
inputs, every particle in one fine cell, particles on the box faces and on
the shell edge, exact d^2 = l^2 ties, a halo that spans the periodic
boundary, coincident particles, and bad inputs that must be rejected with a
status rather than a fault."""
import numpy as np
import pytest

from cm_halofinder_b200 import CmhError, FofConfig, fof, synth
from oracle import cpu
from tests.helpers import assert_same_catalog

pytestmark = pytest.mark.gpu


def _w(pos, L=10.0, l=0.5, b=1.0, nmin=2, periodic=True, vel=None):
    pos = np.ascontiguousarray(pos)
    if vel is None:
        vel = np.random.default_rng(0).normal(0, 300, pos.shape).astype(np.float32)
    return synth.Workload(name="edge", pos=pos, vel=vel, ids=np.arange(len(pos), dtype=np.uint64),
                          lo=(0.0,) * 3, hi=(L,) * 3, linklength=l, boundary=b, nphalomin=nmin,
                          periodic=periodic, cells=max(int(L / (2 * l)), 1))


def _check(w, precision="fp32"):
    ref = cpu.run(w)
    cat = fof(w.pos, w.vel, FofConfig.from_workload(w, precision=precision), members=True)
    assert_same_catalog(cat, ref)
    return cat, ref


@pytest.mark.parametrize("n", [0, 1])
def test_empty_and_single(n):
    pos = np.full((n, 3), 5.0, np.float32)
    cat, _ = _check(_w(pos))
    assert cat.nhalos == 0


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_all_particles_in_one_fine_cell(precision):
    rng = np.random.default_rng(1)
    pos = (5.0 + rng.uniform(0, 0.01, (3000, 3))).astype(np.float32)
    cat, _ = _check(_w(pos), precision)
    assert cat.nhalos == 1 and cat.props[0, 0] == 3000


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_faces_ties_and_coincident(precision):
    """Particles on the box faces (x = 0 and x = L wrap), pairs at exactly the
    linking length (a power of two, so d^2 = l^2 is exact), coincident pairs."""
    l = 0.5
    pts = [[0.0, 1.0, 1.0], [9.75, 1.0, 1.0],          # across the periodic face: 0.25 apart
           [3.0, 3.0, 3.0], [3.5, 3.0, 3.0],            # exactly l apart: linked (d^2 <= l^2)
           [6.0, 6.0, 6.0], [6.0, 6.0, 6.0],            # coincident
           [8.0, 2.0, 2.0], [8.0, 2.5000002, 2.0],      # just beyond l: not linked
           [1.0, 9.999999, 5.0], [1.0, 0.2, 5.0]]       # near the face, 0.200001 apart through it
    pos = np.array(pts, np.float32)
    cat, ref = _check(_w(pos, l=l), precision)
    assert cat.nhalos == ref["halo_head"].shape[0] >= 3


def test_halo_across_the_periodic_corner():
    rng = np.random.default_rng(2)
    c = rng.normal(0, 0.15, (400, 3))
    pos = np.mod(c, 10.0).astype(np.float32)           # a clump centred on the corner
    pos[pos >= np.float32(10.0)] = 0
    cat, _ = _check(_w(pos, l=0.2, nmin=10))
    assert cat.nhalos == 1 and cat.props[0, 0] >= 390   # one halo, built across all 8 corners


def test_nonperiodic_shell_edges():
    """Non-periodic: particles exactly on [lo - b, hi + b] are kept, beyond
    are dropped (read_data.c:409-424)."""
    pos = np.array([[-1.0, 5, 5], [-0.9, 5, 5], [11.0, 5, 5], [10.9, 5, 5],
                    [-1.0000001, 5, 5], [11.000001, 5, 5]], np.float32)
    w = _w(pos, periodic=False, l=0.2)
    cat, ref = _check(w)
    assert cat.stats["n_out"] == ref["stats"]["n_out"] == 2


def test_bad_inputs_are_rejected():
    pos = np.zeros((10, 3), np.float32)
    w = _w(pos)
    with pytest.raises(CmhError, match="INVALID_ARGUMENT"):
        fof(pos, w.vel, FofConfig(lo=(0, 0, 0), hi=(10, 10, 10), boundary=1.0, linklength=-1.0,
                                  nphalomin=2, periodic=True))
    with pytest.raises(CmhError, match="INVALID_ARGUMENT"):
        fof(pos, w.vel, FofConfig(lo=(0, 0, 0), hi=(0, 10, 10), boundary=1.0, linklength=0.5,
                                  nphalomin=2, periodic=True))
    with pytest.raises(ValueError):  # the wrapper checks shapes before any device work
        fof(pos, w.vel[:5], FofConfig.from_workload(w))
