"""One box split over ranks, on one GPU: each rank's share of the routing
(computed with torch on the device) is found by the GPU FoF of that rank's
padded domain in turn, and the union of the ranks' catalogs must be the
single-box GPU catalog (and so the oracle's): the same member ID sets, the
same member counts, centres and mean velocities within 1e-6.  The ranks run
one after another; nothing waits on another rank."""
import numpy as np
import pytest
import torch

from cm_halofinder_b200 import FofConfig, fof, slabs, synth
from cm_halofinder_b200.slabs import SlabSplit, halo_id_sets

pytestmark = pytest.mark.gpu
PROP_TOL = 1e-6


@pytest.mark.parametrize("grid,periodic,precision", [((2, 2, 2), True, "fp32"),
                                                     ((3, 1, 1), True, "fp64"),
                                                     ((2, 2, 1), False, "fp32")])
def test_split_box_matches_single_box(grid, periodic, precision):
    w = synth.make_box(60000, 100.0, 600, 811, nphalomin=5, boundary=5.0)
    w.periodic = periodic
    split = SlabSplit(w.lo, w.hi, grid, w.boundary, periodic=periodic)
    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(w.pos).to(dev)
    vel = torch.from_numpy(w.vel).to(dev)
    ids = torch.from_numpy(w.ids.astype(np.int64)).to(dev)
    # the routing on the device is the routing on the host
    a = split.route(pos)
    b = split.route(pos.cpu())
    for x, y in zip(a[:3], b[:3]):
        assert torch.equal(x.cpu(), y)
    halos = {}
    for r in range(split.nranks):
        p, v, i = split.local_copies(pos, vel, ids, r)
        cfg = slabs.local_config(split, r, w.linklength, w.nphalomin, precision)
        cat = fof(p.cpu().numpy(), v.cpu().numpy(), cfg, members=True)
        for h, s in enumerate(halo_id_sets(cat.member, i.cpu().numpy(), cat.nhalos)):
            assert s not in halos, "a halo owned by two ranks"
            halos[s] = cat.props[h].astype(np.float64)
    single = fof(w.pos, w.vel, FofConfig.from_workload(w, precision=precision), members=True)
    ref = halo_id_sets(single.member, w.ids, single.nhalos)
    assert len(ref) == single.nhalos > 50
    assert set(halos) == set(ref)
    L = np.array(w.hi) - np.array(w.lo)
    for h, s in enumerate(ref):
        got, want = halos[s], single.props[h].astype(np.float64)
        assert got[0] == want[0]
        d = np.abs(got[1:4] - want[1:4])
        if periodic:
            d = np.minimum(d, np.abs(L - d))
        assert (d <= PROP_TOL * np.maximum(np.abs(want[1:4]), 1.0)).all()
        assert np.allclose(got[4:7], want[4:7], rtol=PROP_TOL, atol=PROP_TOL * 300.0)
