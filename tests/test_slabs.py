"""One box split over ranks (cm_halofinder_b200.slabs), on CPU.

Routing: every particle reaches its owner once and, as a ghost, exactly the
ranks whose padded domain holds it or its periodic image (read_data.c:409-521
with the single-box image rule).  Distributed run: gloo ranks, each holding
a share of the particles as if read from its own files, exchange the copies
with one all-to-all, run the oracle's isolated FoF on their padded domain
and keep the halos whose centre of mass they own; the union of their
catalogs must be the single-box oracle catalog: the same member ID sets,
properties within 1e-6 (sums run in a different order)."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest
import torch

from cm_halofinder_b200 import synth
from cm_halofinder_b200.slabs import SlabSplit, halo_id_sets

PROP_TOL = 1e-6


def _box(seed=801, n=12000, L=60.0, periodic=True):
    w = synth.make_box(n, L, 250, seed, nphalomin=5, boundary=4.0)
    if not periodic:
        w.periodic = False
    return w


def _padded(split, rank):
    rmin, rmax = split.domain(rank)
    b = split.boundary
    return np.array(rmin) - b, np.array(rmax) + b


@pytest.mark.parametrize("grid", [(2, 1, 1), (2, 2, 1), (3, 2, 2), (1, 1, 1)])
def test_route_reaches_every_padded_domain_once(grid):
    w = _box()
    split = SlabSplit(w.lo, w.hi, grid, w.boundary, periodic=True)
    pos = torch.from_numpy(w.pos)
    src, dest, shift, n_out = split.route(pos)
    assert n_out == 0
    L = np.array(w.hi) - np.array(w.lo)
    got = {}
    for s, d, sh in zip(src.tolist(), dest.tolist(), shift.tolist()):
        key = (s, d, tuple(sh))
        assert key not in got, "a copy sent twice"
        got[key] = 1
    # owners: one copy with no shift, in the rank whose domain holds the particle
    x = w.pos.astype(np.float64)
    for r in range(split.nranks):
        lo, hi = _padded(split, r)
        for sh in np.array(np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1])).T.reshape(-1, 3):
            y = x + sh * L
            want = np.nonzero(((y > lo) & (y < hi)).all(axis=1))[0]
            have = sorted(s for (s, d, t) in got if d == r and t == tuple(sh))
            assert have == sorted(want.tolist()), (r, sh)


def test_route_isolated_drops_outside_and_never_shifts():
    w = _box(periodic=False)
    pos = w.pos.copy()
    pos[:50, 0] = -w.boundary - 1.0   # beyond the padded box
    split = SlabSplit(w.lo, w.hi, (2, 2, 1), w.boundary, periodic=False)
    src, dest, shift, n_out = split.route(torch.from_numpy(pos))
    assert n_out == 50
    assert int(shift.abs().sum()) == 0
    assert not np.isin(np.arange(50), src.numpy()).any()
    # every kept particle has exactly one owner copy
    own = np.zeros(pos.shape[0], int)
    for r in range(split.nranks):
        rmin, rmax = split.domain(r)
        sel = (dest == r).numpy()
        s = src.numpy()[sel]
        inside = ((pos[s] >= np.array(rmin)) & (pos[s] < np.array(rmax))).all(axis=1)
        own[s[inside]] += 1
    kept = ((pos >= np.array(w.lo)) & (pos < np.array(w.hi))).all(axis=1)
    assert (own[kept] == 1).all()


def test_domains_follow_set_params():
    split = SlabSplit((0.0, 10.0, -5.0), (100.0, 40.0, 5.0), (4, 3, 2), 2.0)
    seen = set()
    for r in range(split.nranks):
        ix, iy, iz = split.coords(r)
        assert r == 4 * 3 * iz + 4 * iy + ix
        seen.add((ix, iy, iz))
        rmin, rmax = split.domain(r)
        assert rmin[0] == ix * (100.0 / 4) + 0.0 and rmax[1] == rmin[1] + 30.0 / 3
    assert len(seen) == 24


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, grid, periodic, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import datetime

    import torch.distributed as dist

    from cm_halofinder_b200 import slabs
    from oracle import cpu
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w = _box(periodic=periodic)
        split = SlabSplit(w.lo, w.hi, grid, w.boundary, periodic=periodic)
        # this rank's share of the input, as read from its own files
        share = np.array_split(np.arange(w.n), world)[rank]
        pos = torch.from_numpy(w.pos[share])
        vel = torch.from_numpy(w.vel[share])
        ids = torch.from_numpy(w.ids[share].astype(np.int64))
        rp, rv, ri, _ = slabs.exchange(dist, split, pos, vel, ids)
        rmin, rmax = split.domain(rank)
        lw = synth.Workload(name="slab", pos=rp.numpy(), vel=rv.numpy(),
                            ids=ri.numpy().astype(np.uint64), lo=rmin, hi=rmax,
                            linklength=w.linklength, boundary=w.boundary,
                            nphalomin=w.nphalomin, periodic=False,
                            cells=max(int((rmax[0] - rmin[0]) / (2 * w.linklength)), 1))
        res = cpu.run(lw)
        nh = res["stats"]["nhalos"]
        sets = halo_id_sets(res["member"], ri.numpy(), nh)
        mine = [(s, res["halo_props"][h].tolist()) for h, s in enumerate(sets)]
        allh = [None] * world
        dist.all_gather_object(allh, mine)
        if rank == 0:
            out.put([h for part in allh for h in part])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("grid,periodic", [((2, 1, 1), True), ((2, 2, 1), True),
                                           ((3, 1, 1), True), ((2, 2, 1), False)])
def test_gloo_ranks_find_the_single_box_catalog(grid, periodic):
    from oracle import cpu
    world = grid[0] * grid[1] * grid[2]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, grid, periodic, out))
             for r in range(world)]
    for p in procs:
        p.start()
    halos = out.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    w = _box(periodic=periodic)
    ref = cpu.run(w)
    nh = ref["stats"]["nhalos"]
    ref_sets = halo_id_sets(ref["member"], w.ids, nh)
    got = {s: p for s, p in halos}
    assert len(got) == len(halos) == nh > 20
    assert set(got) == set(ref_sets)
    L = np.array(w.hi) - np.array(w.lo)
    for h, s in enumerate(ref_sets):
        a, b = np.array(got[s]), ref["halo_props"][h].astype(np.float64)
        assert a[0] == b[0]
        d = np.abs(a[1:4] - b[1:4])
        d = np.minimum(d, np.abs(L - d)) if periodic else d   # centres modulo the box
        assert (d <= PROP_TOL * np.maximum(np.abs(b[1:4]), 1.0)).all()
        assert np.allclose(a[4:7], b[4:7], rtol=PROP_TOL, atol=PROP_TOL * 300.0)
