"""Batched boxes (many domains in one run), graph replay and the capacity
rerun path, against the CPU oracle box by box."""
import numpy as np
import pytest

import cm_halofinder_b200 as cmh

from cm_halofinder_b200 import FofConfig, Plan, fof, synth
from oracle import cpu
from tests.helpers import assert_same_catalog

pytestmark = pytest.mark.gpu


def _boxes(nbox, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nbox):
        n = int(np.exp(rng.uniform(np.log(2000), np.log(20000))))
        L = 1000.0 * (n / 256 ** 3) ** (1 / 3)
        out.append(synth.make_box(n, L, max(1, round(10000 * n / 256 ** 3)), seed * 100 + i,
                                  linkb=float(rng.uniform(0.15, 0.25)), boundary=6.0))
    return out


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_matches_oracle_per_box(precision):
    import torch
    boxes = _boxes(7, 5)
    cfgs = [FofConfig.from_workload(w, precision=precision) for w in boxes]
    pos = [torch.from_numpy(w.pos).cuda() for w in boxes]
    vel = [torch.from_numpy(w.vel).cuda() for w in boxes]
    plan = Plan(cfgs[0])
    cats = plan.run_batch(cfgs, pos, vel)
    for w, cat in zip(boxes, cats):
        ref = cpu.run(w)
        assert cat.stats["n_in"] == w.n
        assert_same_catalog(cat, ref, check_member=False)
    # a second run of the same shape replays the captured graph
    cats2 = plan.run_batch(cfgs, pos, vel)
    for a, b in zip(cats, cats2):
        np.testing.assert_array_equal(a.head, b.head)
        np.testing.assert_array_equal(a.props[:, 0], b.props[:, 0])


def test_graph_replay_single_box():
    import torch
    w = synth.config2(seed=301, scale=40000 / 256 ** 3)
    ref = cpu.run(w)
    plan = Plan(FofConfig.from_workload(w))
    pos = torch.from_numpy(w.pos).cuda()
    vel = torch.from_numpy(w.vel).cuda()
    for _ in range(3):  # eager + capture, then replays
        cat = plan.run(pos, vel, members=True)
        assert_same_catalog(cat, ref)
    plan.set_graph(False)
    cat = plan.run(pos, vel, members=True)
    assert_same_catalog(cat, ref)


def test_image_overflow_reruns_with_room():
    """All particles in one corner: every one has 7 images, far above the
    geometric estimate; the run must notice and repeat with larger buffers."""
    rng = np.random.default_rng(3)
    L, b = 100.0, 2.0
    pos = rng.uniform(0.0, 1.5, (20000, 3)).astype(np.float32)
    vel = rng.normal(0, 300, pos.shape).astype(np.float32)
    w = synth.Workload(name="corner", pos=pos, vel=vel, ids=np.arange(len(pos), dtype=np.uint64),
                       lo=(0.0,) * 3, hi=(L,) * 3, linklength=0.05, boundary=b, nphalomin=5,
                       periodic=True, cells=40)
    cat = fof(w.pos, w.vel, FofConfig.from_workload(w), members=True)
    ref = cpu.run(w)
    assert cat.stats["n_images"] == ref["stats"]["n_images"] == 7 * 20000
    assert_same_catalog(cat, ref)


def test_autotune_keeps_results():
    """The autotuner only changes cell sizes and the dense-top threshold; the
    catalogs after tuning match the oracle box by box."""
    import torch
    boxes = _boxes(5, 9)
    cfgs = [FofConfig.from_workload(w) for w in boxes]
    pos = [torch.from_numpy(w.pos).cuda() for w in boxes]
    vel = [torch.from_numpy(w.vel).cuda() for w in boxes]
    plan = Plan(cfgs[0])
    t = plan.autotune(cfgs, pos, vel, repeats=1)
    assert t["tried"] == 15 and t["ms"] > 0
    assert t["cell_scale"] in (0.5, 0.75, 1.0, 1.5, 2.0) and t["dense_min"] in (8, 16, 32)
    cats = plan.run_batch(cfgs, pos, vel)
    for w, cat in zip(boxes, cats):
        assert_same_catalog(cat, cpu.run(w), check_member=False)


@pytest.mark.parametrize("scale", [0.5, 2.0])
def test_cell_scale_extremes(scale):
    """The coarsest and finest cell grids the tuner tries give the same
    catalog (set here through an explicit cell-size factor)."""
    w = synth.config2(seed=311, scale=30000 / 256 ** 3)
    ref = cpu.run(w)
    sep = (float(np.prod(np.array(w.hi) - np.array(w.lo))) / w.n) ** (1 / 3)
    h = w.linklength * (1 - 2 ** -20) / 3 ** 0.5
    k = max(2, min(32, int(round(sep / h * scale))))
    cat = fof(w.pos, w.vel, FofConfig.from_workload(w, cell_factor=k), members=True)
    assert cat.stats["cell_factor"] == k
    assert_same_catalog(cat, ref)


def test_host_inputs_repeated_runs_overlap_velocity_copy():
    """Host-resident inputs: velocities are copied on a side stream while the
    first stages run; eager, captured and replayed runs all match."""
    w = synth.config2(seed=321, scale=40000 / 256 ** 3)
    ref = cpu.run(w)
    plan = Plan(FofConfig.from_workload(w))
    for i in range(4):
        vel = w.vel if i % 2 == 0 else w.vel.copy()  # a fresh host buffer every other run
        cat = plan.run(w.pos, vel, members=True)
        assert_same_catalog(cat, ref)


def test_graph_replay_after_an_eager_run_of_another_shape():
    """Run A is recorded in a graph; run B (another linking length) is issued
    eagerly with graphs off, which replaces the device's box table; A replayed
    afterwards must use A's table again."""
    import torch
    w = synth.config2(seed=401, scale=30000 / 256 ** 3)
    dev = torch.device("cuda", 0)
    pos, vel = torch.from_numpy(w.pos).to(dev), torch.from_numpy(w.vel).to(dev)
    cfg_a = FofConfig.from_workload(w)
    cfg_b = FofConfig.from_workload(w)
    cfg_b.linklength = 1.3 * w.linklength
    ref_a = cpu.run(w)
    plan = Plan(cfg_a)
    try:
        for _ in range(2):
            assert_same_catalog(plan.run(pos, vel, members=True), ref_a)
        plan.set_graph(False)
        plan.set_config(cfg_b)
        cat_b = plan.run(pos, vel, members=True)
        # the longer length gathers more particles into the halos
        assert cat_b.props[:, 0].sum() > ref_a["halo_props"][:, 0].sum()
        plan.set_graph(True)
        plan.set_config(cfg_a)
        for _ in range(2):
            assert_same_catalog(plan.run(pos, vel, members=True), ref_a)
    finally:
        plan.close()


def test_prefetched_host_inputs():
    """Host inputs copied ahead with prefetch(): each run uses the copy staged
    for its arrays (one step ahead, alternating between the plan's two input
    buffers and their two recorded graphs); a run given other arrays drops
    what was staged; a third pending prefetch is refused."""
    import torch
    ws = [synth.config2(seed=420 + i, scale=25000 / 256 ** 3) for i in range(2)]
    refs = [cpu.run(w) for w in ws]
    host = [(torch.from_numpy(w.pos).pin_memory().numpy(),
             torch.from_numpy(w.vel).pin_memory().numpy()) for w in ws]
    plan = Plan(FofConfig.from_workload(ws[0]))
    try:
        order = [0, 0, 0, 0, 0]
        plan.prefetch(*host[order[0]])
        for i, k in enumerate(order):
            if i + 1 < len(order):
                plan.prefetch(*host[order[i + 1]])
            assert_same_catalog(plan.run(*host[k], members=True), refs[k])
        # staged for box 0, run on box 1: the staged copy is dropped
        plan.set_config(FofConfig.from_workload(ws[1]))
        plan.prefetch(*host[0])
        assert_same_catalog(plan.run(*host[1], members=True), refs[1])
        plan.prefetch(*host[1])
        plan.prefetch(*host[1])
        with pytest.raises(cmh.CmhError):
            plan.prefetch(*host[1])
        for _ in range(2):
            assert_same_catalog(plan.run(*host[1], members=True), refs[1])
    finally:
        plan.close()


def test_host_batch_with_prefetch():
    """A batch of host-resident boxes: copied inside the call, or staged one
    step ahead with prefetch_batch (both input buffers in turn); every box
    matches the oracle.  A batch mixing host and device boxes is refused."""
    import torch
    boxes = _boxes(5, 9)
    refs = [cpu.run(w) for w in boxes]
    cfgs = [FofConfig.from_workload(w) for w in boxes]
    hpos = [torch.from_numpy(w.pos).pin_memory().numpy() for w in boxes]
    hvel = [torch.from_numpy(w.vel).pin_memory().numpy() for w in boxes]
    plan = Plan(cfgs[0])
    try:
        def check(cats):
            for cat, ref in zip(cats, refs):
                assert_same_catalog(cat, ref, check_member=False)
        check(plan.run_batch(cfgs, hpos, hvel))          # copied in the call
        plan.prefetch_batch(hpos, hvel)
        for i in range(4):
            if i + 1 < 4:
                plan.prefetch_batch(hpos, hvel)
            check(plan.run_batch(cfgs, hpos, hvel))
        # staged for these boxes, run on a subset: the staged copy is dropped
        plan.prefetch_batch(hpos, hvel)
        cats = plan.run_batch(cfgs[:3], hpos[:3], hvel[:3])
        for cat, ref in zip(cats, refs[:3]):
            assert_same_catalog(cat, ref, check_member=False)
        mpos = [torch.from_numpy(boxes[0].pos).cuda()] + hpos[1:]
        mvel = [torch.from_numpy(boxes[0].vel).cuda()] + hvel[1:]
        with pytest.raises(cmh.CmhError) as e:
            plan.run_batch(cfgs, mpos, mvel)
        assert e.value.status == 1
        with pytest.raises(ValueError):
            plan.run_batch(cfgs, mpos, hvel)
    finally:
        plan.close()


def _shell_box(seed, n=20000):
    """A periodic box whose particles all lie within Boundarysize of the
    faces on every axis: about 7 images per particle, far above the plan's
    first capacity estimate, so the first run overflows and is repeated."""
    w = synth.make_box(n, 100.0, 40, seed, boundary=10.0)
    rng = np.random.default_rng(seed)
    x = (w.pos.astype(np.float64) * 0.09) % 9.0
    flip = rng.random(x.shape) < 0.5
    w.pos = np.where(flip, 99.99 - x, x).astype(np.float32)
    return w


def test_one_input_buffer_prefetch():
    """One input buffer: the next run's copies wait until the current run
    has read its inputs (positions after ingest, velocities after the sums),
    in both the eager and the replayed runs; a run that overflows its
    capacity and repeats gets its own inputs copied again; every catalog
    matches the oracle."""
    import torch
    ws = [_shell_box(501), synth.config2(seed=502, scale=20000 / 256 ** 3)]
    refs = [cpu.run(w) for w in ws]
    host = [(torch.from_numpy(w.pos).pin_memory().numpy(),
             torch.from_numpy(w.vel).pin_memory().numpy()) for w in ws]
    plan = Plan(FofConfig.from_workload(ws[0]))
    try:
        plan.set_input_buffers(1)
        # box 0 overflows on its first run, with box 1's copies already queued
        plan.prefetch(*host[0])
        plan.prefetch(*host[1])
        assert_same_catalog(plan.run(*host[0], members=True), refs[0])
        plan.set_config(FofConfig.from_workload(ws[1]))
        assert_same_catalog(plan.run(*host[1], members=True), refs[1])
        # a stream of runs of one box: eager, captured, then replays
        plan.prefetch(*host[1])
        for i in range(5):
            if i + 1 < 5:
                plan.prefetch(*host[1])
            assert_same_catalog(plan.run(*host[1], members=True), refs[1])
        # a run on device-resident particles between them leaves the staged
        # copies alone (it records no free events to wait for)
        dpos = torch.from_numpy(ws[1].pos).cuda()
        dvel = torch.from_numpy(ws[1].vel).cuda()
        plan.prefetch(*host[1])
        plan.prefetch(*host[1])
        assert_same_catalog(plan.run(dpos, dvel, members=True), refs[1])
        for _ in range(2):
            assert_same_catalog(plan.run(*host[1], members=True), refs[1])
        with pytest.raises(cmh.CmhError):
            plan.set_input_buffers(3)
    finally:
        plan.close()


def test_dense_slots_beyond_capacity_then_grown():
    """Every top cell of two or more fine cells dense (dense_min 1, large top
    cells): the first run has far more dense top cells than slots, leaves
    the rest to the sparse path and asks for more slots; every run, before
    and after the growth, eager and replayed, matches the oracle."""
    import torch
    w = synth.config2(seed=511, scale=200000 / 256 ** 3)
    ref = cpu.run(w)
    pos = torch.from_numpy(w.pos).cuda()
    vel = torch.from_numpy(w.vel).cuda()
    plan = Plan(FofConfig.from_workload(w))
    try:
        plan.set_tuning({"cell_scale": 2.0, "dense_min": 1})
        cats = [plan.run(pos, vel, members=True) for _ in range(3)]
        assert cats[0].stats["n_dense_tops"] > 200000 // 1024 + 1024
        for cat in cats:
            assert_same_catalog(cat, ref)
    finally:
        plan.close()


def test_one_input_buffer_batch_prefetch():
    """prefetch_batch with one input buffer: the next batch's copies wait
    until the current batch has read its inputs."""
    import torch
    boxes = _boxes(4, 13)
    refs = [cpu.run(w) for w in boxes]
    cfgs = [FofConfig.from_workload(w) for w in boxes]
    hpos = [torch.from_numpy(w.pos).pin_memory().numpy() for w in boxes]
    hvel = [torch.from_numpy(w.vel).pin_memory().numpy() for w in boxes]
    plan = Plan(cfgs[0])
    try:
        plan.set_input_buffers(1)
        plan.prefetch_batch(hpos, hvel)
        for i in range(4):
            if i + 1 < 4:
                plan.prefetch_batch(hpos, hvel)
            cats = plan.run_batch(cfgs, hpos, hvel)
            for cat, ref in zip(cats, refs):
                assert_same_catalog(cat, ref, check_member=False)
    finally:
        plan.close()
