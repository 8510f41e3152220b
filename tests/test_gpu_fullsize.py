"""The workloads bench.py times, at full size, against the oracle.

The oracle's results on exactly these inputs (same generator, same seeds)
are committed as summaries in tests/golden/fullsize_*.npz by
tests/golden/make_fullsize.py, since the oracle needs minutes at these
sizes.  Each test regenerates the input, checks that it is the one the
fixture was made from (SHA-256 of the arrays), runs the CUDA path through
the C ABI and compares:

* the counts: dropped, images, processed, groups (singletons included),
  candidates, halos;
* per halo in catalog order: the head (lowest processing index) and n
  exactly, mean position and velocity within helpers.PROP_RTOL;
* per halo the count and hash of its member-ID set (golden_io.member_digests),
  i.e. bit-exact membership of every input particle.

Workloads: the 64^3 box with FP64 positions, the 256^3 box of the headline
number, the 50M-particle lightcone with a variable linking length, the 64
boxes of the batched run (through the batched entry point, and box by box
for the member sets), and the 1024^3 box's parameters over one eighth of
its volume (134M particles)."""
import json

import numpy as np
import pytest

from cm_halofinder_b200 import FofConfig, Plan, fof, synth
from tests import golden_io
from tests.helpers import PROP_RTOL, prop_errors

pytestmark = pytest.mark.gpu

WORKLOADS = {
    "c1": lambda: [synth.config1(seed=1)],
    "c2": lambda: [synth.config2(seed=2)],
    "c3": lambda: [synth.config3(seed=3)],
    "c4": lambda: synth.config4(seed=4),
    "c5s": lambda: [synth.config5(seed=5, scale=1 / 8)],
}
_cache = {}


def workload(name):
    """(boxes, fixture), the boxes checked against the fixture's input hash."""
    if name not in _cache:
        _cache.clear()                      # one workload in memory at a time
        fx = golden_io.load_fullsize(name)
        boxes = WORKLOADS[name]()
        assert len(boxes) == len(fx["input_sha256"])
        for w, digest in zip(boxes, fx["input_sha256"]):
            assert golden_io.input_digest(w.pos, w.vel) == str(digest), \
                f"{w.name}: the generator no longer gives the fixture's input"
        _cache[name] = (boxes, fx)
    return _cache[name]


def box_slice(fx, b):
    o = fx["box_offsets"]
    return slice(int(o[b]), int(o[b + 1]))


def check_catalog(cat, fx, b, members=True):
    sl = box_slice(fx, b)
    keys = [str(k) for k in fx["stat_keys"]]
    exp = dict(zip(keys, fx["stats"][b].tolist()))
    nh = exp["nhalos"]
    assert cat.nhalos == nh, (cat.nhalos, nh)
    np.testing.assert_array_equal(cat.head, fx["head"][sl])
    np.testing.assert_array_equal(cat.props[:, 0], fx["record"][sl, 0])
    err = prop_errors(cat.props[:, :7], fx["record"][sl])
    assert err[0] == 0 and np.all(err[1:] <= PROP_RTOL), err
    if members:
        cnt, hsh = golden_io.member_digests(cat.member, nh)
        np.testing.assert_array_equal(cnt, fx["member_count"][sl])
        np.testing.assert_array_equal(hsh, fx["member_hash"][sl])
    return exp


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_fullsize_box_matches_oracle(name, precision):
    boxes, fx = workload(name)
    w = boxes[0]
    cat = fof(w.pos, w.vel, FofConfig.from_workload(w, precision=precision), members=True)
    exp = check_catalog(cat, fx, 0)
    for k in ("n_in", "n_out", "n_images", "n_proc", "n_groups", "n_candidates"):
        assert cat.stats[k] == exp[k], (k, cat.stats[k], exp[k])
    if precision == "fp32":
        assert cat.stats["n_rechecks"] <= cat.stats["n_pair_tests"]


def test_fullsize_headline_box_through_plan_and_graph():
    """The bench's own path for the 256^3 box: a plan, device-resident
    inputs, the autotuner's choice applied, the run replayed from its
    CUDA graph."""
    import torch
    boxes, fx = workload("c2")
    w = boxes[0]
    dev = torch.device("cuda", 0)
    pos = torch.from_numpy(w.pos).to(dev)
    vel = torch.from_numpy(w.vel).to(dev)
    cfg = FofConfig.from_workload(w, precision="fp32")
    plan = Plan(cfg, pos_dtype=np.float32)
    try:
        for tuning in ({"cell_scale": 0.5, "dense_min": 32}, {"cell_scale": 1.0, "dense_min": 8}):
            plan.set_tuning(tuning)
            for _ in range(2):              # eager run, then the graph replay
                cat = plan.run(pos, vel, members=True, out="host")
                check_catalog(cat, fx, 0)
    finally:
        plan.close()


def test_fullsize_batched_boxes_match_oracle():
    """The 64 boxes of the batched run through cmh_plan_run_batch (graph
    replay on the second call), then each box alone with its members."""
    import torch
    boxes, fx = workload("c4")
    keys = [str(k) for k in fx["stat_keys"]]
    dev = torch.device("cuda", 0)
    cfgs = [FofConfig.from_workload(w, precision="fp32") for w in boxes]
    pos = [torch.from_numpy(w.pos).to(dev) for w in boxes]
    vel = [torch.from_numpy(w.vel).to(dev) for w in boxes]
    plan = Plan(cfgs[0], pos_dtype=np.float32)
    try:
        for _ in range(2):
            cats = plan.run_batch(cfgs, pos, vel)
            for b, cat in enumerate(cats):
                exp = check_catalog(cat, fx, b, members=False)
                for k in ("n_in", "n_out", "n_images", "n_proc"):
                    assert cat.stats[k] == exp[k], (b, k)
            # groups and candidates are counted over the whole run
            tot = fx["stats"].sum(axis=0)
            assert cats[0].stats["n_groups"] == tot[keys.index("n_groups")]
            assert cats[0].stats["n_candidates"] == tot[keys.index("n_candidates")]
    finally:
        plan.close()
    del pos, vel
    params = json.loads(str(fx["params"]))
    assert len(params) == len(boxes)
    for b, w in enumerate(boxes):
        cat = fof(w.pos, w.vel, cfgs[b], members=True)
        check_catalog(cat, fx, b)


def test_fullsize_1024_parameters_eighth_volume_match_oracle():
    """The 1024^3 box's parameters (mean density, clump density, Nphalomin
    20) over one eighth of its volume: 134M particles in L = 1000, one
    shot from host arrays, every halo's member set against the oracle."""
    boxes, fx = workload("c5s")
    w = boxes[0]
    cat = fof(w.pos, w.vel, FofConfig.from_workload(w, precision="fp32"), members=True)
    exp = check_catalog(cat, fx, 0)
    for k in ("n_in", "n_out", "n_images", "n_proc", "n_groups", "n_candidates"):
        assert cat.stats[k] == exp[k], (k, cat.stats[k], exp[k])
    _cache.clear()
