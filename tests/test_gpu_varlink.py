"""Variable linking length (lightcone) on the GPU against the CPU oracle:
exact membership, heads and order, properties within 1e-6."""
import numpy as np
import pytest

from cm_halofinder_b200 import FofConfig, Plan, fof, synth
from oracle import cpu
from tests.helpers import assert_same_catalog

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_lightcone_matches_oracle(precision):
    n = 60000
    w = synth.make_lightcone(n, 1400.0 * (n / 50_000_000) ** (1 / 3), 400, 41)
    ref = cpu.run(w)
    cat = fof(w.pos, w.vel, FofConfig.from_workload(w, precision=precision), members=True)
    assert ref["stats"]["nhalos"] > 20
    assert_same_catalog(cat, ref)


def test_lightcone_fp64_positions():
    n = 30000
    w = synth.make_lightcone(n, 1400.0 * (n / 50_000_000) ** (1 / 3), 200, 43)
    w.pos = w.pos.astype(np.float64) + np.float64(1e-9)
    ref = cpu.run(w)
    cat = fof(w.pos, w.vel, FofConfig.from_workload(w), members=True)
    assert_same_catalog(cat, ref)


@pytest.mark.parametrize("origin", [(0.0, 0.0, 0.0), (30.0, 0.0, 0.0)])
def test_lower_cell_rule(origin):
    tab = np.array([1.0, 1.0, 2.0, 2.0])
    pos = np.array([[14.5, 0.5, 0.5], [16.0, 0.5, 0.5], [40.0, 40.0, 40.0]], np.float32)
    w = synth.Workload(name="pair", pos=pos, vel=np.zeros_like(pos),
                       ids=np.arange(3, dtype=np.uint64), lo=(0.0,) * 3, hi=(60.0,) * 3,
                       linklength=2.0, boundary=0.0, nphalomin=2, periodic=False, cells=20,
                       varlink={"origin": origin, "rmax": 30.0, "table": tab})
    ref = cpu.run(w)
    for precision in ("fp32", "fp64"):
        cat = fof(w.pos, w.vel, FofConfig.from_workload(w, precision=precision), members=True)
        assert_same_catalog(cat, ref)
    assert cat.nhalos == (1 if origin[0] > 0 else 0)


def test_batch_mixes_fixed_and_variable_lengths():
    import torch
    n = 20000
    boxes = [synth.make_lightcone(n, 1400.0 * (n / 50_000_000) ** (1 / 3), 150, 51),
             synth.config2(seed=52, scale=15000 / 256 ** 3),
             synth.make_lightcone(n // 2, 1400.0 * (n / 2 / 50_000_000) ** (1 / 3), 80, 53),
             synth.config2(seed=54, scale=9000 / 256 ** 3)]
    cfgs = [FofConfig.from_workload(w) for w in boxes]
    pos = [torch.from_numpy(w.pos).cuda() for w in boxes]
    vel = [torch.from_numpy(w.vel).cuda() for w in boxes]
    plan = Plan(cfgs[0])
    for _ in range(2):   # eager + capture, then a replay
        cats = plan.run_batch(cfgs, pos, vel)
        for w, cat in zip(boxes, cats):
            assert_same_catalog(cat, cpu.run(w), check_member=False)


def test_grid_cell_shorter_than_link_is_rejected():
    from cm_halofinder_b200 import CmhError
    n = 5000
    w = synth.make_lightcone(n, 1400.0 * (n / 50_000_000) ** (1 / 3), 20, 55)
    w.cells = 8 * w.cells   # cells shorter than the longest linking length
    with pytest.raises(CmhError, match="INVALID_ARGUMENT"):
        fof(w.pos, w.vel, FofConfig.from_workload(w))
