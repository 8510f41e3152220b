"""The device-side generator of the 1024^3 box and checks that hold at any
size: the FP32 + FP64-recheck form and the plain FP64 form give the same
halos, and a box gives the same halos whatever its particle order."""
import numpy as np
import pytest

from cm_halofinder_b200 import FofConfig, Plan, fof, synth
from oracle import cpu
from tests.helpers import assert_same_catalog

pytestmark = pytest.mark.gpu


def test_device_generated_box_matches_oracle():
    w = synth.config5_device(seed=61, scale=250000 / 1024 ** 3).to_host()
    ref = cpu.run(w)
    assert ref["stats"]["nhalos"] > 30
    cat = fof(w.pos, w.vel, FofConfig.from_workload(w), members=True)
    assert_same_catalog(cat, ref)


def test_forms_agree_at_8m():
    w = synth.config5_device(seed=62, scale=8_000_000 / 1024 ** 3)
    out = {}
    for precision in ("fp32", "fp64"):
        plan = Plan(FofConfig.from_workload(w, precision=precision))
        out[precision] = plan.run(w.pos, w.vel, out="host")
        plan.close()
    a, b = out["fp32"], out["fp64"]
    assert a.nhalos == b.nhalos > 1000
    np.testing.assert_array_equal(a.head, b.head)
    np.testing.assert_array_equal(a.props[:, 0], b.props[:, 0])
    np.testing.assert_allclose(a.props[:, 1:4], b.props[:, 1:4], rtol=1e-6)
    # halo sizes are bounded by the particles and at least the minimum
    assert a.props[:, 0].sum() <= w.n and a.props[:, 0].min() >= w.nphalomin


def test_particle_order_does_not_change_halos():
    """Permuting the input permutes nothing in the catalog but the member
    indices: same halo sizes and centres (heads are processing indices, so
    they follow the permutation)."""
    import torch
    w = synth.config5_device(seed=63, scale=2_000_000 / 1024 ** 3)
    cfg = FofConfig.from_workload(w)
    a = fof(w.pos.cpu().numpy(), w.vel.cpu().numpy(), cfg)
    perm = torch.randperm(w.n, device=w.pos.device)
    b = fof(w.pos[perm].cpu().numpy(), w.vel[perm].cpu().numpy(), cfg)
    assert a.nhalos == b.nhalos
    ka = np.lexsort((a.props[:, 3], a.props[:, 2], a.props[:, 1], a.props[:, 0]))
    kb = np.lexsort((b.props[:, 3], b.props[:, 2], b.props[:, 1], b.props[:, 0]))
    np.testing.assert_array_equal(a.props[ka, 0], b.props[kb, 0])
    np.testing.assert_allclose(a.props[ka, 1:4], b.props[kb, 1:4], rtol=1e-6)
