"""Subsampling on the GPU (FOF.c:205-284): the kept particles must be
exactly those of a numpy restatement of the draw over the oracle's groups
(originals inside the domain, rate by group size against Nphalomin, the
SplitMix64 uniform of Seed and ID or index), and the catalog must not
change.  The reference draws GSL RANLUX numbers along its rings, so its
own sample is not the comparison (parity unpinned)."""
import numpy as np
import pytest

from cm_halofinder_b200 import FofConfig, fof, fof_sampled, synth
from oracle import cpu
from tests.helpers import assert_same_catalog
from tests.subsample_ref import expected_sample

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("periodic,with_ids,precision", [(True, True, "fp32"),
                                                         (True, False, "fp64"),
                                                         (False, True, "fp32")])
def test_sample_matches_the_restated_draw(periodic, with_ids, precision):
    w = synth.make_box(40000, 80.0, 500, 911, nphalomin=8, boundary=4.0)
    w.periodic = periodic
    ids = (w.ids * np.uint64(3) + np.uint64(12345)) if with_ids else None
    cfg = FofConfig.from_workload(w, precision=precision)
    cat, inh, outh = fof_sampled(w.pos, w.vel, cfg, 0.25, 0.02, 77, ids=ids, members=True)
    ref = cpu.run(w)
    assert_same_catalog(cat, ref)
    keys = ids if with_ids else np.arange(w.n, dtype=np.uint64)
    closed = (0, 0, 0) if periodic else (1, 1, 1)
    want_in, want_out = expected_sample(ref, w, 0.25, 0.02, 77, keys, closed)
    np.testing.assert_array_equal(inh, want_in)
    np.testing.assert_array_equal(outh, want_out)
    assert len(inh) > 500 and len(outh) > 50
    # the plain run gives the same catalog
    assert_same_catalog(fof(w.pos, w.vel, cfg, members=True), ref)


def test_rates_zero_and_one():
    w = synth.make_box(20000, 60.0, 300, 912, nphalomin=5, boundary=3.0)
    cfg = FofConfig.from_workload(w)
    _, inh, outh = fof_sampled(w.pos, w.vel, cfg, 1.0, 0.0, 5)
    ref = cpu.run(w)
    want_in, want_out = expected_sample(ref, w, 1.0, 0.0, 5, np.arange(w.n, dtype=np.uint64),
                                        (0, 0, 0))
    np.testing.assert_array_equal(inh, want_in)
    assert len(outh) == 0 and len(want_out) == 0
    # with rate 1 every particle of a big group inside the box is kept
    group = ref["group"]
    size = np.bincount(group)[group]
    n_kept = ref["stats"]["n_kept"]
    assert len(inh) == int((size[:n_kept] >= w.nphalomin).sum())
