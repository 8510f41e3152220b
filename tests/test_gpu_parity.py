"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Membership and catalog order must be identical (bit-exact integer work);
halo properties within 1e-6 (helpers.PROP_RTOL).  Sizes are ones the
oracle finishes in seconds."""
import numpy as np
import pytest

from cm_halofinder_b200 import FofConfig, fof, synth
from oracle import cpu
from tests.band_pairs import make_band_workload
from tests.helpers import assert_same_catalog, prop_errors

pytestmark = pytest.mark.gpu


def run_both(w, precision, props=0, cell_factor=0):
    ref = cpu.run(w, props=props)
    cfg = FofConfig.from_workload(w, precision=precision, properties=props,
                                  cell_factor=cell_factor)
    cat = fof(w.pos, w.vel, cfg, members=True)
    return cat, ref


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_c1_shape_fp64_positions(precision):
    w = synth.config1(seed=101, scale=30000 / 262144)
    cat, ref = run_both(w, precision)
    assert cat.stats["n_proc"] == ref["stats"]["n_proc"]
    assert cat.stats["n_images"] == ref["stats"]["n_images"]
    assert cat.stats["n_groups"] == ref["stats"]["n_groups"]
    assert_same_catalog(cat, ref)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_c2_shape_fp32_positions(precision):
    w = synth.config2(seed=202, scale=60000 / 256 ** 3)
    cat, ref = run_both(w, precision)
    assert cat.stats["n_groups"] == ref["stats"]["n_groups"]
    assert_same_catalog(cat, ref)


@pytest.mark.parametrize("cell_factor", [2, 3, 5, 9, 16])
def test_cell_factor_does_not_change_result(cell_factor):
    w = synth.config2(seed=203, scale=40000 / 256 ** 3)
    cat, ref = run_both(w, "fp32", cell_factor=cell_factor)
    assert cat.stats["cell_factor"] == max(cell_factor, 2)
    assert_same_catalog(cat, ref)


def test_nonperiodic_with_shell_particles():
    w = synth.config2(seed=204, scale=40000 / 256 ** 3)
    w.periodic = False
    # shift part of the box into the shell and some particles outside it
    L = w.hi[0]
    pos = w.pos.astype(np.float64)
    pos[::7] -= 0.5 * w.boundary
    pos[::97] += 3 * w.boundary
    w.pos = pos.astype(np.float32)
    cat, ref = run_both(w, "fp32")
    assert cat.stats["n_out"] == ref["stats"]["n_out"] > 0
    assert_same_catalog(cat, ref)
    del L


def test_properties_inertia_dispersion():
    w = synth.config2(seed=205, scale=40000 / 256 ** 3)
    cat, ref = run_both(w, "fp32", props=3)
    assert cat.props.shape[1] == 19
    assert_same_catalog(cat, ref)
    # second moments: cancellation-limited, compared against the diagonal scale
    got, exp = cat.props.astype(np.float64), ref["halo_props"].astype(np.float64)
    for blk in (7, 13):
        diag = np.abs(exp[:, blk:blk + 3]).mean(axis=1, keepdims=True)
        err = np.abs(got[:, blk:blk + 6] - exp[:, blk:blk + 6]) / np.maximum(diag, 1e-30)
        assert err.max() < 1e-5, (blk, err.max())


def test_repeatable_membership():
    w = synth.config2(seed=206, scale=40000 / 256 ** 3)
    cfg = FofConfig.from_workload(w)
    a = fof(w.pos, w.vel, cfg, members=True)
    b = fof(w.pos, w.vel, cfg, members=True)
    np.testing.assert_array_equal(a.head, b.head)
    np.testing.assert_array_equal(a.member, b.member)
    assert prop_errors(a.props, b.props).max() <= 1e-6


def test_fp32_and_plain_agree_and_rechecks_counted():
    w = synth.config2(seed=207, scale=60000 / 256 ** 3)
    a = fof(w.pos, w.vel, FofConfig.from_workload(w, precision="fp32"), members=True)
    b = fof(w.pos, w.vel, FofConfig.from_workload(w, precision="fp64"), members=True)
    np.testing.assert_array_equal(a.member, b.member)
    np.testing.assert_array_equal(a.head, b.head)
    assert b.stats["n_rechecks"] == 0
    assert 0 <= a.stats["n_rechecks"] <= a.stats["n_pair_tests"]
    # the forms visit the same cell pairs; how many particle pairs a visit
    # tests before its cells are found joined depends on the order in which
    # concurrent unions land (a few per cent apart on a box this small), so
    # the counts agree closely, not exactly; exact counts are asserted on the
    # isolated pairs of test_fp32_band_pairs_are_rechecked
    ta, tb = a.stats["n_pair_tests"], b.stats["n_pair_tests"]
    assert ta > 0 and abs(ta - tb) <= 0.10 * max(ta, tb), (ta, tb)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_fp32_band_pairs_are_rechecked(dtype):
    """Isolated pairs whose FP32 d^2 sits k ulp from fl32(l^2), k in -6..6,
    on both sides of the double threshold (tests/band_pairs.py): the FP32
    form links exactly the pairs the double expression links -- including
    those the FP32 value alone decides wrongly -- and re-checks exactly the
    pairs inside its band (4 ulp, 8 for FP64 positions)."""
    w, cases = make_band_workload(dtype)
    width = 8 if dtype == np.float64 else 4
    ref = cpu.run(w)
    a = fof(w.pos, w.vel, FofConfig.from_workload(w, precision="fp32"), members=True)
    b = fof(w.pos, w.vel, FofConfig.from_workload(w, precision="fp64"), members=True)
    assert_same_catalog(a, ref)
    assert_same_catalog(b, ref)
    assert a.nhalos == sum(l64 for _, l64, _ in cases)
    assert any(l64 != l32 for _, l64, l32 in cases)
    # one test per pair (the pairs are isolated), in both forms
    assert a.stats["n_pair_tests"] == b.stats["n_pair_tests"] == len(cases)
    assert a.stats["n_rechecks"] == sum(abs(k) <= width for k, _, _ in cases) > 0
    assert b.stats["n_rechecks"] == 0
