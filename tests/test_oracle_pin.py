"""Pins the CPU oracle to the reference: the golden fixtures hold what the
reference binary (src_v2, built unmodified) produced; the restatement must
give the same halos (member ID sets, catalog order) and properties."""
import numpy as np
import pytest

from oracle import cpu
from tests import golden_io
from tests.helpers import PROP_RTOL, prop_errors


@pytest.mark.parametrize("name", golden_io.names())
def test_oracle_matches_reference(name):
    w, ref = golden_io.load(name)
    o = cpu.run(w, props=3)
    nh = len(ref["sets"])
    assert o["stats"]["nhalos"] == nh
    assert o["stats"]["n_proc"] == ref["params"]["proc_stats"]["n_proc"]
    # member sets at the processing level (two owned copies of a halo wider
    # than the shell may share particles, as in the reference)
    for h in range(nh):
        proc = np.nonzero(o["group"] == o["halo_head"][h])[0]
        np.testing.assert_array_equal(np.unique(w.ids[o["proc_src"][proc]]), ref["sets"][h])
    if o["stats"]["n_member_conflicts"] == 0:
        sets = golden_io.sets_from_member(o["member"], w.ids, nh)
        for h in range(nh):
            np.testing.assert_array_equal(sets[h], ref["sets"][h])
    # head of each halo: the reference writes it first
    np.testing.assert_array_equal(w.ids[o["proc_src"][o["halo_head"]]], ref["first_id"])
    err = prop_errors(o["halo_props"][:, :7], ref["props"][:, :7])
    assert err[0] == 0 and np.all(err[1:] <= PROP_RTOL), err
    got, exp = o["halo_props"].astype(np.float64), ref["props"].astype(np.float64)
    for blk in (7, 13):
        diag = np.abs(exp[:, blk:blk + 3]).mean(axis=1, keepdims=True)
        e = np.abs(got[:, blk:blk + 6] - exp[:, blk:blk + 6]) / np.maximum(diag, 1e-30)
        assert e.max(initial=0) < 1e-5


def test_fixtures_present():
    assert len(golden_io.names()) >= 5


def test_lattice_ties_are_linked():
    """d^2 == l^2 exactly links (FOF.c:357 returns only for d^2 > l^2)."""
    w, ref = golden_io.load("lattice_ties")
    sizes = sorted(len(s) for s in ref["sets"])
    assert 216 in sizes          # the 6^3 lattice at spacing exactly l is one halo
    a = np.array([0, 0, 0], np.float32)
    b = np.array([0.78125, 0, 0], np.float32)
    assert cpu.lib().cmh_oracle_linked_f32(a.ctypes.data, b.ctypes.data, 0.78125 ** 2) == 1
    c = np.array([np.nextafter(np.float32(0.78125), np.float32(1)), 0, 0], np.float32)
    assert cpu.lib().cmh_oracle_linked_f32(a.ctypes.data, c.ctypes.data, 0.78125 ** 2) == 0
