"""Subsample files (Subsample, FOF.c:432-544) and the info file's sample
counts (Output_Info, FOF.c:917-957), written by the library from given
indices -- no GPU involved."""
import numpy as np
import pytest

import cm_halofinder_b200 as cmh
from cm_halofinder_b200 import _abi
from tests.subsample_ref import read_unformatted, uniforms


def _parts(n=200, seed=3, dtype=np.float32):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 50, (n, 3)).astype(dtype)
    vel = rng.normal(0, 300, (n, 3)).astype(dtype)
    ids = rng.permutation(10 ** 6)[:n].astype(np.uint64) + np.uint64(2 ** 40)
    return pos, vel, ids


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_unformatted_layout(tmp_path, native_lib, dtype):
    pos, vel, ids = _parts(dtype=dtype)
    idx = np.array([5, 17, 18, 150, 199], np.int64)
    cmh.write_subsample(tmp_path / "out", 3, True, pos, vel, idx, ids,
                        cmh.CMH_OUT_UNFORMATTED | cmh.CMH_OUT_PARTICLE_ID)
    p, v, i = read_unformatted(tmp_path / "out_inhalo.3")
    np.testing.assert_array_equal(p, pos[idx].astype(np.float32))
    np.testing.assert_array_equal(v, vel[idx].astype(np.float32))
    np.testing.assert_array_equal(i, ids[idx])
    cmh.write_subsample(tmp_path / "out", 3, False, pos, vel, idx[:2], None,
                        cmh.CMH_OUT_UNFORMATTED)
    p, v, _ = read_unformatted(tmp_path / "out_outhalo.3", with_id=False)
    np.testing.assert_array_equal(p, pos[idx[:2]].astype(np.float32))


def test_ascii_lines_and_empty_sample(tmp_path, native_lib):
    pos, vel, ids = _parts()
    idx = np.array([0, 9], np.int64)
    cmh.write_subsample(tmp_path / "a", 0, True, pos, vel, idx, ids, cmh.CMH_OUT_PARTICLE_ID)
    lines = open(tmp_path / "a_inhalo.0").read().splitlines()
    assert len(lines) == 2
    j = idx[1]
    want = "%15d %15.6f %15.6f %15.6f %15.6f %15.6f %15.6f" % (
        (int(ids[j]),) + tuple(float(np.float32(x)) for x in list(pos[j]) + list(vel[j])))
    assert lines[1] == want
    cmh.write_subsample(tmp_path / "a", 0, False, pos, vel, np.zeros(0, np.int64))
    assert not (tmp_path / "a_outhalo.0").exists()
    with pytest.raises(cmh.CmhError, match="INVALID_ARGUMENT"):
        cmh.write_subsample(tmp_path / "a", 0, True, pos, vel, np.array([500], np.int64))


def test_info_file_carries_the_sample_counts(tmp_path, native_lib):
    rp = _abi.RunParameters()
    rp.Nx, rp.Ny, rp.Nz = 2, 1, 1
    rp.Lxmin, rp.Lymin, rp.Lzmin, rp.Lxmax, rp.Lymax, rp.Lzmax = 0, 0, 0, 100, 50, 50
    cmh.write_info(tmp_path / "r", rp, [3, 4], [10, 20], [7, 0])
    rows = [ln.split() for ln in open(tmp_path / "r.info").read().splitlines()[1:]]
    assert [r[7:] for r in rows] == [["3", "10", "7"], ["4", "20", "0"]]
    cmh.write_info(tmp_path / "s", rp, [3, 4])
    rows = [ln.split() for ln in open(tmp_path / "s.info").read().splitlines()[1:]]
    assert [r[7:] for r in rows] == [["3", "0", "0"], ["4", "0", "0"]]


def test_uniforms_are_uniform():
    u = uniforms(7, np.arange(200000, dtype=np.uint64))
    assert u.min() >= 0.0 and u.max() < 1.0
    hist = np.histogram(u, bins=20, range=(0, 1))[0]
    assert np.all(np.abs(hist - 10000) < 6 * 100)
    assert not np.array_equal(uniforms(8, np.arange(100, dtype=np.uint64)), u[:100])
