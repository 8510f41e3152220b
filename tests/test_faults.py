"""Host-side fault injection (CMH_FAULT) on the CPU: the particle readers
and the catalog writers return CMH_ERR_IO when a file cannot be opened, as
the reference's my_fread/my_fwrite/FatalError stop a run (main.c:83-112),
and work again once the fault is gone.  The GPU-side cases (allocation,
capacity overflow, capped device waits, per-box batch status) are in
test_gpu_faults.py."""
import os

import numpy as np
import pytest

import cm_halofinder_b200 as cmh
from cm_halofinder_b200 import _abi
from tests.test_readers import _data, _rp, _write_ascii

IO = 8


@pytest.fixture
def fault(monkeypatch):
    def set_fault(value):
        if value is None:
            monkeypatch.delenv("CMH_FAULT", raising=False)
        else:
            monkeypatch.setenv("CMH_FAULT", value)
    yield set_fault
    monkeypatch.delenv("CMH_FAULT", raising=False)


@pytest.mark.parametrize("value", ["io", "overflow,io", "io,alloc"])
def test_reader_io_fault(tmp_path, native_lib, fault, value):
    pos, vel, _ = _data(50, 1)
    _write_ascii(tmp_path / "in.0", pos, vel)
    rp = _rp(tmp_path / "in")
    fault(value)
    with pytest.raises(cmh.CmhError) as e:
        cmh.read_particles(rp, "ascii")
    assert e.value.status == IO and "CMH_FAULT" not in _abi.last_error()
    fault(None)
    p, v, _ = cmh.read_particles(rp, "ascii")
    np.testing.assert_allclose(p, pos, rtol=1e-6)


@pytest.mark.parametrize("value", ["alloc", "iox", "overflow", ""])
def test_other_words_leave_files_alone(tmp_path, native_lib, fault, value):
    pos, vel, _ = _data(20, 2)
    _write_ascii(tmp_path / "in.0", pos, vel)
    fault(value)
    p, _, _ = cmh.read_particles(_rp(tmp_path / "in"), "ascii")
    assert p.shape == (20, 3)


def test_writer_io_fault(tmp_path, native_lib, fault):
    props = np.arange(3 * 7, dtype=np.float32).reshape(3, 7) + 10
    cat = cmh.Catalog(props, np.arange(3, dtype=np.uint32), None, {})
    base = str(tmp_path / "halos")
    fault("io")
    with pytest.raises(cmh.CmhError) as e:
        cmh.write_halos(base, 0, cat)
    assert e.value.status == IO
    assert not os.path.exists(base + ".0")
    fault(None)
    cmh.write_halos(base, 0, cat)
    assert os.path.exists(base + ".0")


def test_info_writer_io_fault(tmp_path, native_lib, fault):
    rp = _abi.RunParameters()
    rp.Nx = rp.Ny = rp.Nz = 1
    rp.Lxmax = rp.Lymax = rp.Lzmax = 10.0
    base = str(tmp_path / "run")
    fault("io")
    with pytest.raises(cmh.CmhError) as e:
        cmh.write_info(base, rp, [1])
    assert e.value.status == IO
    fault(None)
    cmh.write_info(base, rp, [1])
    assert os.path.exists(base + ".info")
