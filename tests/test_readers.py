"""Particle readers (read_data.c:100-404): ASCII lines, Gadget-1 snapshots
and PICOLA unformatted lightcones, the two file-naming styles, and the
I/O errors.  Files are written here from the layouts the reference reads."""
import struct

import numpy as np
import pytest

import cm_halofinder_b200 as cmh
from cm_halofinder_b200 import _abi


def _rp(base, nfiles=1, style=0, start=0):
    rp = _abi.RunParameters()
    rp.InputStyle = style
    rp.Ninputfiles = nfiles
    rp.Starting_file = start
    rp.InputFileBase = str(base).encode()
    return rp


def _data(n, seed, dtype=np.float32):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 100, (n, 3)).astype(dtype)
    vel = rng.normal(0, 300, (n, 3)).astype(dtype)
    ids = rng.permutation(10 ** 6)[:n].astype(np.uint64) + np.uint64(2 ** 33)
    return pos, vel, ids


def _write_ascii(path, pos, vel, ids=None):
    fmt = "%.9g" if pos.dtype == np.float32 else "%.17g"
    with open(path, "w") as f:
        for k in range(pos.shape[0]):
            vals = " ".join(fmt % v for v in list(pos[k]) + list(vel[k]))
            f.write((f"{int(ids[k])} " if ids is not None else "") + vals + "\n")


def _rec(f, payload):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def _write_gadget(path, pos, vel, ids=None):
    header = bytearray(256)
    struct.pack_into("<6I", header, 0, 0, pos.shape[0], 0, 0, 0, 0)
    with open(path, "wb") as f:
        _rec(f, bytes(header))
        _rec(f, np.ascontiguousarray(pos, np.float32).tobytes())
        _rec(f, np.ascontiguousarray(vel, np.float32).tobytes())
        if ids is not None:
            _rec(f, np.ascontiguousarray(ids, np.uint64).tobytes())


def _write_picola(path, blocks, with_id):
    with open(path, "wb") as f:
        for pos, vel, ids in blocks:
            n = pos.shape[0]
            _rec(f, struct.pack("<I", n))
            rec = np.zeros(n, dtype=[("id", "<u4"), ("x", "<f4", 3), ("v", "<f4", 3)]
                           if with_id else [("x", "<f4", 3), ("v", "<f4", 3)])
            if with_id:
                rec["id"] = ids.astype(np.uint32)
            rec["x"], rec["v"] = pos, vel
            _rec(f, rec.tobytes())


@pytest.mark.parametrize("with_id", [False, True])
@pytest.mark.parametrize("fp64", [False, True])
def test_ascii_two_files_in_order(tmp_path, native_lib, with_id, fp64):
    dt = np.float64 if fp64 else np.float32
    a, b = _data(50, 1, dt), _data(70, 2, dt)
    base = tmp_path / "snap"
    _write_ascii(f"{base}.3", a[0], a[1], a[2] if with_id else None)
    _write_ascii(f"{base}.4", b[0], b[1], b[2] if with_id else None)
    pos, vel, ids = cmh.read_particles(_rp(base, nfiles=2, start=3), "ascii", with_id, fp64)
    np.testing.assert_array_equal(pos, np.concatenate([a[0], b[0]]))
    np.testing.assert_array_equal(vel, np.concatenate([a[1], b[1]]))
    if with_id:
        np.testing.assert_array_equal(ids, np.concatenate([a[2], b[2]]))
    else:
        assert ids is None


def test_file_list_skips_comments_and_blank_lines(tmp_path, native_lib):
    a, b = _data(5, 3), _data(6, 4)
    _write_ascii(tmp_path / "x.dat", *a[:2])
    _write_ascii(tmp_path / "y.dat", *b[:2])
    lst = tmp_path / "files.txt"
    lst.write_text(f"% the files\n\n{tmp_path / 'x.dat'}\n   \n{tmp_path / 'y.dat'} trailing\n")
    pos, _, _ = cmh.read_particles(_rp(lst, style=1), "ascii")
    np.testing.assert_array_equal(pos, np.concatenate([a[0], b[0]]))


@pytest.mark.parametrize("with_id", [False, True])
def test_gadget1_snapshot(tmp_path, native_lib, with_id):
    a = _data(123, 5)
    _write_gadget(tmp_path / "g.0", a[0], a[1], a[2] if with_id else None)
    pos, vel, ids = cmh.read_particles(_rp(tmp_path / "g"), "gadget1", with_id)
    np.testing.assert_array_equal(pos, a[0])
    np.testing.assert_array_equal(vel, a[1])
    if with_id:
        np.testing.assert_array_equal(ids, a[2])


@pytest.mark.parametrize("with_id", [False, True])
def test_picola_lightcone_blocks(tmp_path, native_lib, with_id):
    blocks = [_data(40, 6), _data(0, 7), _data(17, 8)]
    _write_picola(tmp_path / "lc.0", blocks, with_id)
    pos, vel, ids = cmh.read_particles(_rp(tmp_path / "lc"), "picola_lightcone", with_id)
    np.testing.assert_array_equal(pos, np.concatenate([b[0] for b in blocks]))
    np.testing.assert_array_equal(vel, np.concatenate([b[1] for b in blocks]))
    if with_id:  # 32-bit IDs in this format, zero-extended
        want = np.concatenate([b[2] for b in blocks]).astype(np.uint32).astype(np.uint64)
        np.testing.assert_array_equal(ids, want)


def test_io_errors(tmp_path, native_lib):
    with pytest.raises(cmh.CmhError, match="IO"):
        cmh.read_particles(_rp(tmp_path / "missing"), "ascii")
    a = _data(10, 9)
    _write_gadget(tmp_path / "t.0", *a[:2])
    data = (tmp_path / "t.0").read_bytes()
    (tmp_path / "t.0").write_bytes(data[:-30])  # truncated velocity record
    with pytest.raises(cmh.CmhError, match="IO"):
        cmh.read_particles(_rp(tmp_path / "t"), "gadget1")
    (tmp_path / "bad.0").write_text("1.0 2.0 three 4 5 6\n")
    with pytest.raises(cmh.CmhError, match="IO"):
        cmh.read_particles(_rp(tmp_path / "bad"), "ascii")
