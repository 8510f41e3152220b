"""Run-parameter file (startup.c:109-314) and catalog writers
(FOF.c:546-957) through the C ABI; host code, no GPU needed."""
import os
import struct

import numpy as np
import pytest

import cm_halofinder_b200 as cmh
from cm_halofinder_b200 import _abi
from oracle import cpu, reference
from tests import golden_io

TAGS = """% our own test parameter file
Nx 1
Ny 1
Nz 1
Px 64
Py 64
Pz 64
Lxmin 0.0
Lymin 0.0
Lzmin 0.0
Lxmax 250.0
Lymax 250.0
Lzmax 250.0
Seed 7
Buffer 1.5
Boundarysize 8
Linklength 0.78125
Nphalomin 10
SampInHalos -1
SampOutHalos -1
InputStyle 0
Ninputfiles 1
Starting_file 0
Nread 1
Nwrite 1
InputFileBase /tmp/in
OutputFileBase /tmp/out
"""


def write(tmp_path, text, name="p.txt"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_parse_all_tags(tmp_path, native_lib):
    rp = cmh.read_parameterfile(write(tmp_path, TAGS))
    assert (rp.Nx, rp.Px, rp.Seed, rp.Nwrite) == (1, 64, 7, 1)
    assert rp.Lxmax == 250.0 and rp.Linklength == 0.78125 and rp.Nphalomin == 10
    assert rp.OutputFileBase == b"/tmp/out"


def test_comments_and_short_lines_skipped(tmp_path, native_lib):
    text = "% header\n\n  \nlonely\n" + TAGS.replace("Seed 7", "% Seed 9\nSeed 7")
    rp = cmh.read_parameterfile(write(tmp_path, text))
    assert rp.Seed == 7


@pytest.mark.parametrize("mutate,needle", [
    (lambda t: t + "Bogus 3\n", "Bogus"),
    (lambda t: t + "Seed 8\n", "Seed"),
    (lambda t: t.replace("Nphalomin 10\n", ""), "Nphalomin"),
])
def test_bad_files_are_errors(tmp_path, native_lib, mutate, needle):
    with pytest.raises(cmh.CmhError) as e:
        cmh.read_parameterfile(write(tmp_path, mutate(TAGS)))
    assert e.value.status == 2 and needle in str(e.value)


def test_missing_file(tmp_path, native_lib):
    with pytest.raises(cmh.CmhError) as e:
        cmh.read_parameterfile(str(tmp_path / "nope.txt"))
    assert e.value.status == 2


def test_varlink_tags(tmp_path, native_lib):
    text = TAGS + "Omega 0.25\nOrigin_x 1.5\nOrigin_y 0\nOrigin_z 0\n"
    with pytest.raises(cmh.CmhError):
        cmh.read_parameterfile(write(tmp_path, text))        # not allowed without VARLINK
    rp = cmh.read_parameterfile(write(tmp_path, text), varlink=True)
    assert rp.Omega == 0.25 and rp.Origin_x == 1.5          # float, not the INT typo


REF_EXAMPLE = os.path.join(os.environ.get("CMH_REFERENCE", ""), "files", "run_parameters.dat")


@pytest.mark.skipif(not os.environ.get("CMH_REFERENCE") or not os.path.exists(REF_EXAMPLE),
                    reason="reference sources not given (CMH_REFERENCE)")
def test_reference_example_file_parses(native_lib):
    rp = cmh.read_parameterfile(REF_EXAMPLE)
    assert (rp.Nx, rp.Ny, rp.Nz, rp.Px) == (2, 2, 2, 256)
    assert rp.Linklength == 0.625 and rp.Boundarysize == 35


def test_domain_of_each_task(tmp_path, native_lib):
    rp = cmh.read_parameterfile(write(tmp_path, TAGS.replace("Nx 1", "Nx 2").replace("Nz 1", "Nz 3")))
    cfg = cmh.config_from_run(rp, task=5)
    # task 5 of 2 x 1 x 3: (x, y, z) = (1, 0, 2)  (startup.c:33-47)
    assert cfg.lo[0] == 125.0 and cfg.hi[0] == 250.0
    assert abs(cfg.lo[2] - 2 * 250 / 3) < 1e-12
    with pytest.raises(cmh.CmhError):
        cmh.config_from_run(rp, task=6)


def _oracle_catalog(name, props):
    w, _ = golden_io.load(name)
    o = cpu.run(w, props=props)
    cat = cmh.Catalog(props=o["halo_props"], head=o["halo_head"], member=o["member"],
                      stats={})
    return w, o, cat


def test_write_unformatted_with_particles_roundtrip(tmp_path, native_lib):
    w, o, cat = _oracle_catalog("box_f32_manyhalos", 3)
    # member copies: for this fixture every member is an original particle
    mp = np.zeros((w.n, 3), np.float32)
    proc = np.zeros(w.n, np.uint32)
    for h, head in enumerate(o["halo_head"]):
        for p in np.nonzero(o["group"] == head)[0]:
            s = o["proc_src"][p]
            if o["member"][s] == h:
                mp[s] = o["proc_pos"][p]
                proc[s] = p
    base = str(tmp_path / "cat")
    _write_members(base, cat, w, mp, proc,
                   _abi.CMH_OUT_UNFORMATTED | _abi.CMH_OUT_PARTICLES | _abi.CMH_OUT_PARTICLE_ID)
    halos = reference.read_catalog(base + ".0", 19)
    assert len(halos) == cat.nhalos
    for h, rec in enumerate(halos):
        np.testing.assert_array_equal(rec["props"], cat.props[h])
        ids = np.sort(rec["ids"])
        np.testing.assert_array_equal(ids, np.sort(w.ids[o["member"] == h]))
        # head first, as the reference walks its ring from the head
        assert rec["ids"][0] == w.ids[o["proc_src"][o["halo_head"][h]]]


def _write_members(base, cat, w, mp, proc, flags):
    import ctypes as C
    L = _abi.lib()
    props = np.ascontiguousarray(cat.props, np.float32)
    head = np.ascontiguousarray(cat.head, np.uint32)
    mem = np.ascontiguousarray(cat.member, np.int64)
    c = _abi.Catalog(nhalos=props.shape[0], halosize=props.shape[1], location=0,
                     props=props.ctypes.data_as(C.POINTER(C.c_float)),
                     head=head.ctypes.data_as(C.POINTER(C.c_uint32)),
                     member=mem.ctypes.data_as(C.POINTER(C.c_int64)),
                     member_proc=proc.ctypes.data_as(C.POINTER(C.c_uint32)),
                     member_pos=mp.ctypes.data_as(C.POINTER(C.c_float)))
    c.stats.n_in = w.n
    vel = np.ascontiguousarray(w.vel)
    ids = np.ascontiguousarray(w.ids)
    parts = _abi.Particles(n=w.n, pos_dtype=0, vel_dtype=0, pos=mp.ctypes.data,
                           vel=vel.ctypes.data, id=ids.ctypes.data, location=0)
    _abi.check(L.cmh_write_halos(base.encode(), 0, C.byref(c), C.byref(parts), flags))


def test_write_unformatted_block(tmp_path, native_lib):
    w, o, cat = _oracle_catalog("box_f32_manyhalos", 0)
    base = str(tmp_path / "blk")
    cmh.write_halos(base, 3, cmh.Catalog(cat.props, cat.head, None, {}),
                    flags=_abi.CMH_OUT_UNFORMATTED)
    data = open(base + ".3", "rb").read()
    nh = cat.nhalos
    assert struct.unpack_from("<iii", data, 0) == (4, nh, 4)
    (ln,) = struct.unpack_from("<i", data, 12)
    assert ln == nh * 7 * 4
    block = np.frombuffer(data, np.float32, nh * 7, 16).reshape(nh, 7)
    np.testing.assert_array_equal(block, cat.props)
    assert struct.unpack_from("<i", data, 16 + ln)[0] == ln


def test_write_ascii(tmp_path, native_lib):
    w, o, cat = _oracle_catalog("box_f32_manyhalos", 2)
    base = str(tmp_path / "asc")
    cmh.write_halos(base, 0, cmh.Catalog(cat.props, cat.head, None, {}))
    lines = open(base + ".0").read().splitlines()
    assert len(lines) == cat.nhalos
    first = lines[0].split()
    assert int(first[0]) == int(cat.props[0, 0]) and len(first) == 13
    assert abs(float(first[7]) - cat.props[0, 7]) <= 1e-6 * max(1, abs(cat.props[0, 7]))


def test_no_halos_no_file(tmp_path, native_lib):
    base = str(tmp_path / "empty")
    cmh.write_halos(base, 0, cmh.Catalog(np.zeros((0, 7), np.float32),
                                         np.zeros(0, np.uint32), None, {}))
    assert not os.path.exists(base + ".0")


def test_info_file(tmp_path, native_lib):
    rp = cmh.read_parameterfile(write(tmp_path, TAGS.replace("Nx 1", "Nx 2")))
    base = str(tmp_path / "run")
    cmh.write_info(base, rp, [3, 4])
    lines = open(base + ".info").read().splitlines()
    assert lines[0].startswith("#    FILENUM")
    f = lines[2].split()
    assert f[0] == "1" and float(f[1]) == 125.0 and f[7] == "4"
