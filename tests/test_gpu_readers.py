"""The readers end to end: a Gadget-1 snapshot and a PICOLA unformatted
lightcone file are read by cmh_read_particles and found by the GPU FoF, and
the halos must equal those of the reference program built with the same
reader (oracle/_ref/cmh_ref_gadget_f32, cmh_ref_picola_f32) on the same file:
same halos in the same order, the same members, properties within 1e-6."""
import os
import struct
import subprocess

import numpy as np
import pytest

import cm_halofinder_b200 as cmh
from cm_halofinder_b200 import FofConfig, _abi, fof, synth
from oracle import cpu, reference
from tests.helpers import PROP_RTOL, prop_errors

pytestmark = pytest.mark.gpu
HALOSIZE = 19


def _rec(f, payload):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def _run_ref(binary, w, n, d, extra=()):
    exe = os.path.join(reference.REF_DIR, binary)
    if not os.path.exists(exe):
        pytest.skip(f"{binary} not built")
    pf = os.path.join(d, "params.txt")
    reference.write_params(pf, lo=w.lo, hi=w.hi, boundary=w.boundary, linklength=w.linklength,
                           nphalomin=w.nphalomin, cells=w.cells, n_proc=n,
                           base_in=os.path.join(d, "in"), base_out=os.path.join(d, "ref"))
    with open(pf, "a") as f:
        f.writelines(line + "\n" for line in extra)
    r = subprocess.run([exe, pf], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:]


def _read_noid_catalog(path):
    """Catalog written without PARTICLE_ID: member records hold 6 floats."""
    halos = []
    if not os.path.exists(path):
        return halos
    data = open(path, "rb").read()
    off = 0

    def rec():
        nonlocal off
        (ln,) = struct.unpack_from("<i", data, off)
        body = data[off + 4: off + 4 + ln]
        off += 8 + ln
        return body

    (nh,) = struct.unpack("<i", rec())
    for _ in range(nh):
        props = np.frombuffer(rec(), np.float32).copy()
        pv = np.stack([np.frombuffer(rec(), np.float32) for _ in range(int(props[0]))])
        halos.append({"props": props, "pv": pv})
    return halos


def _ours(w, d, fmt, with_id):
    rp = _abi.RunParameters()
    rp.InputStyle, rp.Ninputfiles, rp.Starting_file = 0, 1, 0
    rp.InputFileBase = os.path.join(d, "in").encode()
    pos, vel, ids = cmh.read_particles(rp, fmt, with_id)
    cfg = FofConfig(lo=w.lo, hi=w.hi, boundary=w.boundary, linklength=w.linklength,
                    nphalomin=w.nphalomin, periodic=False, precision="fp32",
                    properties=cmh.CMH_PROP_INERTIA | cmh.CMH_PROP_DISPERSION)
    return pos, vel, ids, fof(pos, vel, cfg, members=True)


def _check_props(cat, ref):
    assert cat.nhalos == len(ref) > 5
    rp = np.stack([h["props"] for h in ref])
    np.testing.assert_array_equal(cat.props[:, 0], rp[:, 0])
    err = prop_errors(cat.props[:, :7], rp[:, :7])
    assert np.all(err[1:] <= PROP_RTOL), err


def test_gadget1_reader_matches_reference(tmp_path):
    w = synth.make_box(20000, 60.0, 400, 701, nphalomin=5, boundary=3.0)
    src, ppos, _ = cpu.build_proc(w)
    ids = (np.asarray(src, np.uint64) * np.uint64(7) + np.uint64(2 ** 34))
    header = bytearray(256)
    struct.pack_into("<6I", header, 0, 0, ppos.shape[0], 0, 0, 0, 0)
    with open(tmp_path / "in.0", "wb") as f:
        _rec(f, bytes(header))
        _rec(f, np.ascontiguousarray(ppos, np.float32).tobytes())
        _rec(f, np.ascontiguousarray(w.vel[src], np.float32).tobytes())
        _rec(f, ids.tobytes())
    _run_ref("cmh_ref_gadget_f32", w, ppos.shape[0], str(tmp_path))
    ref = reference.read_catalog(str(tmp_path / "ref.0"), HALOSIZE)
    pos, vel, rids, cat = _ours(w, str(tmp_path), "gadget1", True)
    np.testing.assert_array_equal(rids, ids)
    _check_props(cat, ref)
    for h, halo in enumerate(ref):
        np.testing.assert_array_equal(np.sort(rids[cat.member == h]), np.sort(halo["ids"]))


def test_picola_lightcone_reader_matches_reference(tmp_path):
    n = 20000
    w = synth.make_lightcone(n, 1400.0 * (n / 50_000_000) ** (1 / 3), 150, 702)
    w.varlink = None  # a constant linking length: the reader is what is checked
    pos, vel = w.pos, w.vel
    with open(tmp_path / "in.0", "wb") as f:
        for lo, hi in ((0, 7000), (7000, 7000), (7000, n)):   # three blocks, one empty
            _rec(f, struct.pack("<I", hi - lo))
            rec = np.zeros(hi - lo, dtype=[("x", "<f4", 3), ("v", "<f4", 3)])
            rec["x"], rec["v"] = pos[lo:hi], vel[lo:hi]
            _rec(f, rec.tobytes())
    info = tmp_path / "in.info"
    info.write_text(f"# file xmin ymin zmin xmax ymax zmax npart\n0 {w.lo[0]} {w.lo[1]} {w.lo[2]} "
                    f"{w.hi[0]} {w.hi[1]} {w.hi[2]} {n}\n")
    _run_ref("cmh_ref_picola_f32", w, n, str(tmp_path), extra=[f"InputInfoFile {info}"])
    ref = _read_noid_catalog(str(tmp_path / "ref.0"))
    rpos, rvel, _, cat = _ours(w, str(tmp_path), "picola_lightcone", False)
    np.testing.assert_array_equal(rpos, pos)
    _check_props(cat, ref)
    pv = np.concatenate([rpos, rvel], axis=1)
    for h, halo in enumerate(ref):
        got = pv[cat.member == h]
        key = lambda a: np.lexsort(a.T[::-1])  # noqa: E731
        np.testing.assert_array_equal(got[key(got)], halo["pv"][key(halo["pv"])])
