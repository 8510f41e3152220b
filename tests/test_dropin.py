"""The drop-in FOF(): the reference program -- its own main.c, startup.c,
read_data.c and vars.c, unmodified -- with FOF.c replaced by
cm_halofinder_b200/shim/fof_shim.c and linked against libcmh_fof
(tests/dropin/Makefile builds it).  It runs beside the reference's own build
(oracle/_ref) on the same parameter file and input; the catalogs and info
files the two write must agree: same halos in the same order, the same
member particles (ID, position, velocity records), properties within 1e-6.
"""
import os
import subprocess

import numpy as np
import pytest

from cm_halofinder_b200 import synth
from oracle import cpu, reference
from tests.helpers import prop_errors, PROP_RTOL

HERE = os.path.dirname(os.path.abspath(__file__))
DROPIN = os.path.join(HERE, "dropin", "_build")
HALOSIZE = 19  # the parity builds carry INERTIA and DISPERSION


def _exe(name):
    path = os.path.join(DROPIN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (make -C tests/dropin)")
    return path


def _prepare(w, d):
    """Input file and two parameter files (outputs "ref" and "gpu") for one
    rank whose P[] is the pre-ghosted processing array of `w`."""
    src, ppos, _ = cpu.build_proc(w)
    ids = np.asarray(src, np.uint64)  # images carry the ID of their source particle
    reference.write_ascii(os.path.join(d, "in.0"), ids, ppos, w.vel[src])
    out = {}
    for name in ("ref", "gpu"):
        pf = os.path.join(d, f"params_{name}.txt")
        reference.write_params(pf, lo=w.lo, hi=w.hi, boundary=w.boundary,
                               linklength=w.linklength, nphalomin=w.nphalomin,
                               cells=w.cells, n_proc=ppos.shape[0],
                               base_in=os.path.join(d, "in"),
                               base_out=os.path.join(d, name))
        out[name] = pf
    return out


def _run(exe, params):
    r = subprocess.run([exe, params], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:]
    return r


def _compare(d):
    ref = reference.read_catalog(os.path.join(d, "ref.0"), HALOSIZE)
    got = reference.read_catalog(os.path.join(d, "gpu.0"), HALOSIZE)
    assert len(got) == len(ref)
    if ref:
        rp = np.stack([h["props"] for h in ref])
        gp = np.stack([h["props"] for h in got])
        np.testing.assert_array_equal(gp[:, 0], rp[:, 0])
        err = prop_errors(gp[:, :7], rp[:, :7])
        assert np.all(err[1:] <= PROP_RTOL), err
    same_order = True
    for h, g in zip(ref, got):
        np.testing.assert_array_equal(np.sort(g["ids"]), np.sort(h["ids"]))
        # every member record carries the particle's own position and velocity
        kr, kg = np.argsort(h["ids"], kind="stable"), np.argsort(g["ids"], kind="stable")
        np.testing.assert_array_equal(g["pv"][kg], h["pv"][kr])
        same_order &= bool(np.array_equal(g["ids"], h["ids"]))
    with open(os.path.join(d, "ref.info")) as f1, open(os.path.join(d, "gpu.info")) as f2:
        assert f2.read() == f1.read()
    return len(ref), same_order


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["box_f32", "box_f64", "many_small"])
def test_dropin_matches_reference_program(tmp_path, case):
    if case == "box_f32":
        w = synth.config2(seed=401, scale=25000 / 256 ** 3)
    elif case == "box_f64":
        w = synth.config1(seed=402, scale=20000 / 64 ** 3)
    else:
        w = synth.make_box(20000, 60.0, 400, 403, nphalomin=5, boundary=3.0)
    suffix = "f64" if w.pos.dtype == np.float64 else "f32"
    params = _prepare(w, str(tmp_path))
    _run(os.path.join(reference.REF_DIR, f"cmh_ref_{suffix}"), params["ref"])
    _run(_exe(f"cmh_dropin_{suffix}"), params["gpu"])
    nh, _ = _compare(str(tmp_path))
    assert nh > 5


@pytest.mark.gpu
def test_dropin_no_halos_writes_no_catalog(tmp_path):
    rng = np.random.default_rng(404)
    pos = rng.uniform(0, 100.0, (2000, 3)).astype(np.float32)
    w = synth.Workload(name="sparse", pos=pos, vel=np.zeros_like(pos),
                       ids=np.arange(2000, dtype=np.uint64), lo=(0.0,) * 3, hi=(100.0,) * 3,
                       linklength=0.05, boundary=1.0, nphalomin=10, periodic=True, cells=12)
    params = _prepare(w, str(tmp_path))
    _run(os.path.join(reference.REF_DIR, "cmh_ref_f32"), params["ref"])
    _run(_exe("cmh_dropin_f32"), params["gpu"])
    assert not os.path.exists(os.path.join(tmp_path, "ref.0"))
    assert not os.path.exists(os.path.join(tmp_path, "gpu.0"))
    with open(os.path.join(tmp_path, "ref.info")) as f1, open(os.path.join(tmp_path, "gpu.info")) as f2:
        assert f2.read() == f1.read()


@pytest.mark.gpu
def test_dropin_subsamples(tmp_path):
    """SampInHalos / SampOutHalos > 0: the drop-in writes the same catalog
    as the reference (which runs without sampling here: its GSL draw is not
    available), "<base>_inhalo.0" / "_outhalo.0" in Subsample's unformatted
    layout holding exactly the particles the library's own sampled run keeps
    on the same input, and the counts in the info file."""
    from cm_halofinder_b200 import FofConfig, fof_sampled
    from tests.subsample_ref import read_unformatted
    w = synth.make_box(20000, 60.0, 400, 405, nphalomin=5, boundary=3.0)
    params = _prepare(w, str(tmp_path))
    text = open(params["gpu"]).read()
    text = text.replace("SampInHalos -1", "SampInHalos 0.3").replace(
        "SampOutHalos -1", "SampOutHalos 0.05").replace("Seed 1", "Seed 41")
    open(params["gpu"], "w").write(text)
    _run(os.path.join(reference.REF_DIR, "cmh_ref_f32"), params["ref"])
    _run(_exe("cmh_dropin_f32"), params["gpu"])
    # the catalog is the reference's; the info file differs only in the counts
    ref = reference.read_catalog(os.path.join(tmp_path, "ref.0"), HALOSIZE)
    got = reference.read_catalog(os.path.join(tmp_path, "gpu.0"), HALOSIZE)
    assert len(got) == len(ref) > 5
    for h, g in zip(ref, got):
        np.testing.assert_array_equal(np.sort(g["ids"]), np.sort(h["ids"]))
    # the same draw through the library on the program's P[] (the pre-ghosted
    # processing array, run isolated on [lo, hi] with the upper faces closed)
    src, ppos, _ = cpu.build_proc(w)
    ids = np.asarray(src, np.uint64)
    cfg = FofConfig(lo=w.lo, hi=w.hi, boundary=w.boundary, linklength=w.linklength,
                    nphalomin=w.nphalomin, periodic=False)
    _, inh, outh = fof_sampled(ppos, w.vel[src], cfg, 0.3, 0.05, 41, ids=ids)
    for name, idx in (("inhalo", inh), ("outhalo", outh)):
        p, v, i = read_unformatted(os.path.join(tmp_path, f"gpu_{name}.0"))
        np.testing.assert_array_equal(i, ids[idx])
        np.testing.assert_array_equal(p, ppos[idx])
        np.testing.assert_array_equal(v, w.vel[src][idx])
    rows = open(os.path.join(tmp_path, "gpu.info")).read().splitlines()[1].split()
    assert rows[7:] == [str(len(got)), str(len(inh)), str(len(outh))]
    assert len(inh) > 100 and len(outh) > 100


def test_dropin_without_gpu_reports_the_library_error(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    exe = _exe("cmh_dropin_f32")
    w = synth.config2(seed=406, scale=3000 / 256 ** 3)
    params = _prepare(w, str(tmp_path))
    r = subprocess.run([exe, params["gpu"]], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "no usable CUDA device" in r.stdout
    assert not os.path.exists(os.path.join(tmp_path, "gpu.0"))
