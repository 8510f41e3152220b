"""Run the reference's own FoF (oracle/_ref, built from src_v2 by
oracle/Makefile) on a processing array -- test infrastructure only.

The reference runs single-rank and non-periodic (Nx = Ny = Nz = 1), which is
the configuration in which its periodic-image handling is not needed: the
caller hands it a pre-built processing array (originals then images), so the
reference's P[] order equals the processing order and its halo heads are the
same indices.  Input is the ASCII reader of read_data.c:380-400
(``%llu %f %f %f %f %f %f`` in MEMORY_MODE, ``%lf`` otherwise; values are
printed with enough digits to round-trip exactly).  Output is the
OUTPUT_UNFORMATTED + OUTPUT_PARTICLES + PARTICLE_ID catalog of
FOF.c:600-773, parsed by ``read_catalog``.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# The reference tree (its src_v2/ sources) comes from the environment; unset,
# nothing here is rebuilt and the prebuilt binaries in _ref/ are used as found.
REF_SRC = os.environ.get("CMH_REFERENCE") or None


def available(binary="cmh_ref_f32"):
    return os.path.exists(os.path.join(REF_DIR, binary))


def build():
    """Compile the reference binaries (needs the reference sources)."""
    if not REF_SRC or not os.path.isdir(REF_SRC):
        raise FileNotFoundError("reference sources are not present (set CMH_REFERENCE)")
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)


def write_params(path, *, lo, hi, boundary, linklength, nphalomin, cells,
                 n_proc, base_in, base_out):
    lo = [float(x) for x in lo]   # plain floats: repr of a numpy scalar is not a number
    hi = [float(x) for x in hi]
    boundary, linklength, nphalomin = float(boundary), float(linklength), float(nphalomin)
    ext = [hi[a] - lo[a] for a in range(3)]
    # Set_Params sizes P[] as Buffer*(1+extra)*Px*Py*Pz (startup.c:96-104);
    # pick Buffer so that the whole processing array fits.
    buffer = 2.0 * (n_proc + 16) / float(cells) ** 3 + 1.0
    lines = [
        "Nx 1", "Ny 1", "Nz 1",
        f"Px {cells}", f"Py {cells}", f"Pz {cells}",
        f"Lxmin {lo[0]!r}", f"Lymin {lo[1]!r}", f"Lzmin {lo[2]!r}",
        f"Lxmax {hi[0]!r}", f"Lymax {hi[1]!r}", f"Lzmax {hi[2]!r}",
        "Seed 1", f"Buffer {buffer!r}", f"Boundarysize {boundary!r}",
        f"Linklength {linklength!r}", f"Nphalomin {nphalomin!r}",
        "SampInHalos -1", "SampOutHalos -1", "InputStyle 0", "Ninputfiles 1",
        "Starting_file 0", "Nread 1", "Nwrite 1",
        f"InputFileBase {base_in}", f"OutputFileBase {base_out}",
    ]
    del ext
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_ascii(path, ids, pos, vel):
    """One particle per line, with digits enough for an exact round trip."""
    fmt = "%.9g" if pos.dtype == np.float32 else "%.17g"
    arr = np.concatenate([pos.astype(np.float64), vel.astype(np.float64)], axis=1)
    row = " ".join([fmt] * 6)
    with open(path, "w") as f:
        if ids is None:
            f.writelines(row % tuple(a) + "\n" for a in arr.tolist())
        else:
            f.writelines("%d " % i + row % tuple(a) + "\n"
                         for i, a in zip(ids.tolist(), arr.tolist()))


def read_catalog(path, halosize):
    """Parse the OUTPUT_PARTICLES + OUTPUT_UNFORMATTED + PARTICLE_ID catalog:
    [4][nhalos:i32][4] then per halo [4][halosize floats][4] followed by n
    particle records [4][ID:u64][6 floats][4] (FOF.c:603-773)."""
    halos = []
    if not os.path.exists(path):
        return halos
    data = open(path, "rb").read()
    off = 0

    def rec():
        nonlocal off
        (ln,) = struct.unpack_from("<i", data, off)
        body = data[off + 4: off + 4 + ln]
        (ln2,) = struct.unpack_from("<i", data, off + 4 + ln)
        assert ln == ln2, "bad Fortran record"
        off += 8 + ln
        return body

    (nh,) = struct.unpack("<i", rec())
    for _ in range(nh):
        props = np.frombuffer(rec(), np.float32).copy()
        assert props.shape[0] == halosize
        n = int(props[0])
        ids = np.empty(n, np.uint64)
        pv = np.empty((n, 6), np.float32)
        for k in range(n):
            body = rec()
            ids[k] = struct.unpack_from("<Q", body, 0)[0]
            pv[k] = np.frombuffer(body, np.float32, 6, 8)
        halos.append({"props": props, "ids": ids, "pv": pv})
    return halos


class SubBox:
    """One rank's domain of the reference's Nx = Ny = Nz = ndiv decomposition
    of a box (startup.c:33-47) with its ghost shell: for a periodic box the
    shell is filled by the periodic wrap the reference applies to received
    ghosts (read_data.c:792-797); for an isolated domain (a lightcone) the
    shell holds the particles within Boundarysize of the sub-domain, with no
    wrap.  Used to time the reference on bounded samples.  `w.pos` / `w.vel`
    may be numpy arrays or torch tensors on a GPU (the cut is then made
    there and only the sub-domain's particles are copied to the host)."""

    def __init__(self, w, ndiv, index):
        L = w.hi[0] - w.lo[0]
        side = L / ndiv
        ix, iy, iz = index % ndiv, (index // ndiv) % ndiv, index // (ndiv * ndiv)
        lo = np.array([w.lo[0] + ix * side, w.lo[1] + iy * side, w.lo[2] + iz * side])
        b = w.boundary
        if not isinstance(w.pos, np.ndarray):
            import torch
            x = w.pos
            off = torch.tensor(lo - b, dtype=torch.float64, device=x.device)
            keep = torch.ones(x.shape[0], dtype=torch.bool, device=x.device)
            for a in range(3):  # per axis, to bound the temporaries
                y = x[:, a].double() - off[a]
                if w.periodic:
                    y = torch.remainder(y, L)
                keep &= (y >= 0) & (y <= side + 2 * b)
            idx = torch.nonzero(keep).squeeze(1)
            y = x[idx].double() - off
            if w.periodic:
                y = torch.remainder(y, L)
            y = y.cpu().numpy()
            self.pvel = w.vel[idx].cpu().numpy()
            dtype = np.float32 if x.dtype == torch.float32 else np.float64
        else:
            y = w.pos.astype(np.float64) - (lo - b)  # offset from the padded low corner
            if w.periodic:
                y = np.mod(y, L)
            keep = np.all((y >= 0) & (y <= side + 2 * b), axis=1)
            y = y[keep]
            self.pvel = w.vel[keep]
            dtype = w.pos.dtype
        self.ppos = (lo - b + y).astype(dtype)
        self.n_owned = int(np.all((y >= b) & (y < side + b), axis=1).sum())
        self.lo = tuple(lo)
        self.hi = tuple(lo + side)
        self.boundary = b
        self.linklength = w.linklength
        self.nphalomin = w.nphalomin
        # cell size of the global run, lcell = (L + 2b) / Px (FOF.c:50-52)
        lcell = (L + 2 * b) / w.cells
        self.cells = max(int(round((side + 2 * b) / lcell)), 1)


def time_subbox(sb, timeout=None, binary="cmh_ref_f32_timing"):
    """Wall time of the reference process (ASCII read, FOF, binary write) on
    one sub-box; None if it did not finish within `timeout` seconds."""
    exe = os.path.join(REF_DIR, binary)
    d = tempfile.mkdtemp(prefix="cmhref_t_")
    try:
        write_ascii(os.path.join(d, "in.0"), None, sb.ppos, sb.pvel)
        write_params(os.path.join(d, "params.txt"), lo=sb.lo, hi=sb.hi, boundary=sb.boundary,
                     linklength=sb.linklength, nphalomin=sb.nphalomin, cells=sb.cells,
                     n_proc=sb.ppos.shape[0], base_in=os.path.join(d, "in"),
                     base_out=os.path.join(d, "out"))
        t0 = time.perf_counter()
        try:
            r = subprocess.run([exe, os.path.join(d, "params.txt")], capture_output=True,
                               timeout=timeout)
        except subprocess.TimeoutExpired:
            return None, time.perf_counter() - t0
        dt = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference failed ({r.returncode})")
        return dt, dt
    finally:
        for f in os.listdir(d):
            os.unlink(os.path.join(d, f))
        os.rmdir(d)


def run_proc(w, ppos, pvel, pids, *, binary=None, workdir=None, timeout=None):
    """Run the reference FoF on a processing array.  Returns (halos, seconds).

    ``pids`` are the IDs written for each processing particle (images carry
    the ID of their source particle).
    """
    if binary is None:
        binary = "cmh_ref_f64" if ppos.dtype == np.float64 else "cmh_ref_f32"
    exe = os.path.join(REF_DIR, binary)
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    own = workdir is None
    d = tempfile.mkdtemp(prefix="cmhref_") if own else workdir
    try:
        base_in = os.path.join(d, "in")
        base_out = os.path.join(d, "out")
        write_ascii(base_in + ".0", pids, ppos, pvel)
        write_params(os.path.join(d, "params.txt"), lo=w.lo, hi=w.hi,
                     boundary=w.boundary, linklength=w.linklength,
                     nphalomin=w.nphalomin, cells=w.cells, n_proc=ppos.shape[0],
                     base_in=base_in, base_out=base_out)
        t0 = time.perf_counter()
        r = subprocess.run([exe, os.path.join(d, "params.txt")], capture_output=True,
                           text=True, timeout=timeout)
        dt = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference failed ({r.returncode}): {r.stdout[-2000:]}")
        halosize = 19  # parity builds carry INERTIA and DISPERSION
        halos = read_catalog(base_out + ".0", halosize)
        return halos, dt
    finally:
        if own:
            for f in os.listdir(d):
                os.unlink(os.path.join(d, f))
            os.rmdir(d)
