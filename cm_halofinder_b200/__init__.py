"""B200 Friends-of-Friends halo finder: drop-in for CM_Halofinder's FoF path.

Python face of the C ABI in include/cmh_fof.h.  The compute runs in the
native library (cm_halofinder_b200/libcmh_fof.so, hand-written sm_100a
kernels); there is no CPU fallback: importing works without a GPU, running
FoF without one raises ``CmhError(CMH_ERR_NO_DEVICE)``.

Reference interface mirrored here:
* ``read_parameterfile``  <- Read_Parameterfile (src_v2/startup.c:109-314)
* ``fof`` / ``Plan.run``  <- FOF() (src_v2/FOF.c:23-339): cell grid,
  befriending, halo retrieval, Checkhalo ownership and the property sums of
  Output_Halos; ``Catalog`` holds the unformatted halo records
  (FOF.c:836-872) in head order
* ``write_halos`` / ``write_info`` <- Output_Halos / Output_Info
  (FOF.c:546-957)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import (CMH_DEVICE, CMH_FLOAT32, CMH_FLOAT64, CMH_FP32_RECHECK, CMH_HOST,
                   CMH_OUT_PARTICLE_ID, CMH_OUT_PARTICLES, CMH_OUT_UNFORMATTED,
                   CMH_PLAIN_FP64, CMH_PROP_DISPERSION, CMH_PROP_INERTIA, CmhError)

__all__ = [
    "fof", "Plan", "Catalog", "FofConfig", "read_parameterfile", "read_particles",
    "config_from_run", "write_halos", "write_info", "fof_sampled", "write_subsample",
    "CmhError", "CMH_FP32_RECHECK", "CMH_PLAIN_FP64", "CMH_PROP_INERTIA", "CMH_PROP_DISPERSION",
    "CMH_OUT_UNFORMATTED", "CMH_OUT_PARTICLES", "CMH_OUT_PARTICLE_ID", "halosize",
]

PRECISION = {"fp64": CMH_PLAIN_FP64, "plain": CMH_PLAIN_FP64, "fp32": CMH_FP32_RECHECK,
             "fp32_recheck": CMH_FP32_RECHECK}


def halosize(properties=0):
    """Floats per halo record (FOF.c:574-580)."""
    return 7 + (6 if properties & 1 else 0) + (6 if properties & 2 else 0)


@dataclass
class FofConfig:
    """The run parameters FOF() reads, for one domain (Nx = Ny = Nz = 1)."""

    lo: tuple
    hi: tuple
    boundary: float
    linklength: float
    nphalomin: float = 10.0
    periodic: bool = True
    precision: str = "fp32"
    properties: int = 0
    cell_factor: int = 0
    varlink: dict | None = None       # {"origin", "rmax", "table", "ref_cells"}

    def to_c(self):
        p = _abi.FofParams()
        for a in range(3):
            p.lo[a] = float(self.lo[a])
            p.hi[a] = float(self.hi[a])
        p.boundary = float(self.boundary)
        p.linklength = float(self.linklength)
        p.nphalomin = float(self.nphalomin)
        p.periodic = int(bool(self.periodic))
        p.precision = PRECISION[self.precision] if isinstance(self.precision, str) \
            else int(self.precision)
        p.properties = int(self.properties)
        p.cell_factor = int(self.cell_factor)
        p.varlink = 0
        if self.varlink:
            tab = np.ascontiguousarray(self.varlink["table"], np.float64)
            p._keep = tab
            p.varlink = 1
            rc = self.varlink.get("ref_cells", (1, 1, 1))
            if np.isscalar(rc):
                rc = (rc, rc, rc)
            for a in range(3):
                p.origin[a] = float(self.varlink["origin"][a])
                p.ref_cells[a] = int(rc[a])
            p.ltab_n = len(tab)
            p.ltab_rmax = float(self.varlink["rmax"])
            p.ltab = tab.ctypes.data_as(C.POINTER(C.c_double))
        return p

    @classmethod
    def from_workload(cls, w, precision="fp32", properties=0, cell_factor=0):
        vl = None
        if getattr(w, "varlink", None):
            vl = dict(w.varlink)
            vl["ref_cells"] = w.cells
        return cls(lo=w.lo, hi=w.hi, boundary=w.boundary, linklength=w.linklength,
                   nphalomin=w.nphalomin, periodic=w.periodic, precision=precision,
                   properties=properties, cell_factor=cell_factor, varlink=vl)


@dataclass
class Catalog:
    """Owned halos in head order: ``props[h]`` is the reference's unformatted
    record (n, x, y, z, vx, vy, vz [, inertia] [, dispersion])."""

    props: np.ndarray
    head: np.ndarray
    member: np.ndarray | None
    stats: dict

    @property
    def nhalos(self):
        return int(self.props.shape[0])


def _dtype_code(a):
    if a.dtype == np.float32:
        return CMH_FLOAT32
    if a.dtype == np.float64:
        return CMH_FLOAT64
    raise TypeError("positions and velocities must be float32 or float64")


def _host_catalog(cat):
    nh, hs = int(cat.nhalos), int(cat.halosize)
    props = np.ctypeslib.as_array(cat.props, shape=(max(nh, 1), hs))[:nh].copy() \
        if nh else np.zeros((0, hs), np.float32)
    head = np.ctypeslib.as_array(cat.head, shape=(max(nh, 1),))[:nh].copy() \
        if nh else np.zeros(0, np.uint32)
    member = None
    if bool(cat.member):
        n = int(cat.stats.n_in)
        member = np.ctypeslib.as_array(cat.member, shape=(max(n, 1),))[:n].copy()
    return Catalog(props=props, head=head, member=member, stats=cat.stats.as_dict())


def fof(pos, vel, config: FofConfig, ids=None, members=False, stream=None):
    """One-shot FoF on host (numpy) arrays; returns a host Catalog.

    Equivalent of the reference's FOF() for one domain, minus the file
    writers (see write_halos)."""
    L = _abi.lib()
    pos = np.ascontiguousarray(pos)
    vel = np.ascontiguousarray(vel)
    if pos.ndim != 2 or pos.shape[1] != 3 or vel.shape != pos.shape:
        raise ValueError("pos and vel must be (N, 3)")
    parts = _abi.Particles(n=pos.shape[0], pos_dtype=_dtype_code(pos), vel_dtype=_dtype_code(vel),
                           pos=pos.ctypes.data, vel=vel.ctypes.data,
                           id=None if ids is None else np.ascontiguousarray(ids, np.uint64).ctypes.data,
                           location=CMH_HOST)
    p = config.to_c()
    cat = _abi.Catalog()
    _abi.check(L.cmh_fof_run(C.byref(p), C.byref(parts), C.byref(cat), int(members),
                             C.c_void_p(stream or 0)))
    try:
        return _host_catalog(cat)
    finally:
        L.cmh_catalog_free(C.byref(cat))


class Plan:
    """Device-resident repeated runs (cmh_plan_*).  Particles are torch CUDA
    tensors (N, 3) or raw device pointers with explicit dtypes."""

    def __init__(self, config: FofConfig, pos_dtype=np.float32, device=0, max_particles=0):
        self._L = _abi.lib()
        self.config = config
        self._p = config.to_c()
        h = C.c_void_p()
        _abi.check(self._L.cmh_plan_create(C.byref(h), C.byref(self._p), int(max_particles),
                                           CMH_FLOAT64 if np.dtype(pos_dtype) == np.float64
                                           else CMH_FLOAT32, int(device)))
        self._h = h

    def set_config(self, config: FofConfig):
        self.config = config
        self._p = config.to_c()
        _abi.check(self._L.cmh_plan_set_params(self._h, C.byref(self._p)))

    @staticmethod
    def _ptr(t):
        return int(t.data_ptr()) if hasattr(t, "data_ptr") else int(t)

    @staticmethod
    def _tdt(t):
        s = str(getattr(t, "dtype", ""))
        return CMH_FLOAT64 if "float64" in s else CMH_FLOAT32

    def run(self, pos, vel, n=None, members=False, out="host", stream=None,
            pos_dtype=None, vel_dtype=None):
        """Run on torch CUDA tensors (device-resident) or numpy arrays (host;
        copied to the device on `stream` inside the call)."""
        n = int(pos.shape[0]) if n is None else int(n)
        if isinstance(pos, np.ndarray):
            if not (pos.flags.c_contiguous and vel.flags.c_contiguous):
                raise ValueError("host arrays must be C-contiguous")
            parts = _abi.Particles(n=n, pos_dtype=_dtype_code(pos), vel_dtype=_dtype_code(vel),
                                   pos=pos.ctypes.data, vel=vel.ctypes.data, id=None,
                                   location=CMH_HOST)
        else:
            parts = _abi.Particles(n=n,
                                   pos_dtype=self._tdt(pos) if pos_dtype is None else pos_dtype,
                                   vel_dtype=self._tdt(vel) if vel_dtype is None else vel_dtype,
                                   pos=self._ptr(pos), vel=self._ptr(vel), id=None,
                                   location=CMH_DEVICE)
        cat = _abi.Catalog()
        loc = CMH_HOST if out == "host" else CMH_DEVICE
        if stream is None:
            sp = 0
        elif hasattr(stream, "cuda_stream"):
            sp = stream.cuda_stream
        else:
            sp = int(stream)
        _abi.check(self._L.cmh_plan_run(self._h, C.byref(parts), C.byref(cat), int(members),
                                        loc, C.c_void_p(sp)))
        if loc == CMH_DEVICE:
            return cat  # raw struct: device pointers into plan-owned memory
        try:
            return _host_catalog(cat)
        finally:
            self._L.cmh_catalog_free(C.byref(cat))

    def prefetch(self, pos, vel, stream=None):
        """Start copying host (numpy, ideally pinned) arrays to the device
        ahead of a later run(pos, vel) with the same arrays, so that the
        copy overlaps the GPU's current work (cmh_plan_prefetch)."""
        if not (pos.flags.c_contiguous and vel.flags.c_contiguous):
            raise ValueError("host arrays must be C-contiguous")
        parts = _abi.Particles(n=int(pos.shape[0]), pos_dtype=_dtype_code(pos),
                               vel_dtype=_dtype_code(vel), pos=pos.ctypes.data,
                               vel=vel.ctypes.data, id=None, location=CMH_HOST)
        _abi.check(self._L.cmh_plan_prefetch(self._h, C.byref(parts),
                                             C.c_void_p(self._stream(stream))))

    def set_input_buffers(self, n: int):
        """Device copies of host inputs the plan keeps: 2 (default) or 1, for
        workspaces that leave no room for a second (cmh_plan_set_input_buffers);
        with 1, prefetch() copies into the same buffer once the current run
        has read it."""
        _abi.check(self._L.cmh_plan_set_input_buffers(self._h, int(n)))

    def set_graph(self, enable: bool):
        """Replay runs of a repeated shape from a captured CUDA graph."""
        _abi.check(self._L.cmh_plan_set_graph(self._h, int(bool(enable))))

    def _parts(self, positions, velocities):
        """Particle descriptions of the boxes: torch CUDA tensors (device) or
        C-contiguous numpy arrays (host)."""
        nb = len(positions)
        parts = (_abi.Particles * nb)()
        for b in range(nb):
            pos, vel = positions[b], velocities[b]
            if isinstance(pos, np.ndarray) != isinstance(vel, np.ndarray):
                raise ValueError("a box's positions and velocities are both numpy "
                                 "(host) or both torch tensors (device)")
            if isinstance(pos, np.ndarray):
                if not (pos.flags.c_contiguous and vel.flags.c_contiguous):
                    raise ValueError("host arrays must be C-contiguous")
                parts[b] = _abi.Particles(n=int(pos.shape[0]), pos_dtype=_dtype_code(pos),
                                          vel_dtype=_dtype_code(vel), pos=pos.ctypes.data,
                                          vel=vel.ctypes.data, id=None, location=CMH_HOST)
            else:
                parts[b] = _abi.Particles(n=int(pos.shape[0]), pos_dtype=self._tdt(pos),
                                          vel_dtype=self._tdt(vel), pos=self._ptr(pos),
                                          vel=self._ptr(vel), id=None, location=CMH_DEVICE)
        return parts

    def _batch_args(self, configs, positions, velocities):
        nb = len(configs)
        cs = [c.to_c() for c in configs]     # keep the varlink tables alive
        P = (_abi.FofParams * nb)(*cs)
        return nb, P, self._parts(positions, velocities), cs

    def prefetch_batch(self, positions, velocities, stream=None):
        """Start copying the host (numpy, ideally pinned) arrays of a later
        run_batch with the same boxes, in the same order, to the device
        (cmh_plan_prefetch_batch)."""
        parts = self._parts(positions, velocities)
        _abi.check(self._L.cmh_plan_prefetch_batch(self._h, parts, len(positions),
                                                   C.c_void_p(self._stream(stream))))

    @staticmethod
    def _stream(stream):
        if stream is None:
            return 0
        return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)

    def autotune(self, configs, positions, velocities, repeats=2, stream=None):
        """Time the boxes over a grid of cell-size scales and dense-top
        thresholds; the plan keeps the fastest.  Returns the choice."""
        nb, P, parts, _keep = self._batch_args(configs, positions, velocities)
        t = _abi.Tuning()
        _abi.check(self._L.cmh_plan_autotune(self._h, P, parts, nb, int(repeats),
                                             C.c_void_p(self._stream(stream)), C.byref(t)))
        return {"cell_scale": t.cell_scale, "dense_min": t.dense_min, "ms": t.ms,
                "tried": t.tried}

    def set_tuning(self, tuning):
        """Apply a setting returned by autotune() (e.g. to a new plan)."""
        t = _abi.Tuning(cell_scale=float(tuning["cell_scale"]),
                        dense_min=int(tuning["dense_min"]))
        _abi.check(self._L.cmh_plan_set_tuning(self._h, C.byref(t)))

    def run_batch(self, configs, positions, velocities, stream=None, with_status=False):
        """Many independent boxes in one run (one sort, one befriending pass,
        one reduction for all of them); positions/velocities are torch CUDA
        tensors, or numpy arrays for every box (copied to the device inside
        the call, or taken from prefetch_batch).  Returns one host Catalog
        per box.  with_status: each box is
        checked on its own (cmh_plan_run_batch_status) and (catalogs,
        statuses) is returned, a rejected box's catalog being None."""
        nb, P, parts, _keep = self._batch_args(configs, positions, velocities)
        cats = (_abi.Catalog * nb)()
        st = (C.c_int * nb)()
        sp = C.c_void_p(self._stream(stream))
        if with_status:
            rc = self._L.cmh_plan_run_batch_status(self._h, P, parts, nb, cats, st, sp)
        else:
            rc = self._L.cmh_plan_run_batch(self._h, P, parts, nb, cats, sp)
        _abi.check(rc)
        out = []
        for b in range(nb):
            try:
                out.append(_host_catalog(cats[b]) if (not with_status or st[b] == 0) else None)
            finally:
                self._L.cmh_catalog_free(C.byref(cats[b]))
        return (out, [int(x) for x in st]) if with_status else out

    def set_limits(self, union_attempts=-1, lookback_polls=-1):
        """Bounds of the device loops that retry or wait (cmh_plan_set_limits);
        negative keeps the default."""
        lim = _abi.Limits(union_attempts=int(union_attempts), lookback_polls=int(lookback_polls))
        _abi.check(self._L.cmh_plan_set_limits(self._h, C.byref(lim)))

    def close(self):
        if getattr(self, "_h", None):
            self._L.cmh_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_parameterfile(fname, varlink=False):
    """Read a run_parameters file with the reference's rules
    (startup.c:109-314); raises CmhError(CMH_ERR_PARAMETER_FILE) on a
    missing, unknown or repeated tag."""
    rp = _abi.RunParameters()
    _abi.check(_abi.lib().cmh_read_parameterfile(str(fname).encode(), int(varlink),
                                                  C.byref(rp)))
    return rp


_FORMATS = {"ascii": 0, "gadget1": 1, "picola_lightcone": 2}


def read_particles(rp, fmt="ascii", with_id=False, fp64=False):
    """Read every input file of a run (read_data.c:100-404) in the
    reference's file order: returns (pos, vel, ids) host arrays, ids None
    unless with_id.  fmt is "ascii", "gadget1" or "picola_lightcone"."""
    L = _abi.lib()
    parts = _abi.Particles()
    store = C.c_void_p()
    flags = (_abi.CMH_READ_PARTICLE_ID if with_id else 0) | (_abi.CMH_READ_FP64 if fp64 else 0)
    _abi.check(L.cmh_read_particles(C.byref(rp), _FORMATS[fmt], flags, C.byref(parts),
                                    C.byref(store)))
    try:
        n = int(parts.n)
        dt = np.float64 if fp64 else np.float32
        ct = C.c_double if fp64 else C.c_float

        def arr(ptr, shape, ctype, dtype):
            if n == 0:
                return np.zeros(shape, dtype)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=shape).copy()

        pos = arr(parts.pos, (n, 3), ct, dt)
        vel = arr(parts.vel, (n, 3), ct, dt)
        ids = arr(parts.id, (n,), C.c_uint64, np.uint64) if with_id else None
    finally:
        L.cmh_particle_store_free(store)
    return pos, vel, ids


def config_from_run(rp, task=0, periodic=False, precision="fp32", properties=0):
    """FoF parameters of one task's domain (Set_Params, startup.c:33-47)."""
    p = _abi.FofParams()
    _abi.check(_abi.lib().cmh_params_from_run(C.byref(rp), int(task), int(periodic), C.byref(p)))
    return FofConfig(lo=tuple(p.lo), hi=tuple(p.hi), boundary=p.boundary,
                     linklength=p.linklength, nphalomin=p.nphalomin, periodic=bool(p.periodic),
                     precision=precision, properties=properties)


def write_halos(base, task, catalog: Catalog, pos=None, vel=None, ids=None, flags=0):
    """Write "<base>.<task>" in the reference's Output_Halos layout."""
    L = _abi.lib()
    nh, hs = catalog.props.shape
    props = np.ascontiguousarray(catalog.props, np.float32)
    head = np.ascontiguousarray(catalog.head, np.uint32)
    cat = _abi.Catalog(nhalos=nh, halosize=hs, location=CMH_HOST,
                       props=props.ctypes.data_as(C.POINTER(C.c_float)),
                       head=head.ctypes.data_as(C.POINTER(C.c_uint32)))
    keep = [props, head]
    parts = None
    if catalog.member is not None:
        mem = np.ascontiguousarray(catalog.member, np.int64)
        keep.append(mem)
        cat.member = mem.ctypes.data_as(C.POINTER(C.c_int64))
        cat.stats.n_in = mem.shape[0]
    if pos is not None:
        pos = np.ascontiguousarray(pos)
        vel = np.ascontiguousarray(vel)
        idp = None
        if ids is not None:
            ids = np.ascontiguousarray(ids, np.uint64)
            idp = ids.ctypes.data
        keep += [pos, vel, ids]
        parts = _abi.Particles(n=pos.shape[0], pos_dtype=_dtype_code(pos),
                               vel_dtype=_dtype_code(vel), pos=pos.ctypes.data,
                               vel=vel.ctypes.data, id=idp, location=CMH_HOST)
    _abi.check(L.cmh_write_halos(str(base).encode(), int(task), C.byref(cat),
                                 C.byref(parts) if parts is not None else None, int(flags)))


def write_info(base, rp, nhalos_per_task, ninhalo_per_task=None, nouthalo_per_task=None):
    """Write "<base>.info" (Output_Info); the subsample counts default to 0."""
    L = _abi.lib()
    arr = np.ascontiguousarray(nhalos_per_task, np.int64)
    cnt = [None if a is None else np.ascontiguousarray(a, np.int64)
           for a in (ninhalo_per_task, nouthalo_per_task)]
    ptr = [None if a is None else a.ctypes.data_as(C.POINTER(C.c_int64)) for a in cnt]
    _abi.check(L.cmh_write_info_sampled(str(base).encode(), C.byref(rp),
                                        arr.ctypes.data_as(C.POINTER(C.c_int64)), ptr[0],
                                        ptr[1], len(arr)))


def fof_sampled(pos, vel, config: FofConfig, samp_in, samp_out, seed, ids=None,
                members=False, stream=None, closed_hi=None):
    """fof() that also draws the SampInHalos / SampOutHalos subsample
    (FOF.c:205-284): returns (catalog, inhalo, outhalo), the last two the
    input indices of the kept particles, ascending.  closed_hi (per axis)
    defaults to the reference's single-rank run: upper faces included when
    isolated, excluded when periodic."""
    L = _abi.lib()
    pos = np.ascontiguousarray(pos)
    vel = np.ascontiguousarray(vel)
    if pos.ndim != 2 or pos.shape[1] != 3 or vel.shape != pos.shape:
        raise ValueError("pos and vel must be (N, 3)")
    idarr = None if ids is None else np.ascontiguousarray(ids, np.uint64)
    parts = _abi.Particles(n=pos.shape[0], pos_dtype=_dtype_code(pos), vel_dtype=_dtype_code(vel),
                           pos=pos.ctypes.data, vel=vel.ctypes.data,
                           id=None if idarr is None else idarr.ctypes.data, location=CMH_HOST)
    p = config.to_c()
    if closed_hi is None:
        closed_hi = (0, 0, 0) if config.periodic else (1, 1, 1)
    samp = _abi.Sampling(samp_in=float(samp_in), samp_out=float(samp_out), seed=int(seed),
                         closed_hi=(C.c_int32 * 3)(*[int(bool(c)) for c in closed_hi]))
    cat = _abi.Catalog()
    out = _abi.Sample()
    _abi.check(L.cmh_fof_run_sampled(C.byref(p), C.byref(parts), C.byref(samp), C.byref(cat),
                                     int(members), C.byref(out), C.c_void_p(stream or 0)))
    try:
        inh = np.ctypeslib.as_array(out.inhalo, shape=(max(out.n_inhalo, 1),))[:out.n_inhalo].copy()
        outh = np.ctypeslib.as_array(out.outhalo, shape=(max(out.n_outhalo, 1),))[
            :out.n_outhalo].copy()
        return _host_catalog(cat), inh, outh
    finally:
        L.cmh_catalog_free(C.byref(cat))
        L.cmh_sample_free(C.byref(out))


def write_subsample(base, task, inhalo, pos, vel, idx, ids=None, flags=0):
    """Write "<base>_inhalo.<task>" (inhalo true) or "<base>_outhalo.<task>"
    in the layout of Subsample (FOF.c:432-544)."""
    L = _abi.lib()
    pos = np.ascontiguousarray(pos)
    vel = np.ascontiguousarray(vel)
    idx = np.ascontiguousarray(idx, np.int64)
    idarr = None if ids is None else np.ascontiguousarray(ids, np.uint64)
    parts = _abi.Particles(n=pos.shape[0], pos_dtype=_dtype_code(pos), vel_dtype=_dtype_code(vel),
                           pos=pos.ctypes.data, vel=vel.ctypes.data,
                           id=None if idarr is None else idarr.ctypes.data, location=CMH_HOST)
    _abi.check(L.cmh_write_subsample(str(base).encode(), int(task), int(bool(inhalo)),
                                     C.byref(parts), idx.ctypes.data_as(C.POINTER(C.c_int64)),
                                     idx.shape[0], int(flags)))
