"""ctypes wrapper of the CPU restatement (fof_oracle.c) -- test infrastructure.

The restatement follows src_v2/FOF.c of the reference line by line except
that Befriend's ring splice (FOF.c:359-373) is a union-find; see
fof_oracle.h.  It is pinned against the reference binaries in
tests/test_oracle_pin.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libcmh_oracle.so")


class Params(C.Structure):
    _fields_ = [
        ("lo", C.c_double * 3), ("hi", C.c_double * 3),
        ("boundary", C.c_double), ("linklength", C.c_double),
        ("nphalomin", C.c_double), ("periodic", C.c_int),
        ("pos_is_double", C.c_int), ("vel_is_double", C.c_int),
        ("cells", C.c_int * 3), ("props", C.c_int), ("varlink", C.c_int),
        ("origin", C.c_double * 3), ("ltab_n", C.c_int),
        ("ltab_rmax", C.c_double), ("ltab", C.POINTER(C.c_double)),
    ]


class Stats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in (
        "n_in", "n_out", "n_kept", "n_images", "n_proc", "n_groups",
        "n_candidates", "nhalos", "n_edge_warn", "n_pair_tests",
        "n_member_conflicts")]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "libcmh_oracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.cmh_oracle_halosize.restype = C.c_int
        L.cmh_oracle_build_proc.restype = C.c_int64
        L.cmh_oracle_build_proc.argtypes = [C.POINTER(Params), C.c_int64, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.POINTER(Stats)]
        L.cmh_oracle_fof.restype = C.c_int
        L.cmh_oracle_fof.argtypes = [C.POINTER(Params), C.c_int64, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.POINTER(Stats)]
        L.cmh_oracle_linked_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_double]
        L.cmh_oracle_linked_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_double]
        _lib = L
    return _lib


def make_params(w, props=0, periodic=None, cells=None):
    """Oracle parameters from a synth.Workload-like object."""
    p = Params()
    for a in range(3):
        p.lo[a] = w.lo[a]
        p.hi[a] = w.hi[a]
        p.cells[a] = int(cells if cells is not None else w.cells)
    p.boundary = w.boundary
    p.linklength = w.linklength
    p.nphalomin = w.nphalomin
    p.periodic = int(w.periodic if periodic is None else periodic)
    p.pos_is_double = int(w.pos.dtype == np.float64)
    p.vel_is_double = int(w.vel.dtype == np.float64)
    p.props = props
    p.varlink = 0
    if getattr(w, "varlink", None):
        tab = np.ascontiguousarray(w.varlink["table"], np.float64)
        p._ltab_keep = tab
        p.varlink = 1
        for a in range(3):
            p.origin[a] = w.varlink["origin"][a]
        p.ltab_n = len(tab)
        p.ltab_rmax = w.varlink["rmax"]
        p.ltab = tab.ctypes.data_as(C.POINTER(C.c_double))
    return p


def halosize(props):
    return lib().cmh_oracle_halosize(props)


def build_proc(w, periodic=None):
    """Processing array (kept originals, then images) as in fof_oracle.h."""
    p = make_params(w, periodic=periodic)
    pos = np.ascontiguousarray(w.pos)
    st = Stats()
    m = lib().cmh_oracle_build_proc(C.byref(p), pos.shape[0], pos.ctypes.data, None,
                                    None, C.byref(st))
    if m < 0:
        raise ValueError("oracle: bad arguments")
    src = np.empty(m, np.uint32)
    ppos = np.empty((m, 3), pos.dtype)
    lib().cmh_oracle_build_proc(C.byref(p), pos.shape[0], pos.ctypes.data,
                                src.ctypes.data, ppos.ctypes.data, C.byref(st))
    return src, ppos, st.as_dict()


def fof_proc(w, src, ppos, pvel, props=0, n_src=None):
    """FoF over a processing array; returns a dict of numpy arrays."""
    p = make_params(w, props=props)
    m = ppos.shape[0]
    ppos = np.ascontiguousarray(ppos)
    pvel = np.ascontiguousarray(pvel)
    p.pos_is_double = int(ppos.dtype == np.float64)
    p.vel_is_double = int(pvel.dtype == np.float64)
    src = np.ascontiguousarray(src, np.uint32)
    n_src = int(n_src if n_src is not None else (int(src.max()) + 1 if m else 0))
    hs = halosize(props)
    group = np.empty(m, np.int64)
    head = np.empty(max(m, 1), np.uint32)
    props_out = np.empty((max(m, 1), hs), np.float32)
    member = np.empty(max(n_src, 1), np.int64)
    st = Stats()
    rc = lib().cmh_oracle_fof(C.byref(p), m, ppos.ctypes.data, pvel.ctypes.data,
                              src.ctypes.data, n_src, group.ctypes.data,
                              head.ctypes.data, props_out.ctypes.data,
                              member.ctypes.data, C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle FoF failed with code {rc}")
    nh = st.nhalos
    return {"group": group, "halo_head": head[:nh].copy(),
            "halo_props": props_out[:nh].copy(), "member": member[:n_src].copy(),
            "stats": st.as_dict()}


def run(w, props=0):
    """Whole hot path on the CPU: processing array, FoF, catalog."""
    src, ppos, st0 = build_proc(w)
    pvel = w.vel[src]
    out = fof_proc(w, src, ppos, pvel, props=props, n_src=w.n)
    out["proc_src"] = src
    out["proc_pos"] = ppos
    out["stats"].update({k: st0[k] for k in ("n_in", "n_out", "n_kept",
                                             "n_images", "n_proc")})
    return out
