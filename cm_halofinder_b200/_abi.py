"""ctypes mirror of include/cmh_fof.h (the library's C ABI)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcmh_fof.so")

CMH_OK = 0
STATUS = {
    0: "CMH_OK", 1: "CMH_ERR_INVALID_ARGUMENT", 2: "CMH_ERR_PARAMETER_FILE",
    3: "CMH_ERR_CUDA", 4: "CMH_ERR_OUT_OF_MEMORY", 5: "CMH_ERR_DOMAIN",
    6: "CMH_ERR_CAPACITY", 7: "CMH_ERR_DEVICE_TIMEOUT", 8: "CMH_ERR_IO",
    9: "CMH_ERR_NO_DEVICE",
}
CMH_FLOAT32, CMH_FLOAT64 = 0, 1
CMH_PLAIN_FP64, CMH_FP32_RECHECK = 0, 1
CMH_HOST, CMH_DEVICE = 0, 1
CMH_PROP_INERTIA, CMH_PROP_DISPERSION = 1, 2
CMH_OUT_UNFORMATTED, CMH_OUT_PARTICLES, CMH_OUT_PARTICLE_ID = 1, 2, 4
CMH_TAGS_VARLINK, CMH_TAGS_INFOFILE = 1, 2
CMH_FMT_ASCII, CMH_FMT_GADGET1, CMH_FMT_PICOLA_LIGHTCONE = 0, 1, 2
CMH_READ_PARTICLE_ID, CMH_READ_FP64 = 1, 2


class FofParams(C.Structure):
    _fields_ = [
        ("lo", C.c_double * 3), ("hi", C.c_double * 3), ("boundary", C.c_double),
        ("linklength", C.c_double), ("nphalomin", C.c_double), ("periodic", C.c_int32),
        ("precision", C.c_int32), ("properties", C.c_uint32), ("cell_factor", C.c_int32),
        ("varlink", C.c_int32), ("ref_cells", C.c_int32 * 3), ("origin", C.c_double * 3),
        ("ltab_n", C.c_int32), ("ltab_rmax", C.c_double), ("ltab", C.POINTER(C.c_double)),
    ]


class Particles(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("pos_dtype", C.c_int32), ("vel_dtype", C.c_int32),
        ("pos", C.c_void_p), ("vel", C.c_void_p), ("id", C.c_void_p),
        ("location", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in (
        "n_in", "n_out", "n_images", "n_proc", "n_cells", "n_groups", "n_candidates",
        "nhalos", "n_edge_warn", "n_pair_tests", "n_rechecks", "n_member_conflicts")] + [
        ("cell_factor", C.c_int32), ("key_bits", C.c_int32), ("ms_total", C.c_float),
        ("stage_ms", C.c_float * 8), ("n_launches", C.c_int32)] + [
        (k, C.c_int64) for k in ("n_cell_pairs", "n_root_skips", "n_unions", "n_find_steps",
                                 "n_scan_iters", "n_window_iters", "n_dense_tops",
                                 "n_queued", "n_big_tops")]

    STAGES = ("ingest", "sort", "cells", "befriend", "groups", "sums", "catalog", "members")

    def as_dict(self):
        d = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            if k == "stage_ms":
                d[k] = dict(zip(self.STAGES, (float(x) for x in v)))
            elif k == "ms_total":
                d[k] = float(v)
            else:
                d[k] = int(v)
        return d


class Catalog(C.Structure):
    _fields_ = [
        ("nhalos", C.c_int64), ("halosize", C.c_int32), ("location", C.c_int32),
        ("props", C.POINTER(C.c_float)), ("head", C.POINTER(C.c_uint32)),
        ("member", C.POINTER(C.c_int64)), ("member_proc", C.POINTER(C.c_uint32)),
        ("member_pos", C.POINTER(C.c_float)), ("stats", Stats), ("impl", C.c_void_p),
    ]


class Tuning(C.Structure):
    _fields_ = [("cell_scale", C.c_double), ("dense_min", C.c_int32), ("ms", C.c_float),
                ("tried", C.c_int32)]


class Sampling(C.Structure):
    _fields_ = [("samp_in", C.c_double), ("samp_out", C.c_double), ("seed", C.c_int32),
                ("closed_hi", C.c_int32 * 3)]


class Sample(C.Structure):
    _fields_ = [("n_inhalo", C.c_int64), ("inhalo", C.POINTER(C.c_int64)),
                ("n_outhalo", C.c_int64), ("outhalo", C.POINTER(C.c_int64))]


class RunParameters(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("Nx", "Ny", "Nz", "Px", "Py", "Pz")] + [
        (k, C.c_double) for k in ("Lxmin", "Lymin", "Lzmin", "Lxmax", "Lymax", "Lzmax")] + [
        ("Seed", C.c_int32)] + [
        (k, C.c_double) for k in ("Buffer", "Boundarysize", "Linklength", "Nphalomin",
                                  "SampInHalos", "SampOutHalos")] + [
        (k, C.c_int32) for k in ("InputStyle", "Ninputfiles", "Starting_file", "Nread",
                                 "Nwrite")] + [
        ("InputFileBase", C.c_char * 500), ("OutputFileBase", C.c_char * 500)] + [
        (k, C.c_double) for k in ("Omega", "Origin_x", "Origin_y", "Origin_z")] + [
        ("InputInfoFile", C.c_char * 500)]


class Limits(C.Structure):
    _fields_ = [("union_attempts", C.c_int64), ("lookback_polls", C.c_int64)]


# Every symbol include/cmh_fof.h declares, with its ctypes signature.
SIGNATURES = {
    "cmh_abi_version": (C.c_int, []),
    "cmh_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "cmh_fof_run": (C.c_int, [C.POINTER(FofParams), C.POINTER(Particles), C.POINTER(Catalog),
                              C.c_int32, C.c_void_p]),
    "cmh_catalog_free": (None, [C.POINTER(Catalog)]),
    "cmh_plan_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(FofParams), C.c_int64,
                                  C.c_int32, C.c_int32]),
    "cmh_plan_run": (C.c_int, [C.c_void_p, C.POINTER(Particles), C.POINTER(Catalog), C.c_int32,
                               C.c_int32, C.c_void_p]),
    "cmh_plan_set_params": (C.c_int, [C.c_void_p, C.POINTER(FofParams)]),
    "cmh_plan_destroy": (None, [C.c_void_p]),
    "cmh_plan_set_graph": (C.c_int, [C.c_void_p, C.c_int32]),
    "cmh_plan_autotune": (C.c_int, [C.c_void_p, C.POINTER(FofParams), C.POINTER(Particles),
                                    C.c_int32, C.c_int32, C.c_void_p, C.POINTER(Tuning)]),
    "cmh_plan_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    "cmh_plan_run_batch": (C.c_int, [C.c_void_p, C.POINTER(FofParams), C.POINTER(Particles),
                                     C.c_int32, C.POINTER(Catalog), C.c_void_p]),
    "cmh_fof_run_batch": (C.c_int, [C.POINTER(FofParams), C.POINTER(Particles), C.c_int32,
                                    C.POINTER(Catalog), C.c_void_p]),
    "cmh_plan_run_batch_status": (C.c_int, [C.c_void_p, C.POINTER(FofParams),
                                            C.POINTER(Particles), C.c_int32, C.POINTER(Catalog),
                                            C.POINTER(C.c_int), C.c_void_p]),
    "cmh_plan_set_limits": (C.c_int, [C.c_void_p, C.POINTER(Limits)]),
    "cmh_plan_prefetch": (C.c_int, [C.c_void_p, C.POINTER(Particles), C.c_void_p]),
    "cmh_plan_prefetch_batch": (C.c_int, [C.c_void_p, C.POINTER(Particles), C.c_int32,
                                          C.c_void_p]),
    "cmh_plan_set_input_buffers": (C.c_int, [C.c_void_p, C.c_int32]),
    "cmh_fof_labels_noalloc": (C.c_int, [C.POINTER(FofParams), C.c_void_p, C.c_int32,
                                         C.c_int64, C.c_void_p, C.c_void_p]),
    "cmh_read_parameterfile": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(RunParameters)]),
    "cmh_params_from_run": (C.c_int, [C.POINTER(RunParameters), C.c_int32, C.c_int32,
                                      C.POINTER(FofParams)]),
    "cmh_write_halos": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(Catalog),
                                  C.POINTER(Particles), C.c_uint32]),
    "cmh_write_info": (C.c_int, [C.c_char_p, C.POINTER(RunParameters), C.POINTER(C.c_int64),
                                 C.c_int32]),
    "cmh_write_info_sampled": (C.c_int, [C.c_char_p, C.POINTER(RunParameters),
                                         C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                         C.POINTER(C.c_int64), C.c_int32]),
    "cmh_fof_run_sampled": (C.c_int, [C.POINTER(FofParams), C.POINTER(Particles),
                                      C.POINTER(Sampling), C.POINTER(Catalog), C.c_int32,
                                      C.POINTER(Sample), C.c_void_p]),
    "cmh_sample_free": (None, [C.POINTER(Sample)]),
    "cmh_write_subsample": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.POINTER(Particles),
                                      C.POINTER(C.c_int64), C.c_int64, C.c_uint32]),
    "cmh_read_particles": (C.c_int, [C.POINTER(RunParameters), C.c_int32, C.c_uint32,
                                     C.POINTER(Particles), C.POINTER(C.c_void_p)]),
    "cmh_particle_store_free": (None, [C.c_void_p]),
}

_lib = None


class CmhError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def lib():
    """Load the native library; fails loudly if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"native library {LIB_PATH} is missing: run "
                              "`python -m cm_halofinder_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    buf = C.create_string_buffer(2048)
    lib().cmh_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status):
    if status != CMH_OK:
        raise CmhError(status, last_error())
