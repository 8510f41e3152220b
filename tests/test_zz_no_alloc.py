"""The allocation-free entry point (cmh_fof_labels_noalloc) against the
regular one.

It serves callers that cannot allocate device memory, so it takes device
inputs and outputs from the caller and keeps its scratch in a fixed device
array inside the library.  This file is collected last on purpose.  It must
pass alone in a fresh process and after the other tests.

The regular entry point (cmh_fof_run) on the same particles, non-periodic,
with every particle inside [lo, hi), Nphalomin = 1 and no ghost shell, owns
every group and orders its catalog by each group's lowest index.  So the
label of particle i (lowest index of its group) must be the head of i's
catalog entry, exactly.  Two calls in a row, on different inputs, check that
the shared scratch is cleared between calls."""
import ctypes as C

import numpy as np
import pytest

from cm_halofinder_b200 import FofConfig, _abi, fof, synth

pytestmark = pytest.mark.gpu


def _case(seed, n, dtype):
    w = synth.config2(seed=seed, scale=n / 256 ** 3)
    pos = w.pos.astype(dtype)
    cfg = FofConfig(lo=w.lo, hi=w.hi, boundary=0.0, linklength=w.linklength, nphalomin=1,
                    periodic=False, precision="fp64")
    return pos, w.vel, cfg


def _labels_noalloc(pos, cfg):
    import torch
    dev = torch.device("cuda", 0)
    tpos = torch.from_numpy(pos).to(dev)
    lab = torch.full((pos.shape[0],), -1, dtype=torch.int32, device=dev)
    p = cfg.to_c()
    st = _abi.lib().cmh_fof_labels_noalloc(
        C.byref(p), C.c_void_p(tpos.data_ptr()),
        _abi.CMH_FLOAT64 if pos.dtype == np.float64 else _abi.CMH_FLOAT32,
        pos.shape[0], C.c_void_p(lab.data_ptr()),
        C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    _abi.check(st)
    return lab.cpu().numpy().view(np.uint32)


def test_noalloc_labels_match_regular_entry_point_twice():
    for seed, dtype in ((11, np.float32), (12, np.float64)):
        pos, vel, cfg = _case(seed, 30000, dtype)
        label = _labels_noalloc(pos, cfg)
        cat = fof(pos, vel, cfg, members=True)
        assert cat.stats["n_out"] == 0
        assert cat.nhalos == np.unique(label).shape[0]
        # every group owned: member[i] indexes the catalog, whose head is the
        # group's lowest index
        np.testing.assert_array_equal(cat.head[cat.member], label)


def test_noalloc_rejects_oversize_and_periodic():
    import torch
    dev = torch.device("cuda", 0)
    pos = torch.zeros((65537, 3), dtype=torch.float32, device=dev)
    lab = torch.zeros(65537, dtype=torch.int32, device=dev)
    cfg = FofConfig(lo=(0, 0, 0), hi=(1, 1, 1), boundary=0.0, linklength=0.1, periodic=False)
    p = cfg.to_c()
    st = _abi.lib().cmh_fof_labels_noalloc(C.byref(p), C.c_void_p(pos.data_ptr()), 0, 65537,
                                           C.c_void_p(lab.data_ptr()), None)
    assert st == 6 and "65536" in _abi.last_error()
    cfg.periodic = True
    p = cfg.to_c()
    st = _abi.lib().cmh_fof_labels_noalloc(C.byref(p), C.c_void_p(pos.data_ptr()), 0, 10,
                                           C.c_void_p(lab.data_ptr()), None)
    assert st == 1
