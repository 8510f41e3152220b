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


def _call_noalloc(tpos, lab, cfg):
    import torch
    p = cfg.to_c()
    return _abi.lib().cmh_fof_labels_noalloc(
        C.byref(p), C.c_void_p(tpos.data_ptr()),
        _abi.CMH_FLOAT64 if tpos.dtype == torch.float64 else _abi.CMH_FLOAT32,
        tpos.shape[0], C.c_void_p(lab.data_ptr()),
        C.c_void_p(torch.cuda.current_stream(tpos.device).cuda_stream))


def _labels_noalloc(pos, cfg):
    import torch
    dev = torch.device("cuda", 0)
    tpos = torch.from_numpy(pos).to(dev)
    lab = torch.full((pos.shape[0],), -1, dtype=torch.int32, device=dev)
    _abi.check(_call_noalloc(tpos, lab, cfg))
    return lab.cpu().numpy().view(np.uint32)


def _brute_labels(pos, linklength):
    """Lowest index of each particle's group, every pair tested with the
    reference's predicate: the coordinate difference in the storage type,
    then ((dx*dx + dy*dy) + dz*dz) <= l^2 in double."""
    n = pos.shape[0]
    parent = np.arange(n)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    lsq = float(linklength) * float(linklength)
    for i in range(n - 1):
        d = (pos[i + 1:] - pos[i]).astype(np.float64)
        d2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]
        d2 = d2 + d[:, 2] * d[:, 2]
        for j in np.nonzero(~(d2 > lsq))[0] + i + 1:
            a, b = find(i), find(int(j))
            if a != b:
                parent[max(a, b)] = min(a, b)
    return np.array([find(i) for i in range(n)], np.uint32)


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


def test_noalloc_tiny_linklength_in_large_box():
    """A linking length far below the box side: the cell grid is sized by the
    2^18-cell limit, not by the linking length, and stays complete."""
    rng = np.random.default_rng(31)
    L, ll = 1000.0, 4.8e-4
    base = rng.random((700, 3)) * L
    # pairs and triples at 0.2-0.9 l and lone neighbours at 1.1-2 l
    near = base[:400] + rng.normal(size=(400, 3)) * (0.35 * ll / np.sqrt(3))
    far = base[400:600] + rng.choice([-1, 1], (200, 3)) * (1.1 * ll)
    pos = np.clip(np.concatenate([base, near, far]), 0, L).astype(np.float32)
    pos = pos[rng.permutation(pos.shape[0])]
    cfg = FofConfig(lo=(0, 0, 0), hi=(L, L, L), boundary=0.0, linklength=ll, nphalomin=1,
                    periodic=False, precision="fp64")
    label = _labels_noalloc(pos, cfg)
    np.testing.assert_array_equal(label, _brute_labels(pos, ll))
    assert np.unique(label).shape[0] < pos.shape[0]  # some groups formed


def test_noalloc_shell_particles_and_domain_error():
    """Particles in the ghost shell [lo-b, lo) and (hi, hi+b] are grouped
    like the others; a particle beyond the shell is CMH_ERR_DOMAIN."""
    import torch
    w = synth.config2(seed=13, scale=3000 / 256 ** 3)
    b = 6.0
    top = np.float32(w.hi[0] + b)
    if float(top) > w.hi[0] + b:       # the largest float32 not beyond hi + b
        top = np.nextafter(top, np.float32(0))
    pos = w.pos.astype(np.float64)
    pos[::5] -= 0.5 * b        # into the low shell where x < b/2
    pos = np.clip(pos, w.lo[0] - b, float(top)).astype(np.float32)
    pos[1] = top               # on the outer face: inside
    cfg = FofConfig(lo=w.lo, hi=w.hi, boundary=b, linklength=w.linklength, nphalomin=1,
                    periodic=False, precision="fp64")
    label = _labels_noalloc(pos, cfg)
    np.testing.assert_array_equal(label, _brute_labels(pos, w.linklength))
    bad = pos.copy()
    bad[7, 2] = np.float32(w.hi[2] + 1.5 * b)
    dev = torch.device("cuda", 0)
    lab = torch.zeros(bad.shape[0], dtype=torch.int32, device=dev)
    st = _call_noalloc(torch.from_numpy(bad).to(dev), lab, cfg)
    assert st == 5 and "outside" in _abi.last_error()


def test_noalloc_calls_allocate_nothing():
    """Device memory in use does not change across calls (the module and
    its array are loaded by the first call, so the check starts after it)."""
    import torch
    pos, _, cfg = _case(14, 20000, np.float32)
    dev = torch.device("cuda", 0)
    tpos = torch.from_numpy(pos).to(dev)
    lab = torch.zeros(pos.shape[0], dtype=torch.int32, device=dev)
    _abi.check(_call_noalloc(tpos, lab, cfg))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    reserved0 = torch.cuda.memory_reserved(dev)
    for _ in range(3):
        _abi.check(_call_noalloc(tpos, lab, cfg))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    assert torch.cuda.memory_reserved(dev) == reserved0
