"""Generate the golden fixtures: the reference's own FoF run on small seeded
inputs.

    python tests/golden/make_golden.py        (needs oracle/_ref, i.e. the
                                               reference sources, to build)

Each fixture stores the input particles and run parameters, and what the
reference binary (src_v2 built unmodified by oracle/Makefile, single rank,
non-periodic, fed the processing array: originals then periodic images)
wrote: the halo records (n, mean position, mean velocity, inertia and
dispersion tensors as floats) and each halo's member IDs, in catalog order.
The clumpy seeds are picked so that the reference's O(sum m^3) ring merge
finishes in seconds (largest clump recorded in the fixture).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cm_halofinder_b200 import synth  # noqa: E402
from oracle import cpu, reference  # noqa: E402


def lattice_ties():
    """Adversarial: a lattice with spacing exactly the linking length (d^2 ==
    l^2 exactly in double, linked), a lattice one float step wider (not
    linked), a dense knot of coincident particles, a lone particle, pairs
    straddling a face, and points at x = 0 and x = L - ulp."""
    L = 40.0
    ll = 0.78125                         # 25/32: l^2 exact in double
    pts = []
    g = np.arange(6) * ll + 5.0          # linked 6^3 block
    pts += [(x, y, z) for x in g for y in g for z in g]
    step = np.nextafter(np.float32(ll), np.float32(2))   # just beyond l
    g2 = 20.0 + np.arange(4, dtype=np.float32) * step
    pts += [(float(x), float(y), 20.0) for x in g2 for y in g2]
    pts += [(30.0, 30.0, 30.0)] * 15                      # coincident knot
    pts += [(35.0, 5.0, 35.0)]                            # lonely
    pts += [(0.1, 10.0, 10.0), (L - 0.3, 10.0, 10.0), (0.0, 12.0, 12.0),
            (float(np.nextafter(np.float32(L), np.float32(0))), 12.0, 12.0)]
    pts += [(0.2 + 0.5 * i, 33.0, 3.0) for i in range(12)]  # chain across nothing
    pts += [(L - 0.2 - 0.5 * i, 33.0, 3.0) for i in range(12)]  # wraps to the chain
    pos = np.array(pts, np.float32)
    rng = np.random.default_rng(99)
    vel = rng.normal(0, 300, pos.shape).astype(np.float32)
    w = synth.Workload(name="lattice_ties", pos=pos, vel=vel,
                       ids=np.arange(len(pos), dtype=np.uint64), lo=(0.0,) * 3, hi=(L,) * 3,
                       linklength=ll, boundary=3.0, nphalomin=10.0, periodic=True, cells=8,
                       meta={"seed": 99})
    return w


def cases():
    out = []
    w = synth.config2(seed=1003, scale=6000 / 256 ** 3)
    w.name = "box_f32_periodic"
    out.append(w)
    w = synth.config1(seed=1001, scale=6000 / 64 ** 3)
    w.name = "box_f64_periodic"
    out.append(w)
    w = synth.config2(seed=1005, scale=5000 / 256 ** 3)
    w.name = "box_f32_nonperiodic"
    w.periodic = False
    pos = w.pos.astype(np.float64)
    pos[::5] -= 0.6 * w.boundary
    pos[::61] += 4 * w.boundary
    w.pos = pos.astype(np.float32)
    out.append(w)
    w = synth.config5(seed=1007, scale=6000 / 1024 ** 3)
    w.name = "box_f32_min20"
    out.append(w)
    # many small halos: 80 clumps over 9000 particles in a sparser box
    w = synth.make_box(9000, 160.0, 80, 1009, boundary=6.0, name="box_f32_manyhalos")
    out.append(w)
    out.append(lattice_ties())
    return out


def run_reference(w):
    src, ppos, st = cpu.build_proc(w)
    pvel = w.vel[src].astype(ppos.dtype)
    halos, dt = reference.run_proc(w, ppos, pvel, w.ids[src], timeout=600)
    return halos, dt, st


def main():
    if not reference.available("cmh_ref_f32"):
        reference.build()
    for w in cases():
        halos, dt, st = run_reference(w)
        ids = [np.unique(h["ids"]) for h in halos]
        first = np.array([int(h["ids"][0]) for h in halos], np.uint64)
        props = np.array([h["props"] for h in halos], np.float32).reshape(-1, 19)
        offs = np.cumsum([0] + [len(x) for x in ids]).astype(np.int64)
        params = {"lo": list(w.lo), "hi": list(w.hi), "linklength": w.linklength,
                  "boundary": w.boundary, "nphalomin": w.nphalomin,
                  "periodic": bool(w.periodic), "cells": w.cells,
                  "meta": {k: (float(v) if isinstance(v, (float, np.floating)) else v)
                           for k, v in w.meta.items()},
                  "reference_seconds": dt, "proc_stats": st}
        path = os.path.join(HERE, f"{w.name}.npz")
        np.savez_compressed(path, pos=w.pos, vel=w.vel, ids=w.ids,
                            params=np.array(json.dumps(params)), ref_props=props,
                            ref_ids=np.concatenate(ids) if ids else np.zeros(0, np.uint64),
                            ref_offsets=offs, ref_first_id=first)
        print(f"{w.name}: n={w.n} proc={st['n_proc']} halos={len(halos)} "
              f"ref {dt:.2f}s -> {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
