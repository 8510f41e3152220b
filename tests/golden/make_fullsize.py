"""Generate the full-size fixtures: the oracle run once, on the CPU, over
exactly the workloads that bench.py times.

    python tests/golden/make_fullsize.py [c1 c2 c3 c4 c5s]

The oracle (oracle/fof_oracle.c) is the CPU restatement of the reference's
FoF pinned to the reference binaries by tests/test_oracle_pin.py and
tests/test_oracle_live_pin.py.  At these sizes it is too slow for a test
run (the 256^3 box takes about a minute on 8 cores, the others a few), so
its results are committed here as compact summaries:

* the workload's parameters and a SHA-256 of the regenerated input arrays,
* the run's counts (kept, images, processed, groups, candidates, halos),
* per halo in catalog order: its head (lowest processing index), the first
  seven record entries (n, mean position, mean velocity) as float32, and
  the count and order-independent hash of its member-ID set
  (golden_io.member_digests; IDs are input indices).

Workloads (the bench's seeds): c1 = synth.config1(seed=1), the 64^3 box
with FP64 positions; c2 = synth.config2(seed=2), the 256^3 box of the
headline number; c3 = synth.config3(seed=3), the 50M-particle lightcone
with a variable linking length; c4 = synth.config4(seed=4), the 64 boxes of
the batched run (summaries concatenated, with per-box offsets); c5s =
synth.config5(seed=5, scale=1/8), the 1024^3 box's parameters (density,
clump density, Nphalomin 20) over one eighth of its volume: 134M particles
in L = 1000 (the full box is drawn on the GPU by the bench and is beyond
this oracle's memory here).
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cm_halofinder_b200 import synth  # noqa: E402
from oracle import cpu  # noqa: E402
from tests import golden_io  # noqa: E402

WORKLOADS = {
    "c1": lambda: [synth.config1(seed=1)],
    "c2": lambda: [synth.config2(seed=2)],
    "c3": lambda: [synth.config3(seed=3)],
    "c4": lambda: synth.config4(seed=4),
    "c5s": lambda: [synth.config5(seed=5, scale=1 / 8)],
}

STAT_KEYS = ("n_in", "n_out", "n_images", "n_proc", "n_groups", "n_candidates", "nhalos")


def params_of(w):
    p = {"name": w.name, "n": w.n, "lo": list(w.lo), "hi": list(w.hi),
         "linklength": w.linklength, "boundary": w.boundary, "nphalomin": w.nphalomin,
         "periodic": bool(w.periodic), "cells": w.cells,
         "pos_dtype": str(w.pos.dtype), "meta": {k: v for k, v in w.meta.items()
                                                 if isinstance(v, (int, float, str))}}
    if getattr(w, "varlink", None):
        p["varlink"] = {"origin": list(w.varlink["origin"]), "rmax": w.varlink["rmax"],
                        "table_sha256": golden_io.input_digest(w.varlink["table"])}
    return p


def summarise(name):
    boxes = WORKLOADS[name]()
    heads, recs, cnts, hashes, offs, stats, params, digests = [], [], [], [], [0], [], [], []
    t0 = time.time()
    for w in boxes:
        out = cpu.run(w)
        nh = out["stats"]["nhalos"]
        c, h = golden_io.member_digests(out["member"], nh)
        heads.append(out["halo_head"].astype(np.uint32))
        recs.append(out["halo_props"][:, :7].astype(np.float32))
        cnts.append(c)
        hashes.append(h)
        offs.append(offs[-1] + nh)
        stats.append([out["stats"][k] for k in STAT_KEYS])
        params.append(params_of(w))
        digests.append(golden_io.input_digest(w.pos, w.vel))
    dt = time.time() - t0
    np.savez_compressed(
        os.path.join(HERE, f"fullsize_{name}.npz"),
        params=np.array(json.dumps(params)), input_sha256=np.array(digests),
        stat_keys=np.array(STAT_KEYS), stats=np.array(stats, np.int64),
        box_offsets=np.array(offs, np.int64), head=np.concatenate(heads),
        record=np.concatenate(recs), member_count=np.concatenate(cnts),
        member_hash=np.concatenate(hashes))
    print(f"{name}: {len(boxes)} box(es), {sum(s[0] for s in stats)} particles, "
          f"{offs[-1]} halos, oracle {dt:.0f} s", flush=True)


if __name__ == "__main__":
    for name in sys.argv[1:] or list(WORKLOADS):
        summarise(name)
