"""Load the golden fixtures of tests/golden (made by make_golden.py)."""
import glob
import json
import os

import numpy as np

from cm_halofinder_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = json.loads(str(z["params"]))
    w = synth.Workload(name=name, pos=z["pos"], vel=z["vel"], ids=z["ids"], lo=tuple(p["lo"]),
                       hi=tuple(p["hi"]), linklength=p["linklength"], boundary=p["boundary"],
                       nphalomin=p["nphalomin"], periodic=p["periodic"], cells=p["cells"],
                       meta=p.get("meta", {}))
    offs = z["ref_offsets"]
    ref_sets = [z["ref_ids"][offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]
    return w, {"props": z["ref_props"], "sets": ref_sets, "first_id": z["ref_first_id"],
               "params": p}


def sets_from_member(member, ids, nh):
    """Member ID set of each halo (catalog order) from a per-particle map."""
    out = [[] for _ in range(nh)]
    for i in np.nonzero(member >= 0)[0]:
        out[member[i]].append(ids[i])
    return [np.unique(np.array(s, np.uint64)) for s in out]
