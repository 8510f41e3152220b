"""Load the golden fixtures of tests/golden (made by make_golden.py)."""
import glob
import json
import os

import numpy as np

from cm_halofinder_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    """The reference-binary fixtures (not the full-size oracle summaries)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("fullsize_"))


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


# ---- full-size fixtures (made by golden/make_fullsize.py) -----------------

def _mix64(x):
    """SplitMix64's output mix of uint64 values (Steele, Lea & Flood 2014)."""
    z = np.asarray(x, np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def member_digests(member, nh):
    """Per halo: the number of input particles mapped to it and the sum
    (mod 2^64) of the mixed indices of those particles -- a hash of the
    halo's member-ID set that does not depend on member order."""
    member = np.asarray(member)
    idx = np.nonzero(member >= 0)[0]
    h = member[idx]
    counts = np.bincount(h, minlength=nh).astype(np.int64)
    sums = np.zeros(nh, np.uint64)
    np.add.at(sums, h, _mix64(idx.astype(np.uint64)))
    return counts, sums


def input_digest(*arrays):
    """SHA-256 of the arrays' bytes: the regenerated input must be the one
    the fixture was made from."""
    import hashlib
    d = hashlib.sha256()
    for a in arrays:
        d.update(np.ascontiguousarray(a).tobytes())
    return d.hexdigest()


def load_fullsize(name):
    z = np.load(os.path.join(GOLDEN, f"fullsize_{name}.npz"))
    return {k: z[k] for k in z.files}
