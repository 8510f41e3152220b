"""Test-side restatement of the subsample draw and a reader of the files
Subsample (FOF.c:432-544) writes."""
import os
import struct

import numpy as np

M1, M2, M3 = np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB), np.uint64(
    0x9E3779B97F4A7C15)
SEEDMUL = np.uint64(0xD1B54A32D192ED03)


def uniforms(seed, keys):
    """u(seed, key): SplitMix64's output mix of key ^ (seed * C), top 53
    bits times 2^-53 (every product wraps modulo 2^64)."""
    k = np.asarray(keys, np.uint64)
    s = np.uint64(np.int64(seed).astype(np.uint64))
    with np.errstate(over="ignore"):
        z = k ^ (s * SEEDMUL)
        z = z + M3
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def expected_sample(ref, w, samp_in, samp_out, seed, keys, closed):
    """The kept input indices (in, out) from an oracle run: originals
    inside [lo, hi) ([lo, hi] on closed axes), by their group's size."""
    group = ref["group"]
    size = np.bincount(group, minlength=group.max() + 1 if group.size else 1)[group]
    n_kept = ref["stats"]["n_kept"]
    src = ref["proc_src"][:n_kept].astype(np.int64)
    x = ref["proc_pos"][:n_kept].astype(np.float64)
    lo, hi = np.array(w.lo), np.array(w.hi)
    inside = (x >= lo).all(axis=1)
    for a in range(3):
        inside &= (x[:, a] <= hi[a]) if closed[a] else (x[:, a] < hi[a])
    big = ~(size[:n_kept].astype(np.float64) < w.nphalomin)
    u = uniforms(seed, np.asarray(keys, np.uint64)[src])
    keep_in = inside & big & (u < samp_in)
    keep_out = inside & ~big & (u < samp_out)
    return np.sort(src[keep_in]), np.sort(src[keep_out])


def read_unformatted(path, with_id=True):
    """[4][n][4] [len][3n floats][len] [len][3n floats][len] ([len][n u64][len])."""
    data = open(path, "rb").read()
    off = 0

    def rec():
        nonlocal off
        (ln,) = struct.unpack_from("<i", data, off)
        body = data[off + 4: off + 4 + ln]
        (ln2,) = struct.unpack_from("<i", data, off + 4 + ln)
        assert ln2 == ln
        off += 8 + ln
        return body

    (n,) = struct.unpack("<I", rec())
    pos = np.frombuffer(rec(), np.float32).reshape(n, 3)
    vel = np.frombuffer(rec(), np.float32).reshape(n, 3)
    ids = np.frombuffer(rec(), np.uint64) if with_id else None
    assert off == len(data)
    return pos, vel, ids


def exists(path):
    return os.path.exists(path)
