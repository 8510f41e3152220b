"""Seeded synthetic particle sets for the FoF halo finder.

No public dataset is involved: the reference reads N-body snapshots
(read_data.c:207-404), and the workloads here are seeded stand-ins with the
shapes, sizes and value distributions of the five benchmark configurations:

* a fraction (60 %) of the particles sits in Plummer clumps whose particle
  counts follow dN/dM ~ M^-1.9 on [10, 5000], rescaled (largest-remainder
  rounding) so that the clumps hold exactly that fraction -- the drawn masses
  alone cannot (their mean is ~78), and the factor is recorded in ``meta``;
* the Plummer scale radius is 0.05 * (M / 10)^(1/3) Mpc/h for a clump of M
  particles (after rescaling); radii are r_s / sqrt(u^(-2/3) - 1) with u
  uniform on (0, 0.999]; directions isotropic; centres uniform;
* the rest is a uniform background;
* velocities are Gaussian, sigma = 300 km/s per component, float32;
* IDs are 0..N-1 in array order; the array order is a random permutation.

Everything is drawn from ``numpy.random.default_rng(seed)`` so the arrays are
reproducible from (config, seed, scale).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SIGMA_V = 300.0


@dataclass
class Workload:
    """One box (or lightcone) of particles plus its FoF run parameters."""

    name: str
    pos: np.ndarray            # (N, 3) float32 or float64
    vel: np.ndarray            # (N, 3) float32
    ids: np.ndarray            # (N,) uint64
    lo: tuple                  # box lower corner (Lxmin, Lymin, Lzmin)
    hi: tuple                  # box upper corner
    linklength: float
    boundary: float            # Boundarysize (ghost-shell width)
    nphalomin: float
    periodic: bool
    cells: int                 # Px = Py = Pz of the reference's cell grid
    varlink: dict | None = None
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])


def _clump_masses(rng, n_clumps, target, mmin=10.0, mmax=5000.0, alpha=1.9):
    u = rng.random(n_clumps)
    a1 = 1.0 - alpha
    m = (mmin ** a1 + u * (mmax ** a1 - mmin ** a1)) ** (1.0 / a1)
    scale = target / m.sum()
    ms = m * scale
    base = np.floor(ms).astype(np.int64)
    rem = int(target - base.sum())
    if rem > 0:
        order = np.argsort(-(ms - base), kind="stable")
        base[order[:rem]] += 1
    return base, float(scale)


def _plummer_offsets(rng, counts, rs):
    n = int(counts.sum())
    r_s = np.repeat(rs, counts)
    u = 0.999 * (1.0 - rng.random(n))
    r = r_s / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d * r[:, None]


def make_box(n, L, n_clumps, seed, *, pos_dtype=np.float32, linkb=0.2,
             nphalomin=10, boundary=10.0, clump_frac=0.6, name="box"):
    """Periodic box of side L with n particles and n_clumps Plummer clumps."""
    rng = np.random.default_rng(seed)
    target = int(round(clump_frac * n))
    n_clumps = max(int(n_clumps), 1)
    counts, scale = _clump_masses(rng, n_clumps, target)
    rs = 0.05 * np.cbrt(np.maximum(counts, 1) / 10.0)
    centres = rng.random((n_clumps, 3)) * L
    cl = np.repeat(centres, counts, axis=0) + _plummer_offsets(rng, counts, rs)
    bg = rng.random((n - target, 3)) * L
    pos = np.concatenate([cl, bg], axis=0)
    pos = np.mod(pos, L)
    pos = pos.astype(pos_dtype)
    pos[pos >= pos_dtype(L)] = 0          # float rounding of L - tiny
    perm = rng.permutation(n)
    pos = np.ascontiguousarray(pos[perm])
    vel = rng.normal(0.0, SIGMA_V, (n, 3)).astype(np.float32)
    ids = np.arange(n, dtype=np.uint64)
    sep = L / n ** (1.0 / 3.0)
    cells = max(int(round(n ** (1.0 / 3.0))), 1)
    return Workload(name=name, pos=pos, vel=vel, ids=ids, lo=(0.0, 0.0, 0.0),
                    hi=(float(L),) * 3, linklength=linkb * sep,
                    boundary=float(boundary), nphalomin=float(nphalomin),
                    periodic=True, cells=cells,
                    meta={"seed": seed, "n_clumps": n_clumps,
                          "mass_scale": scale, "largest_clump": int(counts.max()),
                          "mean_separation": sep, "linkb": linkb})


def lightcone_linklength_table(n_total, R, n_tab=4097, linkb=0.2, ratio=3.0):
    """l(r) = linkb * nbar(r)^(-1/3) for nbar falling linearly by `ratio`
    from r = 0 to r = R, normalised to n_total particles in the sphere."""
    c = (1.0 - 1.0 / ratio) / R            # nbar(r) = n0 (1 - c r)
    # N = 4 pi n0 (R^3/3 - c R^4/4)
    n0 = n_total / (4.0 * math.pi * (R ** 3 / 3.0 - c * R ** 4 / 4.0))
    r = np.linspace(0.0, R, n_tab)
    nbar = n0 * (1.0 - c * r)
    return r, linkb * nbar ** (-1.0 / 3.0), n0, c


def make_lightcone(n, R, n_clumps, seed, *, boundary=5.0, cells=None,
                   nphalomin=10, clump_frac=0.6, name="lightcone"):
    """Sphere of radius R around the observer at the origin; nbar(r) falls
    linearly by 3x from r = 0 to R; variable linking length l(r)."""
    rng = np.random.default_rng(seed)
    r_tab, l_tab, n0, c = lightcone_linklength_table(n, R)

    def radii(k):
        # pdf ~ r^2 (1 - c r) on [0, R]: inverse CDF on a fine grid
        g = np.linspace(0.0, R, 1 << 16)
        cdf = g ** 3 / 3.0 - c * g ** 4 / 4.0
        cdf /= cdf[-1]
        return np.interp(rng.random(k), cdf, g)

    def directions(k):
        d = rng.standard_normal((k, 3))
        return d / np.linalg.norm(d, axis=1, keepdims=True)

    target = int(round(clump_frac * n))
    counts, scale = _clump_masses(rng, max(int(n_clumps), 1), target)
    rs = 0.05 * np.cbrt(np.maximum(counts, 1) / 10.0)
    centres = directions(len(counts)) * radii(len(counts))[:, None]
    cl = np.repeat(centres, counts, axis=0) + _plummer_offsets(rng, counts, rs)
    bg = directions(n - target) * radii(n - target)[:, None]
    pos = np.concatenate([cl, bg], axis=0)
    # keep the shell: clump members thrown outside r = R are clipped onto it
    rr = np.linalg.norm(pos, axis=1)
    out = rr > R
    pos[out] *= (R / rr[out])[:, None] * (1.0 - 1e-7)
    pos = pos.astype(np.float32)
    perm = rng.permutation(n)
    pos = np.ascontiguousarray(pos[perm])
    vel = rng.normal(0.0, SIGMA_V, (n, 3)).astype(np.float32)
    ids = np.arange(n, dtype=np.uint64)
    lmax = float(l_tab.max())
    if cells is None:
        cells = max(int((2 * R + 2 * boundary) / (4.0 * lmax)), 1)
    return Workload(name=name, pos=pos, vel=vel, ids=ids, lo=(-R,) * 3,
                    hi=(R,) * 3, linklength=lmax, boundary=float(boundary),
                    nphalomin=float(nphalomin), periodic=False, cells=cells,
                    varlink={"origin": (0.0, 0.0, 0.0), "rmax": float(R),
                             "table": np.ascontiguousarray(l_tab, np.float64)},
                    meta={"seed": seed, "n_clumps": int(n_clumps),
                          "mass_scale": scale, "n0": n0})


# ---------------------------------------------------------------------------
# The five benchmark configurations (full size at scale = 1).
# ---------------------------------------------------------------------------

def config1(seed=1, scale=1.0):
    """Periodic L=250, N=64^3, FP64 positions, 1,500 clumps, min 10."""
    n = max(int(round(64 ** 3 * scale)), 64)
    L = 250.0 * (n / 64 ** 3) ** (1.0 / 3.0)
    return make_box(n, L, round(1500 * n / 64 ** 3), seed, pos_dtype=np.float64,
                    boundary=8.0, name="c1_box64")


def config2(seed=2, scale=1.0):
    """Periodic L=1000, N=256^3, FP32 positions, 10,000 clumps, min 10."""
    n = max(int(round(256 ** 3 * scale)), 64)
    L = 1000.0 * (n / 256 ** 3) ** (1.0 / 3.0)
    return make_box(n, L, round(10000 * n / 256 ** 3), seed, boundary=10.0,
                    name="c2_box256")


def config3(seed=3, scale=1.0):
    """Lightcone, N=50M in a sphere of radius 1400, variable linking length."""
    n = max(int(round(50_000_000 * scale)), 64)
    R = 1400.0 * (n / 50_000_000) ** (1.0 / 3.0)
    # clump count at the C2 clump density (10^4 per 256^3 particles)
    return make_lightcone(n, R, round(10000 * n / 256 ** 3), seed,
                          name="c3_lightcone")


def config4(seed=4, scale=1.0, nbox=64):
    """64 independent periodic boxes, N log-uniform in [1e4, 4e6] (scaled),
    constant mean density, linking parameter uniform in [0.15, 0.25]."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(1e4), math.log(4e6), nbox)) * scale
    bs = rng.uniform(0.15, 0.25, nbox)
    boxes = []
    for i in range(nbox):
        n = max(int(round(ns[i])), 64)
        L = 1000.0 * (n / 256 ** 3) ** (1.0 / 3.0)
        boxes.append(make_box(n, L, max(round(10000 * n / 256 ** 3), 1),
                              seed * 1000 + i, linkb=float(bs[i]), boundary=8.0,
                              name=f"c4_box{i}"))
    return boxes


def config5(seed=5, scale=1.0):
    """Periodic L=2000, N=1024^3, FP32, 500,000 clumps, min 20 (CPU, numpy:
    only for down-scaled use; the full size is generated on the device)."""
    n = max(int(round(1024 ** 3 * scale)), 64)
    L = 2000.0 * (n / 1024 ** 3) ** (1.0 / 3.0)
    w = make_box(n, L, round(500000 * n / 1024 ** 3), seed, nphalomin=20,
                 boundary=10.0, name="c5_box1024")
    return w


def make_box_device(n, L, n_clumps, seed, *, device=0, linkb=0.2, nphalomin=10,
                    boundary=10.0, clump_frac=0.6, name="box", chunk=1 << 26):
    """make_box() drawn on a CUDA device with torch (same distributions, its
    own random stream), for sizes whose host generation would take minutes:
    positions float32, velocities float32, both torch tensors on `device`.
    Clump members and background are drawn in chunks of `chunk` particles;
    the array order is then a random permutation, as on the host."""
    import torch

    dev = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
    rng = np.random.default_rng(seed)
    target = int(round(clump_frac * n))
    n_clumps = max(int(n_clumps), 1)
    counts, scale = _clump_masses(rng, n_clumps, target)
    rs = 0.05 * np.cbrt(np.maximum(counts, 1) / 10.0)
    centres = rng.random((n_clumps, 3)) * L
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    cum = torch.from_numpy(np.cumsum(counts)).to(dev)
    rs_t = torch.from_numpy(rs).to(dev)
    cen_t = torch.from_numpy(centres).to(dev)
    pos = torch.empty((n, 3), dtype=torch.float32, device=dev)
    Lf = torch.tensor(L, dtype=torch.float32).item()

    def store(s, p):
        p = torch.remainder(p, L).to(torch.float32)
        p[p >= Lf] = 0.0                      # float rounding of L - tiny
        pos[s:s + p.shape[0]] = p

    for s in range(0, target, chunk):
        e = min(s + chunk, target)
        idx = torch.arange(s, e, device=dev)
        cl = torch.searchsorted(cum, idx, right=True)
        u = 0.999 * (1.0 - torch.rand(e - s, generator=g, device=dev, dtype=torch.float64))
        r = rs_t[cl] / torch.sqrt(u ** (-2.0 / 3.0) - 1.0)
        d = torch.randn((e - s, 3), generator=g, device=dev, dtype=torch.float64)
        d /= torch.linalg.norm(d, dim=1, keepdim=True)
        store(s, cen_t[cl] + d * r[:, None])
        del idx, cl, u, r, d
    for s in range(target, n, chunk):
        e = min(s + chunk, n)
        store(s, torch.rand((e - s, 3), generator=g, device=dev, dtype=torch.float64) * L)
    perm = torch.randperm(n, generator=g, device=dev)
    pos = pos[perm]
    del perm
    vel = torch.randn((n, 3), generator=g, device=dev, dtype=torch.float32) * SIGMA_V
    torch.cuda.empty_cache()
    sep = L / n ** (1.0 / 3.0)
    return DeviceWorkload(name=name, pos=pos, vel=vel, lo=(0.0, 0.0, 0.0), hi=(float(L),) * 3,
                          linklength=linkb * sep, boundary=float(boundary),
                          nphalomin=float(nphalomin), periodic=True,
                          cells=max(int(round(n ** (1.0 / 3.0))), 1),
                          meta={"seed": seed, "n_clumps": n_clumps, "mass_scale": scale,
                                "largest_clump": int(counts.max()), "mean_separation": sep,
                                "linkb": linkb, "generated_on": str(dev)})


@dataclass
class DeviceWorkload:
    """A Workload whose pos / vel are torch tensors on a CUDA device."""

    name: str
    pos: object
    vel: object
    lo: tuple
    hi: tuple
    linklength: float
    boundary: float
    nphalomin: float
    periodic: bool
    cells: int
    varlink: dict | None = None
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    def to_host(self) -> Workload:
        """The same particles as a host Workload (for checks at small sizes)."""
        import numpy as _np
        pos = self.pos.cpu().numpy()
        return Workload(name=self.name, pos=pos, vel=self.vel.cpu().numpy(),
                        ids=_np.arange(pos.shape[0], dtype=_np.uint64), lo=self.lo,
                        hi=self.hi, linklength=self.linklength, boundary=self.boundary,
                        nphalomin=self.nphalomin, periodic=self.periodic, cells=self.cells,
                        varlink=self.varlink, meta=dict(self.meta))


def config5_device(seed=5, scale=1.0, device=0):
    """config5 at full size (1024^3 = 1.07e9 particles, 25.8 GB of float32
    positions and velocities) generated on the device."""
    n = max(int(round(1024 ** 3 * scale)), 64)
    L = 2000.0 * (n / 1024 ** 3) ** (1.0 / 3.0)
    return make_box_device(n, L, round(500000 * n / 1024 ** 3), seed, device=device,
                           nphalomin=20, boundary=10.0, name="c5_box1024")
