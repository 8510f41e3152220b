"""One box split over ranks, the way the reference's MPI run splits it.

The box [Lmin, Lmax] is cut into Nx x Ny x Nz domains, one per rank
(startup.c:33-47): rank = Nx Ny iz + Nx iy + ix, rmin = i (L / N) + Lmin and
rmax = rmin + L / N per axis, each padded by Boundarysize.  Every particle
goes to the rank that owns it and, as a ghost, to the ranks whose padded
domain it lies in (read_data.c:409-521):

* particles outside the box (periodic) or outside the padded box (isolated)
  are dropped and counted;
* the owner per axis is floor(N ((x - Lmin) / L)) (isolated: -1 -> 0), with
  N -> N - 1;
* per axis the neighbour is floor(N ((x - Lmin + k b) / L)) for k = -1 then
  +1 when it differs from the owner (the later one wins; isolated: none past
  the box), and the particle goes to every combination of its neighbour
  axes;
* a copy that crosses a periodic face (neighbour index wrapped from N to 0
  or from -1 to N - 1) is shifted by -L or +L, computed in double and stored
  in the position type: the image rule of the single-box run
  (read_data.c:785-797 gives the same values for Lmin = 0).  Where an axis is
  not split (N = 1), the neighbour across a periodic face is the rank itself
  and the copy is that image; the reference's receive-side wrap, which only
  moves coordinates outside the receiving rank's padded domain, would keep it
  unshifted there.

Each rank then runs the isolated FoF of its padded domain and keeps the
halos whose centre of mass lies in [rmin, rmax) (Checkhalo, FOF.c:378-430):
with Boundarysize above the largest halo extent, the union of the ranks'
catalogs is the single-box catalog.  The exchange is one all-to-all of the
copies (counts first), over NCCL for CUDA tensors or gloo for CPU tensors;
routing is torch arithmetic in float64 on the tensors' own device.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class SlabSplit:
    """The domains of a box split over Nx * Ny * Nz ranks."""

    lo: tuple
    hi: tuple
    split: tuple            # (Nx, Ny, Nz)
    boundary: float
    periodic: bool = True

    @property
    def nranks(self) -> int:
        return int(self.split[0] * self.split[1] * self.split[2])

    def coords(self, rank: int) -> tuple:
        nx, ny, _ = self.split
        iz = rank // (nx * ny)
        iy = (rank - nx * ny * iz) // nx
        ix = rank - nx * iy - nx * ny * iz
        return ix, iy, iz

    def domain(self, rank: int) -> tuple:
        """(rmin, rmax) of a rank, in the reference's double arithmetic."""
        idx = self.coords(rank)
        rmin, rmax = [], []
        for a in range(3):
            w = (float(self.hi[a]) - float(self.lo[a])) / float(self.split[a])
            r0 = idx[a] * w + float(self.lo[a])
            rmin.append(r0)
            rmax.append(r0 + w)
        return tuple(rmin), tuple(rmax)

    def route(self, pos):
        """Copies of the particles: (source index, destination rank, shift per
        axis in units of L) as torch tensors on pos's device, and the number
        of particles dropped outside the box."""
        import torch
        dev = pos.device
        x = pos.to(torch.float64)
        lo = torch.tensor([float(v) for v in self.lo], dtype=torch.float64, device=dev)
        hi = torch.tensor([float(v) for v in self.hi], dtype=torch.float64, device=dev)
        L = hi - lo
        N = torch.tensor(list(self.split), dtype=torch.int64, device=dev)
        Nd = N.to(torch.float64)
        b = float(self.boundary)
        if self.periodic:
            inside = ((x >= lo) & (x <= hi)).all(dim=1)
        else:
            inside = ((x >= lo - b) & (x <= hi + b)).all(dim=1)
        src = torch.nonzero(inside).flatten()
        n_out = int(x.shape[0] - src.numel())
        x = x[src]
        own = torch.floor(Nd * ((x - lo) / L)).to(torch.int64)
        if not self.periodic:
            own = torch.where(own < 0, own + 1, own)
        own = torch.where(own >= N, own - 1, own)
        sub = torch.zeros_like(own)
        for k in (-1, 1):
            nb = torch.floor(Nd * (((x - lo) + k * b) / L)).to(torch.int64)
            take = nb != own
            if not self.periodic:
                take &= (nb >= 0) & (nb < N)
            sub = torch.where(take, torch.full_like(sub, k), sub)
        srcs, dests, shifts = [], [], []
        for combo in range(8):  # bit a: move along axis a to the neighbour
            use = torch.tensor([(combo >> a) & 1 for a in range(3)], dtype=torch.int64,
                               device=dev)
            ok = ((sub != 0) | (use == 0)).all(dim=1)
            step = sub * use
            cell = own + step
            shift = torch.zeros_like(cell)
            if self.periodic:
                shift = torch.where(cell >= N, -torch.ones_like(cell), shift)
                shift = torch.where(cell < 0, torch.ones_like(cell), shift)
                cell = torch.where(cell >= N, cell - N, cell)
                cell = torch.where(cell < 0, cell + N, cell)
            rank = N[0] * N[1] * cell[:, 2] + N[0] * cell[:, 1] + cell[:, 0]
            srcs.append(src[ok])
            dests.append(rank[ok])
            shifts.append(shift[ok])
        return torch.cat(srcs), torch.cat(dests), torch.cat(shifts), n_out

    def copy_positions(self, pos, src, shift):
        """Positions of the copies: x + shift L in double, stored in pos's type."""
        import torch
        lo = torch.tensor([float(v) for v in self.lo], dtype=torch.float64, device=pos.device)
        hi = torch.tensor([float(v) for v in self.hi], dtype=torch.float64, device=pos.device)
        L = hi - lo
        x = pos[src]
        moved = x.to(torch.float64) + shift.to(torch.float64) * L
        return torch.where(shift != 0, moved.to(pos.dtype), x)

    def local_copies(self, pos, vel, ids, rank):
        """Without a process group: the copies one rank receives from all the
        particles (every rank's share at once), in the order of an exchange
        from a single sender."""
        src, dest, shift, _ = self.route(pos)
        sel = dest == rank
        s, sh = src[sel], shift[sel]
        return self.copy_positions(pos, s, sh), vel[s], ids[s]


def exchange(dist, split: SlabSplit, pos, vel, ids):
    """All-to-all of the copies over the process group: each rank routes the
    particles it holds and receives its own domain's particles and ghosts
    (senders in rank order, each sender's copies in its particle order): one
    exchange of the counts, then one of the copies packed as rows of bytes.
    pos / vel are (n, 3) tensors, ids (n,) int64; all on one device (CUDA
    for NCCL, CPU for gloo).  Returns the received (pos, vel, ids) and the
    particles this rank dropped outside the box."""
    import torch
    world = dist.get_world_size()
    if world != split.nranks:
        raise ValueError(f"the split has {split.nranks} domains for {world} ranks")
    src, dest, shift, n_out = split.route(pos)
    order = torch.argsort(dest, stable=True)
    src, dest, shift = src[order], dest[order], shift[order]
    send = torch.bincount(dest, minlength=world).to(torch.int64)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send)
    sc, rc = send.tolist(), recv.tolist()
    m = int(sum(rc))
    # one exchange of packed rows (position, velocity, ID bytes side by side)
    # instead of one per array
    parts = [split.copy_positions(pos, src, shift), vel[src], ids[src].reshape(-1, 1)]
    widths = [a.shape[1] * a.element_size() for a in parts]
    rows = torch.cat([a.contiguous().view(torch.uint8).reshape(a.shape[0], w)
                      for a, w in zip(parts, widths)], dim=1)
    got = torch.empty((m, rows.shape[1]), dtype=torch.uint8, device=rows.device)
    dist.all_to_all_single(got, rows, rc, sc)
    out, c = [], 0
    for a, w in zip(parts, widths):
        out.append(got[:, c:c + w].contiguous().view(a.dtype).reshape((m,) + tuple(a.shape[1:])))
        c += w
    return out[0], out[1], out[2].reshape(m), n_out


def local_config(split: SlabSplit, rank: int, linklength: float, nphalomin: float,
                 precision: str = "fp32", properties: int = 0):
    """The FoF configuration of one rank's domain: isolated, padded by
    Boundarysize, owning the halos whose centre of mass lies in it."""
    from . import FofConfig
    rmin, rmax = split.domain(rank)
    return FofConfig(lo=rmin, hi=rmax, boundary=float(split.boundary),
                     linklength=float(linklength), nphalomin=float(nphalomin), periodic=False,
                     precision=precision, properties=properties)


def halo_id_sets(member: np.ndarray, ids: np.ndarray, nhalos: int) -> list:
    """Member ID sets of a catalog, halo by halo (member: halo index per
    particle, -1 outside)."""
    member = np.asarray(member)
    ids = np.asarray(ids)
    order = np.argsort(member, kind="stable")
    m = member[order]
    starts = np.searchsorted(m, np.arange(nhalos))
    ends = np.searchsorted(m, np.arange(nhalos), side="right")
    return [frozenset(ids[order[s:e]].tolist()) for s, e in zip(starts, ends)]
