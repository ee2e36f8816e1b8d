"""z-slab decomposition of one lattice over several ranks (devices or processes).

Rank r owns the planes k0 + 1 .. k0 + nk of the global lattice (`split`: n cut
as evenly as possible, the lower ranks one plane more) as a library-owned AB
Lattice of extents (l, m, nk).  Its z faces at the cuts read the entering
populations from its halo planes as stored (bgk_lattice_set_zhalo), so after
every step the ranks exchange face planes:

  * the 5 populations with c_z = +1 of plane nk go to the upper neighbour's
    plane 0 (its nodes at k = 1 pull them),
  * the 5 populations with c_z = -1 of plane 1 go to the lower neighbour's
    plane nk + 1.

The periodic case wraps z from the last rank to the first; with walls in z
(driven cavity, channel) the outer faces keep the case's rule (bounce-back,
lid).  Every node then computes exactly what it computes in the undivided
lattice, so the assembled state is bit-identical to it (tested on one GPU
with all slabs in one process).  Per step each cut moves 2 x 5 planes of
nx * ny values; a plane is one contiguous region of a population array, so
the exchange sends and receives in place, with no packing.

Transports: `DistTransport` (torch.distributed point-to-point: NCCL between
GPUs over NVLink, gloo between CPU processes) and `LocalTransport` (all slabs
in one process, device-to-device copies).

The reference runs on one GPU; this decomposition has no counterpart there.
It serves lattices larger than one device's memory.
"""
from __future__ import annotations

from . import fields as F

UP = [d for d in range(18) if F.CZ[d] == 1]      # populations that cross a cut upwards
DOWN = [d for d in range(18) if F.CZ[d] == -1]   # ... and downwards


def split(n: int, parts: int):
    """[(k0, nk)] per rank: planes k0 + 1 .. k0 + nk of 1..n."""
    if parts < 1 or n < parts:
        raise ValueError(f"cannot split {n} planes over {parts} ranks")
    base, extra = divmod(n, parts)
    out, k0 = [], 0
    for r in range(parts):
        nk = base + (1 if r < extra else 0)
        out.append((k0, nk))
        k0 += nk
    return out


def neighbours(rank: int, size: int, periodic_z: bool):
    """(lower, upper) neighbour ranks; None where the slab face is the lattice's own z face."""
    if size == 1:
        return None, None
    lower = rank - 1 if rank > 0 else (size - 1 if periodic_z else None)
    upper = rank + 1 if rank < size - 1 else (0 if periodic_z else None)
    return lower, upper


def zhalo_flags(rank: int, size: int, periodic_z: bool) -> int:
    lower, upper = neighbours(rank, size, periodic_z)
    return (1 if lower is not None else 0) | (2 if upper is not None else 0)


def exchange_plan(nk: int, lower, upper):
    """The face planes one rank sends and receives after a step, as
    (op, population, plane, peer, tag) with op 'send' or 'recv'.  Between any
    two ranks the sends of one and the receives of the other come in the same
    order (NCCL matches point-to-point operations by order, gloo by tag)."""
    plan = []
    for d in UP:
        if upper is not None:
            plan.append(("send", d, nk, upper, d))
        if lower is not None:
            plan.append(("recv", d, 0, lower, d))
    for d in DOWN:
        if lower is not None:
            plan.append(("send", d, 1, lower, 32 + d))
        if upper is not None:
            plan.append(("recv", d, nk + 1, upper, 32 + d))
    return plan


class DistTransport:
    """Face-plane exchange over torch.distributed (one slab per process)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group

    def exchange(self, slab) -> None:
        dist = self.dist
        ops = []
        for op, d, k, peer, tag in exchange_plan(slab.nk, slab.lower, slab.upper):
            fn = dist.isend if op == "send" else dist.irecv
            ops.append(dist.P2POp(fn, slab.plane(d, k), peer, group=self.group, tag=tag))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


class LocalTransport:
    """Face-plane exchange between slabs held by one process (device copies
    on the current stream, after every slab's step was launched)."""

    def exchange_all(self, slabs) -> None:
        by_rank = {s.rank: s for s in slabs}
        for s in slabs:
            for op, d, k, peer, _ in exchange_plan(s.nk, s.lower, s.upper):
                if op != "send":
                    continue
                dst = by_rank[peer]
                k_dst = 0 if d in UP else dst.nk + 1
                dst.plane(d, k_dst).copy_(s.plane(d, k))


class Slab:
    """One rank's slab of an (l, m, n) lattice: a Lattice of extents
    (l, m, nk) with halo-reading faces at its cuts."""

    def __init__(self, rank: int, size: int, l: int, m: int, n: int, bcase: str = "periodic", **lattice_kw):
        from .lattice import Lattice
        if bcase in ("inflow", 3):
            raise ValueError("z slabs do not support the inflow case")
        if lattice_kw.get("pattern", "ab") not in ("ab", 0):
            raise ValueError("z slabs need the AB pattern")
        self.rank, self.size = rank, size
        self.l, self.m, self.n = l, m, n
        self.k0, self.nk = split(n, size)[rank]
        periodic_z = bcase in ("periodic", 1)
        self.lower, self.upper = neighbours(rank, size, periodic_z)
        self.lat = Lattice(l, m, self.nk, bcase=bcase, **lattice_kw)
        self.lat.set_zhalo(zhalo_flags(rank, size, periodic_z))

    def plane(self, pop: int, k: int):
        return self.lat.plane(pop, k)

    def upload_global(self, state) -> None:
        """This slab's planes of a global state (19, n+2, m+2, l+2) in the
        reference layout; the halo planes are filled by the next exchange."""
        self.lat.upload(state[:, self.k0:self.k0 + self.nk + 2])

    def download_interior(self):
        """(19, nk, m, l) interior of the current state."""
        st = self.lat.download()
        return st[:, 1:self.nk + 1, 1:self.m + 1, 1:self.l + 1]

    def close(self) -> None:
        self.lat.close()


class SlabLattice:
    """The distributed lattice as one rank sees it: its slab, the exchange
    after every step, and FP64 moments summed over the ranks in rank order."""

    def __init__(self, l: int, m: int, n: int, bcase: str = "periodic", group=None, **lattice_kw):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        rank = dist.get_rank(group) if dist.is_initialized() else 0
        size = dist.get_world_size(group) if dist.is_initialized() else 1
        self.slab = Slab(rank, size, l, m, n, bcase=bcase, **lattice_kw)
        self.transport = DistTransport(group) if size > 1 else None

    def exchange(self) -> None:
        if self.transport is not None:
            self.transport.exchange(self.slab)

    def upload_global(self, state) -> None:
        self.slab.upload_global(state)
        self.exchange()

    def step(self, nsteps: int = 1) -> None:
        for _ in range(int(nsteps)):
            self.slab.lat.step(1)
            self.exchange()

    def moments(self):
        """Global FP64 sums (rho, u_x, u_y, u_z, 0.5 |u|^2): each rank's sums,
        gathered and added in rank order (the same bits on every rank)."""
        import numpy as np
        import torch
        local = torch.tensor(self.slab.lat.moments(), dtype=torch.float64)
        if self.transport is None:
            return local.numpy()
        dev = torch.device("cuda", torch.cuda.current_device()) if self.dist.get_backend(self.group) == "nccl" \
            else torch.device("cpu")
        parts = [torch.zeros(5, dtype=torch.float64, device=dev) for _ in range(self.dist.get_world_size(self.group))]
        self.dist.all_gather(parts, local.to(dev), group=self.group)
        total = np.zeros(5)
        for p in parts:
            total = total + p.cpu().numpy()
        return total

    def close(self) -> None:
        self.slab.close()
