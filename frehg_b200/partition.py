"""One domain over several GPUs: the (i, j) slab decomposition and its halos.

The reference decomposes the grid over (i, j) only -- every rank owns full
z-columns, the coupling and post-allocation unit -- with the block rule
``n_local = N / P + (p < N % P)`` and a one-cell halo in i and j
(``src/core/Grid.hpp:5-8``, ``src/core/Grid.cpp:22-24, 92-140``).  Its
``HaloExchanger`` settles the i-halo columns first and then sends full-width
rows, so the corner cells travel inside the south / north messages
(``src/core/HaloExchanger.cpp:200-262``).  This module restates both over
``torch.distributed`` point-to-point messages, which run over NCCL between
GPUs (CUDA tensors) and over gloo on the host (CPU tensors, as the tests
use it):

* :class:`SlabPartition` -- the process grid (``MPI_Dims_create``'s balanced
  factorisation with the larger count on the larger extent), each rank's
  block, neighbours and global offsets, and the scatter / gather of fields
  in the halo layout ``(ny + 2, nx + 2, nz)``;
* :class:`HaloExchange` -- the two-phase exchange of any number of cell
  fields of one rank, packed into one message per direction (k, the
  unit-stride axis, stays contiguous inside every packed plane).

:mod:`frehg_b200.dcg` builds the distributed predictor solve on them.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

WEST, EAST, SOUTH, NORTH = 0, 1, 2, 3


def block_size(n: int, p: int, r: int) -> int:
    """Cells of block r of n split over p blocks (Grid::blockSize)."""
    return n // p + (1 if r < n % p else 0)


def block_start(n: int, p: int, r: int) -> int:
    """First cell of block r (Grid::blockStart)."""
    return r * (n // p) + min(r, n % p)


def dims_create(size: int) -> tuple:
    """The balanced two-factor split MPI_Dims_create(size, 2) returns: the
    factors as close as possible, the larger first."""
    best = (size, 1)
    for a in range(1, int(size ** 0.5) + 1):
        if size % a == 0:
            best = (size // a, a)
    return best


def choose_grid(nx: int, ny: int, size: int, px: int = 0, py: int = 0) -> tuple:
    """The process grid of Grid::chooseDecomposition: an explicit request
    (both, or one that divides the rank count), else the balanced split with
    the larger count on the larger extent, falling back to the most
    balanced factorisation that leaves no block empty."""
    if px > 0 and py > 0:
        if px * py != size:
            raise ValueError(f"decomposition {px} x {py} needs {px * py} ranks, have {size}")
        return px, py
    if px > 0:
        if size % px:
            raise ValueError(f"mpi_nx = {px} does not divide {size} ranks")
        return px, size // px
    if py > 0:
        if size % py:
            raise ValueError(f"mpi_ny = {py} does not divide {size} ranks")
        return size // py, py
    large, small = dims_create(size)
    px, py = (large, small) if nx >= ny else (small, large)
    if px > nx or py > ny:
        best, score = None, -1
        for cx in range(1, size + 1):
            if size % cx:
                continue
            cy = size // cx
            if cx > nx or cy > ny:
                continue
            s = min(nx // cx, ny // cy)
            if s > score:
                best, score = (cx, cy), s
        if best is None:
            raise ValueError(f"{size} ranks cannot split a {nx} x {ny} grid")
        px, py = best
    return px, py


@dataclass(frozen=True)
class Block:
    rank: int
    pi: int
    pj: int
    i0: int  # first owned global column (0-based interior index)
    j0: int
    nx: int  # owned columns
    ny: int
    neighbor: tuple  # (west, east, south, north) rank or None


class SlabPartition:
    """The (i, j) block decomposition of an nx x ny x nz grid over `size`
    ranks; rank r sits at (r % px, r // px)."""

    def __init__(self, nx: int, ny: int, nz: int, size: int, px: int = 0, py: int = 0):
        self.nx, self.ny, self.nz, self.size = nx, ny, nz, size
        self.px, self.py = choose_grid(nx, ny, size, px, py)
        self.blocks: List[Block] = [self._block(r) for r in range(size)]

    def _block(self, r: int) -> Block:
        px, py = self.px, self.py
        pi, pj = r % px, r // px
        nb = (r - 1 if pi > 0 else None, r + 1 if pi + 1 < px else None,
              r - px if pj > 0 else None, r + px if pj + 1 < py else None)
        return Block(r, pi, pj, block_start(self.nx, px, pi), block_start(self.ny, py, pj),
                     block_size(self.nx, px, pi), block_size(self.ny, py, pj), nb)

    def local_shape(self, rank: int, nz: Optional[int] = None) -> tuple:
        b = self.blocks[rank]
        return (b.ny + 2, b.nx + 2, self.nz if nz is None else nz)

    def local_slice(self, rank: int):
        """Slices of the global halo layout that rank's local halo layout
        (its block plus a one-cell ring) covers."""
        b = self.blocks[rank]
        return slice(b.j0, b.j0 + b.ny + 2), slice(b.i0, b.i0 + b.nx + 2)

    def scatter(self, field: np.ndarray, rank: int) -> np.ndarray:
        """Rank's local field (halo ring included, filled from the global
        field's neighbouring cells or its domain ghosts)."""
        sj, si = self.local_slice(rank)
        return np.ascontiguousarray(field[sj, si])

    def gather(self, locals_: Sequence[np.ndarray]) -> np.ndarray:
        """The global interior from every rank's local interior (ghost ring 0)."""
        shape = (self.ny + 2, self.nx + 2) + tuple(locals_[0].shape[2:])
        out = np.zeros(shape, dtype=locals_[0].dtype)
        for r, a in enumerate(locals_):
            b = self.blocks[r]
            out[1 + b.j0:1 + b.j0 + b.ny, 1 + b.i0:1 + b.i0 + b.nx] = a[1:-1, 1:-1]
        return out

    def edges(self, rank: int) -> Dict[str, bool]:
        """Which sides of the block are the domain's edges (their halos hold
        boundary ghosts, not a neighbour's cells)."""
        nb = self.blocks[rank].neighbor
        return {"west": nb[WEST] is None, "east": nb[EAST] is None,
                "south": nb[SOUTH] is None, "north": nb[NORTH] is None}


class HaloExchange:
    """The two-phase one-cell halo exchange of a rank's cell fields
    (HaloExchanger::exchangeSelected): phase 1 sends the owned edge columns
    west / east and fills the i-halo columns, phase 2 sends full-width rows
    (i-halo included) south / north, so the corner cells arrive with them.
    Fields are torch tensors of the local halo layout (ny + 2, nx + 2, nz),
    all on one device; each direction's planes of every field travel as one
    packed message.  Domain-edge halos are left alone (they hold boundary
    ghosts).  Messages pair opposite directions, as the reference's tags do;
    every rank posts its receives and sends of a phase before waiting."""

    def __init__(self, part: SlabPartition, rank: int, dist, group=None):
        self.part, self.rank, self.dist, self.group = part, rank, dist, group
        self.block = part.blocks[rank]

    @staticmethod
    def _planes(f, side: int, send: bool):
        # owned edge plane (send) or halo plane (receive) of one side
        if side == WEST:
            return f[1:-1, 1 if send else 0]
        if side == EAST:
            return f[1:-1, -2 if send else -1]
        if side == SOUTH:
            return f[1 if send else 0, :]
        return f[-2 if send else -1, :]

    def _phase(self, fields, sides):
        import torch
        reqs, recvs = [], []
        for side in sides:
            peer = self.block.neighbor[side]
            if peer is None:
                continue
            bufs = [self._planes(f, side, True).reshape(-1) for f in fields]
            send = torch.cat(bufs).contiguous()
            recv = torch.empty_like(send)
            reqs.append(self.dist.irecv(recv, src=peer, group=self.group))
            reqs.append(self.dist.isend(send, dst=peer, group=self.group))
            recvs.append((side, recv))
        for q in reqs:
            q.wait()
        for side, recv in recvs:
            off = 0
            for f in fields:
                dst = self._planes(f, side, False)
                n = dst.numel()
                dst.copy_(recv[off:off + n].view_as(dst))
                off += n

    def exchange(self, fields) -> None:
        fields = list(fields)
        self._phase(fields, (WEST, EAST))
        self._phase(fields, (SOUTH, NORTH))
