"""z-slab decomposition of the Newton-step residual across ranks.

The reference runs MPI ranks over contiguous ranges of its global rows and
gives every rank the whole unknown vector (UpdateAll's VecScatterCreateToAll,
compsim/PetscAUX.cpp:186-198). Here each rank holds one slab of z layers
plus one ghost layer on each side that has a neighbour, as its own device
grid:

* ``slab_ranges`` splits the layers evenly; ``sub_deck`` cuts a deck to a
  slab with its ghosts (per-cell arrays by layer, DK by layer; block heights
  are recomputed from the slab's own bottom, so height differences, which is
  all gravity uses, are unchanged);
* before every residual evaluation each rank receives the unknowns of its
  ghost layers from the neighbouring ranks (``exchange_ghost_unknowns``:
  point-to-point sends of one layer of unknowns, both continua, over
  ``torch.distributed`` -- NCCL between GPUs, gloo between CPU processes),
  then unpacks and evaluates its whole local grid; properties of ghost cells
  are recomputed locally from the exchanged unknowns;
* PCoeff, the unknowns' pressure scale, is the maximum over all ranks
  (``torch.distributed.all_reduce`` with MAX);
* the rows of the owned layers are the rank's part of the global residual
  (``owned_blocks``); ghost rows are discarded (their outer faces are
  missing).

Decks with wells are not split: a rate-controlled well distributes its rate
over all its completions, which would couple slabs.
"""
from __future__ import annotations

import copy

import numpy as np


def slab_ranges(nz: int, ranks: int):
    """Owned layer ranges [z0, z1) of each rank (contiguous, sizes differing
    by at most one)."""
    if ranks < 1 or ranks > nz:
        raise ValueError("need 1 <= ranks <= nz")
    cuts = [nz * r // ranks for r in range(ranks + 1)]
    return [(cuts[r], cuts[r + 1]) for r in range(ranks)]


def ghost_range(nz: int, z0: int, z1: int):
    """Layers [lo, hi) a slab's grid holds: its own plus one ghost layer on
    each side that has a neighbour."""
    return max(z0 - 1, 0), min(z1 + 1, nz)


def sub_deck(d, lo: int, hi: int):
    """The deck restricted to layers [lo, hi)."""
    if d.wells_i is not None and len(d.wells_i):
        raise ValueError("decks with wells are not split into slabs")
    s = copy.copy(d)
    nxy = d.nx * d.ny
    a, b = lo * nxy, hi * nxy
    s.nz = hi - lo
    s.dk = np.array(d.dk[lo:hi], dtype=float)
    for k in ("tor", "por", "fpor", "p0", "fp0", "sw0", "fsw0"):
        v = getattr(d, k)
        if v is not None:
            setattr(s, k, np.array(np.asarray(v)[..., a:b]))
    for k in ("perm", "fperm", "z0", "fz0"):
        v = getattr(d, k)
        if v is not None:
            setattr(s, k, np.array(np.asarray(v)[:, a:b]))
    return s


def owned_blocks(nx: int, ny: int, nz_local: int, z0: int, z1: int, lo: int):
    """(local, global-layer) block index ranges of the owned layers: for each
    continuum, local blocks [m n_loc + (z0-lo) nxy, m n_loc + (z1-lo) nxy)."""
    nxy = nx * ny
    n_loc = nxy * nz_local
    return [(m * n_loc + (z0 - lo) * nxy, m * n_loc + (z1 - lo) * nxy) for m in (0, 1)]


def layer_rows(rowoff_local, nx: int, ny: int, nz_local: int, layer: int):
    """Row ranges [(r0, r1)] of one local layer, matrix then fracture."""
    nxy = nx * ny
    n_loc = nxy * nz_local
    return [(int(rowoff_local[m * n_loc + layer * nxy]), int(rowoff_local[m * n_loc + (layer + 1) * nxy]))
            for m in (0, 1)]


def exchange_ghost_unknowns(x_local, rowoff_local, nx: int, ny: int, nz_local: int, has_lower: bool,
                            has_upper: bool, rank: int, group=None):
    """Fill the ghost layers' unknowns of x_local (a torch tensor in the
    local row layout) from the neighbouring ranks: the first owned layer goes
    to rank - 1 (its upper ghost), the last owned layer to rank + 1 (its lower
    ghost).  Row counts of the ghost layers follow the local labels, which the
    ranks keep equal by exchanging state at every layout change."""
    import torch
    import torch.distributed as dist
    ops = []
    lo_g = 1 if has_lower else 0
    last_owned = nz_local - 1 - (1 if has_upper else 0)

    def rows_of(layer):
        return [(a, b) for a, b in layer_rows(rowoff_local, nx, ny, nz_local, layer)]

    def pack(layer):
        return torch.cat([x_local[a:b] for a, b in rows_of(layer)])

    recv = {}
    if has_lower:
        send_down = pack(lo_g)
        ghost = rows_of(0)
        recv["lower"] = torch.empty(sum(b - a for a, b in ghost), dtype=x_local.dtype, device=x_local.device)
        ops += [dist.P2POp(dist.isend, send_down, rank - 1, group),
                dist.P2POp(dist.irecv, recv["lower"], rank - 1, group)]
    if has_upper:
        send_up = pack(last_owned)
        ghost = rows_of(nz_local - 1)
        recv["upper"] = torch.empty(sum(b - a for a, b in ghost), dtype=x_local.dtype, device=x_local.device)
        ops += [dist.P2POp(dist.isend, send_up, rank + 1, group),
                dist.P2POp(dist.irecv, recv["upper"], rank + 1, group)]
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    for side, layer in (("lower", 0), ("upper", nz_local - 1)):
        if side in recv:
            off = 0
            for a, b in rows_of(layer):
                x_local[a:b] = recv[side][off:off + (b - a)]
                off += b - a
    return x_local


def global_pcoeff(local_pcoeff: float, group=None, device=None) -> float:
    """PCoeff over all ranks (CalcPCoeff's maximum, compsim/Init_Calcs.cpp:
    1118-1130)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([local_pcoeff], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


class Slab:
    """One rank's part of a z-slab run: its device grid (owned layers plus
    ghosts), the ghost exchange and the global PCoeff around the residual."""

    def __init__(self, d, rank: int, world: int, group=None):
        from . import Grid
        self.deck, self.rank, self.world, self.group = d, rank, world, group
        self.z0, self.z1 = slab_ranges(d.nz, world)[rank]
        self.lo, self.hi = ghost_range(d.nz, self.z0, self.z1)
        self.grid = Grid(sub_deck(d, self.lo, self.hi))
        self._rowoff = None

    def refresh_layout(self, device=None):
        """Row layout of the current labels and the global PCoeff (every rank
        calls it at the same point)."""
        rows, pc = self.grid.refresh_layout()
        self.grid.set_controls(self.deck.dt, global_pcoeff(pc, self.group, device))
        self._rowoff = self.grid.row_offsets()
        return rows

    def owned_rows(self):
        """Local row ranges of the owned layers, matrix then fracture."""
        nl = self.grid.cells
        nxy = self.deck.nx * self.deck.ny
        return [(int(self._rowoff[m * nl + (self.z0 - self.lo) * nxy]),
                 int(self._rowoff[m * nl + (self.z1 - self.lo) * nxy])) for m in (0, 1)]

    def frac_start(self) -> int:
        """First local row of the fracture continuum."""
        return int(self._rowoff[self.grid.cells])

    def global_offsets(self, device=None):
        """This rank's global row offsets per continuum (an all-gather of the
        ranks' owned row counts)."""
        import torch
        import torch.distributed as dist
        own = self.owned_rows()
        mine = torch.tensor([own[0][1] - own[0][0], own[1][1] - own[1][0]], dtype=torch.int64, device=device)
        every = [torch.zeros_like(mine) for _ in range(self.world)]
        dist.all_gather(every, mine, group=self.group)
        return global_offsets([tuple(t.tolist()) for t in every], self.rank)

    def jacobian_coo_global(self, vals, offsets):
        """(rows, cols, values) of the owned rows of the local Jacobian values
        in the global numbering, the triplets a multi-rank PETSc matrix takes
        (MatSetValuesCOO with global indices)."""
        r, c, v = self.grid.jacobian_coo(vals)
        own = self.owned_rows()
        keep = ((r >= own[0][0]) & (r < own[0][1])) | ((r >= own[1][0]) & (r < own[1][1]))
        fs = self.frac_start()
        return (to_global(r[keep], fs, own, offsets), to_global(c[keep], fs, own, offsets), v[keep])

    def form_function(self, x_local, f_local, sim_time: float):
        """Exchange the ghost layers' unknowns, then UpdateAll + residual on
        the whole local grid; the owned rows of f_local are this rank's part."""
        exchange_ghost_unknowns(x_local, self._rowoff, self.deck.nx, self.deck.ny, self.hi - self.lo,
                                self.z0 > 0, self.z1 < self.deck.nz, self.rank, self.group)
        self.grid.form_function(x_local, f_local, sim_time)


def global_offsets(owned_counts, rank: int):
    """Global row offset of a rank's first owned row in each continuum, from
    every rank's owned row counts [(matrix, fracture)] in rank order: the
    global numbering holds all matrix rows (rank by rank) before all fracture
    rows."""
    owned_counts = [tuple(int(v) for v in c) for c in owned_counts]
    all_matrix = sum(c[0] for c in owned_counts)
    before = [sum(c[m] for c in owned_counts[:rank]) for m in (0, 1)]
    return before[0], all_matrix + before[1]


def to_global(idx, frac_start: int, owned_local, offsets):
    """Global row indices of local row indices idx.  Within one continuum a
    slab's rows -- lower ghost layer, owned layers, upper ghost layer -- are
    consecutive in the global numbering, so each continuum maps by one shift:
    the distance between the rank's first owned row there, locally and
    globally.  frac_start: the first local fracture row; owned_local: the
    local owned row ranges (Slab.owned_rows); offsets: global_offsets."""
    idx = np.asarray(idx)
    return np.where(idx >= frac_start, idx + (offsets[1] - owned_local[1][0]),
                    idx + (offsets[0] - owned_local[0][0]))
