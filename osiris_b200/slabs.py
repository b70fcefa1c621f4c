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
  missing);
* the linear solve is distributed the way PETSc distributes KSPBCGS +
  PCVPBJACOBI over MPI ranks: every rank iterates on its slab's Jacobian,
  the dot products are summed over the ranks, and the search vectors' ghost
  layers are refreshed from the neighbours before each matrix-vector product
  (``SlabSolve``, ``solve_slabs``; the device stages are osr_dksp_* of the C
  library, the sums an all-reduce on the launching stream).

Wells go to every slab with their completions cut to the slab's layers. A
rate-controlled (or latched) well splits its rate over all its completions
by sums over its completed layers; each rank takes those sums over its owned
layers (osr_grid_well_sums), the ranks add them (all-reduce) and every slab
evaluates its completions with the totals (osr_grid_set_well_sums), so a
well crossing slabs sees the sums of the whole reservoir.
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
    """The deck restricted to layers [lo, hi).  Every well is kept (the
    ranks hold the same well list), its completed layers cut to [lo, hi) and
    renumbered; a well with none there keeps an empty range (first layer
    after the last)."""
    s = copy.copy(d)
    if d.wells_i is not None and len(d.wells_i):
        wi = np.array(d.wells_i, dtype=np.int64)
        k0, k1 = np.maximum(wi[:, 3], lo) - lo, np.minimum(wi[:, 4], hi - 1) - lo
        empty = k0 > k1
        wi[:, 3] = np.where(empty, 1, k0)
        wi[:, 4] = np.where(empty, 0, k1)
        s.wells_i = wi
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

    def ksp_solve(self, vals, b, x, check_every: int = 8, **opts) -> dict:
        """Distributed solve of the global Newton system: this rank's slab
        Jacobian vals, right-hand side b and solution x in the local row
        layout (ghost rows of x are not set)."""
        part = SlabSolve(self.grid, self.deck.nx, self.deck.ny, self.z0, self.z1, self.lo, self.hi)
        try:
            part.begin(vals, b, x, **opts)
            return solve_slabs([part], RankComm(self.rank, self.group), check_every)
        finally:
            part.close()

    def form_function(self, x_local, f_local, sim_time: float):
        """Exchange the ghost layers' unknowns, then UpdateAll + residual on
        the whole local grid (with the wells' layer sums added over the
        ranks); the owned rows of f_local are this rank's part.  The grid's
        Jacobian evaluated next uses the same sums."""
        exchange_ghost_unknowns(x_local, self._rowoff, self.deck.nx, self.deck.ny, self.hi - self.lo,
                                self.z0 > 0, self.z1 < self.deck.nz, self.rank, self.group)
        self.grid.update_all(x_local)
        self.sum_wells(x_local.device)
        self.grid.residual(f_local, None, sim_time)

    def sum_wells(self, device=None):
        """The wells' layer sums over the owned layers, added over the ranks
        and handed to the grid (no-op without wells)."""
        import torch
        import torch.distributed as dist
        nw = 0 if self.deck.wells_i is None else len(self.deck.wells_i)
        if nw == 0:
            return
        if getattr(self, "_wsums", None) is None or self._wsums.device != torch.device(device):
            self._wsums = torch.zeros((nw, 2, 5), dtype=torch.float64, device=device)
        self.grid.well_sums(self.z0 - self.lo, self.z1 - self.lo, self._wsums)
        dist.all_reduce(self._wsums, op=dist.ReduceOp.SUM, group=self.group)
        self.grid.set_well_sums(self._wsums)


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


class SlabSolve:
    """One slab's part of the distributed linear solve (osr_dksp_*): the
    handle, the search vectors p and s whose ghost rows ``solve_slabs``
    refreshes, and the partial sums ``dots`` it sums over the slabs."""

    def __init__(self, grid, nx: int, ny: int, z0: int, z1: int, lo: int, hi: int):
        import ctypes

        from . import _check, lib
        self.grid, self.nx, self.ny = grid, nx, ny
        self.nz_local = hi - lo
        self.has_lower, self.has_upper = z0 > lo, z1 < hi
        nxy, nl = nx * ny, grid.cells
        self.owned = [(z0 - lo) * nxy, (z1 - lo) * nxy, nl + (z0 - lo) * nxy, nl + (z1 - lo) * nxy]
        h = ctypes.c_void_p()
        _check(lib().osr_dksp_create(grid._h, ctypes.byref(h)), "osr_dksp_create")
        self._h = h
        self.rowoff = None
        self.p = self.s = self.dots = None

    def close(self):
        from . import lib
        if self._h:
            lib().osr_dksp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self, device):
        import torch
        return torch.cuda.current_stream(device).cuda_stream

    def begin(self, vals, b, x, **opts):
        """Set-up of J x = b on this slab from x = 0 (vectors in the slab's
        local row layout, on the device)."""
        import ctypes

        import torch

        from . import _check, _vp, ksp_opts, lib
        self.rowoff = self.grid.row_offsets()
        rows = int(self.rowoff[-1])
        self.p = torch.zeros(rows, dtype=torch.float64, device=x.device)
        self.s = torch.zeros_like(self.p)
        self.dots = torch.zeros(4, dtype=torch.float64, device=x.device)
        self._dev = x.device
        o = ksp_opts(**opts)
        owned = (ctypes.c_long * 4)(*self.owned)
        self._keep = (vals, b, x)
        _check(lib().osr_dksp_begin(self._h, _vp(vals.data_ptr()), _vp(b.data_ptr()), _vp(x.data_ptr()),
                                    _vp(self.p.data_ptr()), _vp(self.s.data_ptr()), owned, ctypes.byref(o),
                                    _vp(self.dots.data_ptr()), _vp(self._stream(self._dev))), "osr_dksp_begin")

    def stage(self, k: int):
        from . import _check, _vp, lib
        _check(lib().osr_dksp_stage(self._h, int(k), _vp(self._stream(self._dev))), "osr_dksp_stage")

    def info(self) -> dict:
        import ctypes

        from . import KspInfo, _check, _vp, lib
        i = KspInfo()
        _check(lib().osr_dksp_info(self._h, ctypes.byref(i), _vp(self._stream(self._dev))), "osr_dksp_info")
        return {"reason": i.reason, "its": i.its, "rnorm0": i.rnorm0, "rnorm": i.rnorm}


class RankComm:
    """The sums and ghost exchanges of ``solve_slabs`` between ranks, over
    ``torch.distributed`` (NCCL between GPUs, gloo between CPU processes);
    each rank passes its one part."""

    def __init__(self, rank: int, group=None):
        self.rank, self.group = rank, group

    def sum(self, parts, k: int):
        import torch.distributed as dist
        dist.all_reduce(parts[0].dots[:k], op=dist.ReduceOp.SUM, group=self.group)

    def exchange(self, parts, name: str):
        q = parts[0]
        exchange_ghost_unknowns(getattr(q, name), q.rowoff, q.nx, q.ny, q.nz_local, q.has_lower, q.has_upper,
                                self.rank, self.group)


# the collective after each stage of one iteration: a sum of k partial sums,
# or a ghost refresh of a search vector
_STAGES = ((1, ("exchange", "p")), (2, ("sum", 1)), (3, ("exchange", "s")), (4, ("sum", 3)), (5, ("sum", 2)),
           (6, None))


def solve_slabs(parts, comm, check_every: int = 8) -> dict:
    """Run the distributed iteration to its end on parts whose ``begin`` was
    called: every stage on every part, then the stage's collective through
    ``comm`` (``sum(parts, k)``, ``exchange(parts, name)``); the state is
    read back every ``check_every`` iterations.  Every rank takes the same
    steps in the same order, so the collectives match across ranks."""
    comm.sum(parts, 1)
    for q in parts:
        q.stage(0)
    while True:
        info = parts[0].info()
        if info["reason"] != 0:
            return info
        for _ in range(max(1, check_every)):
            for k, after in _STAGES:
                for q in parts:
                    q.stage(k)
                if after is not None:
                    getattr(comm, after[0])(parts, after[1])
