"""Distributed linear solve over z-slabs (osiris_b200.slabs.solve_slabs), CPU
only: gloo ranks (world sizes 2 and 3) each iterate on their slab of a
block-structured system (variable block sizes from one-phase and two-phase
labels, 7-point coupling plus the other continuum, like the Newton
Jacobian), summing the dot products over the ranks and refreshing the
search vectors' ghost layers.  The owned rows of every rank's solution must
equal the one-rank solution of the whole system within 1e-10 of its largest
entry, with the same outcome and iteration count within one.  Every slab's
stage arithmetic is the CPU restatement in dksp_cpu.py, so what is checked
here is the driver and its collectives; the device stages are checked
against the single-grid device solve in test_dksp_gpu.py."""
import os
import socket

import numpy as np
import pytest
import scipy.sparse as sp
import torch.multiprocessing as tmp

from dksp_cpu import CpuPart, LocalComm
from osiris_b200 import slabs

NX, NY, NZ, NC = 3, 3, 6, 3


def _labels():
    return np.random.default_rng(7).choice([-1, 0, 1], size=2 * NX * NY * NZ)


def _sizes(lab):
    return np.where(lab == 0, 2 * NC + 4, NC + 3)


def _neighbours(b):
    n, nxy = NX * NY * NZ, NX * NY
    m, c = divmod(b, n)
    ix, iy, iz = c % NX, (c // NX) % NY, c // nxy
    out = [(1 - m) * n + c]
    for d, ok in ((-1, ix > 0), (1, ix < NX - 1), (-NX, iy > 0), (NX, iy < NY - 1), (-nxy, iz > 0),
                  (nxy, iz < NZ - 1)):
        if ok:
            out.append(b + d)
    return out


def _system():
    """Global matrix (CSR), right-hand side and block row offsets."""
    rng = np.random.default_rng(11)
    lab = _labels()
    size = _sizes(lab)
    off = np.concatenate([[0], np.cumsum(size)])
    rows = int(off[-1])
    R, C, V = [], [], []
    for b in range(len(lab)):
        o0, o1 = off[b], off[b + 1]
        coupl = 0.0
        for nb in _neighbours(b):
            blk = rng.uniform(-1, 1, (o1 - o0, size[nb])) * 0.35
            coupl += np.abs(blk).sum(axis=1)
            rr, cc = np.meshgrid(np.arange(o0, o1), np.arange(off[nb], off[nb + 1]), indexing="ij")
            R.append(rr.ravel()), C.append(cc.ravel()), V.append(blk.ravel())
        own = rng.uniform(-1, 1, (o1 - o0, o1 - o0))
        own[np.diag_indices(o1 - o0)] = np.abs(own).sum(axis=1) + 0.05 * coupl + 0.1
        rr, cc = np.meshgrid(np.arange(o0, o1), np.arange(o0, o1), indexing="ij")
        R.append(rr.ravel()), C.append(cc.ravel()), V.append(own.ravel())
    A = sp.csr_matrix((np.concatenate(V), (np.concatenate(R), np.concatenate(C))), shape=(rows, rows))
    b = rng.uniform(-1, 1, rows)
    return A, b, off, lab


def _local(world, rank):
    """Rank's CpuPart (its slab: owned layers plus ghosts; ghost block rows
    are identity rows) and the global rows of its owned rows."""
    A, b, off, lab = _system()
    n, nxy = NX * NY * NZ, NX * NY
    z0, z1 = slabs.slab_ranges(NZ, world)[rank]
    lo, hi = slabs.ghost_range(NZ, z0, z1)
    gblocks = [m * n + c for m in (0, 1) for c in range(lo * nxy, hi * nxy)]
    lsize = _sizes(lab[gblocks])
    loff = np.concatenate([[0], np.cumsum(lsize)])
    grow = np.concatenate([np.arange(off[g], off[g + 1]) for g in gblocks])
    gmap = -np.ones(int(off[-1]), np.int64)
    gmap[grow] = np.arange(len(grow))
    owned_b = slabs.owned_blocks(NX, NY, hi - lo, z0, z1, lo)
    owned = np.zeros(len(gblocks), bool)
    for b0, b1 in owned_b:
        owned[b0:b1] = True
    Ac = A.tocoo()
    lr, lc = gmap[Ac.row], gmap[Ac.col]
    keep = (lr >= 0) & (lc >= 0)
    keep &= owned[np.searchsorted(loff, np.maximum(lr, 0), side="right") - 1]
    rows = int(loff[-1])
    ghost_rows = np.concatenate([np.arange(loff[i], loff[i + 1]) for i in range(len(gblocks)) if not owned[i]]
                                + [np.zeros(0, np.int64)])
    Al = sp.csr_matrix((np.concatenate([Ac.data[keep], np.ones(len(ghost_rows))]),
                        (np.concatenate([lr[keep], ghost_rows]), np.concatenate([lc[keep], ghost_rows]))),
                       shape=(rows, rows))
    bl = np.where(np.isin(np.arange(rows), ghost_rows), 0.0, b[grow])
    part = CpuPart(Al, loff, [owned_b[0][0], owned_b[0][1], owned_b[1][0], owned_b[1][1]], NX, NY, hi - lo,
                   z0 > lo, z1 < hi)
    own_rows = np.concatenate([np.arange(loff[b0], loff[b1]) for b0, b1 in owned_b])
    return part, bl, grow[own_rows], own_rows


def _one_rank():
    part, bl, grows, own_rows = _local(1, 0)
    part.begin(bl)
    info = slabs.solve_slabs([part], LocalComm(), check_every=4)
    x = np.zeros(int(_system()[2][-1]))
    x[grows] = part.x[own_rows]
    return x, info


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        part, bl, grows, own_rows = _local(world, rank)
        part.begin(bl)
        info = slabs.solve_slabs([part], slabs.RankComm(rank), check_every=4)
        out[rank] = (grows.tolist(), part.x[own_rows].tolist(), info)
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_one_rank_solves_the_system():
    A, b, _, _ = _system()
    x, info = _one_rank()
    assert info["reason"] in (2, 3), info
    assert np.abs(A @ x - b).max() <= 1e-9 * np.abs(b).max()


def test_lockstep_slabs_match_one_rank():
    """The slabs of 2 and 3 ranks held in one process (LocalComm)."""
    x1, info1 = _one_rank()
    for world in (2, 3):
        parts, maps = [], []
        for rank in range(world):
            part, bl, grows, own_rows = _local(world, rank)
            part.begin(bl)
            parts.append(part)
            maps.append((grows, own_rows))
        info = slabs.solve_slabs(parts, LocalComm(), check_every=4)
        x = np.zeros_like(x1)
        for part, (grows, own_rows) in zip(parts, maps):
            x[grows] = part.x[own_rows]
        assert info["reason"] == info1["reason"] and abs(info["its"] - info1["its"]) <= 1, (info, info1)
        assert np.abs(x - x1).max() <= 1e-10 * np.abs(x1).max()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_match_one_rank(world):
    x1, info1 = _one_rank()
    ctx = tmp.get_context("spawn")
    out = ctx.Manager().dict()
    tmp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    x = np.zeros_like(x1)
    infos = []
    for r in range(world):
        grows, vals, info = out[r]
        x[np.asarray(grows)] = vals
        infos.append(info)
    assert all(i == infos[0] for i in infos), infos          # every rank took the same steps
    assert infos[0]["reason"] == info1["reason"] and abs(infos[0]["its"] - info1["its"]) <= 1, (infos[0], info1)
    assert np.abs(x - x1).max() <= 1e-10 * np.abs(x1).max()
