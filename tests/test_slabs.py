"""z-slab decomposition (osiris_b200/slabs.py), CPU only: layer ranges,
sub-decks, and the ghost-layer exchange of unknowns between gloo ranks
(world sizes 2 and 3, variable block sizes from one-phase and two-phase
labels): after the exchange every rank's local vector is the global vector
restricted to its layers, ghosts included."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

from osiris_b200 import deck, slabs

NX, NY, NZ, NC = 3, 2, 7, 3


def _layout(labels):
    sizes = np.where(labels == 0, 2 * NC + 4, NC + 3)
    return np.concatenate([[0], np.cumsum(sizes)])


def _labels():
    rng = np.random.default_rng(1)
    return rng.choice([-1, 0, 1], size=2 * NX * NY * NZ)   # matrix blocks, then fracture blocks


def _local_labels(lab, lo, hi):
    n, nxy = NX * NY * NZ, NX * NY
    return np.concatenate([lab[lo * nxy:hi * nxy], lab[n + lo * nxy:n + hi * nxy]])


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lab = _labels()
    gro = _layout(lab)
    xg = np.arange(gro[-1], dtype=float) + 0.5
    z0, z1 = slabs.slab_ranges(NZ, world)[rank]
    lo, hi = slabs.ghost_range(NZ, z0, z1)
    nzl = hi - lo
    lro = _layout(_local_labels(lab, lo, hi))
    nxy, n = NX * NY, NX * NY * NZ
    # the global rows of every local block, matrix then fracture
    want = np.concatenate([xg[gro[m * n + lo * nxy]:gro[m * n + hi * nxy]] for m in (0, 1)])
    x = torch.full((lro[-1],), float("nan"), dtype=torch.float64)
    for (a, b) in [(lro[m * nzl * nxy + (z0 - lo) * nxy], lro[m * nzl * nxy + (z1 - lo) * nxy]) for m in (0, 1)]:
        x[a:b] = torch.from_numpy(want[a:b])
    slabs.exchange_ghost_unknowns(x, lro, NX, NY, nzl, z0 > 0, z1 < NZ, rank)
    out[rank] = bool(np.array_equal(x.numpy(), want))
    pc = slabs.global_pcoeff(float(rank + 1))
    out[world + rank] = pc == float(world)
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_ghost_exchange_and_pcoeff(world):
    ctx = tmp.get_context("spawn")
    out = ctx.Manager().dict()
    tmp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert all(out[r] for r in range(world)), dict(out)
    assert all(out[world + r] for r in range(world)), dict(out)


def test_ranges_and_sub_deck(tmp_path):
    assert slabs.slab_ranges(7, 3) == [(0, 2), (2, 4), (4, 7)]
    assert slabs.ghost_range(7, 2, 4) == (1, 5) and slabs.ghost_range(7, 0, 2) == (0, 3)
    path = os.path.join(str(tmp_path), "d.dat")
    deck.write_deck(path, deck.config_deck(nx=3, ny=2, nz=5, wells=False))
    d = deck.parse_deck(path)
    s = slabs.sub_deck(d, 1, 4)
    nxy = 6
    assert s.nz == 3 and np.array_equal(s.dk, d.dk[1:4])
    assert np.array_equal(s.perm, d.perm[:, nxy:4 * nxy]) and np.array_equal(s.z0, d.z0[:, nxy:4 * nxy])
    assert np.array_equal(s.por, d.por[nxy:4 * nxy])
    # wells are kept with their completed layers cut to the slab and renumbered
    path2 = os.path.join(str(tmp_path), "w.dat")
    spec = deck.config_deck(nx=3, ny=2, nz=5)
    spec["wells"][1][3:5] = [4, 5]                  # producer completed in layers 4..5 (1-based)
    deck.write_deck(path2, spec)
    dw = deck.parse_deck(path2)
    assert dw.wells_i[:, 3:5].tolist() == [[0, 4], [3, 4]]
    sw = slabs.sub_deck(dw, 1, 4)
    assert sw.wells_i[:, 3:5].tolist() == [[0, 2], [2, 2]]
    assert np.array_equal(sw.wells_i[:, :3], dw.wells_i[:, :3]) and np.array_equal(sw.wells_f, dw.wells_f)
    s0 = slabs.sub_deck(dw, 0, 2)
    assert s0.wells_i[:, 3:5].tolist() == [[0, 1], [1, 0]]   # no producer layer here: an empty range
    assert dw.wells_i[:, 3:5].tolist() == [[0, 4], [3, 4]]   # the deck itself is unchanged


def test_global_offsets_and_mapping():
    counts = [(10, 6), (8, 4), (12, 9)]           # owned rows (matrix, fracture) per rank
    assert slabs.global_offsets(counts, 0) == (0, 30)
    assert slabs.global_offsets(counts, 1) == (10, 36)
    assert slabs.global_offsets(counts, 2) == (18, 40)
    # rank 1 with ghost layers: local matrix rows [0, 14) (4 ghost + 8 owned + 2 ghost),
    # local fracture rows [14, 24) (3 ghost + 4 owned + 3 ghost)
    own = [(4, 12), (17, 21)]
    offs = slabs.global_offsets(counts, 1)
    g = slabs.to_global(np.array([0, 4, 11, 13, 14, 17, 20, 23]), 14, own, offs)
    assert g.tolist() == [6, 10, 17, 19, 33, 36, 39, 42]
