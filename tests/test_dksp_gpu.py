"""Distributed linear solve on the device (osr_dksp_*, driven by
osiris_b200.slabs.solve_slabs).

* One slab owning the whole grid: the staged iteration performs the
  single-grid solve's arithmetic, so its solution, outcome and iteration
  count equal osr_grid_ksp_solve's bit for bit.
* The same through Slab.ksp_solve on a one-rank NCCL group (the sums are an
  NCCL all-reduce on the launching stream).
* 2 and 3 slabs of the grid (each its own device grid: owned layers plus
  ghosts, state cut from the single grid, its own residual and Jacobian)
  held in one process and stepped in lockstep (dksp_cpu.LocalComm adds the
  slabs' sums and copies ghost layers): the owned rows of the solution match
  the single-grid solution within 1e-8 of its largest entry, with the same
  outcome and an iteration count within two.  No kernel waits on another
  rank here."""
import os

import numpy as np
import pytest

import osiris_b200 as osr
from dksp_cpu import LocalComm
from osiris_b200 import deck, slabs

pytestmark = pytest.mark.gpu

CASES = {
    "twophase_10MPa_cdif0": lambda: deck.config_deck(nx=6, ny=5, nz=7, cdif=0.0, ipress=1e7, seed=3, wells=False),
    "oil_20MPa_diffusion": lambda: deck.config_deck(nx=5, ny=4, nz=6, cdif=None, wells=False, seed=4),
}
T = 3600.0
FIELDS = ("sat", "x", "y", "z", "label", "rho")
OPTS = dict(rtol=1e-12, max_it=2000)


def _single(name, tmp_path, dev):
    import torch
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    d = deck.parse_deck(path)
    G = osr.Grid(d)
    G.initialize(dev)
    rows, pcoeff = G.layout()
    x0 = torch.zeros(rows, dtype=torch.float64, device=dev)
    G.init_guess(x0)
    xp = x0.cpu().numpy() * (1 + 1e-3 * np.random.default_rng(2).uniform(-1, 1, rows))
    f = torch.zeros(rows, dtype=torch.float64, device=dev)
    G.form_function(torch.tensor(xp, device=dev), f, T)
    J = G.alloc_jacobian(dev)
    assert G.jacobian(J, T) == 0
    return d, G, rows, pcoeff, xp, f, J


@pytest.mark.parametrize("name", list(CASES))
def test_one_slab_equals_single_grid_solve(name, tmp_path, cuda_device):
    import torch
    d, G, rows, _, _, f, J = _single(name, tmp_path, cuda_device)
    x_ref = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    info_ref = G.ksp_solve(J, f, x_ref, **OPTS)
    part = slabs.SlabSolve(G, d.nx, d.ny, 0, d.nz, 0, d.nz)
    x = torch.full((rows,), float("nan"), dtype=torch.float64, device=cuda_device)
    part.begin(J, f, x, **OPTS)
    info = slabs.solve_slabs([part], LocalComm())
    part.close()
    assert info_ref["reason"] in (2, 3) and info_ref["its"] > 5, info_ref
    assert info == info_ref
    assert torch.equal(x, x_ref)


def test_slab_solve_single_rank_nccl(tmp_path, cuda_device):
    import socket

    import torch
    import torch.distributed as dist
    name = "twophase_10MPa_cdif0"
    d, G, rows, _, xp, _, _ = _single(name, tmp_path, cuda_device)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=cuda_device)
    try:
        S = slabs.Slab(d, 0, 1)
        S.grid.initialize(cuda_device)
        assert S.refresh_layout(cuda_device) == rows
        JS = S.grid.alloc_jacobian(cuda_device)
        fs = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
        S.grid.form_function(torch.tensor(xp, device=cuda_device), fs, T)
        assert S.grid.jacobian(JS, T) == 0
        x_ref = torch.zeros_like(fs)
        info_ref = S.grid.ksp_solve(JS, fs, x_ref, **OPTS)
        xs = torch.full_like(fs, float("nan"))
        info = S.ksp_solve(JS, fs, xs, **OPTS)
        torch.cuda.synchronize()
        assert info_ref["reason"] in (2, 3) and info_ref["its"] > 5, info_ref
        assert info == info_ref
        assert torch.equal(xs, x_ref)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", list(CASES))
def test_lockstep_slabs_match_single_grid(name, world, tmp_path, cuda_device):
    import torch
    d, G, rows, pcoeff, xp, f, J = _single(name, tmp_path, cuda_device)
    x_ref = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    info_ref = G.ksp_solve(J, f, x_ref, **OPTS)
    state = {f"{m}.{k}": G.get(f"{m}.{k}") for m in "mf" for k in FIELDS + ("P",)}
    gro = G.row_offsets()
    n, nxy = G.cells, d.nx * d.ny
    parts, maps, keep = [], [], []
    for z0, z1 in slabs.slab_ranges(d.nz, world):
        lo, hi = slabs.ghost_range(d.nz, z0, z1)
        S = osr.Grid(slabs.sub_deck(d, lo, hi))
        a, b = lo * nxy, hi * nxy
        for mi, m in enumerate("mf"):
            cut = {k: state[f"{m}.{k}"][..., a:b] for k in FIELDS + ("P",)}
            S.set_state(mi, cut["P"][1], cut["sat"], cut["x"], cut["y"], cut["z"], cut["label"], cut["rho"])
            S.set_pressures(mi, cut["P"])
        lrows, _ = S.refresh_layout()
        S.set_controls(d.dt, pcoeff)
        lro = S.row_offsets()
        xl = np.concatenate([xp[gro[m * n + a]:gro[m * n + b]] for m in (0, 1)])
        fl = torch.zeros(lrows, dtype=torch.float64, device=cuda_device)
        S.form_function(torch.tensor(xl, device=cuda_device), fl, T)
        JS = S.alloc_jacobian(cuda_device)
        assert S.jacobian(JS, T) == 0
        part = slabs.SlabSolve(S, d.nx, d.ny, z0, z1, lo, hi)
        xs = torch.zeros(lrows, dtype=torch.float64, device=cuda_device)
        part.begin(JS, fl, xs, **OPTS)
        parts.append(part)
        nl = S.cells
        own = [(int(lro[m * nl + (z0 - lo) * nxy]), int(lro[m * nl + (z1 - lo) * nxy])) for m in (0, 1)]
        glob = [(int(gro[m * n + z0 * nxy]), int(gro[m * n + z1 * nxy])) for m in (0, 1)]
        maps.append((xs, own, glob))
        keep.append((S, JS, fl))
    info = slabs.solve_slabs(parts, LocalComm())
    torch.cuda.synchronize()
    x = np.full(rows, np.nan)
    for xs, own, glob in maps:
        xh = xs.cpu().numpy()
        for (la, lb), (ga, gb) in zip(own, glob):
            assert lb - la == gb - ga
            x[ga:gb] = xh[la:lb]
    for p in parts:
        p.close()
    xr = x_ref.cpu().numpy()
    assert info["reason"] == info_ref["reason"] and abs(info["its"] - info_ref["its"]) <= 2, (info, info_ref)
    err = np.abs(x - xr).max() / np.abs(xr).max()
    print(f"{name} world {world}: its {info['its']} (single grid {info_ref['its']}), max error {err:.2e}")
    assert err <= 1e-8
