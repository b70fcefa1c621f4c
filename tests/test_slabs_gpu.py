"""z-slab residual on one GPU: the slabs of a 2- and 3-rank decomposition
are evaluated one after another (each its own device grid: owned layers plus
ghost layers, PCoeff of the whole grid, its unknowns gathered from the global
vector as the ghost exchange delivers them); the rows of every slab's owned
layers must equal the single-grid residual's rows within 1e-12 of each row's
absolute term sum.  No kernel waits on another rank here."""
import os

import numpy as np
import pytest

import osiris_b200 as osr
from osiris_b200 import deck, slabs

pytestmark = pytest.mark.gpu

CASES = {
    "twophase_10MPa_cdif0": lambda: deck.config_deck(nx=6, ny=5, nz=7, cdif=0.0, ipress=1e7, seed=3, wells=False),
    "oil_20MPa_diffusion": lambda: deck.config_deck(nx=5, ny=4, nz=6, cdif=None, wells=False, seed=4),
}
T = 3600.0
FIELDS = ("sat", "x", "y", "z", "label", "rho")


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", list(CASES))
def test_slab_residual_rows_match_single_grid(name, world, tmp_path, cuda_device):
    import torch
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    d = deck.parse_deck(path)
    G = osr.Grid(d)
    G.initialize(cuda_device)
    rows, pcoeff = G.layout()
    state = {f"{m}.{k}": G.get(f"{m}.{k}") for m in "mf" for k in FIELDS + ("P",)}
    x0 = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    G.init_guess(x0)
    xp = x0.cpu().numpy() * (1 + 1e-3 * np.random.default_rng(2).uniform(-1, 1, rows))
    f = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    scale = torch.zeros_like(f)
    G.form_function(torch.tensor(xp, device=cuda_device), f, T)
    G.residual(f, scale, T)
    f, scale = f.cpu().numpy(), scale.cpu().numpy()
    gro = G.row_offsets()
    n, nxy = G.cells, d.nx * d.ny
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
        assert len(xl) == lrows
        fl = torch.zeros(lrows, dtype=torch.float64, device=cuda_device)
        S.form_function(torch.tensor(xl, device=cuda_device), fl, T)
        fl = fl.cpu().numpy()
        nl = S.cells
        for m in (0, 1):
            ga, gb = gro[m * n + z0 * nxy], gro[m * n + z1 * nxy]
            la, lb = lro[m * nl + (z0 - lo) * nxy], lro[m * nl + (z1 - lo) * nxy]
            assert gb - ga == lb - la
            err = np.abs(fl[la:lb] - f[ga:gb])
            bad = err > 1e-12 * scale[ga:gb] + 1e-300
            assert not bad.any(), (z0, z1, m, int(bad.sum()), float((err / (scale[ga:gb] + 1e-300)).max()))


def test_slab_wrapper_single_rank_nccl(tmp_path, cuda_device):
    """The Slab wrapper on a one-rank NCCL group (no neighbours, PCoeff
    through the all-reduce) gives the single grid's residual exactly."""
    import socket

    import torch
    import torch.distributed as dist
    path = os.path.join(str(tmp_path), "d.dat")
    deck.write_deck(path, CASES["twophase_10MPa_cdif0"]())
    d = deck.parse_deck(path)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=cuda_device)
    try:
        G = osr.Grid(d)
        G.initialize(cuda_device)
        rows, _ = G.layout()
        x = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
        G.init_guess(x)
        f = torch.zeros_like(x)
        S = slabs.Slab(d, 0, 1)
        S.grid.initialize(cuda_device)
        assert S.refresh_layout(cuda_device) == rows
        fl = torch.zeros_like(x)
        G.form_function(x.clone(), f, T)
        S.form_function(x.clone(), fl, T)
        torch.cuda.synchronize()
        assert S.owned_rows()[0][0] == 0 and S.owned_rows()[1][1] == rows
        assert torch.equal(f, fl)
        offs = S.global_offsets(cuda_device)
        assert offs == (0, S.frac_start())
        J = G.alloc_jacobian(cuda_device)
        assert G.jacobian(J, T) == 0
        JS = S.grid.alloc_jacobian(cuda_device)
        assert S.grid.jacobian(JS, T) == 0
        r, c, v = S.jacobian_coo_global(JS, offs)
        rg, cg, vg = G.jacobian_coo(J)
        assert np.array_equal(r, rg) and np.array_equal(c, cg) and np.array_equal(v, vg)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", list(CASES))
def test_slab_jacobian_rows_match_single_grid(name, world, tmp_path, cuda_device):
    """The owned rows of every slab's Jacobian, mapped to the global
    numbering (slabs.global_offsets / to_global), rebuild the single grid's
    Jacobian: every entry within 1e-12 of its row's largest."""
    import scipy.sparse as sp
    import torch
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    d = deck.parse_deck(path)
    G = osr.Grid(d)
    G.initialize(cuda_device)
    rows, pcoeff = G.layout()
    state = {f"{m}.{k}": G.get(f"{m}.{k}") for m in "mf" for k in FIELDS + ("P",)}
    x0 = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    G.init_guess(x0)
    xp = x0.cpu().numpy() * (1 + 1e-3 * np.random.default_rng(2).uniform(-1, 1, rows))
    f = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    G.form_function(torch.tensor(xp, device=cuda_device), f, T)
    J = G.alloc_jacobian(cuda_device)
    assert G.jacobian(J, T) == 0
    A = sp.csr_matrix((lambda r, c, v: (v, (r, c)))(*G.jacobian_coo(J)), shape=(rows, rows))
    gro = G.row_offsets()
    n, nxy = G.cells, d.nx * d.ny
    parts = []
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
        nl = S.cells
        own = [(int(lro[m * nl + (z0 - lo) * nxy]), int(lro[m * nl + (z1 - lo) * nxy])) for m in (0, 1)]
        parts.append((S, JS, own, int(lro[nl])))
    counts = [(o[0][1] - o[0][0], o[1][1] - o[1][0]) for _, _, o, _ in parts]
    R, C, V = [], [], []
    for rank, (S, JS, own, fs) in enumerate(parts):
        r, c, v = S.jacobian_coo(JS)
        keep = ((r >= own[0][0]) & (r < own[0][1])) | ((r >= own[1][0]) & (r < own[1][1]))
        offs = slabs.global_offsets(counts, rank)
        R.append(slabs.to_global(r[keep], fs, own, offs))
        C.append(slabs.to_global(c[keep], fs, own, offs))
        V.append(v[keep])
    B = sp.csr_matrix((np.concatenate(V), (np.concatenate(R), np.concatenate(C))), shape=(rows, rows))
    D = abs(A - B)
    scale = np.maximum(abs(A).max(axis=1).toarray().ravel(), 1e-300)
    worst = (D.max(axis=1).toarray().ravel() / scale).max()
    assert worst <= 1e-12, worst


WELL_CASES = {
    "all_well_types_9MPa": (lambda: deck.all_wells_deck(), False),
    "all_well_types_13MPa_latched": (lambda: deck.all_wells_deck(ipress=13e6, cdif=0.0), True),
    "plain_wells_5x4x6": (lambda: deck.config_deck(nx=5, ny=4, nz=6, ipress=1e7, seed=5), False),
}


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", list(WELL_CASES))
def test_slab_wells_match_single_grid(name, world, tmp_path, cuda_device):
    """Slabs of decks whose wells cross the slab boundaries (every well type,
    rate latches on and off): each slab keeps the wells cut to its layers,
    takes the wells' layer sums over its owned layers, and the slabs' sums
    are added (as the ranks' all-reduce does) and handed back before the
    residual and Jacobian.  The owned rows of every slab's residual match the
    single grid within 1e-12 of each row's absolute term sum, and its
    Jacobian rows rebuild the single grid's within 1e-12 of each row's
    largest entry."""
    import scipy.sparse as sp
    import torch
    make, latched = WELL_CASES[name]
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, make())
    d = deck.parse_deck(path)
    assert len(d.wells_i) > 0
    G = osr.Grid(d)
    G.initialize(cuda_device)
    nw = len(d.wells_i)
    if latched:
        for w in range(nw):
            G.set_well_condition(w, True)
    rows, pcoeff = G.layout()
    state = {f"{m}.{k}": G.get(f"{m}.{k}") for m in "mf" for k in FIELDS + ("P",)}
    x0 = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    G.init_guess(x0)
    xp = x0.cpu().numpy() * (1 + 1e-3 * np.random.default_rng(2).uniform(-1, 1, rows))
    f = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    scale = torch.zeros_like(f)
    G.update_all(torch.tensor(xp, device=cuda_device))
    G.residual(f, scale, T)
    J = G.alloc_jacobian(cuda_device)
    assert G.jacobian(J, T) == 0
    A = sp.csr_matrix((lambda r, c, v: (v, (r, c)))(*G.jacobian_coo(J)), shape=(rows, rows))
    f, scale = f.cpu().numpy(), scale.cpu().numpy()
    gro = G.row_offsets()
    n, nxy = G.cells, d.nx * d.ny
    slabs_ = []
    for z0, z1 in slabs.slab_ranges(d.nz, world):
        lo, hi = slabs.ghost_range(d.nz, z0, z1)
        S = osr.Grid(slabs.sub_deck(d, lo, hi))
        if latched:
            for w in range(nw):
                S.set_well_condition(w, True)
        a, b = lo * nxy, hi * nxy
        for mi, m in enumerate("mf"):
            cut = {k: state[f"{m}.{k}"][..., a:b] for k in FIELDS + ("P",)}
            S.set_state(mi, cut["P"][1], cut["sat"], cut["x"], cut["y"], cut["z"], cut["label"], cut["rho"])
            S.set_pressures(mi, cut["P"])
        lrows, _ = S.refresh_layout()
        S.set_controls(d.dt, pcoeff)
        xl = np.concatenate([xp[gro[m * n + a]:gro[m * n + b]] for m in (0, 1)])
        S.update_all(torch.tensor(xl, device=cuda_device))
        part = torch.zeros((nw, 2, 5), dtype=torch.float64, device=cuda_device)
        S.well_sums(z0 - lo, z1 - lo, part)
        slabs_.append((S, z0, z1, lo, hi, lrows, part))
    total = sum(p for *_, p in slabs_)
    R, C, V = [], [], []
    counts = []
    owned = []
    for S, z0, z1, lo, hi, lrows, _ in slabs_:
        S.set_well_sums(total)
        fl = torch.zeros(lrows, dtype=torch.float64, device=cuda_device)
        S.residual(fl, None, T)
        fl = fl.cpu().numpy()
        lro = S.row_offsets()
        nl = S.cells
        own = [(int(lro[m * nl + (z0 - lo) * nxy]), int(lro[m * nl + (z1 - lo) * nxy])) for m in (0, 1)]
        for m in (0, 1):
            ga, gb = gro[m * n + z0 * nxy], gro[m * n + z1 * nxy]
            la, lb = own[m]
            assert gb - ga == lb - la
            err = np.abs(fl[la:lb] - f[ga:gb])
            bad = err > 1e-12 * scale[ga:gb] + 1e-300
            assert not bad.any(), (z0, z1, m, int(bad.sum()), float((err / (scale[ga:gb] + 1e-300)).max()))
        JS = S.alloc_jacobian(cuda_device)
        assert S.jacobian(JS, T) == 0
        owned.append((S, JS, own, int(lro[nl])))
        counts.append((own[0][1] - own[0][0], own[1][1] - own[1][0]))
    for rank, (S, JS, own, fs) in enumerate(owned):
        r, c, v = S.jacobian_coo(JS)
        keep = ((r >= own[0][0]) & (r < own[0][1])) | ((r >= own[1][0]) & (r < own[1][1]))
        offs = slabs.global_offsets(counts, rank)
        R.append(slabs.to_global(r[keep], fs, own, offs))
        C.append(slabs.to_global(c[keep], fs, own, offs))
        V.append(v[keep])
    B = sp.csr_matrix((np.concatenate(V), (np.concatenate(R), np.concatenate(C))), shape=(rows, rows))
    D = abs(A - B)
    jscale = np.maximum(abs(A).max(axis=1).toarray().ravel(), 1e-300)
    worst = (D.max(axis=1).toarray().ravel() / jscale).max()
    assert worst <= 1e-12, worst


def test_slab_wrapper_wells_single_rank_nccl(tmp_path, cuda_device):
    """Slab.form_function on a deck with wells, on a one-rank NCCL group:
    the wells' layer sums go through the all-reduce and back to the grid;
    the residual matches the single grid's within 1e-12 of each row's
    absolute term sum, and the Jacobian evaluated next (same sums) within
    1e-12 of each row's largest entry."""
    import socket

    import torch
    import torch.distributed as dist
    path = os.path.join(str(tmp_path), "w.dat")
    deck.write_deck(path, deck.all_wells_deck())
    d = deck.parse_deck(path)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=cuda_device)
    try:
        G = osr.Grid(d)
        G.initialize(cuda_device)
        rows, _ = G.layout()
        x = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
        G.init_guess(x)
        f, scale = torch.zeros_like(x), torch.zeros_like(x)
        G.update_all(x.clone())
        G.residual(f, scale, T)
        J = G.alloc_jacobian(cuda_device)
        assert G.jacobian(J, T) == 0
        S = slabs.Slab(d, 0, 1)
        S.grid.initialize(cuda_device)
        assert S.refresh_layout(cuda_device) == rows
        fl = torch.zeros_like(x)
        S.form_function(x.clone(), fl, T)
        JS = S.grid.alloc_jacobian(cuda_device)
        assert S.grid.jacobian(JS, T) == 0
        torch.cuda.synchronize()
        err = (fl - f).abs().cpu().numpy()
        assert np.all(err <= 1e-12 * scale.cpu().numpy() + 1e-300), float(err.max())
        dv = (JS - J).abs().cpu().numpy()
        assert dv.max() <= 1e-12 * np.abs(J.cpu().numpy()).max()
    finally:
        dist.destroy_process_group()
