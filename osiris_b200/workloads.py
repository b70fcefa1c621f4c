"""Seeded synthetic workloads with the shapes of the reference's benchmark cases.

The reference publishes no dataset; these generators are the whole workload.
Every draw uses ``numpy.random.default_rng`` with a fixed seed so tests,
fixtures and the bench see the same cells.

``flash_fluid_srk6`` / ``flash_cells``: the standalone batched flash
(1,048,576 cells, SRK, 6 components).  Component table (seed 2): Tc ~ U(150,
700) K, Pc ~ U(1.5, 5) MPa, omega ~ U(0, 0.6), kij ~ U(0, 0.1) symmetric with a
zero diagonal.  Cells (seed 3): P ~ U(5, 40) MPa, T ~ U(300, 450) K,
z ~ Dirichlet(1).

``fluid_c1_nc4_nc10``: the small plain case's 3-component PR fluid
(C1/nC4/nC10: Tc 190.6/425.1/617.7 K, Pc 4.599/3.796/2.110 MPa, omega
0.011/0.200/0.490, kij = 0.04 for C1-nC10, else 0).
"""
from __future__ import annotations

import numpy as np

FLASH_CELLS = 1_048_576


def flash_table(nc: int, seed: int):
    rng = np.random.default_rng(seed)
    tc = rng.uniform(150.0, 700.0, nc)
    pc = rng.uniform(1.5e6, 5.0e6, nc)
    acf = rng.uniform(0.0, 0.6, nc)
    k = rng.uniform(0.0, 0.1, (nc, nc))
    k = np.triu(k, 1)
    kij = k + k.T
    return tc, pc, acf, kij


def flash_fluid_srk6():
    """(tc, pc, acf, kij, eos) of the 6-component SRK batched-flash case."""
    tc, pc, acf, kij = flash_table(6, 2)
    return tc, pc, acf, kij, 1


def flash_cells(n: int, nc: int, seed: int = 3):
    """P [n] Pa, T [n] K, z [nc, n] for n cells.  The first n cells of a larger
    draw are NOT the same as a smaller draw; tests that need a subset of the
    full case slice the full draw."""
    rng = np.random.default_rng(seed)
    P = rng.uniform(5e6, 40e6, n)
    T = rng.uniform(300.0, 450.0, n)
    z = np.ascontiguousarray(rng.dirichlet(np.ones(nc), n).T)
    return P, T, z


INSTANCES = 4096


def batched_instances(n_inst: int = INSTANCES, seed: int = 4, cells_lo: float = 1e3, cells_hi: float = 6.4e4,
                      nc_lo: int = 3, nc_hi: int = 12):
    """The uneven-instance workload: n_inst independent flash instances, each
    with log-uniform cell count in [cells_lo, cells_hi], component count
    uniform in {nc_lo..nc_hi}, PR or SRK with equal odds, and its own seeded
    component table drawn as ``flash_table``'s.  Returns a list of dicts
    (nc, eos, tc, pc, acf, kij, cells, seed)."""
    rng = np.random.default_rng(seed)
    cells = np.exp(rng.uniform(np.log(cells_lo), np.log(cells_hi), n_inst)).astype(np.int64)
    ncs = rng.integers(nc_lo, nc_hi + 1, n_inst)
    eos = rng.integers(0, 2, n_inst)
    out = []
    for i in range(n_inst):
        s = int(seed) * 1_000_003 + i
        tc, pc, acf, kij = flash_table(int(ncs[i]), s)
        out.append(dict(nc=int(ncs[i]), eos=int(eos[i]), tc=tc, pc=pc, acf=acf, kij=kij, cells=int(cells[i]), seed=s))
    return out


def instance_group(instances, nc: int, seed: int = 5):
    """The instances with nc components, concatenated: (members, start [m+1],
    P [n], T [n], z [nc, n]) with P ~ U(5, 40) MPa, T ~ U(300, 450) K and
    z ~ Dirichlet(1) per cell (seeded per group)."""
    members = [d for d in instances if d["nc"] == nc]
    start = np.zeros(len(members) + 1, np.int64)
    start[1:] = np.cumsum([d["cells"] for d in members])
    n = int(start[-1])
    rng = np.random.default_rng(seed * 1000 + nc)
    P = rng.uniform(5e6, 40e6, n)
    T = rng.uniform(300.0, 450.0, n)
    g = rng.standard_gamma(1.0, (nc, n))
    z = np.ascontiguousarray(g / g.sum(axis=0, keepdims=True))
    return members, start, P, T, z


def fluid_c1_nc4_nc10():
    tc = np.array([190.6, 425.1, 617.7])
    pc = np.array([4.599e6, 3.796e6, 2.110e6])
    acf = np.array([0.011, 0.200, 0.490])
    kij = np.zeros((3, 3))
    kij[0, 2] = kij[2, 0] = 0.04
    return tc, pc, acf, kij, 0


def flash_bytes_per_cell(nc: int, derivs: bool = True, iters: bool = True) -> int:
    """Algorithmic HBM bytes per flashed cell: inputs P, T, z read once;
    outputs label, L, x, y, Zl, Zg (+ iteration counters, + derivative
    blocks) written once."""
    b_in = (nc + 2) * 8
    b_out = 1 + 8 + 2 * nc * 8 + 2 * 8
    if iters:
        b_out += 2 * 4
    if derivs:
        b_out += (2 * nc * nc + 2 * nc) * 8
    return b_in + b_out


# ----------------------------------------------------------------------------
# Full Newton-step assembly: 128 x 128 x 32 dual-porosity grid, PR, 8
# components with the seeded table of the batched flash (seed 2), all cells
# two-phase.
# ----------------------------------------------------------------------------
ASSEMBLY_GRID = (128, 128, 32)


def assembly_deck(nx: int = 128, ny: int = 128, nz: int = 32, nc: int = 8, seed: int = 2, cdif=0.0):
    """A ``deck.Deck`` for the assembly workload.  Component criticals as the
    batched flash's table; molecular weight ~ U(16, 250), Z_c 0.27 (so V_c =
    Z_c R T_c / P_c), parachor ~ U(70, 700); matrix porosity 0.2, fracture 0.01,
    log-normal matrix permeability (median 10 mD, sigma_ln 0.5), fracture
    permeability 1000 mD, 50 m x 50 m x 5 m blocks, the sample deck's
    saturation tables, no wells.  Initial state is set by ``assembly_state``."""
    from .deck import Deck, SAMPLE_SGT, SAMPLE_SWT
    rng = np.random.default_rng(seed)
    tc, pc, acf, kij = flash_table(nc, seed)
    n = nx * ny * nz
    d = Deck()
    d.nx, d.ny, d.nz, d.pnc, d.unc, d.eos = nx, ny, nz, nc, 0, 0
    d.restemp, d.wat_ro, d.wat_mu = 360.0, 1000.0, 1.0
    d.di, d.dj, d.dk = np.full(nx, 50.0), np.full(ny, 50.0), np.full(nz, 5.0)
    d.tor = np.ones(n)
    d.por, d.fpor = np.full(n, 0.2), np.full(n, 0.01)
    d.perm = np.exp(np.log(10.0) + 0.5 * rng.standard_normal((3, n)))
    d.fperm = np.full((3, n), 1000.0)
    d.cdif = cdif
    d.sigma, d.lf, d.re_f = 1.0, 0.01, 1e6
    d.refp, d.cpor, d.dcpor = 101325.0, 0.0, 0.0
    d.tc, d.pc, d.acf = tc, pc, acf
    d.mw = rng.uniform(16.0, 250.0, nc)
    d.zc = np.full(nc, 0.27)
    d.vc = d.zc * 8.3144621 * tc / pc * 1e6
    d.parachor = rng.uniform(70.0, 700.0, nc)
    d.kij = kij
    d.swt = np.array(SAMPLE_SWT, dtype=float)
    d.sgt = np.array(SAMPLE_SGT, dtype=float)
    d.wells_i = np.zeros((0, 5), dtype=np.int32)
    d.wells_f = np.zeros((0, nc + 6))
    d.dt = 3600.0
    d.total_time = 17520 * 3600.0   # the sample deck's TOTALT (2 years)
    return d


def assembly_state(grid, d, device, seed: int = 4, noise: float = 0.005):
    """Initial two-phase state of the assembly workload on the device: one
    feed composition and the middle of its two-phase pressure range (found by
    a flash sweep), seeded pressure noise (+-0.5 % by default; the time-stepping
    workload starts without it), water saturation 0.2 in the
    matrix and 0 in the fracture; phase split, compositions and densities from
    the device flash.  Returns the pressure the sweep chose."""
    import torch
    from . import Fluid, flash
    rng = np.random.default_rng(seed)
    nc, n = d.nc, d.cells
    z0 = rng.dirichlet(np.ones(nc))
    fl = Fluid(d.tc, d.pc, d.acf, d.kij, d.eos)
    sweep = np.linspace(1e6, 40e6, 256)
    Ps = torch.tensor(sweep, device=device)
    Ts = torch.full_like(Ps, d.restemp)
    zs = torch.tensor(np.repeat(z0[:, None], len(sweep), axis=1), device=device)
    lab = flash(fl, Ps, Ts, zs)["label"].cpu().numpy()
    two = sweep[lab == 0]
    if len(two) == 0:
        raise RuntimeError("the seeded feed has no two-phase pressure range")
    p0 = float(np.median(two))
    R = 8.3144621
    for med, sw in ((0, 0.2), (1, 0.0)):
        P = torch.tensor(p0 * (1 + noise * rng.uniform(-1, 1, n)), device=device)
        T = torch.full_like(P, d.restemp)
        z = torch.tensor(np.repeat(z0[:, None], n, axis=1), device=device)
        o = flash(fl, P, T, z)
        L, Zl, Zg = o["L"], o["Zl"], o["Zg"]
        newD = Zl * L / (Zl * L + Zg * (1 - L))
        sat = torch.stack([torch.full_like(P, sw), newD * (1 - sw), (1 - newD) * (1 - sw)])
        rho = torch.stack([P / (Zl * R * T), P / (Zg * R * T)])
        grid.set_state(med, P.cpu().numpy(), sat.cpu().numpy(), o["x"].cpu().numpy(), o["y"].cpu().numpy(),
                       z.cpu().numpy(), o["label"].cpu().numpy(), rho.cpu().numpy())
    return p0


def assembly_spec(d) -> dict:
    """``deck.write_deck`` spec of an assembly deck ``d`` for readers of the
    reference's deck format: the same grid, rock, saturation tables and
    controls.  The keywords cannot carry a seeded component table (named
    components come from the library, user components from SG/TB
    correlations), so the components are placeholder library names and the
    table is replaced after loading; the initial state is likewise a
    placeholder for ``assembly_state``'s.  ``parse_deck`` of the written text
    with ``d``'s component table reproduces ``d``."""
    from .deck import COMPONENT_LIBRARY, TIME_FACTOR
    names = list(COMPONENT_LIBRARY)[:d.nc]
    z = np.full(d.nc, 1.0 / d.nc)
    return dict(grid=(d.nx, d.ny, d.nz), di=d.di, dj=d.dj, dk=d.dk, por=d.por, fpor=d.fpor, permi=d.perm[0],
                permj=d.perm[1], permk=d.perm[2], fpermi=d.fperm[0], fpermj=d.fperm[1], fpermk=d.fperm[2],
                lf=d.lf, re_f=d.re_f, model="PR" if d.eos == 0 else "SRK", comps=names, bic=np.zeros((d.nc, d.nc)),
                sgt=d.sgt, swt=d.swt, refp=d.refp, cpor=d.cpor, dcpor=d.dcpor, wells=[],
                restemp_c=d.restemp - 273.15, wat_ro=d.wat_ro, wat_mu=d.wat_mu, dt=d.dt / TIME_FACTOR,
                totalt=d.total_time / TIME_FACTOR, dtmax=d.dtmax,
                cdif=d.cdif, ipress=2e7, iws=0.2, igc=z.tolist(), fipress=2e7, fiws=0.0, figc=z.tolist())


def with_table(parsed, d):
    """``parsed`` (a ``Deck`` read from ``assembly_spec(d)``'s text) with
    ``d``'s component table."""
    for k in ("tc", "pc", "acf", "mw", "vc", "zc", "parachor", "kij"):
        setattr(parsed, k, np.array(getattr(d, k), dtype=float))
    return parsed
