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
