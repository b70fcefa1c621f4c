"""Generate the golden flash fixtures from the reference itself.

The reference simulator (khazali/Osiris) ships no tests or golden vectors.
These fixtures are outputs of its own SuccFalsh (compsim/Init_Calcs.cpp:571),
compiled unmodified from source by ``oracle/Makefile`` and driven through
``oracle/ref_driver.cpp``, on seeded inputs:

* ``flash_srk6.npz``  -- 2048 cells of the batched-flash case (SRK, 6
  components, seeds 2/3), plus edge cells: zero feed fractions, both ends of
  the pressure and temperature ranges, a nearly pure feed.
* ``flash_pr3.npz``   -- the small plain case's PR C1/nC4/nC10 fluid at
  T = 360 K over a pressure sweep, feed (0.5, 0.2, 0.3) and random feeds.

Run from the repository root where the reference sources are available:
``make -C oracle ref && python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from osiris_b200 import workloads  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def _edge_cells(nc: int, rng):
    P, T, Z = [], [], []
    for p in (5e6, 40e6):
        for t in (300.0, 450.0):
            z = rng.dirichlet(np.ones(nc))
            P.append(p); T.append(t); Z.append(z)
    for zero in range(nc):  # one component absent
        z = rng.dirichlet(np.ones(nc))
        z[zero] = 0.0
        z /= z.sum()
        P.append(rng.uniform(5e6, 40e6)); T.append(rng.uniform(300, 450)); Z.append(z)
    for lead in range(nc):  # nearly pure feed
        z = np.full(nc, 1e-6)
        z[lead] = 1 - 1e-6 * (nc - 1)
        P.append(rng.uniform(5e6, 40e6)); T.append(rng.uniform(300, 450)); Z.append(z)
    return np.array(P), np.array(T), np.ascontiguousarray(np.array(Z).T)


def _run(fl, P, T, z, path, meta):
    r = oracle.ref_flash_batch(fl, P, T, z)
    np.savez_compressed(path, tc=fl.tc, pc=fl.pc, acf=fl.acf, kij=fl.kij, eos=fl.eos, P=P, T=T, z=z, **r, **meta)
    print(path, "cells", P.shape[0], "labels", np.bincount(r["label"] + 1, minlength=3))


def main():
    tc, pc, acf, kij, eos = workloads.flash_fluid_srk6()
    fl = oracle.Fluid(tc, pc, acf, kij, eos)
    P, T, z = workloads.flash_cells(2048, 6, seed=3)
    eP, eT, ez = _edge_cells(6, np.random.default_rng(7))
    _run(fl, np.concatenate([P, eP]), np.concatenate([T, eT]), np.concatenate([z, ez], axis=1),
         os.path.join(OUT, "flash_srk6.npz"), dict(n_edge=eP.shape[0]))

    tc, pc, acf, kij, eos = workloads.fluid_c1_nc4_nc10()
    fl = oracle.Fluid(tc, pc, acf, kij, eos)
    sweep = np.linspace(2e6, 30e6, 57)
    rng = np.random.default_rng(11)
    zr = rng.dirichlet(np.ones(3), 200).T
    P = np.concatenate([sweep, rng.uniform(5e6, 40e6, 200)])
    T = np.full(P.shape[0], 360.0)
    z = np.concatenate([np.tile(np.array([[0.5], [0.2], [0.3]]), (1, sweep.shape[0])), zr], axis=1)
    _run(fl, P, T, np.ascontiguousarray(z), os.path.join(OUT, "flash_pr3.npz"), dict(n_sweep=sweep.shape[0]))


if __name__ == "__main__":
    main()
