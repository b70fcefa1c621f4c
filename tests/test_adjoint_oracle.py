"""The oracle's restatement of the flash adjoint (orc_flash_adjoint) against
central finite differences of the flash polished to the exact equilibrium
(orc_flash_polish), on the CPU.  This pins the restatement the device
adjoint is compared with.  Bar: 1e-6 relative on kij directions (h = 1e-6)."""
import numpy as np

import oracle
from osiris_b200 import workloads


def test_oracle_adjoint_matches_central_differences():
    tc, pc, acf, kij, eos = workloads.flash_fluid_srk6()
    P, T, z = workloads.flash_cells(1500, 6, seed=41)
    fl = oracle.Fluid(tc, pc, acf, kij, eos)
    base = oracle.flash_batch(fl, P, T, z)
    keep = (base["iters"] < 500) & (base["label"] == 0)
    P, T, z = P[keep], T[keep], np.ascontiguousarray(z[:, keep])
    r0 = oracle.flash_batch(fl, P, T, z)
    assert oracle.flash_polish(fl, P, T, z, r0) == 0
    rng = np.random.default_rng(3)
    xb, yb, Lb = rng.standard_normal(r0["x"].shape), rng.standard_normal(r0["y"].shape), rng.standard_normal(len(P))
    kb, zb, pb, bad = oracle.flash_adjoint(fl, P, T, z, r0, xb, yb, Lb)
    assert bad == 0

    def obj(k):
        f = oracle.Fluid(tc, pc, acf, k, eos)
        r = oracle.flash_batch(f, P, T, z)
        assert oracle.flash_polish(f, P, T, z, r) == 0
        return (xb * r["x"]).sum() + (yb * r["y"]).sum() + (Lb * r["L"]).sum()

    h = 1e-6
    for _ in range(4):
        V = rng.standard_normal((6, 6))
        np.fill_diagonal(V, 0)
        fd = (obj(kij + h * V) - obj(kij - h * V)) / (2 * h)
        ad = (kb * V).sum()
        assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)
