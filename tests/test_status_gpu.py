"""Per-cell status codes and failures injected on the host.

* osr_flash_status on the batched flash's workload: MAXIT exactly on the
  cells that stopped at the 500-step cap, nothing else flagged; cells whose
  pressure is set to NaN on the host before the upload come back NAN (the
  flash returns, with NaN values, for those cells only) and the first bad
  cell is the lowest flagged index.
* osr_grid_status and the time step: a NaN written into one matrix cell's
  oil pressure on the host is reported at that block; the next pass is
  rejected, Dt is divided by 1.5 and the backup state comes back, as the
  reference's main loop does on the same injected state (its acceptance
  test (vnorm - vnorm) != 0, compsim/PetscAUX.cpp:703, and TimeStepCtrl /
  RestoreBackups, compsim/Do_Time_Step.cpp:391-470); the pass after that is
  accepted with the same Dt and time on both sides.
No GPU fault is involved: the failures are values, made on the host.
"""
import os

import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from osiris_b200 import deck, workloads

pytestmark = pytest.mark.gpu


def test_flash_status_codes_and_injected_nan(cuda_device):
    import torch
    tc, pc, acf, kij, eos = workloads.flash_fluid_srk6()
    f = osr.Fluid(tc, pc, acf, kij, eos)
    P, T, z = workloads.flash_cells(200_000, 6, seed=3)
    dev = cuda_device
    out = osr.flash(f, torch.from_numpy(P).to(dev), torch.from_numpy(T).to(dev), torch.from_numpy(z).to(dev))
    r = osr.flash_status(out, 6)
    it = out["iters"].cpu().numpy()
    assert r["counts"]["MAXIT"] == int((it >= 500).sum())
    assert r["counts"]["NAN"] == 0 and r["counts"]["NOROOT"] == 0
    st = r["status"].cpu().numpy()
    assert np.array_equal(np.flatnonzero(st == 1), np.flatnonzero(it >= 500))
    # NaN pressures injected on the host
    bad = np.array([11, 4_567, 123_456])
    Pn = P.copy()
    Pn[bad] = np.nan
    out2 = osr.flash(f, torch.from_numpy(Pn).to(dev), torch.from_numpy(T).to(dev), torch.from_numpy(z).to(dev))
    r2 = osr.flash_status(out2, 6)
    st2 = r2["status"].cpu().numpy()
    assert (st2[bad] == 2).all()
    assert r2["counts"]["NAN"] == len(bad)
    flagged = np.flatnonzero(st2 != 0)
    assert r2["first_bad"] == flagged.min()
    keep = np.setdiff1d(np.arange(len(P)), bad)
    for k in ("L", "x", "y"):
        a, b = out[k].cpu().numpy(), out2[k].cpu().numpy()
        assert np.array_equal(a[..., keep], b[..., keep]), k


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")
def test_injected_nan_rejects_the_pass_as_the_reference_does(tmp_path, cuda_device):
    from oracle import steps
    path = os.path.join(str(tmp_path), "plain.dat")
    deck.write_deck(path, deck.config_deck(cdif=0.0))
    R = oracle.RefDeck(path)
    G = osr.Grid(deck.parse_deck(path))
    G.initialize(cuda_device)
    sim = osr.Sim.from_deck(G)
    R.create_backups(0.0)
    assert G.status() == (0, -1)
    cell = 37
    Pr = R.get("m.P").copy()
    Pr[1, cell] = np.nan
    R.set("m.P", Pr)
    Pg = G.get("m.P").copy()
    Pg[1, cell] = np.nan
    G.set_pressures(0, Pg)
    assert G.status() == (2, cell)
    o = steps.ref_pass(R, 0.0)
    d = sim.step()
    assert not o["accepted"] and not d["accepted"]
    assert (d["sim_time"], d["dt"]) == (o["sim_time"], o["dt"])
    assert G.status() == (0, -1)
    assert np.isfinite(G.get("m.P")).all()
    o2 = steps.ref_pass(R, o["sim_time"])
    d2 = sim.step()
    assert o2["accepted"] and d2["accepted"]
    assert (d2["sim_time"], d2["dt"]) == (o2["sim_time"], o2["dt"])
    for m in "mf":
        assert np.array_equal(G.get(f"{m}.label"), R.get(f"{m}.label"))
        a, b = G.get(f"{m}.P")[1], R.get(f"{m}.P")[1]
        assert np.abs(a - b).max() <= 1e-8 * np.abs(b).max(), m
