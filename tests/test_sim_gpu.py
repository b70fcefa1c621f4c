"""GPU parity of time stepping (osr_sim_*) against the reference's main loop.

Both runs start from the reference's initial state of the same deck.  The
CPU side is the reference itself pass by pass (oracle/steps.py: InitGuess2,
FormFunction, FormJacobian, UpdateAll(x, true), CreateBackups, TimeStepCtrl
with RestoreBackups) with an exact sparse solve in place of PETSc's KSP; the
device side is osr_sim_step with its BiCGStab + block-Jacobi solve.  Every
pass must take the same decision (accepted or not) with the same simulation
time, Dt and row count (exactly: the time arithmetic is the same), and after
every accepted pass both continua's phase labels must be identical and the
oil pressures, saturations and phase compositions within 1e-9 (pressures
relative), through ten accepted passes.
"""
import os

import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from oracle import steps
from osiris_b200 import deck

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")]

CASES = {
    # the small plain case: 10x10x3, C1/nC4/nC10 at 20 MPa, gas injector and producer
    "config1_cdif0": lambda: deck.config_deck(cdif=0.0),
    "config1_diffusion": lambda: deck.config_deck(cdif=None),
    # two-phase at 10 MPa with a 2 h first step: three rejected passes (restore, Dt / 1.5) before the
    # first accepted one, then the DTMAX clamp
    "twophase_10MPa_rejections": lambda: dict(deck.config_deck(nx=6, ny=5, nz=3, cdif=0.0, ipress=1e7, seed=3),
                                              dt=2.0),
    "twophase_12MPa_diffusion": lambda: deck.config_deck(nx=6, ny=5, nz=3, cdif=None, ipress=1.2e7, seed=3),
    # the reference's sample deck (10x10x5, five components)
    "sample_12MPa": lambda: deck.sample_deck(),
}


@pytest.mark.parametrize("name", list(CASES))
def test_run_matches_reference_main_loop(name, tmp_path, cuda_device):
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    R = oracle.RefDeck(path)
    G = osr.Grid(deck.parse_deck(path))
    for mi, m in enumerate("mf"):
        G.set_state(mi, R.get(f"{m}.P")[1], R.get(f"{m}.sat"), R.get(f"{m}.x"), R.get(f"{m}.y"), R.get(f"{m}.z"),
                    R.get(f"{m}.label"), R.get(f"{m}.rho"))
    sim = osr.Sim.from_deck(G)
    t = 0.0
    assert sim.time() == (0.0, R.scalar("Dt"))
    R.create_backups(t)
    accepted = passes = 0
    worst = {"P": 0.0, "sat": 0.0, "x": 0.0, "y": 0.0}
    while accepted < 10:
        passes += 1
        assert passes <= 30, "too many rejected passes"
        o = steps.ref_pass(R, t)
        t = o["sim_time"]
        d = sim.step()
        assert d["accepted"] == o["accepted"], (passes, d, o)
        assert (d["sim_time"], d["dt"], d["rows"], bool(d["finished"])) == (o["sim_time"], o["dt"], o["rows"],
                                                                              o["finished"]), (passes, d, o)
        assert abs(d["vnorm"] - o["vnorm"]) <= 1e-6 * o["vnorm"], (passes, d, o)
        if not o["accepted"]:
            continue
        accepted += 1
        for m in "mf":
            assert np.array_equal(G.get(f"{m}.label"), R.get(f"{m}.label")), (passes, m)
            Pd, Pr = G.get(f"{m}.P")[1], R.get(f"{m}.P")[1]
            worst["P"] = max(worst["P"], float(np.abs(Pd - Pr).max() / np.abs(Pr).max()))
            for k in ("sat", "x", "y"):
                worst[k] = max(worst[k], float(np.abs(G.get(f"{m}.{k}") - R.get(f"{m}.{k}")).max()))
        assert all(v <= 1e-9 for v in worst.values()), (passes, worst)
