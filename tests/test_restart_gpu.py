"""Restart of a device run: after three passes the device run's restart file
holds the reference's state after the same three passes (within 1e-9, labels,
time, Dt and marker index identical); loading it into a freshly started grid
restores exactly that state, and the restored run steps on."""
import os

import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from oracle import steps
from osiris_b200 import deck, restart

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")]


def test_device_restart_round_trip(tmp_path, cuda_device):
    path = os.path.join(str(tmp_path), "deck.dat")
    deck.write_deck(path, deck.config_deck(nx=5, ny=4, nz=3, cdif=0.0, ipress=1e7, seed=3))
    R = oracle.RefDeck(path)
    d = deck.parse_deck(path)
    G = osr.Grid(d)
    G.initialize(cuda_device)
    sim = osr.Sim.from_deck(G)
    t = 0.0
    R.create_backups(t)
    for _ in range(3):
        t = steps.ref_pass(R, t)["sim_time"]
        sim.step()
    ref_file = R.write_rst(str(tmp_path), t)
    mine = os.path.join(str(tmp_path), "device.rst")
    restart.write_rst(mine, G, sim)
    a = restart.read_rst(mine, d.nx, d.ny, d.nz, d.nc)
    b = restart.read_rst(ref_file, d.nx, d.ny, d.nz, d.nc)
    assert (a["sim_time"], a["dt"], a["tsm_ctrl"]) == (b["sim_time"], b["dt"], b["tsm_ctrl"])
    for m in "mf":
        assert np.array_equal(a[f"{m}.label"], b[f"{m}.label"])
        assert np.abs(a[f"{m}.P"][1] - b[f"{m}.P"][1]).max() <= 1e-9 * np.abs(b[f"{m}.P"][1]).max()
        for k in ("sat", "x", "y"):
            assert np.abs(a[f"{m}.{k}"] - b[f"{m}.{k}"]).max() <= 1e-9, (m, k)
    # restore into a fresh start-up grid and step on
    G2 = osr.Grid(d)
    G2.initialize(cuda_device)
    t2, dt2, tsm2, _ = restart.restore(G2, mine)
    for m in "mf":
        for k in ("sat", "x", "y", "label"):
            assert np.array_equal(G2.get(f"{m}.{k}"), a[f"{m}.{k}"]), (m, k)
        assert np.array_equal(G2.get(f"{m}.P")[1], a[f"{m}.P"][1])
    sim2 = osr.Sim.from_deck(G2)
    sim2.restart(t2, dt2, tsm2)
    assert sim2.time() == (t2, dt2) and sim2.marker_index() == tsm2
    o = sim2.step()
    assert o["accepted"] and o["sim_time"] == t2 + dt2, o
