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


def test_c_abi_restart_and_listing_match_python_writers(tmp_path, cuda_device):
    """The C ABI's restart writer and reader (osr_sim_write_restart /
    osr_sim_read_restart) and state listing (osr_grid_write_listing), for a
    C++ host, against the package's writers (which the tests above and
    tests/test_restart.py hold to the reference's own files): the files
    are byte for byte identical, and reading restores the same state, clock
    and marker as restart.restore + Sim.restart."""
    from osiris_b200.output import StateListing
    path = os.path.join(str(tmp_path), "deck.dat")
    deck.write_deck(path, deck.config_deck(nx=5, ny=4, nz=3, cdif=0.0, ipress=1e7, seed=3))
    d = deck.parse_deck(path)
    G = osr.Grid(d)
    G.initialize(cuda_device)
    sim = osr.Sim.from_deck(G)
    lc, lp = os.path.join(str(tmp_path), "c.txt"), os.path.join(str(tmp_path), "py.txt")
    listing = StateListing(lp)
    t = 0.0
    G.write_listing(lc, t, True)
    listing.write_grid(G, t)
    for _ in range(3):
        t = sim.step()["sim_time"]
        G.write_listing(lc, t, False)
        listing.write_grid(G, t)
    listing.close()
    assert open(lc, "rb").read() == open(lp, "rb").read()
    rc, rp = os.path.join(str(tmp_path), "c.rst"), os.path.join(str(tmp_path), "py.rst")
    sim.write_restart(rc, 123.5)
    restart.write_rst(rp, G, sim, 123.5)
    assert open(rc, "rb").read() == open(rp, "rb").read()
    # read back into fresh start-up runs: the C ABI reader and the package's restore
    G2, G3 = osr.Grid(d), osr.Grid(d)
    G2.initialize(cuda_device)
    G3.initialize(cuda_device)
    sim2, sim3 = osr.Sim.from_deck(G2), osr.Sim.from_deck(G3)
    assert sim2.read_restart(rc) == 123.5
    t3, dt3, tsm3, _ = restart.restore(G3, rp)
    sim3.restart(t3, dt3, tsm3)
    assert sim2.time() == sim3.time() == sim.time() and sim2.marker_index() == sim3.marker_index()
    for m in "mf":
        for k in ("P", "sat", "x", "y", "label", "rho", "mu", "kr"):
            assert np.array_equal(G2.get(f"{m}.{k}"), G3.get(f"{m}.{k}"), equal_nan=True), (m, k)
    assert G2.row_offsets().tolist() == G3.row_offsets().tolist()
    assert sim2.step() == sim3.step()
    with pytest.raises(osr.OsrError):
        sim2.read_restart(lc)   # not a restart file
