"""Deck reader (osiris_b200.deck) against the reference's Data_Input.

The reference compiled from source reads the same written deck; every array
and scalar the grid path consumes must come out bit-identical.  CPU only.
"""
import os

import numpy as np
import pytest

import oracle
from osiris_b200 import deck, workloads

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")

SPECS = {
    "plain_diffusion": lambda: deck.config_deck(cdif=None, seed=7),
    "plain_cdif": lambda: deck.config_deck(cdif=1e-8, nx=4, ny=3, nz=2, seed=3),
    "sample": lambda: deck.sample_deck(),
}


def _write(tmp_path, name):
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, SPECS[name]())
    return path


@needs_ref
@pytest.mark.parametrize("name", list(SPECS))
def test_parser_matches_reference(name, tmp_path):
    path = _write(tmp_path, name)
    R = oracle.RefDeck(path)
    d = deck.parse_deck(path)
    assert (d.nx, d.ny, d.nz, d.nc) == (R.nx, R.ny, R.nz, R.nc)
    assert d.eos == (0 if R.pr else 1)
    fl = R.get("fluid")
    for col, arr in ((2, d.mw), (3, d.acf), (4, d.pc), (5, d.tc)):
        assert np.array_equal(arr, fl[:, col]), col
    assert np.array_equal(1 - d.kij, R.get("bic"))
    assert np.array_equal(np.concatenate([d.di, d.dj, d.dk]), R.get("gridDim"))
    for a, b in (("por", "m.por"), ("fpor", "f.por"), ("perm", "m.perm"), ("fperm", "f.perm")):
        assert np.array_equal(getattr(d, a), R.get(b)), a
    for m, p0, sw0, z0 in (("m", d.p0, d.sw0, d.z0), ("f", d.fp0, d.fsw0, d.fz0)):
        assert np.array_equal(R.get(f"{m}.P")[1], p0)
        assert np.array_equal(R.get(f"{m}.sat")[0], sw0)
        assert np.array_equal(R.get(f"{m}.z"), z0)
    assert (R.nswt, R.nsgt, R.nwells) == (len(d.swt), len(d.sgt), len(d.wells_i))
    assert R.scalar("resTemp") == d.restemp
    assert (R.scalar("watRo"), R.scalar("watMu")) == (d.wat_ro, d.wat_mu)
    assert (R.scalar("refP"), R.scalar("cpor"), R.scalar("dcpor")) == (d.refp, d.cpor, d.dcpor)
    assert (R.scalar("Lf"), R.scalar("Re_f"), R.scalar("SigmaMF")) == (d.lf, d.re_f, d.sigma)
    assert R.scalar("Dt") == d.dt
    if d.cdif is None:
        assert R.cdif == 0
    else:
        assert R.cdif == 1 and R.scalar("CDiffCoef") == d.cdif


@pytest.mark.parametrize("name", list(SPECS))
def test_write_parse_roundtrip(name, tmp_path):
    spec = SPECS[name]()
    d = deck.parse_deck(_write(tmp_path, name))
    nx, ny, nz = spec["grid"]
    assert (d.nx, d.ny, d.nz) == (nx, ny, nz)
    assert d.cells == nx * ny * nz
    assert d.z0.shape == (d.nc, d.cells) and np.allclose(d.z0.sum(axis=0), 1.0)
    assert d.perm.shape == (3, d.cells) and (d.perm > 0).all()
    assert d.kij.shape == (d.nc, d.nc) and np.array_equal(d.kij, d.kij.T)
    assert d.wells_f.shape == (len(d.wells_i), d.nc + 6)


def test_spec_round_trip(tmp_path):
    """The written deck, read back with the seeded table, is the bench's deck
    (apart from the placeholder initial state and the time controls)."""
    d = workloads.assembly_deck(6, 5, 4)
    path = os.path.join(str(tmp_path), "a.dat")
    deck.write_deck(path, workloads.assembly_spec(d))
    q = workloads.with_table(deck.parse_deck(path), d)
    skip = {"p0", "fp0", "sw0", "fsw0", "z0", "fz0", "extra", "initcond", "pnc", "unc"}
    for k, v in vars(d).items():
        if k not in skip:
            assert np.array_equal(np.asarray(v), np.asarray(getattr(q, k))), k
    assert q.nc == d.nc


def test_missing_required_keyword(tmp_path):
    path = _write(tmp_path, "sample")
    text = open(path).read().replace("GRID", "GRIX")
    bad = os.path.join(str(tmp_path), "bad.dat")
    open(bad, "w").write(text)
    with pytest.raises(deck.DeckError):
        deck.parse_deck(bad)


@needs_ref
@pytest.mark.parametrize("spec", ["plain", "all_wells", "sample", "no_wells"])
def test_time_markers_match_reference(spec, tmp_path):
    """The run's time markers and first Dt (Data_Input + ManageTSMarker)."""
    s = {"plain": deck.config_deck, "all_wells": deck.all_wells_deck, "sample": deck.sample_deck,
         "no_wells": lambda: deck.config_deck(wells=False)}[spec]()
    path = os.path.join(str(tmp_path), spec + ".dat")
    deck.write_deck(path, s)
    R = oracle.RefDeck(path)
    m_ref, ctrl = R.time_markers()
    m, dt = deck.time_markers(deck.parse_deck(path))
    assert ctrl == 0
    assert np.array_equal(m, m_ref), (m, m_ref)
    assert dt == R.scalar("Dt")
