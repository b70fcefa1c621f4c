"""The C++ deck reader of the C ABI (osr_deck_open / osr_deck_model /
osr_deck_initial_state / osr_deck_times) against the package's reader
(osiris_b200.deck.parse_deck), which tests/test_deck.py pins to the
reference's own Data_Input.  Every value must be identical.  Decks cover
INITCOND 0 (k*v repeat groups), 1 (per layer) and 3 (constant), pseudo
components (SG/TB/MW/AC/... with the Cavett correlations), CON/VAR/IVAR/KVAR
arrays, TOR, CDIF, all nine well types, and malformed decks.  CPU only: the
reader does no device work.
"""
import os

import numpy as np
import pytest

import osiris_b200 as osr
from osiris_b200 import deck, workloads

PSEUDO = """GRID 3 2 2
DI VAR 10 20 30
DJ CON 15
DK VAR 5 7
TOR IVAR 1 1.5 2
POR VAR 0.2 0.2 0.2 0.2 0.2 0.2 0 0.2 0.2 0.2 0.2 0.2
FPOR CON 0.01
PERMI VAR 1 2 3 4 5 6 7 8 9 10 11 12
PERMJ CON 10
PERMK KVAR 3 4
FPERMI CON 100
FPERMJ IVAR 100 200 300
FPERMK CON 50
Lf 0.5
Re_f 1000
MODEL SRK
NC 2 2
COMPNAME C1 CO2
SG 0.78 0.85
TB 600 800
MW 120 250
BIC 0.01 0.02 0.03 0.04 0.05 0.06
SWT 2
0.2 0 1 0
1 1 0 0
SGT 2
0 0 1 0
0.8 1 0 0
WELLS 2
8 1 1 1 2 50 14000000 0 0.1 1 0 0 0 1 17520
0 3 2 1 1 7000000 10 0 0.1 1 17520
RESTEMP 90
WATERPROPS 1000 1
DT 0.01
TOTALT 100
SIGMA 2
CDIF 1e-9
INITCOND 0
IPRESS 6*2e7 6*2.1e7
FIPRESS 12*2e7
IWS 12*0.2
FIWS 12*0
IGC 12*0.4 12*0.3 12*0.2 12*0.1
FIGC 12*0.4 12*0.3 12*0.2 12*0.1
"""

SPECS = {
    "plain_diffusion": lambda: deck.config_deck(cdif=None, seed=7),
    "plain_cdif": lambda: deck.config_deck(cdif=1e-8, nx=4, ny=3, nz=2, seed=3),
    "sample": lambda: deck.sample_deck(),
    "all_wells": lambda: deck.all_wells_deck(),
    "layers": lambda: deck.config_deck(nx=2, ny=3, nz=4, ipress=[8e6, 9e6, 1e7, 2e7],
                                       igc=[(0.5, 0.2, 0.3), (0.4, 0.3, 0.3), (0.6, 0.2, 0.2), (0.5, 0.25, 0.25)]),
    "assembly": lambda: workloads.assembly_spec(workloads.assembly_deck(6, 5, 4)),
}

FIELDS = ("di", "dj", "dk", "por", "fpor", "perm", "fperm", "tor", "mw", "tc", "pc", "vc", "acf", "parachor", "zc",
          "kij", "swt", "sgt", "wells_i", "wells_f", "p0", "fp0", "sw0", "fsw0", "z0", "fz0")
SCALARS = ("nx", "ny", "nz", "nc", "eos", "restemp", "wat_ro", "wat_mu", "refp", "cpor", "dcpor", "lf", "re_f",
           "sigma", "cdif", "dt", "total_time", "dtmax", "initcond")


def _compare(path):
    d = deck.parse_deck(path)
    c = osr.read_deck(path)
    for k in SCALARS:
        assert c[k] == getattr(d, k), (k, c[k], getattr(d, k))
    for k in FIELDS:
        a, b = np.asarray(getattr(d, k)), c[k]
        assert a.shape == b.shape, (k, a.shape, b.shape)
        assert np.array_equal(a, b), (k, np.argwhere(a != b)[:4])
    return d


@pytest.mark.parametrize("name", list(SPECS))
def test_cpp_reader_equals_package_reader(name, tmp_path):
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, SPECS[name]())
    _compare(path)


def test_cpp_reader_pseudo_components_initcond0(tmp_path):
    path = os.path.join(str(tmp_path), "pseudo.dat")
    open(path, "w").write(PSEUDO)
    d = _compare(path)
    assert d.initcond == 0 and d.unc == 2 and d.cdif == 1e-9
    assert d.por[6] == 1e-11   # zero porosity becomes the floor


@pytest.mark.parametrize("edit, reason", [
    (("GRID", "GRIX"), "No GRID keyword"),
    (("MODEL SRK", "MODEL VDW"), "Incorrect EOS keyword format"),
    (("COMPNAME C1 CO2", "COMPNAME C1 XX9"), "Unknown Component XX9"),
    (("TOR IVAR", "TOR JVAR"), "JVAR"),
    (("INITCOND 0", "INITCOND 2"), "INITCOND 2 is not supported"),
    (("PERMJ CON", "PERMJ FOO"), "Incorrect PERMJ keyword format"),
])
def test_cpp_reader_rejects_malformed_decks(edit, reason, tmp_path):
    path = os.path.join(str(tmp_path), "bad.dat")
    open(path, "w").write(PSEUDO.replace(*edit))
    with pytest.raises(deck.DeckError):
        deck.parse_deck(path)
    with pytest.raises(osr.OsrError, match=reason):
        osr.read_deck(path)


def test_cpp_reader_truncated_and_missing_file(tmp_path):
    path = os.path.join(str(tmp_path), "cut.dat")
    open(path, "w").write(PSEUDO[:PSEUDO.index("IGC") + 10])
    with pytest.raises(osr.OsrError, match="deck ends inside"):
        osr.read_deck(path)
    with pytest.raises(osr.OsrError, match="cannot open"):
        osr.read_deck(os.path.join(str(tmp_path), "none.dat"))
