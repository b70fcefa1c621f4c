"""GPU parity of the device start-up (Grid.initialize) against the
reference's: INITCOND state, AllFlash of every cell-medium, then
UpdateDependencies(true) (phase control, PCoeff, PJac, properties).

Labels and row offsets identical; pressures within 1e-12 relative;
saturations and the compositions of the phases present within 1e-9; densities
within 1e-9 relative (the device flash agrees with the reference's SuccFalsh
to rounding).  Decks: the small plain case (all oil), two-phase layers, every
pairing of gas-only / two-phase / oil-only matrix and fracture layers
(INITCOND 1), and the reference's sample deck.
"""
import os

import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from osiris_b200 import deck

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")]

G_, O_ = (0.9, 0.07, 0.03), (0.5, 0.2, 0.3)
_ST = {-1: (8e6, G_), 1: (2e7, O_), 0: (8e6, O_)}
_PAIRS = [(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1)]

CASES = {
    "config1": lambda: deck.config_deck(cdif=0.0),
    "twophase_10MPa": lambda: deck.config_deck(nx=6, ny=5, nz=3, cdif=0.0, ipress=1e7, seed=3),
    "state_pairs": lambda: deck.config_deck(
        nx=2, ny=3, nz=9, ipress=[_ST[a][0] for a, _ in _PAIRS], igc=[_ST[a][1] for a, _ in _PAIRS],
        fipress=[_ST[b][0] for _, b in _PAIRS], figc=[_ST[b][1] for _, b in _PAIRS], cdif=None),
    "sample_12MPa": lambda: deck.sample_deck(),
}


@pytest.mark.parametrize("name", list(CASES))
def test_initialize_matches_reference_startup(name, tmp_path, cuda_device):
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    R = oracle.RefDeck(path)
    G = osr.Grid(deck.parse_deck(path))
    G.initialize(cuda_device)
    rows, pcoeff = G.layout()
    assert pcoeff == R.scalar("PCoeff")
    assert np.array_equal(G.row_offsets(), R.get("rowoff").astype(np.int64))
    for m in "mf":
        lab = R.get(f"{m}.label")
        assert np.array_equal(G.get(f"{m}.label"), lab), m
        P, Pr = G.get(f"{m}.P"), R.get(f"{m}.P")
        assert np.abs(P - Pr).max() <= 1e-12 * np.abs(Pr).max(), m
        assert np.abs(G.get(f"{m}.sat") - R.get(f"{m}.sat")).max() <= 1e-9, m
        for k, present in (("x", lab >= 0), ("y", lab <= 0)):
            err = np.abs(G.get(f"{m}.{k}") - R.get(f"{m}.{k}"))[:, present]
            assert err.size == 0 or err.max() <= 1e-9, (m, k, err.max())
        rho, rr = G.get(f"{m}.rho"), R.get(f"{m}.rho")
        for ph, present in ((0, lab >= 0), (1, lab <= 0)):
            e = np.abs(rho[ph] - rr[ph])[present] / np.abs(rr[ph][present]).max() if present.any() else np.zeros(1)
            assert e.max() <= 1e-9, (m, ph, e.max())


@pytest.mark.parametrize("name", list(CASES))
def test_osr_create_equals_package_startup(name, tmp_path, cuda_device):
    """osr_create (C++ deck reader + start-up in one C call) forms exactly
    the state Grid.initialize forms from the package's reader."""
    import torch
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    with torch.cuda.device(cuda_device):
        C = osr.Grid.create(path)
    G = osr.Grid(deck.parse_deck(path))
    G.initialize(cuda_device)
    assert C.layout() == G.layout()
    assert np.array_equal(C.row_offsets(), G.row_offsets())
    for m in "mf":
        for f in osr.Grid.FIELD_PLANES:
            a, b = C.get(f"{m}.{f}"), G.get(f"{m}.{f}")
            assert np.array_equal(a, b, equal_nan=True), (m, f)
