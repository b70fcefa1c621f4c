"""GPU parity of the residual path (FormFunction) against the reference.

Both sides start from the same deck state: the reference compiled from source
opens the deck and runs its initialisation; the device grid receives that
state (pressures, saturations, compositions, labels and the densities from
which the interfacial tension of the next update is formed).  The row layout
and PCoeff must agree exactly, InitGuess2 must give the same unknowns, and
after both sides unpack the same perturbed unknown vector (UpdateAll) the
residual rows must agree within 1e-10 of the sum of the absolute values of
each row's terms (the device reports that sum per row).
"""
import os

import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from osiris_b200 import deck

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")]

CASES = {
    "oil_20MPa_cdif0": (lambda: deck.config_deck(nx=5, ny=4, nz=3, cdif=0.0), 3600.0),
    "twophase_8MPa_diffusion": (lambda: deck.config_deck(nx=5, ny=4, nz=3, cdif=None, ipress=8e6), 3600.0),
    "twophase_8MPa_cdif0": (lambda: deck.config_deck(nx=4, ny=4, nz=2, cdif=0.0, ipress=8e6, seed=5), 7200.0),
    "sample_12MPa": (lambda: deck.sample_deck(), 3600.0),
    "sample_6MPa": (lambda: deck.sample_deck(ipress=6e6), 0.0),
    "all_well_types_9MPa": (lambda: deck.all_wells_deck(), 3600.0),
    "all_well_types_9MPa_latched": (lambda: deck.all_wells_deck(), 3600.0),
    "all_well_types_13MPa_latched": (lambda: deck.all_wells_deck(ipress=13e6, cdif=0.0), 7200.0),
    "all_well_types_20MPa_oil": (lambda: deck.all_wells_deck(ipress=20e6), 3600.0),
}


def test_well_radius_matches_calc_re(tmp_path, cuda_device):
    R, G = open_pair(tmp_path, "all_well_types_9MPa")
    for w in range(R.nwells):
        assert G.well_radius(w) == R.calc_re(w), w


def open_pair(tmp_path, name):
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name][0]())
    R = oracle.RefDeck(path)
    G = osr.Grid(deck.parse_deck(path))
    for mi, m in enumerate("mf"):
        G.set_state(mi, R.get(f"{m}.P")[1], R.get(f"{m}.sat"), R.get(f"{m}.x"), R.get(f"{m}.y"), R.get(f"{m}.z"),
                    R.get(f"{m}.label"), R.get(f"{m}.rho"))
    if name.endswith("_latched"):
        for w in range(R.nwells):
            R.set_well_condition(w, True)
            G.set_well_condition(w, True)
    return R, G


@pytest.mark.parametrize("name", list(CASES))
def test_layout_and_init_guess(name, tmp_path, cuda_device):
    import torch
    R, G = open_pair(tmp_path, name)
    rows, pcoeff = G.refresh_layout()
    assert pcoeff == R.scalar("PCoeff")
    assert np.array_equal(G.row_offsets(), R.get("rowoff").astype(np.int64))
    x_ref = R.init_guess()
    assert rows == len(x_ref)
    d_x = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    G.init_guess(d_x)
    torch.cuda.synchronize()
    assert np.array_equal(d_x.cpu().numpy(), x_ref)


@pytest.mark.parametrize("name", list(CASES))
def test_form_function_matches_reference(name, tmp_path, cuda_device):
    import torch
    R, G = open_pair(tmp_path, name)
    t = CASES[name][1]
    rows, _ = G.refresh_layout()
    x0 = R.init_guess()
    rng = np.random.default_rng(11)
    xp = x0 * (1 + 1e-3 * rng.uniform(-1, 1, x0.shape))
    f_ref = R.form_function(xp, t)
    d_x = torch.tensor(xp, device=cuda_device)
    d_f = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    d_s = torch.zeros_like(d_f)
    G.form_function(d_x, d_f, t)
    G.residual(d_f, d_s, t)
    torch.cuda.synchronize()
    f = d_f.cpu().numpy()
    scale = d_s.cpu().numpy()
    err = np.abs(f - f_ref)
    bad = err > 1e-10 * scale + 1e-300
    rowoff = R.get("rowoff").astype(np.int64)
    where = [(int(r), int(np.searchsorted(rowoff, r, side="right") - 1), f[r], f_ref[r], scale[r])
             for r in np.nonzero(bad)[0][:10]]
    assert not bad.any(), (int(bad.sum()), rows, where)
