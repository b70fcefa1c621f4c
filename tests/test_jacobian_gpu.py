"""GPU parity of the Jacobian path (FormJacobian) against the reference.

Decks cover two-phase, oil-only and gas-only cells of both continua, every
pairing of matrix and fracture states, diffusion on and off, and all nine
well types with and without the rate-limit latch.

Both sides start from the same deck state and assemble the Jacobian at the
same perturbed unknown vector; the reference's MatSetValues triplets and the
device block-sparse output (plus its overflow entries) are summed into dense
matrices and compared entry by entry:
|J - J_ref| <= 1e-9 * max|J_ref row| (the reference's entries are sums of
many hand-derived terms; the bar is relative to the row's largest entry).
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


def _pairs_deck(cdif, wells):
    """Nine layers: every (matrix, fracture) pairing of gas-only, two-phase and
    oil-only states."""
    return deck.config_deck(nx=2, ny=3, nz=9, ipress=[_ST[a][0] for a, _ in _PAIRS], igc=[_ST[a][1] for a, _ in _PAIRS],
                            fipress=[_ST[b][0] for _, b in _PAIRS], figc=[_ST[b][1] for _, b in _PAIRS],
                            wells=wells, cdif=cdif)


CASES = {
    "state_pairs_diffusion": (lambda: _pairs_deck(None, False), 3600.0),
    "state_pairs_cdif0_wells": (lambda: _pairs_deck(0.0, True), 3600.0),
    "oil_twophase_layers_wells": (lambda: deck.config_deck(nx=4, ny=3, nz=3, ipress=[8e6, 2e7, 8e6],
                                                           fipress=[2e7, 8e6, 8e6], cdif=None), 3600.0),
    "sample_12MPa": (lambda: deck.sample_deck(), 3600.0),
    "all_well_types_20MPa_oil": (lambda: deck.all_wells_deck(ipress=20e6), 3600.0),
    "twophase_cdif0_no_wells": (lambda: deck.config_deck(nx=4, ny=3, nz=3, cdif=0.0, ipress=8e6, wells=False), 3600.0),
    "twophase_diffusion_no_wells": (lambda: deck.config_deck(nx=4, ny=4, nz=3, cdif=None, ipress=8e6, wells=False,
                                                             seed=8), 3600.0),
    "twophase_diffusion_wells": (lambda: deck.config_deck(nx=5, ny=4, nz=3, cdif=None, ipress=8e6), 3600.0),
    "all_well_types_9MPa": (lambda: deck.all_wells_deck(), 3600.0),
    "all_well_types_9MPa_latched": (lambda: deck.all_wells_deck(cdif=0.0), 7200.0),
}


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


def dense(rows, cols, vals, n):
    J = np.zeros((n, n))
    np.add.at(J, (rows, cols), vals)
    return J


@pytest.mark.parametrize("name", list(CASES))
def test_form_jacobian_matches_reference(name, tmp_path, cuda_device):
    import torch
    R, G = open_pair(tmp_path, name)
    t = CASES[name][1]
    n, _ = G.refresh_layout()
    x0 = R.init_guess()
    rng = np.random.default_rng(5)
    xp = x0 * (1 + 1e-2 * rng.uniform(-1, 1, x0.shape))
    Jr = dense(*R.form_jacobian(xp, t), n)
    Jb = G.alloc_jacobian(cuda_device)
    status = G.form_jacobian(torch.tensor(xp, device=cuda_device), Jb, t)
    assert status == 0, osr.lib().osr_status_string(status)
    Jg = dense(*G.jacobian_coo(Jb), n)
    scale = np.maximum(np.abs(Jr).max(axis=1, keepdims=True), 1e-300)
    err = np.abs(Jg - Jr) / scale
    bad = np.argwhere(err > 1e-9)
    assert len(bad) == 0, (len(bad), [(int(r), int(c), Jg[r, c], Jr[r, c]) for r, c in bad[:8]])

