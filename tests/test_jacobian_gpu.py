"""GPU parity of the Jacobian path (FormJacobian) against the reference.

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

CASES = {
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


def test_one_phase_cells_are_reported(tmp_path, cuda_device):
    import torch
    path = os.path.join(str(tmp_path), "oil.dat")
    deck.write_deck(path, deck.config_deck(nx=3, ny=3, nz=2, cdif=0.0, ipress=2e7))
    d = deck.parse_deck(path)
    R = oracle.RefDeck(path)
    G = osr.Grid(d)
    for mi, m in enumerate("mf"):
        G.set_state(mi, R.get(f"{m}.P")[1], R.get(f"{m}.sat"), R.get(f"{m}.x"), R.get(f"{m}.y"), R.get(f"{m}.z"),
                    R.get(f"{m}.label"), R.get(f"{m}.rho"))
    n, _ = G.refresh_layout()
    d_x = torch.zeros(n, dtype=torch.float64, device=cuda_device)
    G.init_guess(d_x)
    Jb = G.alloc_jacobian(cuda_device)
    assert G.form_jacobian(d_x, Jb, 3600.0) == 6   # OSR_ERR_UNSUPPORTED
