"""GPU parity of the Jacobian path (FormJacobian) against the reference.

Decks cover two-phase, oil-only and gas-only cells of both continua, every
pairing of matrix and fracture states, diffusion on and off, and all nine
well types with and without the rate-limit latch.

Both sides start from the same deck state and assemble the Jacobian at the
same perturbed unknown vector; the reference's MatSetValues triplets and the
device values, placed by the device pattern (the COO triplets a PETSc
adapter hands to MatSetValuesCOO), are summed into dense matrices and
compared entry by entry: |J - J_ref| <= 1e-9 * max|J_ref row| (the
reference's entries are sums of many hand-derived terms; the bar is relative
to the row's largest entry), and per entry |J - J_ref| <= 1e-8 |J_ref|
wherever |J_ref| > 1e-12 max|J_ref row| (entries below that floor are sums
that cancel to rounding level in the reference itself).  NaN is accepted only where the reference's own
matrix holds NaN at the same entry (its well-derivative terms give 0/0 on the
diagonal of some completion cells of the all-well-types decks); everywhere
else a NaN is a failure.  Every stored value must be written by the call: two
calls into buffers pre-filled with different patterns (NaN, 7.0) must agree
bit for bit.
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
    Jb.fill_(float("nan"))
    status = G.form_jacobian(torch.tensor(xp, device=cuda_device), Jb, t)
    assert status == 0, osr.lib().osr_status_string(status)
    J2 = torch.full_like(Jb, 7.0)
    assert G.jacobian(J2, t) == 0
    torch.cuda.synchronize()
    assert torch.equal(Jb.view(torch.int64), J2.view(torch.int64)), "values left unwritten or not repeatable"
    Jg = dense(*G.jacobian_coo(Jb), n)
    scale = np.maximum(np.abs(np.nan_to_num(Jr)).max(axis=1, keepdims=True), 1e-300)
    err = np.abs(Jg - Jr) / scale
    bad = np.argwhere(~(err <= 1e-9) & ~(np.isnan(Jg) & np.isnan(Jr)))
    assert len(bad) == 0, (len(bad), [(int(r), int(c), Jg[r, c], Jr[r, c]) for r, c in bad[:8]])
    # per entry, relative to the entry itself above the row floor
    sig = np.isfinite(Jr) & (np.abs(Jr) > 1e-12 * scale)
    rel = np.where(sig, np.abs(Jg - Jr) / np.where(sig, np.abs(Jr), 1.0), 0.0)
    r, c = np.unravel_index(int(np.argmax(rel)), rel.shape)
    print(f"{name}: {int(sig.sum())} entries above the floor, worst per-entry relative error {rel[r, c]:.3e} "
          f"at ({r}, {c}): {Jg[r, c]!r} vs {Jr[r, c]!r}")
    badrel = np.argwhere(rel > 1e-8)
    assert len(badrel) == 0, (len(badrel), [(int(r), int(c), Jg[r, c], Jr[r, c], np.abs(Jr[r]).max())
                                            for r, c in badrel[:8]])



def test_pattern_covers_every_reference_entry(tmp_path, cuda_device):
    """Pattern positions are unique per block row and in range, and every
    (row, column) the reference assembles has a position."""
    R, G = open_pair(tmp_path, "state_pairs_cdif0_wells")
    n, _ = G.refresh_layout()
    x0 = R.init_guess()
    rr, rc, _ = R.form_jacobian(x0, 3600.0)
    rows, cols = G.jacobian_pattern(cuda_device)
    r, c = rows.cpu().numpy().ravel(), cols.cpu().numpy().ravel()
    keep = r >= 0
    assert (c[keep] >= 0).all() and (r[keep] < n).all() and (c[keep] < n).all()
    mine = set(zip(r[keep].tolist(), c[keep].tolist()))
    missing = set(zip(rr.tolist(), rc.tolist())) - mine
    assert not missing, sorted(missing)[:10]


@pytest.mark.parametrize("name", ["state_pairs_diffusion", "sample_12MPa", "all_well_types_9MPa_latched"])
def test_transpose_product_matches_reference(name, tmp_path, cuda_device):
    """J^T lambda (osr_grid_jacobian_apply_transpose) against the reference's
    own matrix transposed: within 1e-9 of sum_r |J_ref[r, c]| |lambda_r| per
    entry (the row bar of the matrix test carried through the sum), and
    within 1e-12 of the same scale against the device values' own COO
    product (rounding of the atomic sums only)."""
    import torch
    R, G = open_pair(tmp_path, name)
    t = CASES[name][1]
    n, _ = G.refresh_layout()
    x0 = R.init_guess()
    rng = np.random.default_rng(6)
    xp = x0 * (1 + 1e-2 * rng.uniform(-1, 1, x0.shape))
    Jr = np.nan_to_num(dense(*R.form_jacobian(xp, t), n))
    Jb = G.alloc_jacobian(cuda_device)
    assert G.form_jacobian(torch.tensor(xp, device=cuda_device), Jb, t) == 0
    lam = rng.standard_normal(n)
    y = torch.zeros(n, dtype=torch.float64, device=cuda_device)
    G.jacobian_apply_transpose(Jb, torch.tensor(lam, device=cuda_device), y)
    torch.cuda.synchronize()
    y = y.cpu().numpy()
    Jg = dense(*G.jacobian_coo(Jb), n)
    finite = np.isfinite(Jg).all(axis=0)
    scale = np.abs(Jr).T @ np.abs(lam) + 1e-300
    mine = np.nan_to_num(Jg).T @ lam
    assert np.all(np.abs(y - mine)[finite] <= 1e-12 * scale[finite])
    err = (np.abs(y - Jr.T @ lam) / scale)[finite]
    print(f"{name}: {int(finite.sum())} of {n} columns finite, worst scaled error {err.max():.2e}")
    assert err.max() <= 1e-9
