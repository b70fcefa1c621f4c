"""Fugacity derivatives against the reference's own Jacobian.

The reference has no standalone fugacity-derivative function: the
derivatives live in the fugacity rows of a two-phase block of its analytic
Jacobian (IteratorJacobian, compsim/Petsc_Functions.cpp:30243-30372).  Row i
of such a block is the derivative of x_i phi_i^L P_o - y_i phi_i^V P_g:

    column x_k:  P_o phi_i^L (delta_ik + x_i dlnphi_dx[0][i][k])
    column y_k: -P_g phi_i^V (delta_ik + y_i dlnphi_dx[1][i][k])
    column P:    PCoeff (x_i phi_i^L (1 + P_o dlnphi_dP[0][i])
                         - y_i phi_i^V (1 + P_g dlnphi_dP[1][i]))

The deck is the small plain case's fluid (PR, C1/nC4/nC10) in two-phase
layers at 6-11 MPa with the gas-oil capillary pressure column zeroed, so
P_g = P_o exactly.  The reference assembles at its start-up state, whose
compositions are its flash's renormalised to sum to one when the unknowns
are unpacked (compsim/PetscAUX.cpp:176-498) and whose Z is P / (rho R T)
from its property sweep.

* At that state (the reference's x, y, Z), the rows rebuilt from the
  derivatives must equal the reference's entries within 1e-10 of the block's
  largest fugacity-row entry, and every other entry of those rows must be
  below that bar: the oracle's derivatives (CPU) and the device's
  (osr_fugacity_derivs, GPU).
* The device flash run on every block's (P_o, T, z) returns its derivative
  blocks at its own, unrenormalised compositions (sum - 1 up to a few 1e-9,
  the Rachford-Rice stopping rule); the rows rebuilt from those outputs must
  agree within 1e-10 + 10 max|sum - 1| of the block maximum.

phi itself comes from the oracle's EOS at the composition and Z used (test
infrastructure).
"""
import os

import numpy as np
import pytest

import oracle
from osiris_b200 import deck

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")

LAYER_P = [6e6, 7e6, 8e6, 9e6, 10e6, 11e6]
LAYER_Z = [(0.5, 0.2, 0.3), (0.55, 0.2, 0.25), (0.45, 0.25, 0.3), (0.6, 0.15, 0.25), (0.5, 0.25, 0.25),
           (0.65, 0.15, 0.2)]
BAR = 1e-10
R_GAS = 8.3144621


def _open(tmp_path):
    spec = deck.config_deck(nx=3, ny=2, nz=len(LAYER_P), cdif=0.0, wells=False, ipress=LAYER_P,
                            igc=[list(z) for z in LAYER_Z])
    spec["sgt"] = [[r[0], r[1], r[2], 0.0] for r in deck.SAMPLE_SGT]
    path = os.path.join(str(tmp_path), "fugrows.dat")
    deck.write_deck(path, spec)
    return oracle.RefDeck(path), deck.parse_deck(path)


def _reference(R, d):
    """The reference's Jacobian (dense) and the state it was assembled at."""
    P0 = np.concatenate([R.get("m.P"), R.get("f.P")], axis=1)[1].copy()
    x0 = R.init_guess()
    rows, cols, vals = R.form_jacobian(x0, 3600.0)
    n = len(x0)
    J = np.zeros((n, n))
    np.add.at(J, (rows, cols), vals)
    P = np.concatenate([R.get("m.P"), R.get("f.P")], axis=1)
    rho = np.concatenate([R.get("m.rho"), R.get("f.rho")], axis=1)
    s = dict(J=J, rowoff=R.get("rowoff").astype(np.int64), PCoeff=R.scalar("PCoeff"), P0=P0, Po=P[1], Pg=P[2],
             lab=np.concatenate([R.get("m.label"), R.get("f.label")]).astype(np.int64),
             z=np.ascontiguousarray(np.concatenate([R.get("m.z"), R.get("f.z")], axis=1)),
             x=np.ascontiguousarray(np.concatenate([R.get("m.x"), R.get("f.x")], axis=1)),
             y=np.ascontiguousarray(np.concatenate([R.get("m.y"), R.get("f.y")], axis=1)))
    s["Zl"] = P[1] / (rho[0] * R_GAS * d.restemp)
    s["Zg"] = P[2] / (rho[1] * R_GAS * d.restemp)
    s["T"] = np.full(len(P0), d.restemp)
    assert np.array_equal(s["Po"], s["Pg"]), "gas-oil capillary pressure must be zero on this deck"
    return s


def _rows_error(ref, d, x, y, Zl, Zg, dx, dp):
    """Worst |rebuilt - reference| / block max over the two-phase blocks, and
    the worst entry of those rows outside the block's own columns."""
    J, nc = ref["J"], d.nc
    fl = oracle.Fluid(d.tc, d.pc, d.acf, d.kij, d.eos)
    two = np.flatnonzero(ref["lab"] == 0)
    assert len(two) >= 12, "the deck must hold two-phase blocks"
    worst = np.zeros(len(two))
    other = 0.0
    eye = np.eye(nc)
    for q, b in enumerate(two):
        o = int(ref["rowoff"][b])
        Po, Pg = ref["Po"][b], ref["Pg"][b]
        lnl, _, _ = oracle.fugacity(fl, Po, d.restemp, x[:, b], Zl[b])
        lng, _, _ = oracle.fugacity(fl, Pg, d.restemp, y[:, b], Zg[b])
        phl, phg = np.exp(lnl), np.exp(lng)
        mine = np.zeros((nc, 2 * nc + 1))
        mine[:, :nc] = Po * phl[:, None] * (eye + x[:, b][:, None] * dx[0, :, :, b])
        mine[:, nc:2 * nc] = -Pg * phg[:, None] * (eye + y[:, b][:, None] * dx[1, :, :, b])
        mine[:, 2 * nc] = ref["PCoeff"] * (x[:, b] * phl * (1 + Po * dp[0, :, b]) - y[:, b] * phg * (1 + Pg * dp[1, :, b]))
        scale = np.abs(J[o:o + nc]).max()
        worst[q] = np.abs(mine - J[o:o + nc, o:o + 2 * nc + 1]).max() / scale
        rest = J[o:o + nc].copy()
        rest[:, o:o + 2 * nc + 1] = 0
        other = max(other, np.abs(rest).max() / scale)
    return worst, other, two


def test_oracle_derivatives_rebuild_reference_fugacity_rows(tmp_path):
    R, d = _open(tmp_path)
    ref = _reference(R, d)
    fl = oracle.Fluid(d.tc, d.pc, d.acf, d.kij, d.eos)
    dx, dp = oracle.flash_derivs(fl, ref["Po"], ref["T"], ref["x"], ref["y"], ref["Zl"], ref["Zg"])
    worst, other, two = _rows_error(ref, d, ref["x"], ref["y"], ref["Zl"], ref["Zg"], dx, dp)
    print(f"oracle: fugacity rows of {len(two)} two-phase blocks, worst {worst.max():.3e} of the block maximum")
    assert worst.max() <= BAR and other <= BAR, (worst.max(), other)


@pytest.mark.gpu
def test_device_derivatives_rebuild_reference_fugacity_rows(tmp_path, cuda_device):
    import torch
    import osiris_b200 as osr
    R, d = _open(tmp_path)
    ref = _reference(R, d)
    f = osr.Fluid(d.tc, d.pc, d.acf, d.kij, d.eos)
    dev = {k: torch.from_numpy(np.ascontiguousarray(ref[k])).to(cuda_device) for k in ("Po", "T", "x", "y", "Zl", "Zg")}
    out = osr.fugacity_derivs(f, dev["Po"], dev["T"], dev["x"], dev["y"], dev["Zl"], dev["Zg"])
    torch.cuda.synchronize()
    dx, dp = out["dlnphi_dx"].cpu().numpy(), out["dlnphi_dP"].cpu().numpy()
    worst, other, two = _rows_error(ref, d, ref["x"], ref["y"], ref["Zl"], ref["Zg"], dx, dp)
    print(f"device: fugacity rows of {len(two)} two-phase blocks, worst {worst.max():.3e} of the block maximum")
    assert worst.max() <= BAR and other <= BAR, (worst.max(), other)


@pytest.mark.gpu
def test_device_flash_outputs_rebuild_reference_fugacity_rows(tmp_path, cuda_device):
    import torch
    import osiris_b200 as osr
    R, d = _open(tmp_path)
    ref = _reference(R, d)
    f = osr.Fluid(d.tc, d.pc, d.acf, d.kij, d.eos)
    g = osr.flash(f, torch.from_numpy(ref["P0"]).to(cuda_device), torch.from_numpy(ref["T"]).to(cuda_device),
                  torch.from_numpy(ref["z"]).to(cuda_device), derivs=True)
    torch.cuda.synchronize()
    g = {k: v.cpu().numpy() for k, v in g.items()}
    two = np.flatnonzero(ref["lab"] == 0)
    assert (g["label"][two] == 0).all()
    worst, other, two = _rows_error(ref, d, g["x"], g["y"], g["Zl"], g["Zg"], g["dlnphi_dx"], g["dlnphi_dP"])
    drift = np.maximum(np.abs(g["x"].sum(axis=0) - 1), np.abs(g["y"].sum(axis=0) - 1))[two]
    print(f"flash outputs: worst {worst.max():.3e} of the block maximum, max |sum - 1| {drift.max():.2e}")
    assert (worst <= BAR + 10 * drift).all(), [(int(b), w, s) for b, w, s in zip(two, worst, drift) if w > BAR + 10 * s]
    assert other <= BAR
