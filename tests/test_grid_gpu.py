"""GPU parity of the grid path's property sweeps against the reference.

Each case writes a deck, loads it into the reference compiled from source
(oracle.RefDeck: Data_Input and the main program's initialisation), perturbs
the reference's own initial guess, unpacks it with the reference's UpdateAll
(which also runs its UpdateDependencies), and feeds the same unpacked state --
plus the densities of the previous update, from which the interfacial tension
is formed -- to osr_grid_update_dependencies.  Every property field of both
media is then compared.

Bar: |gpu - ref| <= 1e-9 |ref| + 1e-12 max|ref over the field plane|; the
absolute term covers values that cancel to rounding residue (a table
interpolation at its first node gives ~1e-18 instead of 0).  Upstream flags
(transS) must agree on interior faces except where the reference's phase
potential is within rounding of zero.
"""
import os

import numpy as np
import pytest

import oracle
import osiris_b200 as osr
from osiris_b200 import deck

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")]

FIELDS = ["P", "ift", "kr", "dkr", "pc", "rho", "mu", "dE", "pre", "diff", "gam", "trans", "wtran", "dwtran", "iftran"]

CASES = {
    "plain_20MPa_cdif0": lambda: deck.config_deck(cdif=0.0),
    "plain_8MPa_diffusion": lambda: deck.config_deck(cdif=None, ipress=8e6),
    "plain_12MPa_srk_like": lambda: deck.config_deck(cdif=0.0, ipress=12e6, seed=4),
    "sample_12MPa": lambda: deck.sample_deck(),
    "sample_6MPa": lambda: deck.sample_deck(ipress=6e6),
}


def _interior(R):
    c = np.arange(R.cells)
    ix, iy, iz = c % R.nx, (c // R.nx) % R.ny, c // (R.nx * R.ny)
    return np.stack([ix < R.nx - 1, iy < R.ny - 1, iz < R.nz - 1])


def _close(a, b):
    planes = b.reshape(-1, b.shape[-1]) if b.ndim > 1 else b[None]
    scale = np.abs(np.where(np.isfinite(planes), planes, 0)).max(axis=1, keepdims=True)
    a2 = a.reshape(planes.shape)
    ok = (np.abs(a2 - planes) <= 1e-9 * np.abs(planes) + 1e-12 * scale) | (np.isnan(a2) & np.isnan(planes))
    return ok


def load_case(tmp_path, name, seed=0, amp=0.01):
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    R = oracle.RefDeck(path)
    rho_prev = {m: R.get(f"{m}.rho") for m in "mf"}
    x0 = R.init_guess()
    rng = np.random.default_rng(seed)
    R.update_all(x0 * (1 + amp * rng.uniform(-1, 1, x0.shape)), False)
    G = osr.Grid(deck.parse_deck(path))
    for mi, m in enumerate("mf"):
        G.set_state(mi, R.get(f"{m}.P")[1], R.get(f"{m}.sat"), R.get(f"{m}.x"), R.get(f"{m}.y"), R.get(f"{m}.z"),
                    R.get(f"{m}.label"), rho_prev[m])
    return R, G


@pytest.mark.parametrize("name", list(CASES))
def test_property_sweeps_match_reference(name, tmp_path, cuda_device):
    R, G = load_case(tmp_path, name)
    G.update_dependencies()
    inter = _interior(R)
    report = []
    for m in "mf":
        for fld in FIELDS:
            a, b = G.get(f"{m}.{fld}"), R.get(f"{m}.{fld}")
            if fld == "trans":
                a, b = a[:, inter], b[:, inter]
            elif fld in ("wtran", "dwtran"):
                a, b = a[inter], b[inter]
            ok = _close(a, b)
            if not ok.all():
                report.append((f"{m}.{fld}", int((~ok).sum()), ok.size))
        sa, sb = G.get(f"{m}.transS")[:, inter], R.get(f"{m}.transS")[:, inter]
        agree = (sa == sb).mean()
        assert agree >= 0.99, (m, agree)
    assert not report, report

