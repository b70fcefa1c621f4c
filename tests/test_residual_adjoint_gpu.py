"""The residual's adjoint with respect to the matrix continuum's per-cell
log-permeability (osr_grid_residual_logk_vjp) against central finite
differences of the device residual.

For seeded directions v over the matrix cells, the grid is rebuilt from the
deck with k_x, k_y, k_z of every matrix cell scaled by exp(+-h v_c)
(h = 1e-6), brought to the same start-up state, and the residual formed at
the same perturbed unknowns; (lambda . F(+h) - lambda . F(-h)) / 2h must
equal gk . v within 1e-6 relative, for a seeded lambda.  Decks: two-phase
layers with and without diffusive transfer, every matrix/fracture state
pairing, no wells (well productivity indices are held fixed by the
product).  The product is also deterministic and independent of lambda on
rows it does not reach (the fugacity and constraint rows)."""
import os

import numpy as np
import pytest

import osiris_b200 as osr
from osiris_b200 import deck

pytestmark = pytest.mark.gpu

G_, O_ = (0.9, 0.07, 0.03), (0.5, 0.2, 0.3)
_ST = {-1: (8e6, G_), 1: (2e7, O_), 0: (8e6, O_)}
_PAIRS = [(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1)]

CASES = {
    "twophase_cdif0": lambda: deck.config_deck(nx=5, ny=4, nz=3, cdif=0.0, ipress=8e6, wells=False, seed=3),
    "twophase_diffusion": lambda: deck.config_deck(nx=4, ny=4, nz=3, cdif=None, ipress=8e6, wells=False, seed=8),
    "state_pairs": lambda: deck.config_deck(
        nx=2, ny=3, nz=9, ipress=[_ST[a][0] for a, _ in _PAIRS], igc=[_ST[a][1] for a, _ in _PAIRS],
        fipress=[_ST[b][0] for _, b in _PAIRS], figc=[_ST[b][1] for _, b in _PAIRS], cdif=None, wells=False),
}
H = 1e-6
T_SIM = 3600.0


def _grid(d, dev):
    G = osr.Grid(d)
    G.initialize(dev)
    return G


def _residual(G, xp, dev):
    import torch
    f = torch.zeros(len(xp), dtype=torch.float64, device=dev)
    G.form_function(torch.tensor(xp, device=dev), f, T_SIM)
    torch.cuda.synchronize()
    return f.cpu().numpy()


@pytest.mark.parametrize("name", list(CASES))
def test_logk_vjp_matches_central_differences(name, tmp_path, cuda_device):
    import copy
    import torch
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    d = deck.parse_deck(path)
    G = _grid(d, cuda_device)
    rows, _ = G.layout()
    x0 = torch.zeros(rows, dtype=torch.float64, device=cuda_device)
    G.init_guess(x0)
    rng = np.random.default_rng(11)
    xp = x0.cpu().numpy() * (1 + 1e-3 * rng.uniform(-1, 1, rows))
    _residual(G, xp, cuda_device)
    lam = torch.tensor(rng.standard_normal(rows), device=cuda_device)
    gk = torch.empty(d.cells, dtype=torch.float64, device=cuda_device)
    G.residual_logk_vjp(lam, gk, T_SIM)
    gk2 = torch.empty_like(gk)
    G.residual_logk_vjp(lam, gk2, T_SIM)
    torch.cuda.synchronize()
    assert torch.equal(gk, gk2)
    g = gk.cpu().numpy()
    lamh = lam.cpu().numpy()
    worst = 0.0
    for _ in range(6):
        v = rng.standard_normal(d.cells)
        fs = []
        for sgn in (1, -1):
            dd = copy.deepcopy(d)
            dd.perm = d.perm * np.exp(sgn * H * v)[None, :]
            Gs = _grid(dd, cuda_device)
            assert Gs.layout()[0] == rows
            fs.append(_residual(Gs, xp, cuda_device))
            Gs.close()
        fd = float(lamh @ (fs[0] - fs[1])) / (2 * H)
        ad = float(g @ v)
        err = abs(ad - fd) / abs(fd)
        worst = max(worst, err)
        assert err <= 1e-6, (ad, fd, err)
    print(f"{name}: 6 directions, worst relative difference from central differences {worst:.2e}")
