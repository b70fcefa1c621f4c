"""The adjoint system of the Newton step: J^T mu = c solved on the device
(osr_grid_ksp_solve_transpose: BiCGStab with the transposed product and the
transposed inverse diagonal blocks) at the Jacobian of one pass of the
reference's time step (InitGuess2, FormFunction, FormJacobian from the deck's
start-up state), against scipy's sparse solve of the device matrix
transposed: within 1e-8 of the largest entry of the solution."""
import os

import numpy as np
import pytest

import osiris_b200 as osr
from osiris_b200 import deck

pytestmark = pytest.mark.gpu

CASES = {
    "twophase_cdif0": lambda: deck.config_deck(nx=4, ny=4, nz=3, cdif=0.0, ipress=8e6, wells=False, seed=3),
    "twophase_diffusion": lambda: deck.config_deck(nx=4, ny=3, nz=3, cdif=None, ipress=8e6, wells=False, seed=8),
}
T_SIM = 0.0
KSP = dict(rtol=1e-13, max_it=4000)


def _pass(d, dev):
    """The pass from the deck's start-up state: grid, x0, J, dx, x1."""
    import torch
    G = osr.Grid(d)
    G.initialize(dev)
    G.set_controls(d.dt, 0.0)
    rows, _ = G.layout()
    x0 = torch.zeros(rows, dtype=torch.float64, device=dev)
    G.init_guess(x0)
    f = torch.zeros_like(x0)
    G.form_function(x0.clone(), f, T_SIM)
    J = G.alloc_jacobian(dev)
    assert G.jacobian(J, T_SIM) == 0
    dx = torch.zeros_like(x0)
    info = G.ksp_solve(J, f, dx, **KSP)
    assert info["reason"] in (2, 3), info
    return G, x0, J, dx, x0 - dx


@pytest.mark.parametrize("name", list(CASES))
def test_transposed_solve_matches_sparse_solve(name, tmp_path, cuda_device):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    import torch
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    G, x0, J, dx, _ = _pass(deck.parse_deck(path), cuda_device)
    n = len(x0)
    c = np.random.default_rng(3).standard_normal(n)
    mu = torch.zeros_like(x0)
    info = G.ksp_solve_transpose(J, torch.tensor(c, device=cuda_device), mu, **KSP)
    assert info["reason"] in (2, 3), info
    r, cc, v = G.jacobian_coo(J)
    A = sp.csr_matrix((v, (r, cc)), shape=(n, n))
    ref = spla.spsolve(A.T.tocsc(), c)
    err = np.abs(mu.cpu().numpy() - ref).max() / np.abs(ref).max()
    print(f"{name}: {info['its']} iterations, max error {err:.2e}")
    assert err <= 1e-8
