"""GPU parity of the device linear solve (osr_grid_jacobian_apply,
osr_grid_ksp_solve) -- the KSPSolve of the reference's SolveNonLinear
(compsim/PetscAUX.cpp:631-698: KSPBCGS, PCVPBJACOBI, RELTOL 1e-18, ABSTOL
1e-50, DIVTOL 1e3, MAXITERS 5000).

* MatMult: J v on the device's compact Jacobian against the reference's own
  assembled matrix (its MatSetValues triplets) times the same v, per row
  within 1e-12 of sum_j |J_ij v_j|.
* Solve: the device solution of J dx = F at a perturbed state against an
  exact sparse solve of the reference's own J and F (scipy spsolve), within
  1e-7 of |dx|_inf.
* Iteration semantics: the device solver and the CPU restatement
  (oracle/linear.py) on the device's matrix reach the same PETSc reason with
  iteration counts within 10 % (+3), and agree on the iterate after a fixed
  small number of iterations (DIVERGED_ITS) to 1e-9; a zero right-hand side
  converges at iteration 0 with reason CONVERGED_ATOL and a zero solution.
Decks without wells' 0/0 diagonal entries (the all-well-types decks carry
NaN in the reference's own matrix).
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle
import osiris_b200 as osr
from oracle import linear
from osiris_b200 import deck

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")]

G_, O_ = (0.9, 0.07, 0.03), (0.5, 0.2, 0.3)
_ST = {-1: (8e6, G_), 1: (2e7, O_), 0: (8e6, O_)}
_PAIRS = [(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1)]

CASES = {
    "state_pairs_cdif0_wells": lambda: deck.config_deck(
        nx=2, ny=3, nz=9, ipress=[_ST[a][0] for a, _ in _PAIRS], igc=[_ST[a][1] for a, _ in _PAIRS],
        fipress=[_ST[b][0] for _, b in _PAIRS], figc=[_ST[b][1] for _, b in _PAIRS], wells=True, cdif=0.0),
    "sample_12MPa": lambda: deck.sample_deck(),
    "twophase_diffusion_wells": lambda: deck.config_deck(nx=5, ny=4, nz=3, cdif=None, ipress=8e6),
    "twophase_cdif0_no_wells": lambda: deck.config_deck(nx=4, ny=3, nz=3, cdif=0.0, ipress=8e6, wells=False),
}
T = 3600.0


def setup_case(tmp_path, name, device):
    import torch
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, CASES[name]())
    R = oracle.RefDeck(path)
    G = osr.Grid(deck.parse_deck(path))
    for mi, m in enumerate("mf"):
        G.set_state(mi, R.get(f"{m}.P")[1], R.get(f"{m}.sat"), R.get(f"{m}.x"), R.get(f"{m}.y"), R.get(f"{m}.z"),
                    R.get(f"{m}.label"), R.get(f"{m}.rho"))
    n, _ = G.refresh_layout()
    x0 = R.init_guess()
    xp = x0 * (1 + 1e-3 * np.random.default_rng(3).uniform(-1, 1, x0.shape))
    d_x = torch.tensor(xp, device=device)
    d_f = torch.zeros(n, dtype=torch.float64, device=device)
    G.form_function(d_x, d_f, T)
    J = G.alloc_jacobian(device)
    assert G.jacobian(J, T) == 0
    torch.cuda.synchronize()
    return R, G, n, xp, d_f, J


def ref_system(R, xp, n):
    f = R.form_function(xp, T)
    r, c, v = R.form_jacobian(xp, T)
    return sp.csr_matrix((v, (r, c)), shape=(n, n)), f


@pytest.mark.parametrize("name", list(CASES))
def test_matmult_matches_reference_matrix(name, tmp_path, cuda_device):
    import torch
    R, G, n, xp, _, J = setup_case(tmp_path, name, cuda_device)
    A, _ = ref_system(R, xp, n)
    v = np.random.default_rng(4).uniform(-1, 1, n)
    y = torch.zeros(n, dtype=torch.float64, device=cuda_device)
    G.jacobian_apply(J, torch.tensor(v, device=cuda_device), y)
    torch.cuda.synchronize()
    y = y.cpu().numpy()
    yr = A @ v
    scale = abs(A) @ np.abs(v)
    bad = ~(np.abs(y - yr) <= 1e-12 * scale + 1e-300)
    assert not bad.any(), (int(bad.sum()), [(int(i), y[i], yr[i]) for i in np.nonzero(bad)[0][:6]])


@pytest.mark.parametrize("name", list(CASES))
def test_solve_matches_exact_solution_of_reference_system(name, tmp_path, cuda_device):
    import torch
    R, G, n, xp, d_f, J = setup_case(tmp_path, name, cuda_device)
    A, f = ref_system(R, xp, n)
    dx_ref = spla.spsolve(A.tocsc(), f)
    d_dx = torch.full((n,), float("nan"), dtype=torch.float64, device=cuda_device)
    info = G.ksp_solve(J, d_f, d_dx)
    dx = d_dx.cpu().numpy()
    assert info["reason"] in (linear.CONVERGED_RTOL, linear.CONVERGED_ATOL), info
    err = np.abs(dx - dx_ref).max() / np.abs(dx_ref).max()
    assert err <= 1e-7, (err, info)


@pytest.mark.parametrize("name", ["state_pairs_cdif0_wells", "twophase_diffusion_wells"])
def test_iteration_semantics_match_restatement(name, tmp_path, cuda_device):
    import torch
    R, G, n, xp, d_f, J = setup_case(tmp_path, name, cuda_device)
    r, c, v = G.jacobian_coo(J)
    A = sp.csr_matrix((v, (r, c)), shape=(n, n))
    f = d_f.cpu().numpy()
    offs = G.row_offsets()
    d_dx = torch.zeros(n, dtype=torch.float64, device=cuda_device)
    info = G.ksp_solve(J, d_f, d_dx)
    x_np, reason, its, r0, _ = linear.bcgs_vpbjacobi(A, f, offs)
    assert info["reason"] == reason, (info, reason, its)
    assert abs(info["its"] - its) <= max(3, 0.1 * its), (info, its)
    assert abs(info["rnorm0"] - r0) <= 1e-12 * r0
    # a fixed number of iterations: the iterates agree
    for k in (1, 4):
        info = G.ksp_solve(J, d_f, d_dx, max_it=k, check_every=1)
        x_np, reason, its, _, _ = linear.bcgs_vpbjacobi(A, f, offs, max_it=k)
        assert (info["reason"], info["its"]) == (reason, its) == (linear.DIVERGED_ITS, k)
        x = d_dx.cpu().numpy()
        assert np.abs(x - x_np).max() <= 1e-9 * np.abs(x_np).max(), k
    # the whole solve as one graph (the cap a whole number of 8-iteration
    # batches) and the host-driven batches (a cap that is not) run the same
    # kernels in the same order: identical iterates
    info_g = G.ksp_solve(J, d_f, d_dx, max_it=5000)
    xg = d_dx.clone()
    info_h = G.ksp_solve(J, d_f, d_dx, max_it=4999)
    assert (info_g["reason"], info_g["its"]) == (info_h["reason"], info_h["its"])
    assert torch.equal(xg, d_dx)
    # zero right-hand side
    info = G.ksp_solve(J, torch.zeros_like(d_f), d_dx)
    assert (info["reason"], info["its"], info["rnorm0"]) == (linear.CONVERGED_ATOL, 0, 0.0)
    assert not d_dx.any()


def test_matmult_large_grid_form(tmp_path, cuda_device):
    """Grids of at least 148 x 2048 block rows use the two-lane-per-block-row
    product: on 64x64x37 (303,104 block rows, the device start-up state of
    the plain case) J v must match the host product of the same values placed
    by the pattern, per row within 1e-12 of sum_j |J_ij v_j|."""
    import torch
    path = os.path.join(str(tmp_path), "large.dat")
    deck.write_deck(path, deck.config_deck(nx=64, ny=64, nz=37, cdif=0.0))
    G = osr.Grid(deck.parse_deck(path))
    G.initialize(cuda_device)
    n, _ = G.layout()
    assert 2 * G.cells >= 148 * 2048
    J = G.alloc_jacobian(cuda_device)
    assert G.jacobian(J, T) == 0
    v = np.random.default_rng(6).uniform(-1, 1, n)
    y = torch.zeros(n, dtype=torch.float64, device=cuda_device)
    G.jacobian_apply(J, torch.tensor(v, device=cuda_device), y)
    torch.cuda.synchronize()
    y = y.cpu().numpy()
    r, c, vals = G.jacobian_coo(J)
    prod = vals * v[c]
    yr = np.bincount(r, weights=prod, minlength=n)
    scale = np.bincount(r, weights=np.abs(prod), minlength=n)
    bad = ~(np.abs(y - yr) <= 1e-12 * scale + 1e-300)
    assert not bad.any(), (int(bad.sum()), [(int(i), y[i], yr[i]) for i in np.nonzero(bad)[0][:6]])
