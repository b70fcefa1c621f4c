"""The C ABI driven from a compiled C++ program (tests/cpp/boundary_test.cpp,
built by tests/cpp/Makefile): the reference's own Data_Input start-up,
InitGuess2, FormFunction and FormJacobian against osr_create and the PETSc
adapter of include/osiris_b200_petsc.hpp (OsrInitGuess, OsrFormFunction,
OsrSetJacobianPattern, OsrFormJacobian) on the oracle's PETSc-lite Vec and
Mat.  Row layout and the VPBJacobi block sizes identical; unknowns from
InitGuess2 within 1e-9 (the two start-ups flash independently); at the same
perturbed unknowns, residual rows within 1e-10 of the row's |terms| and
Jacobian entries within 1e-9 of the reference row's largest entry.  Decks: two-phase layers with diffusion and
wells, every matrix/fracture state pairing, all nine well types, the
reference's sample deck.
"""
import os
import subprocess

import pytest

import oracle
from osiris_b200 import deck

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.ref_available(), reason="reference library missing")]

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp")
G_, O_ = (0.9, 0.07, 0.03), (0.5, 0.2, 0.3)
_ST = {-1: (8e6, G_), 1: (2e7, O_), 0: (8e6, O_)}
_PAIRS = [(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1)]

DECKS = {
    "twophase_diffusion_wells": lambda: deck.config_deck(nx=5, ny=4, nz=3, cdif=None, ipress=8e6),
    "state_pairs": lambda: deck.config_deck(
        nx=2, ny=3, nz=9, ipress=[_ST[a][0] for a, _ in _PAIRS], igc=[_ST[a][1] for a, _ in _PAIRS],
        fipress=[_ST[b][0] for _, b in _PAIRS], figc=[_ST[b][1] for _, b in _PAIRS], cdif=0.0, wells=True),
    "all_well_types_9MPa": lambda: deck.all_wells_deck(),
    "sample_12MPa": lambda: deck.sample_deck(),
}


@pytest.fixture(scope="module")
def boundary_binary():
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return os.path.join(HERE, "_build", "boundary_test")


@pytest.mark.parametrize("name", list(DECKS))
def test_cpp_caller_matches_reference_callbacks(name, boundary_binary, tmp_path, cuda_device):
    path = os.path.join(str(tmp_path), name + ".dat")
    deck.write_deck(path, DECKS[name]())
    r = subprocess.run([boundary_binary, path], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert ": ok" in r.stdout
