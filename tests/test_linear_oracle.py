"""The CPU restatement of the reference's linear solve (oracle/linear.py):
BiCGStab + variable-point-block Jacobi against a direct solve, and PETSc's
reason codes on the edge cases.  CPU only."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import linear


def _system(seed=0, blocks=(20, 11, 20, 11, 20)):
    rng = np.random.default_rng(seed)
    offs = np.concatenate([[0], np.cumsum(blocks)])
    n = offs[-1]
    A = sp.random(n, n, density=0.05, random_state=seed, format="lil")
    for lo, hi in zip(offs[:-1], offs[1:]):
        A[lo:hi, lo:hi] = rng.standard_normal((hi - lo, hi - lo)) + 8 * np.eye(hi - lo)
    return A.tocsr(), rng.standard_normal(n), offs


def test_converges_to_direct_solution():
    A, b, offs = _system()
    x, reason, its, r0, rn = linear.bcgs_vpbjacobi(A, b, offs, rtol=1e-14)
    assert reason == linear.CONVERGED_RTOL and 0 < its < 200
    xd = spla.spsolve(A.tocsc(), b)
    assert np.abs(x - xd).max() <= 1e-10 * np.abs(xd).max()
    assert rn <= 1e-14 * r0


def test_zero_rhs_converges_at_iteration_zero():
    A, b, offs = _system(1)
    x, reason, its, r0, rn = linear.bcgs_vpbjacobi(A, 0 * b, offs)
    assert (reason, its, r0) == (linear.CONVERGED_ATOL, 0, 0.0) and not x.any()


def test_iteration_cap():
    A, b, offs = _system(2)
    x, reason, its, _, _ = linear.bcgs_vpbjacobi(A, b, offs, max_it=3)
    assert (reason, its) == (linear.DIVERGED_ITS, 3)


def test_singular_block_fails_the_preconditioner():
    A, b, offs = _system(3)
    A = A.tolil()
    A[0, :] = 0
    _, reason, its, _, _ = linear.bcgs_vpbjacobi(A.tocsr(), b, offs)
    assert (reason, its) == (linear.DIVERGED_PC_FAILED, 0)
