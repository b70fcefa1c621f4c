"""CPU restatement of the reference's linear solve (test infrastructure only).

SolveNonLinear (compsim/PetscAUX.cpp:631-646) configures PETSc: SNESKSPONLY
(one linear solve per Newton step, x <- x - J^-1 F(x)), KSPBCGS with
PCVPBJACOBI over the PJac block sizes (FormJacobian's
MatSetVariableBlockSizes, compsim/PetscAUX.cpp:160-162) and the deck's
RELTOL / ABSTOL / DIVTOL / MAXITERS (defaults 1e-18, 1e-50, 1e3, 5000,
compsim/Data_Input.cpp:232-266).  PETSc is a third-party library the
reference links against and does not ship (no version is pinned in the
reference tree); its BiCGStab is restated here from the published algorithm
(van der Vorst 1992) in PETSc's left-preconditioned arrangement with the
KSPConvergedDefault test, as the device solver restates it.  Parity of the
device solve is anchored on the reference's own matrix and residual through
an exact sparse solve; this restatement pins the iteration semantics (reason
codes, iteration counts, iterates after a fixed number of steps).
"""
from __future__ import annotations

import numpy as np

CONVERGED_RTOL, CONVERGED_ATOL = 2, 3
DIVERGED_ITS, DIVERGED_DTOL, DIVERGED_BREAKDOWN, DIVERGED_NANORINF, DIVERGED_PC_FAILED = -3, -4, -5, -9, -11


def block_inverses(A, offsets):
    """Inverse of every diagonal block [offsets[i], offsets[i+1]) of the
    sparse matrix A (PCVPBJACOBI set-up); None when a block is singular."""
    A = A.tocsr()
    inv = []
    for lo, hi in zip(offsets[:-1], offsets[1:]):
        D = A[lo:hi, lo:hi].toarray()
        try:
            inv.append(np.linalg.inv(D))
        except np.linalg.LinAlgError:
            return None
    return inv


def _apply(inv, offsets, r):
    z = np.empty_like(r)
    for B, lo, hi in zip(inv, offsets[:-1], offsets[1:]):
        z[lo:hi] = B @ r[lo:hi]
    return z


def bcgs_vpbjacobi(A, b, offsets, rtol=1e-18, atol=1e-50, dtol=1e3, max_it=5000):
    """Left-preconditioned BiCGStab from x = 0.  Returns (x, reason, its,
    rnorm0, rnorm); reason is PETSc's KSPConvergedReason value."""
    A = A.tocsr()
    n = A.shape[0]
    x = np.zeros(n)
    inv = block_inverses(A, offsets)
    if inv is None:
        return x, DIVERGED_PC_FAILED, 0, np.nan, np.nan
    B = lambda v: _apply(inv, offsets, v)  # noqa: E731
    r = B(b)
    dp = float(np.sqrt(r @ r))
    rnorm0 = dp
    ttol = max(rtol * rnorm0, atol)

    def test(rn, its):
        if not np.isfinite(rn):
            return DIVERGED_NANORINF
        if rn <= ttol:
            return CONVERGED_ATOL if rn < atol else CONVERGED_RTOL
        if its > 0 and dtol > 0 and rn >= dtol * rnorm0:
            return DIVERGED_DTOL
        return 0

    reason = test(dp, 0)
    if reason:
        return x, reason, 0, rnorm0, dp
    rp = r.copy()
    p = np.zeros(n)
    v = np.zeros(n)
    rhoold = alpha = omegaold = 1.0
    its = 0
    while True:
        rho = float(r @ rp)
        beta = (rho / rhoold) * (alpha / omegaold)
        p = r + beta * p - omegaold * beta * v
        v = B(A @ p)
        d1 = float(v @ rp)
        if not np.isfinite(d1):
            return x, DIVERGED_NANORINF, its, rnorm0, dp
        if d1 == 0.0:
            return x, DIVERGED_BREAKDOWN, its, rnorm0, dp
        alpha = rho / d1
        s = r - alpha * v
        t = B(A @ s)
        d1, d2 = float(s @ t), float(t @ t)
        if d2 == 0.0:
            if float(s @ s) != 0.0:
                return x, DIVERGED_BREAKDOWN, its, rnorm0, dp
            x = x + alpha * p
            return x, CONVERGED_RTOL, its + 1, rnorm0, 0.0
        omega = d1 / d2
        x = x + alpha * p + omega * s
        r = s - omega * t
        dp = float(np.sqrt(r @ r))
        rhoold, omegaold = rho, omega
        its += 1
        reason = test(dp, its)
        if reason:
            return x, reason, its, rnorm0, dp
        if rho == 0.0:
            return x, DIVERGED_BREAKDOWN, its, rnorm0, dp
        if its >= max_it:
            return x, DIVERGED_ITS, its, rnorm0, dp
