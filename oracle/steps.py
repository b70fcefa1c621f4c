"""One pass of the reference's main loop on the CPU (test infrastructure only).

compsim/PrimeSim.cpp:93-104: SolveNonLinear (compsim/PetscAUX.cpp:566-731)
then TimeStepCtrl (compsim/Do_Time_Step.cpp:391-470).  Everything runs in the
reference compiled from source (InitGuess2, FormFunction, FormJacobian,
UpdateAll(x, true), CreateBackups, TimeStepCtrl with RestoreBackups and
PJac) except the linear solve: PETSc's KSP is not part of the reference, so
J dx = F is solved exactly (scipy's sparse LU); the device's iterative solve
converges to the same dx within the system's conditioning.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

TOLMAIN = 1e-2   # compsim/Functions.h:241


def ref_pass(R, t: float) -> dict:
    """One pass at simulation time t on the RefDeck R; returns the outcome
    and the new time."""
    x0 = R.init_guess()
    n = len(x0)
    f = R.form_function(x0, t)
    r, c, v = R.form_jacobian(x0, t)
    if np.isfinite(f).all() and np.isfinite(v).all():
        A = sp.csc_matrix((v, (r, c)), shape=(n, n))
        with np.errstate(all="ignore"):
            dx = spla.spsolve(A, f)
    else:
        # a non-finite system: PETSc's KSP ends with a NaN residual and the
        # reference rejects the pass on its NaN test; the sparse LU is not
        # asked to factor it
        dx = np.full(n, np.nan)
    vnorm = float(np.abs(dx).sum() / n)
    ok = bool(np.isfinite(vnorm) and vnorm <= TOLMAIN)
    if ok:
        R.update_all(x0 - dx, True)
        R.create_backups(t)
    flag, t_new = R.time_step_ctrl(t, rejected=not ok)
    return {"accepted": ok, "sim_time": t_new, "dt": R.scalar("Dt"), "finished": flag == 1, "vnorm": vnorm,
            "rows": n}
