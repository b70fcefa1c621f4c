/* PETSc-lite shim for the CPU oracle (test infrastructure only).
 *
 * The reference simulator is compiled unmodified from its own sources against
 * the stub headers in oracle/stubs/.  This file supplies the few PETSc, MPI
 * and LAPACKE symbols those sources link against:
 *   - Vec: a host array owned by the caller of the oracle driver;
 *   - Mat: a triplet list with ADD_VALUES semantics (MatSetValues), which is
 *     what the reference's IteratorJacobian writes through
 *     (compsim/Petsc_Functions.cpp:42065);
 *   - LAPACKE_dgesv: partial-pivoting LU, the dense solve behind MKLS
 *     (compsim/MKL_Solver.Cpp:66-90) used by the saturation-pressure Newton
 *     fallback and the interface-equilibrium Newton;
 *   - everything else (solver set-up, options, barriers): no-ops.
 * Nothing here is part of the product; only tests, smoke() and the bench's
 * CPU-baseline leg load the library built from it. */
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <vector>
#include "petscsnes.h"
#include "mpi.h"
#include "lapacke.h"

#include "shim_types.h"

/* The stub headers declare these with C++ linkage (the reference includes
 * them from C++ translation units), so they are defined with C++ linkage. */
PetscErrorCode VecGetArrayRead(Vec x, const PetscScalar **a) { *a = x->a; return 0; }
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar **) { return 0; }
PetscErrorCode VecGetArray(Vec x, PetscScalar **a) { *a = x->a; return 0; }
PetscErrorCode VecRestoreArray(Vec, PetscScalar **) { return 0; }
PetscErrorCode VecGetOwnershipRange(Vec x, PetscInt *lo, PetscInt *hi) { *lo = 0; *hi = x->n; return 0; }

PetscErrorCode MatSetValues(Mat m, PetscInt nr, const PetscInt *rows, PetscInt nc, const PetscInt *cols,
                            const PetscScalar *vals, InsertMode) {
    for (int i = 0; i < nr; i++)
        for (int j = 0; j < nc; j++) {
            m->r.push_back(rows[i]);
            m->c.push_back(cols[j]);
            m->v.push_back(vals[i * nc + j]);
        }
    return 0;
}
PetscErrorCode MatZeroEntries(Mat m) { m->r.clear(); m->c.clear(); m->v.clear(); return 0; }

PetscErrorCode PetscBarrier(PetscObject) { return 0; }
PetscErrorCode PetscOptionsSetValue(void *, const char *, const char *) { return 0; }
PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *) { return 0; }
PetscErrorCode PetscFinalize(void) { return 0; }
PetscErrorCode PetscPrintf(MPI_Comm, const char *, ...) { return 0; }

PetscErrorCode VecCreateMPI(MPI_Comm, PetscInt, PetscInt, Vec *) { return 0; }
PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt, Vec *) { return 0; }
PetscErrorCode VecDuplicate(Vec, Vec *) { return 0; }
PetscErrorCode VecDestroy(Vec *) { return 0; }
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
PetscErrorCode VecNorm(Vec, NormType, PetscReal *r) { *r = 0; return 0; }
PetscErrorCode VecScatterCreateToAll(Vec, VecScatter *, Vec *) { return 0; }
PetscErrorCode VecScatterBegin(VecScatter, Vec, Vec, InsertMode, ScatterMode) { return 0; }
PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode) { return 0; }
PetscErrorCode VecScatterDestroy(VecScatter *) { return 0; }
PetscErrorCode MatCreateAIJ(MPI_Comm, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, const PetscInt *, PetscInt,
                            const PetscInt *, Mat *) { return 0; }
PetscErrorCode MatSetOption(Mat, MatOption, PetscBool) { return 0; }
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatSetVariableBlockSizes(Mat, PetscInt, PetscInt *) { return 0; }
PetscErrorCode MatDestroy(Mat *) { return 0; }
PetscErrorCode SNESCreate(MPI_Comm, SNES *) { return 0; }
PetscErrorCode SNESDestroy(SNES *) { return 0; }
PetscErrorCode SNESSetFunction(SNES, Vec, PetscErrorCode (*)(SNES, Vec, Vec, void *), void *) { return 0; }
PetscErrorCode SNESSetJacobian(SNES, Mat, Mat, PetscErrorCode (*)(SNES, Vec, Mat, Mat, void *), void *) { return 0; }
PetscErrorCode SNESSetComputeInitialGuess(SNES, PetscErrorCode (*)(SNES, Vec, void *), void *) { return 0; }
PetscErrorCode SNESSetType(SNES, SNESType) { return 0; }
PetscErrorCode SNESSetTolerances(SNES, PetscReal, PetscReal, PetscReal, PetscInt, PetscInt) { return 0; }
PetscErrorCode SNESSetFromOptions(SNES) { return 0; }
PetscErrorCode SNESGetKSP(SNES, KSP *) { return 0; }
PetscErrorCode SNESGetLineSearch(SNES, SNESLineSearch *) { return 0; }
PetscErrorCode SNESLineSearchSetType(SNESLineSearch, SNESLineSearchType) { return 0; }
PetscErrorCode SNESLineSearchSetFromOptions(SNESLineSearch) { return 0; }
PetscErrorCode SNESSolve(SNES, Vec, Vec) { return 0; }
PetscErrorCode SNESGetConvergedReason(SNES, SNESConvergedReason *r) { *r = SNES_CONVERGED_ITS; return 0; }
PetscErrorCode SNESGetIterationNumber(SNES, PetscInt *n) { *n = 1; return 0; }
PetscErrorCode SNESGetSolutionUpdate(SNES, Vec *) { return 0; }
PetscErrorCode KSPSetType(KSP, KSPType) { return 0; }
PetscErrorCode KSPSetTolerances(KSP, PetscReal, PetscReal, PetscReal, PetscInt) { return 0; }
PetscErrorCode KSPGetPC(KSP, PC *) { return 0; }
PetscErrorCode KSPGetConvergedReason(KSP, KSPConvergedReason *r) { *r = KSP_CONVERGED_RTOL; return 0; }
PetscErrorCode KSPGetIterationNumber(KSP, PetscInt *n) { *n = 1; return 0; }
PetscErrorCode PCSetType(PC, PCType) { return 0; }

int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
int MPI_Gather(const void *, int, MPI_Datatype, void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }

/* Column-major LU with partial pivoting, overwriting a with the factors and b
 * with the solution; returns k>0 when U(k,k) is exactly zero (LAPACK's info). */
lapack_int LAPACKE_dgesv(int, lapack_int n, lapack_int nrhs, double *a, lapack_int lda, lapack_int *ipiv, double *b,
                         lapack_int ldb) {
    lapack_int info = 0;
    for (int k = 0; k < n; k++) {
        int p = k;
        double best = fabs(a[k + k * lda]);
        for (int i = k + 1; i < n; i++) {
            double v = fabs(a[i + k * lda]);
            if (v > best) { best = v; p = i; }
        }
        ipiv[k] = p + 1;
        if (a[p + k * lda] == 0.0) { if (!info) info = k + 1; continue; }
        if (p != k) {
            for (int j = 0; j < n; j++) { double t = a[k + j * lda]; a[k + j * lda] = a[p + j * lda]; a[p + j * lda] = t; }
            for (int j = 0; j < nrhs; j++) { double t = b[k + j * ldb]; b[k + j * ldb] = b[p + j * ldb]; b[p + j * ldb] = t; }
        }
        double piv = a[k + k * lda];
        for (int i = k + 1; i < n; i++) {
            double l = a[i + k * lda] / piv;
            a[i + k * lda] = l;
            for (int j = k + 1; j < n; j++) a[i + j * lda] -= l * a[k + j * lda];
            for (int j = 0; j < nrhs; j++) b[i + j * ldb] -= l * b[k + j * ldb];
        }
    }
    if (info) return info;
    for (int j = 0; j < nrhs; j++)
        for (int i = n - 1; i >= 0; i--) {
            double s = b[i + j * ldb];
            for (int k = i + 1; k < n; k++) s -= a[i + k * lda] * b[k + j * ldb];
            b[i + j * ldb] = s / a[i + i * lda];
        }
    return 0;
}
