/* Minimal stand-in for the PETSc system header, written for this repository.
 * Test infrastructure only: it lets the reference simulator's sources compile
 * unmodified as a CPU oracle.  Only the types, constants and functions those
 * sources name are declared; oracle/ref_shim.cpp implements the handful that
 * the hot path really calls (vector array access, MatSetValues, barriers) and
 * turns the rest into no-ops. */
#pragma once
#include <cstdio>
#include <cstring>
#include <cmath>
#include <cstdlib>

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscBool;
typedef int MPI_Comm;

#define PETSC_COMM_WORLD 0
#define PETSC_COMM_SELF 1
#define PETSC_FALSE 0
#define PETSC_TRUE 1
#define PETSC_DECIDE (-1)
#define PETSC_DEFAULT (-2)
#define PETSC_DETERMINE (-1)
#define PETSC_NULL 0

#define CHKERRQ(e) do { if (e) return (e); } while (0)

typedef struct _p_PetscObject *PetscObject;

PetscErrorCode PetscBarrier(PetscObject);
PetscErrorCode PetscOptionsSetValue(void *, const char *, const char *);
PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *);
PetscErrorCode PetscFinalize(void);
PetscErrorCode PetscPrintf(MPI_Comm, const char *, ...);
