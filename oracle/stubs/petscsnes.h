/* Minimal stand-in for PETSc's SNES/KSP/Vec/Mat headers, written for this
 * repository (test infrastructure only; see petscsys.h).  Vec and Mat are
 * concrete host structures defined in oracle/ref_shim.cpp: a Vec is a plain
 * array, a Mat collects (row, col, value) triplets with ADD semantics, which
 * is all the reference's residual and Jacobian callbacks need. */
#pragma once
#include "petscsys.h"

typedef struct _p_Vec *Vec;
typedef struct _p_Mat *Mat;
typedef struct _p_SNES *SNES;
typedef struct _p_KSP *KSP;
typedef struct _p_PC *PC;
typedef struct _p_VecScatter *VecScatter;
typedef struct _p_SNESLineSearch *SNESLineSearch;
typedef const char *SNESType;
typedef const char *KSPType;
typedef const char *PCType;
typedef const char *SNESLineSearchType;

typedef enum { SNES_CONVERGED_ITERATING = 0, SNES_CONVERGED_FNORM_ABS = 2, SNES_CONVERGED_ITS = 5,
               SNES_DIVERGED_FUNCTION_DOMAIN = -1 } SNESConvergedReason;
typedef enum { KSP_CONVERGED_ITERATING = 0, KSP_CONVERGED_RTOL = 2, KSP_CONVERGED_ATOL = 3,
               KSP_DIVERGED_ITS = -3 } KSPConvergedReason;
typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;
typedef enum { SCATTER_FORWARD = 0, SCATTER_REVERSE = 1 } ScatterMode;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { MAT_NEW_NONZERO_ALLOCATION_ERR = 19 } MatOption;
typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_INFINITY = 3 } NormType;

#define SNESKSPONLY "ksponly"
#define SNESNEWTONLS "newtonls"
#define SNESLINESEARCHBT "bt"
#define KSPBCGS "bcgs"
#define KSPGMRES "gmres"
#define PCVPBJACOBI "vpbjacobi"
#define PCMINIMALRESIDUAL "minimalresidual"

/* implemented by the shim */
PetscErrorCode VecGetArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecGetArray(Vec, PetscScalar **);
PetscErrorCode VecRestoreArray(Vec, PetscScalar **);
PetscErrorCode VecGetOwnershipRange(Vec, PetscInt *, PetscInt *);
PetscErrorCode MatSetValues(Mat, PetscInt, const PetscInt *, PetscInt, const PetscInt *, const PetscScalar *, InsertMode);
PetscErrorCode MatZeroEntries(Mat);

/* accepted and ignored by the shim (outside the hot path) */
PetscErrorCode VecCreateMPI(MPI_Comm, PetscInt, PetscInt, Vec *);
PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt, Vec *);
PetscErrorCode VecDuplicate(Vec, Vec *);
PetscErrorCode VecDestroy(Vec *);
PetscErrorCode VecAssemblyBegin(Vec);
PetscErrorCode VecAssemblyEnd(Vec);
PetscErrorCode VecNorm(Vec, NormType, PetscReal *);
PetscErrorCode VecScatterCreateToAll(Vec, VecScatter *, Vec *);
PetscErrorCode VecScatterBegin(VecScatter, Vec, Vec, InsertMode, ScatterMode);
PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode);
PetscErrorCode VecScatterDestroy(VecScatter *);
PetscErrorCode MatCreateAIJ(MPI_Comm, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, const PetscInt *, PetscInt, const PetscInt *, Mat *);
PetscErrorCode MatSetOption(Mat, MatOption, PetscBool);
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType);
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType);
PetscErrorCode MatSetVariableBlockSizes(Mat, PetscInt, PetscInt *);
PetscErrorCode MatDestroy(Mat *);
PetscErrorCode SNESCreate(MPI_Comm, SNES *);
PetscErrorCode SNESDestroy(SNES *);
PetscErrorCode SNESSetFunction(SNES, Vec, PetscErrorCode (*)(SNES, Vec, Vec, void *), void *);
PetscErrorCode SNESSetJacobian(SNES, Mat, Mat, PetscErrorCode (*)(SNES, Vec, Mat, Mat, void *), void *);
PetscErrorCode SNESSetComputeInitialGuess(SNES, PetscErrorCode (*)(SNES, Vec, void *), void *);
PetscErrorCode SNESSetType(SNES, SNESType);
PetscErrorCode SNESSetTolerances(SNES, PetscReal, PetscReal, PetscReal, PetscInt, PetscInt);
PetscErrorCode SNESSetFromOptions(SNES);
PetscErrorCode SNESGetKSP(SNES, KSP *);
PetscErrorCode SNESGetLineSearch(SNES, SNESLineSearch *);
PetscErrorCode SNESLineSearchSetType(SNESLineSearch, SNESLineSearchType);
PetscErrorCode SNESLineSearchSetFromOptions(SNESLineSearch);
PetscErrorCode SNESSolve(SNES, Vec, Vec);
PetscErrorCode SNESGetConvergedReason(SNES, SNESConvergedReason *);
PetscErrorCode SNESGetIterationNumber(SNES, PetscInt *);
PetscErrorCode SNESGetSolutionUpdate(SNES, Vec *);
PetscErrorCode KSPSetType(KSP, KSPType);
PetscErrorCode KSPSetTolerances(KSP, PetscReal, PetscReal, PetscReal, PetscInt);
PetscErrorCode KSPGetPC(KSP, PC *);
PetscErrorCode KSPGetConvergedReason(KSP, KSPConvergedReason *);
PetscErrorCode KSPGetIterationNumber(KSP, PetscInt *);
PetscErrorCode PCSetType(PC, PCType);
