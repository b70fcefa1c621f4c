/* The CUDA-vector and COO-assembly calls of PETSc that the osiris_b200
 * adapter (include/osiris_b200_petsc.hpp) makes, over the oracle's
 * PETSc-lite Vec (a host array) and Mat (a triplet list with ADD semantics).
 * Test infrastructure only: the boundary test compiles the adapter against
 * these and compares what reaches the Vec and Mat with the reference's own
 * callbacks. */
#pragma once
#include <cstddef>
#include <petscsnes.h>

typedef std::ptrdiff_t PetscCount;

PetscErrorCode VecCUDAGetArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecCUDARestoreArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecCUDAGetArrayWrite(Vec, PetscScalar **);
PetscErrorCode VecCUDARestoreArrayWrite(Vec, PetscScalar **);
PetscErrorCode MatSetPreallocationCOO(Mat, PetscCount, PetscInt *, PetscInt *);
PetscErrorCode MatSetValuesCOO(Mat, const PetscScalar *, InsertMode);
