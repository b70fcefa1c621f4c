// PETSc SNES adapter over the osiris_b200 C ABI: the reference simulator's
// FormFunction / FormJacobian / InitGuess2 callbacks (compsim/PetscAUX.cpp:
// 59-173, 878-964) with the device doing the work.  Header-only; a host
// program that uses PETSc includes it after <petscsnes.h> (PETSc built with
// CUDA, so that VecCUDAGetArrayRead/Write and the COO assembly calls exist).
//
// Registration, as the reference's SolveNonLinear does it
// (compsim/PetscAUX.cpp:619-622):
//
//   osr_grid *g;  osr_create("test.dat", stream, &g);
//   OsrSnesCtx c{g};
//   OsrSetJacobianPattern(B, &c);           // after every row-layout change
//   SNESSetFunction(snes, r, OsrFormFunction, &c);
//   SNESSetJacobian(snes, B, B, OsrFormJacobian, &c);
//   SNESSetComputeInitialGuess(snes, OsrInitGuess, &c);
//   ... c.sim_time = SimulationTime before each SNESSolve ...
//
// The vectors need no permutation: row order, unknown order and the PCoeff
// scaling of the pressure unknown are the reference's (PJac,
// compsim/Init_Calcs.cpp:1013-1116).  B is a COO-assembled matrix (AIJ or
// AIJCUSPARSE); duplicates of a (row, column) pair are summed as the
// reference's MatSetValues(..., ADD_VALUES) sums them.  Its variable block
// sizes for PCVPBJACOBI (compsim/PetscAUX.cpp:147-163) come from the same
// row layout.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "osiris_b200.h"

#ifndef OSR_PETSC_CHECK
#define OSR_PETSC_CHECK(call)                 \
    do {                                      \
        PetscErrorCode osr_e_ = (call);       \
        if (osr_e_) return osr_e_;            \
    } while (0)
#endif
#ifndef OSR_PETSC_LIB_ERROR
#define OSR_PETSC_LIB_ERROR 76   /* PETSC_ERR_LIB */
#endif

struct OsrSnesCtx {
    osr_grid *g = nullptr;
    double sim_time = 0;          // SimulationTime of the step being solved
    void *stream = nullptr;       // cudaStream_t of the device work
    double *d_vals = nullptr;     // compact Jacobian values (device), nvals doubles
    long nvals = 0;
    osr_status last = OSR_OK;     // status of the last device call
};

// InitGuess2: the unknowns of the current state (PCoeff-scaled pressure).
inline PetscErrorCode OsrInitGuess(SNES, Vec x, void *ctx) {
    OsrSnesCtx *c = (OsrSnesCtx *)ctx;
    PetscScalar *dx = nullptr;
    OSR_PETSC_CHECK(VecCUDAGetArrayWrite(x, &dx));
    c->last = osr_grid_init_guess(c->g, dx, c->stream);
    OSR_PETSC_CHECK(VecCUDARestoreArrayWrite(x, &dx));
    return c->last == OSR_OK ? 0 : OSR_PETSC_LIB_ERROR;
}

// FormFunction: UpdateAll(x, false) with the property sweeps, then every
// residual row, on the device.
inline PetscErrorCode OsrFormFunction(SNES, Vec x, Vec f, void *ctx) {
    OsrSnesCtx *c = (OsrSnesCtx *)ctx;
    const PetscScalar *dx = nullptr;
    PetscScalar *df = nullptr;
    OSR_PETSC_CHECK(VecCUDAGetArrayRead(x, &dx));
    OSR_PETSC_CHECK(VecCUDAGetArrayWrite(f, &df));
    c->last = osr_grid_form_function(c->g, dx, df, c->sim_time, c->stream);
    OSR_PETSC_CHECK(VecCUDARestoreArrayWrite(f, &df));
    OSR_PETSC_CHECK(VecCUDARestoreArrayRead(x, &dx));
    return c->last == OSR_OK ? 0 : OSR_PETSC_LIB_ERROR;
}

// The COO pattern and the VPBJacobi block sizes of the current row layout;
// call once, and again after every phase change (osr_grid_refresh_layout).
inline PetscErrorCode OsrSetJacobianPattern(Mat B, OsrSnesCtx *c) {
    int bs = 0, entries = 0, ovf = 0, d[4] = {0, 0, 0, 0};
    if (osr_grid_jacobian_shape(c->g, &bs, &entries, &ovf) != OSR_OK || osr_grid_dims(c->g, d) != OSR_OK)
        return OSR_PETSC_LIB_ERROR;
    const long cells = (long)d[0] * d[1] * d[2];
    const long nvals = (2 * cells + 31) / 32 * 32 * (long)entries;   // values, chunked by 32 block rows
    if (nvals != c->nvals) {
        if (c->d_vals) cudaFree(c->d_vals);
        c->d_vals = nullptr;
        if (cudaMalloc((void **)&c->d_vals, (size_t)nvals * sizeof(double)) != cudaSuccess)
            return OSR_PETSC_LIB_ERROR;
        c->nvals = nvals;
    }
    long *d_row = nullptr, *d_col = nullptr;
    if (cudaMalloc((void **)&d_row, (size_t)nvals * sizeof(long)) != cudaSuccess ||
        cudaMalloc((void **)&d_col, (size_t)nvals * sizeof(long)) != cudaSuccess) {
        cudaFree(d_row);
        return OSR_PETSC_LIB_ERROR;
    }
    // -1 marks values the reference's matrix does not hold; COO ignores them
    c->last = osr_grid_jacobian_pattern(c->g, d_row, d_col, c->stream);
    std::vector<long> hr((size_t)nvals), hc((size_t)nvals);
    cudaStreamSynchronize((cudaStream_t)c->stream);
    cudaMemcpy(hr.data(), d_row, (size_t)nvals * sizeof(long), cudaMemcpyDeviceToHost);
    cudaMemcpy(hc.data(), d_col, (size_t)nvals * sizeof(long), cudaMemcpyDeviceToHost);
    cudaFree(d_row);
    cudaFree(d_col);
    if (c->last != OSR_OK) return OSR_PETSC_LIB_ERROR;
    std::vector<PetscInt> pi((size_t)nvals), pj((size_t)nvals);
    for (long k = 0; k < nvals; k++) {
        pi[(size_t)k] = (PetscInt)hr[(size_t)k];
        pj[(size_t)k] = (PetscInt)hc[(size_t)k];
    }
    OSR_PETSC_CHECK(MatSetPreallocationCOO(B, (PetscCount)nvals, pi.data(), pj.data()));
    // block sizes of PCVPBJACOBI: one block per cell-medium, 2N+4 rows when
    // two-phase, N+3 when one-phase (compsim/PetscAUX.cpp:160-163)
    std::vector<long> off((size_t)(2 * cells + 1));
    if (osr_grid_row_offsets(c->g, off.data()) != OSR_OK) return OSR_PETSC_LIB_ERROR;
    std::vector<PetscInt> bsz((size_t)(2 * cells));
    for (long b = 0; b < 2 * cells; b++) bsz[(size_t)b] = (PetscInt)(off[(size_t)b + 1] - off[(size_t)b]);
    OSR_PETSC_CHECK(MatSetVariableBlockSizes(B, (PetscInt)(2 * cells), bsz.data()));
    return 0;
}

// FormJacobian: UpdateAll(x, false) with the property sweeps, then every
// value of the matrix (each written once per call, zeros included, so no
// MatZeroEntries), handed to B through the COO pattern.
inline PetscErrorCode OsrFormJacobian(SNES, Vec x, Mat, Mat B, void *ctx) {
    OsrSnesCtx *c = (OsrSnesCtx *)ctx;
    const PetscScalar *dx = nullptr;
    OSR_PETSC_CHECK(VecCUDAGetArrayRead(x, &dx));
    c->last = osr_grid_form_jacobian(c->g, dx, c->sim_time, c->d_vals, c->stream);
    OSR_PETSC_CHECK(VecCUDARestoreArrayRead(x, &dx));
    if (c->last != OSR_OK) return OSR_PETSC_LIB_ERROR;
    cudaStreamSynchronize((cudaStream_t)c->stream);
    OSR_PETSC_CHECK(MatSetValuesCOO(B, c->d_vals, INSERT_VALUES));
    return 0;
}

inline void OsrSnesCtxRelease(OsrSnesCtx *c) {
    if (c->d_vals) cudaFree(c->d_vals);
    c->d_vals = nullptr;
    c->nvals = 0;
}
