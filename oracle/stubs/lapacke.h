/* Minimal stand-in for lapacke.h (test infrastructure only).  The shim
 * provides LAPACKE_dgesv as a partial-pivoting LU solve (column-major, one
 * or more right-hand sides); it differs from a tuned LAPACK only by rounding. */
#pragma once
#define LAPACK_COL_MAJOR 102
#define LAPACK_ROW_MAJOR 101
typedef int lapack_int;
lapack_int LAPACKE_dgesv(int layout, lapack_int n, lapack_int nrhs, double *a, lapack_int lda,
                         lapack_int *ipiv, double *b, lapack_int ldb);
