/* Restated CPU oracle for the cubic-EOS flash (test infrastructure only).
 *
 * Plain C restatement of the reference simulator's flash arithmetic, used by
 * the tests and the bench's CPU-baseline leg to check the CUDA library.  Its
 * own parity is pinned against the reference compiled from source
 * (oracle/_ref/libosiris_ref.so): the flash outputs agree bit for bit.
 *
 * Array layout: per-cell scalars [n]; per-component fields [nc][n];
 * derivative blocks [2][nc][nc][n] (phase, i, k) and [2][nc][n] (phase, i),
 * phase 0 = liquid (oil), 1 = vapour (gas). */
#ifndef OSIRIS_FLASH_ORACLE_H
#define OSIRIS_FLASH_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_NC 16

typedef struct {
    int nc;
    int eos; /* 0 = Peng-Robinson, 1 = Soave-Redlich-Kwong */
    const double *tc, *pc, *acf; /* [nc]: K, Pa, - */
    const double *kij;           /* [nc*nc], symmetric, zero diagonal */
} orc_fluid;

double orc_solve_z(double a1, double a2, double a3, int gas);
void orc_eos_params(const orc_fluid *f, double T, double *a, double *b);

/* Flash n cells.  Optional outputs may be NULL.  iters receives the number of
 * successive-substitution iterations, rr_iters the total Rachford-Rice Newton
 * iterations.  Returns 0. */
int orc_flash_batch(const orc_fluid *f, long n, const double *P, const double *T, const double *z,
                    signed char *label, double *L, double *x, double *y, double *Zl, double *Zg,
                    int *iters, int *rr_iters);

/* Fugacity coefficients and their derivatives for one phase composition w at
 * pressure P and temperature T, with Z the phase's compressibility root:
 * lnphi[i], dlnphi_dx[i*nc+k] = d ln(phi_i)/d w_k (mole fractions treated as
 * independent, as in the reference's Jacobian), dlnphi_dP[i]. */
void orc_fugacity(const orc_fluid *f, double P, double T, const double *w, double Z, double *lnphi,
                  double *dlnphi_dx, double *dlnphi_dP);

/* Derivatives for n flashed cells (SoA), both phases: dlnphi_dx [2][nc][nc][n],
 * dlnphi_dP [2][nc][n]. */
int orc_flash_derivs_batch(const orc_fluid *f, long n, const double *P, const double *T, const double *x,
                           const double *y, const double *Zl, const double *Zg, double *dlnphi_dx,
                           double *dlnphi_dP);

/* Two-phase cells (label 0) of a flash result polished in place: Newton's
 * method on the equal-fugacity, material-balance and Rachford-Rice
 * equations to rounding, Zl and Zg recomputed.  Returns the number of cells
 * whose iteration did not settle (left unchanged). */
int orc_flash_polish(const orc_fluid *f, long n, const double *P, const double *T, const double *z,
                     const signed char *label, double *L, double *x, double *y, double *Zl, double *Zg);

/* Implicit-function adjoint of the flash: given cotangents xbar, ybar
 * [nc][n] and Lbar [n] on a flash result, kij_bar [nc*nc] (summed over the
 * cells) and optionally z_bar [nc][n] and P_bar [n].  One-phase cells pass
 * the present phase's cotangent to z and contribute nothing else.  Returns
 * the number of two-phase cells whose system was singular (skipped). */
int orc_flash_adjoint(const orc_fluid *f, long n, const double *P, const double *T, const double *z,
                      const signed char *label, const double *L, const double *x, const double *y, const double *Zl,
                      const double *Zg, const double *xbar, const double *ybar, const double *Lbar, double *kij_bar,
                      double *z_bar, double *P_bar);

#ifdef __cplusplus
}
#endif
#endif
