/* Restated CPU oracle for the cubic-EOS flash (test infrastructure only).
 *
 * Each function restates one piece of the reference simulator's arithmetic,
 * in the same operation order, so that compiled with the same flags (no
 * fused multiply-add) it reproduces the reference's results bit for bit; the
 * tests pin that against oracle/_ref/libosiris_ref.so.  It is never linked
 * into, or called by, the CUDA library.
 *
 * Constants follow compsim/Functions.h:196-289 (RGAS, SQRT2, PI,
 * NEWTON_TOL, FLASH_TOL, DZERO, MAX_FLASH_N_ITR). */
#include <math.h>
#include <string.h>
#include "flash_oracle.h"

#define R_GAS 8.3144621
#define SQRT_2 1.4142135623730950488016887
#define PI_C 3.1415926535897932384626433
#define RR_TOL 1e-8      /* NEWTON_TOL */
#define SS_TOL 1e-14     /* FLASH_TOL */
#define L_ZERO 1e-20     /* DZERO */
#define RR_MAXIT 100     /* MAX_FLASH_N_ITR */
#define SS_MAXIT 500     /* hard-coded cap, compsim/Init_Calcs.cpp:714 */

/* Cubic Z^3 + a1 Z^2 + a2 Z + a3 = 0: trigonometric roots when the
 * discriminant is negative, Cardano otherwise; vapour takes the largest
 * root, liquid the smallest positive one.  compsim/Globals.cpp:212-264. */
double orc_solve_z(double a1, double a2, double a3, int gas) {
    double Q = (3 * a2 - a1 * a1) / 9;
    double J = (9 * a1 * a2 - 27 * a3 - 2 * a1 * a1 * a1) / 54;
    double D = Q * Q * Q + J * J;
    double Z;
    if (D < 0) {
        double s = 2 * sqrt(-Q);
        double a13 = a1 / 3;
        double t = acos(J / sqrt(-Q * Q * Q)) / 3;
        double r1 = s * cos(t) - a13;
        double r2 = s * cos(t + 2 * PI_C / 3) - a13;
        double r3 = s * cos(t + 4 * PI_C / 3) - a13;
        if (gas) {
            if ((r1 >= r2) && (r1 >= r3)) Z = r1;
            else if ((r2 >= r1) && (r2 >= r3)) Z = r2;
            else Z = r3;
        } else {
            if ((r1 <= r2) && (r1 <= r3) && (r1 > 0)) Z = r1;
            else if ((r2 <= r1) && (r2 <= r3) && (r2 > 0)) Z = r2;
            else Z = r3;
        }
    } else if (D == 0) {
        double t = (J > 0) ? pow(J, 1.0 / 3) : -pow(-J, 1.0 / 3);
        double r1 = 2 * t - a1 / 3;
        double r2 = -t - a1 / 3;
        if (gas) Z = (r2 >= r1) ? r2 : r1;
        else Z = ((r2 <= r1) && (r2 > 0)) ? r2 : r1;
    } else {
        double s = sqrt(D);
        double t = J + s;
        Z = (t > 0) ? pow(t, 1.0 / 3) : -pow(-t, 1.0 / 3);
        t = J - s;
        if (t > 0) Z += pow(t, 1.0 / 3);
        else Z -= pow(-t, 1.0 / 3);
        Z -= a1 / 3;
    }
    return Z;
}

/* a_i(T) and b_i for PR or SRK, compsim/Init_Calcs.cpp:81-96. */
void orc_eos_params(const orc_fluid *f, double T, double *a, double *b) {
    for (int i = 0; i < f->nc; i++) {
        double tc = f->tc[i], pc = f->pc[i], w = f->acf[i];
        double tr = T / tc;
        double ac, m;
        if (f->eos) {
            ac = 0.42747 * R_GAS * R_GAS * tc * tc / pc;
            m = 0.48508 + 1.55171 * w - 0.15613 * w * w;
            b[i] = 0.08664 * R_GAS * tc / pc;
        } else {
            ac = 0.457235 * R_GAS * R_GAS * tc * tc / pc;
            m = 0.3796 + 1.485 * w - 0.1644 * w * w + 0.01667 * w * w * w;
            b[i] = 0.077796 * R_GAS * tc / pc;
        }
        a[i] = ac * (1 + m * (1 - sqrt(tr))) * (1 + m * (1 - sqrt(tr)));
    }
}

/* sqrt(a_i a_j) (1 - k_ij), the mixing-rule table the reference evaluates
 * inline (compsim/Init_Calcs.cpp:641); bic = 1 - kij as the BIC keyword
 * stores it (compsim/Data_Input.cpp:985). */
static void mix_table(const orc_fluid *f, const double *a, double *aij) {
    int nc = f->nc;
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < nc; j++) aij[i * nc + j] = sqrt(a[i] * a[j]) * (1 - f->kij[i * nc + j]);
}

static void eos_uw(int eos, double B, double *U, double *W, double *d1, double *d2) {
    if (eos) { *U = B; *W = 0; *d1 = 1; *d2 = 0; }
    else { *U = 2 * B; *W = B; *d1 = 1 + SQRT_2; *d2 = 1 - SQRT_2; }
}

/* One cell of the reference's SuccFalsh (compsim/Init_Calcs.cpp:571-738). */
static void flash_cell(const orc_fluid *f, const double *a, const double *b, const double *aij, double P, double T,
                       const double *z, signed char *label, double *Lout, double *x, double *y, double *Zlo,
                       double *Zgo, int *iters, int *rr_iters) {
    int nc = f->nc;
    double K[ORC_MAX_NC];
    double L = 0, Lb = 10, ESum, Zl = 0, Zg = 0;
    int k = 0, rr_total = 0;
    const double RT = R_GAS * T;
    for (int i = 0; i < nc; i++)
        K[i] = (f->pc[i] / P) * exp(5.37 * (1 + f->acf[i]) * (1 - f->tc[i] / T));
    do {
        double t;
        int j = 0;
        L = 0.6;
        do { /* Rachford-Rice Newton, compsim/Init_Calcs.cpp:592-606 */
            double F = 0, dF = 0;
            for (int i = 0; i < nc; i++) {
                double td;
                if (K[i] >= 0) td = (1 - K[i]) / (L + (1 - L) * K[i]);
                else td = 1 / (L - 1);
                F += z[i] * td;
                dF -= z[i] * td * td;
            }
            t = F / dF;
            L -= t;
            j++;
        } while (((t * t) > RR_TOL) && (j < RR_MAXIT));
        rr_total += j;
        if (L > 1) L = 1;
        else if (L < 0) L = 0;
        ESum = fabs(Lb - L);
        Lb = L;
        for (int i = 0; i < nc; i++) {
            if (K[i] >= 0) {
                x[i] = z[i] / (L + K[i] * (1 - L));
                y[i] = K[i] * x[i];
            } else {
                x[i] = 0;
                y[i] = z[i] / (1 - L);
            }
        }
        double Al = 0, Bl = 0, Ag = 0, Bg = 0;
        for (int i = 0; i < nc; i++) {
            Bl += x[i] * b[i];
            Bg += y[i] * b[i];
            for (int jj = 0; jj < nc; jj++) {
                double s = aij[i * nc + jj];
                Al += x[i] * x[jj] * s;
                Ag += y[i] * y[jj] * s;
            }
        }
        double Cal = Al, Cbl = Bl, Cag = Ag, Cbg = Bg;
        Al *= P / (R_GAS * R_GAS * T * T);
        Bl *= P / (R_GAS * T);
        Ag *= P / (R_GAS * R_GAS * T * T);
        Bg *= P / (R_GAS * T);
        double Ul, Wl, Ug, Wg, d1, d2;
        eos_uw(f->eos, Bl, &Ul, &Wl, &d1, &d2);
        eos_uw(f->eos, Bg, &Ug, &Wg, &d1, &d2);
        Zl = orc_solve_z(-(1 + Bl - Ul), Al - Bl * Ul - Ul - Wl * Wl, -(Al * Bl - Bl * Wl * Wl - Wl * Wl), 0);
        Zg = orc_solve_z(-(1 + Bg - Ug), Ag - Bg * Ug - Ug - Wg * Wg, -(Ag * Bg - Bg * Wg * Wg - Wg * Wg), 1);
        /* terms of ln(phi_i) that do not depend on i (the reference
         * re-evaluates them per component with the same result) */
        double DDl = Al / (Bl * (d1 - d2)), DDg = Ag / (Bg * (d1 - d2));
        double FFl = log((Zl + d2 * Bl) / (Zl + d1 * Bl)), FFg = log((Zg + d2 * Bg) / (Zg + d1 * Bg));
        double LZBl = log(Zl - Bl), LZBg = log(Zg - Bg);
        for (int i = 0; i < nc; i++) {
            double tl = 0, tg = 0;
            for (int jj = 0; jj < nc; jj++) {
                tl += x[jj] * aij[i * nc + jj];
                tg += y[jj] * aij[i * nc + jj];
            }
            double t1l = b[i] / Cbl, t1g = b[i] / Cbg;
            double EEl = 2 * tl / Cal - t1l, EEg = 2 * tg / Cag - t1g;
            double phiL = exp(t1l * (Zl - 1) - LZBl + DDl * EEl * FFl);
            double phiG = exp(t1g * (Zg - 1) - LZBg + DDg * EEg * FFg);
            double fL = x[i] * phiL, fG = y[i] * phiG;
            if (z[i]) {
                if (fG) K[i] *= fL / fG;
                else K[i] = -1;
                if (fL != fL) K[i] = -1;
                if (fG != fG) K[i] = 1;
            }
        }
        k++;
    } while ((ESum > SS_TOL) && (k < SS_MAXIT));
    (void)RT;
    if (fabs(L) < L_ZERO) *label = -1;
    else if (fabs(1 - L) < L_ZERO) *label = 1;
    else *label = 0;
    *Lout = L;
    *Zlo = Zl;
    *Zgo = Zg;
    if (iters) *iters = k;
    if (rr_iters) *rr_iters = rr_total;
}

int orc_flash_batch(const orc_fluid *f, long n, const double *P, const double *T, const double *z,
                    signed char *label, double *L, double *x, double *y, double *Zl, double *Zg, int *iters,
                    int *rr_iters) {
    int nc = f->nc;
    if (nc < 1 || nc > ORC_MAX_NC) return -1;
    double a[ORC_MAX_NC], b[ORC_MAX_NC], aij[ORC_MAX_NC * ORC_MAX_NC];
    double lastT = -1;
    for (long c = 0; c < n; c++) {
        if (T[c] != lastT) {
            orc_eos_params(f, T[c], a, b);
            mix_table(f, a, aij);
            lastT = T[c];
        }
        double zc[ORC_MAX_NC], xc[ORC_MAX_NC], yc[ORC_MAX_NC], Lc, zl, zg;
        signed char lab;
        int it, rr;
        for (int i = 0; i < nc; i++) zc[i] = z[(long)i * n + c];
        flash_cell(f, a, b, aij, P[c], T[c], zc, &lab, &Lc, xc, yc, &zl, &zg, &it, &rr);
        if (label) label[c] = lab;
        if (L) L[c] = Lc;
        for (int i = 0; i < nc; i++) {
            if (x) x[(long)i * n + c] = xc[i];
            if (y) y[(long)i * n + c] = yc[i];
        }
        if (Zl) Zl[c] = zl;
        if (Zg) Zg[c] = zg;
        if (iters) iters[c] = it;
        if (rr_iters) rr_iters[c] = rr;
    }
    return 0;
}

/* ln(phi_i) and its derivatives for one phase, following the reference's
 * fugacity rows of the analytic Jacobian (compsim/Petsc_Functions.cpp:
 * 30243-30372) with dZ/dP and dZ/dw_k from the implicit derivative of the
 * cubic (compsim/Do_Cycle.cpp:517-552). */
static void fugacity_core(const orc_fluid *f, const double *b, const double *aij, double P, double T,
                          const double *w, double Z, double *lnphi, double *dx, double *dp) {
    int nc = f->nc;
    double Ca = 0, Cb = 0;
    for (int i = 0; i < nc; i++) {
        Cb += w[i] * b[i];
        for (int j = 0; j < nc; j++) Ca += w[i] * w[j] * aij[i * nc + j];
    }
    double A = Ca * (P / (R_GAS * R_GAS * T * T));
    double B = Cb * (P / (R_GAS * T));
    double dAdp = Ca / (R_GAS * R_GAS * T * T);
    double dBdp = Cb / (R_GAS * T);
    double U, W, d1, d2, dUdp, dWdp;
    eos_uw(f->eos, B, &U, &W, &d1, &d2);
    if (f->eos) { dUdp = dBdp; dWdp = 0; }
    else { dUdp = 2 * dBdp; dWdp = dBdp; }
    double den = 3 * Z * Z - 2 * Z * (1 + B - U) + A - B * U - U - W * W;
    double dZdp = -(dAdp * (Z - B) + dBdp * (-Z * Z - U * Z - A + W * W) + dUdp * (Z * Z - B * Z - Z) +
                    dWdp * (-2 * W * Z + 2 * B * W + 2 * W)) / den;
    double DD = A / (B * (d1 - d2));
    double FF = log((Z + d2 * B) / (Z + d1 * B));
    double dDDdp = (B * dAdp - A * dBdp) / (B * B * (d1 - d2));
    double dFFdp = (dZdp + d2 * dBdp) / (Z + d2 * B) - (dZdp + d1 * dBdp) / (Z + d1 * B);
    double dBBdp = (dBdp - dZdp) / (Z - B);
    double dAdx[ORC_MAX_NC], dBdx[ORC_MAX_NC], dZdx[ORC_MAX_NC];
    for (int k = 0; k < nc; k++) {
        double s = 0;
        for (int n = 0; n < nc; n++) s += w[n] * aij[k * nc + n];
        dAdx[k] = s * (2 * P / (R_GAS * R_GAS * T * T));
        dBdx[k] = b[k] * P / (R_GAS * T);
        double dUdx, dWdx;
        if (f->eos) { dUdx = dBdx[k]; dWdx = 0; }
        else { dUdx = 2 * dBdx[k]; dWdx = dBdx[k]; }
        dZdx[k] = -(dAdx[k] * (Z - B) + dBdx[k] * (-Z * Z - U * Z - A + W * W) + dUdx * (Z * Z - B * Z - Z) +
                    dWdx * (-2 * W * Z + 2 * B * W + 2 * W)) / den;
    }
    for (int i = 0; i < nc; i++) {
        double t = 0;
        for (int j = 0; j < nc; j++) t += w[j] * aij[i * nc + j];
        double t1 = b[i] / Cb;
        double EE = 2 * t / Ca - t1;
        if (lnphi) lnphi[i] = t1 * (Z - 1) - log(Z - B) + DD * EE * FF;
        if (dp) {
            double dAAdp = b[i] * dZdp / Cb;
            dp[i] = dAAdp + dBBdp + EE * (dDDdp * FF + DD * dFFdp);
        }
        if (dx) {
            for (int k = 0; k < nc; k++) {
                double dAA = -b[k] * b[i] * (Z - 1) / (Cb * Cb) + b[i] * dZdx[k] / Cb;
                double dBB = (dBdx[k] - dZdx[k]) / (Z - B);
                double dDD = (dAdx[k] * B - dBdx[k] * A) / (B * B * (d1 - d2));
                double dFF = (dZdx[k] + d2 * dBdx[k]) / (Z + d2 * B) - (dZdx[k] + d1 * dBdx[k]) / (Z + d1 * B);
                double dEE = 2 * (aij[i * nc + k] / Ca - dAdx[k] * (R_GAS * R_GAS * T * T) * t / (P * Ca * Ca)) +
                             b[i] * b[k] / (Cb * Cb);
                dx[i * nc + k] = dAA + dBB + dDD * EE * FF + DD * dEE * FF + DD * EE * dFF;
            }
        }
    }
}

void orc_fugacity(const orc_fluid *f, double P, double T, const double *w, double Z, double *lnphi,
                  double *dlnphi_dx, double *dlnphi_dP) {
    double a[ORC_MAX_NC], b[ORC_MAX_NC], aij[ORC_MAX_NC * ORC_MAX_NC];
    orc_eos_params(f, T, a, b);
    mix_table(f, a, aij);
    fugacity_core(f, b, aij, P, T, w, Z, lnphi, dlnphi_dx, dlnphi_dP);
}

int orc_flash_derivs_batch(const orc_fluid *f, long n, const double *P, const double *T, const double *x,
                           const double *y, const double *Zl, const double *Zg, double *dlnphi_dx,
                           double *dlnphi_dP) {
    int nc = f->nc;
    if (nc < 1 || nc > ORC_MAX_NC) return -1;
    double a[ORC_MAX_NC], b[ORC_MAX_NC], aij[ORC_MAX_NC * ORC_MAX_NC];
    double lastT = -1;
    long nn = (long)nc * nc;
    for (long c = 0; c < n; c++) {
        if (T[c] != lastT) {
            orc_eos_params(f, T[c], a, b);
            mix_table(f, a, aij);
            lastT = T[c];
        }
        for (int ph = 0; ph < 2; ph++) {
            const double *src = ph ? y : x;
            double w[ORC_MAX_NC], dx[ORC_MAX_NC * ORC_MAX_NC], dp[ORC_MAX_NC];
            for (int i = 0; i < nc; i++) w[i] = src[(long)i * n + c];
            fugacity_core(f, b, aij, P[c], T[c], w, ph ? Zg[c] : Zl[c], NULL, dx, dp);
            for (long e = 0; e < nn; e++) dlnphi_dx[((long)ph * nn + e) * n + c] = dx[e];
            for (int i = 0; i < nc; i++) dlnphi_dP[((long)ph * nc + i) * n + c] = dp[i];
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * Converged flash sensitivities (test infrastructure for the device
 * adjoint).  A two-phase cell's flash result u = (x, y, L) solves
 *   G_i = ln x_i + ln phi_i^L(x) - ln y_i - ln phi_i^V(y) = 0   (equal fugacity)
 *   H_i = z_i - L x_i - (1 - L) y_i = 0                        (material balance)
 *   S   = sum_i (x_i - y_i) = 0                                (Rachford-Rice)
 * to the reference's stopping tolerances (compsim/Init_Calcs.cpp:571-738).
 * orc_flash_polish solves these equations to rounding by Newton's method
 * from the flash's result, so that finite differences of its output are the
 * derivatives of the exact solution; orc_flash_adjoint restates the
 * implicit-function adjoint of the same equations. */

/* Gaussian elimination with partial pivoting on a row-major n x n system;
 * returns -1 when a pivot is exactly zero. */
static int solve_dense(int n, double *A, double *b) {
    for (int k = 0; k < n; k++) {
        int p = k;
        for (int i = k + 1; i < n; i++)
            if (fabs(A[i * n + k]) > fabs(A[p * n + k])) p = i;
        if (A[p * n + k] == 0) return -1;
        if (p != k) {
            for (int j = 0; j < n; j++) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
            double t = b[k]; b[k] = b[p]; b[p] = t;
        }
        for (int i = k + 1; i < n; i++) {
            double l = A[i * n + k] / A[k * n + k];
            if (l == 0) continue;
            for (int j = k; j < n; j++) A[i * n + j] -= l * A[k * n + j];
            b[i] -= l * b[k];
        }
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = b[i];
        for (int j = i + 1; j < n; j++) s -= A[i * n + j] * b[j];
        b[i] = s / A[i * n + i];
    }
    return 0;
}

/* Compressibility of one phase composition (the flash's root choice). */
static double phase_root(const orc_fluid *f, const double *b, const double *aij, double P, double T, const double *w,
                         int gas) {
    int nc = f->nc;
    double Ca = 0, Cb = 0;
    for (int i = 0; i < nc; i++) {
        Cb += w[i] * b[i];
        for (int j = 0; j < nc; j++) Ca += w[i] * w[j] * aij[i * nc + j];
    }
    double A = Ca * P / (R_GAS * R_GAS * T * T), B = Cb * P / (R_GAS * T);
    double U, W, d1, d2;
    eos_uw(f->eos, B, &U, &W, &d1, &d2);
    return orc_solve_z(-(1 + B - U), A - B * U - U - W * W, -(A * B - B * W * W - W * W), gas);
}

int orc_flash_polish(const orc_fluid *f, long n, const double *P, const double *T, const double *z,
                     const signed char *label, double *L, double *x, double *y, double *Zl, double *Zg) {
    int nc = f->nc, m = 2 * nc + 1, failed = 0;
    double a[ORC_MAX_NC], b[ORC_MAX_NC], aij[ORC_MAX_NC * ORC_MAX_NC];
    double lastT = -1;
    for (long c = 0; c < n; c++) {
        if (label[c] != 0) continue;
        if (T[c] != lastT) {
            orc_eos_params(f, T[c], a, b);
            mix_table(f, a, aij);
            lastT = T[c];
        }
        double u[2 * ORC_MAX_NC + 1];
        for (int i = 0; i < nc; i++) {
            u[i] = x[(long)i * n + c];
            u[nc + i] = y[(long)i * n + c];
        }
        u[2 * nc] = L[c];
        int ok = 0, extra = -1;   /* once the step is small, two more steps settle the last bits */
        for (int it = 0; it < 30 && !ok; it++) {
            double J[(2 * ORC_MAX_NC + 1) * (2 * ORC_MAX_NC + 1)] = {0}, r[2 * ORC_MAX_NC + 1];
            double lnl[ORC_MAX_NC], lng[ORC_MAX_NC], dxl[ORC_MAX_NC * ORC_MAX_NC], dxg[ORC_MAX_NC * ORC_MAX_NC];
            double zl = phase_root(f, b, aij, P[c], T[c], u, 0), zg = phase_root(f, b, aij, P[c], T[c], u + nc, 1);
            fugacity_core(f, b, aij, P[c], T[c], u, zl, lnl, dxl, NULL);
            fugacity_core(f, b, aij, P[c], T[c], u + nc, zg, lng, dxg, NULL);
            double Lc = u[2 * nc];
            for (int i = 0; i < nc; i++) {
                r[i] = -(log(u[i]) + lnl[i] - log(u[nc + i]) - lng[i]);
                r[nc + i] = -(z[(long)i * n + c] - Lc * u[i] - (1 - Lc) * u[nc + i]);
                for (int k = 0; k < nc; k++) {
                    J[i * m + k] = (i == k ? 1 / u[i] : 0) + dxl[i * nc + k];
                    J[i * m + nc + k] = -(i == k ? 1 / u[nc + i] : 0) - dxg[i * nc + k];
                }
                J[(nc + i) * m + i] = -Lc;
                J[(nc + i) * m + nc + i] = -(1 - Lc);
                J[(nc + i) * m + 2 * nc] = u[nc + i] - u[i];
                J[2 * nc * m + i] = 1;
                J[2 * nc * m + nc + i] = -1;
            }
            double s = 0;
            for (int i = 0; i < nc; i++) s += u[i] - u[nc + i];
            r[2 * nc] = -s;
            if (solve_dense(m, J, r)) break;
            double step = 0, size = 0;
            for (int q = 0; q < m; q++) {
                u[q] += r[q];
                step = fmax(step, fabs(r[q]));
                size = fmax(size, fabs(u[q]));
            }
            if (extra < 0 && step <= 1e-11 * fmax(size, 1e-300)) extra = 2;
            else if (extra > 0 && --extra == 0) ok = 1;
        }
        if (!ok) { failed++; continue; }
        for (int i = 0; i < nc; i++) {
            x[(long)i * n + c] = u[i];
            y[(long)i * n + c] = u[nc + i];
        }
        L[c] = u[2 * nc];
        Zl[c] = phase_root(f, b, aij, P[c], T[c], u, 0);
        Zg[c] = phase_root(f, b, aij, P[c], T[c], u + nc, 1);
    }
    return failed;
}

/* sum_i wt_i d ln(phi_i)/d k_mn for one phase, added into kbar[m nc + n]:
 * k_mn enters through sqrt(a_m a_n)(1 - k_mn) in the mixing sum and in the
 * i = m row of sum_j w_j a_ij, and Z follows A implicitly through the cubic. */
static void lnphi_kij_vjp(const orc_fluid *f, const double *a, const double *b, const double *aij, double P,
                          double T, const double *w, double Z, const double *wt, double *kbar) {
    int nc = f->nc;
    double Ca = 0, Cb = 0, t[ORC_MAX_NC];
    for (int i = 0; i < nc; i++) {
        Cb += w[i] * b[i];
        t[i] = 0;
        for (int j = 0; j < nc; j++) t[i] += w[j] * aij[i * nc + j];
        Ca += w[i] * t[i];
    }
    double pa = P / (R_GAS * R_GAS * T * T), A = Ca * pa, B = Cb * P / (R_GAS * T);
    double U, W, d1, d2;
    eos_uw(f->eos, B, &U, &W, &d1, &d2);
    double fp = 3 * Z * Z - 2 * Z * (1 + B - U) + A - B * U - U - W * W;
    double dZdA = -(Z - B) / fp;
    double DD = A / (B * (d1 - d2)), FF = log((Z + d2 * B) / (Z + d1 * B));
    double dFF = 1 / (Z + d2 * B) - 1 / (Z + d1 * B);
    double gZ = 0, gDD = 0, gCa = 0, gs[ORC_MAX_NC];
    for (int i = 0; i < nc; i++) {
        double t1 = b[i] / Cb, EE = 2 * t[i] / Ca - t1;
        gZ += wt[i] * (t1 - 1 / (Z - B) + DD * EE * dFF);
        gDD += wt[i] * FF * EE;
        gCa += wt[i] * DD * FF * (-2 * t[i] / (Ca * Ca));
        gs[i] = wt[i] * DD * FF * 2 / Ca;
    }
    gCa += gZ * dZdA * pa + gDD * DD / Ca;
    for (int p = 0; p < nc; p++)
        for (int q = 0; q < nc; q++) {
            double sq = sqrt(a[p] * a[q]);
            kbar[p * nc + q] -= gCa * w[p] * w[q] * sq + gs[p] * w[q] * sq;
        }
}

int orc_flash_adjoint(const orc_fluid *f, long n, const double *P, const double *T, const double *z,
                      const signed char *label, const double *L, const double *x, const double *y, const double *Zl,
                      const double *Zg, const double *xbar, const double *ybar, const double *Lbar, double *kij_bar,
                      double *z_bar, double *P_bar) {
    int nc = f->nc, m = nc + 1, singular = 0;
    double a[ORC_MAX_NC], b[ORC_MAX_NC], aij[ORC_MAX_NC * ORC_MAX_NC];
    double lastT = -1;
    for (int e = 0; e < nc * nc; e++) kij_bar[e] = 0;
    for (long c = 0; c < n; c++) {
        if (z_bar)
            for (int i = 0; i < nc; i++) z_bar[(long)i * n + c] = 0;
        if (P_bar) P_bar[c] = 0;
        if (label[c] != 0) {
            /* one phase: the present phase is the feed, nothing depends on k */
            if (z_bar)
                for (int i = 0; i < nc; i++)
                    z_bar[(long)i * n + c] = label[c] > 0 ? xbar[(long)i * n + c] : ybar[(long)i * n + c];
            continue;
        }
        if (T[c] != lastT) {
            orc_eos_params(f, T[c], a, b);
            mix_table(f, a, aij);
            lastT = T[c];
        }
        double xs[ORC_MAX_NC], ys[ORC_MAX_NC], dxl[ORC_MAX_NC * ORC_MAX_NC], dxg[ORC_MAX_NC * ORC_MAX_NC];
        double dpl[ORC_MAX_NC], dpg[ORC_MAX_NC], d[ORC_MAX_NC], xb[ORC_MAX_NC], yb[ORC_MAX_NC];
        int live[ORC_MAX_NC];
        for (int i = 0; i < nc; i++) {
            xs[i] = x[(long)i * n + c];
            ys[i] = y[(long)i * n + c];
            xb[i] = xbar[(long)i * n + c];
            yb[i] = ybar[(long)i * n + c];
            d[i] = ys[i] - xs[i];
            live[i] = xs[i] > 0 && ys[i] > 0;
        }
        double Lc = L[c];
        fugacity_core(f, b, aij, P[c], T[c], xs, Zl[c], NULL, dxl, dpl);
        fugacity_core(f, b, aij, P[c], T[c], ys, Zg[c], NULL, dxg, dpg);
        double M[(ORC_MAX_NC + 1) * (ORC_MAX_NC + 1)], r[ORC_MAX_NC + 1];
        double rN = Lbar[c];
        for (int k = 0; k < nc; k++) {
            double ck = 0;
            for (int i = 0; i < nc; i++) {
                double Ax = (i == k && live[i] ? 1 / xs[i] : 0) + dxl[k * nc + i];
                double Ay = (i == k && live[i] ? 1 / ys[i] : 0) + dxg[k * nc + i];
                M[i * m + k] = live[i] && live[k] ? (1 - Lc) * Ax + Lc * Ay : (i == k ? 1.0 : 0.0);
                ck += live[i] ? d[i] * (Ax - Ay) : 0;
            }
            M[k * m + nc] = live[k] ? 1.0 : 0.0;
            M[nc * m + k] = live[k] ? ck : 0.0;
            r[k] = live[k] ? (1 - Lc) * xb[k] - Lc * yb[k] : 0.0;
            rN += live[k] ? d[k] * (xb[k] + yb[k]) : 0;
        }
        M[nc * m + nc] = 0;
        r[nc] = rN;
        if (solve_dense(m, M, r)) { singular++; continue; }
        double wl[ORC_MAX_NC], wg[ORC_MAX_NC];
        double pb = 0;
        for (int i = 0; i < nc; i++) {
            double lg = live[i] ? r[i] : 0;
            wl[i] = -lg;
            wg[i] = lg;
            pb -= lg * (dpl[i] - dpg[i]);
            if (z_bar && live[i]) {
                /* lambda_H = (Dx + Phi_x^T - Dy - Phi_y^T) lambda_G - xbar - ybar */
                double lh = -xb[i] - yb[i] + r[i] / xs[i] - r[i] / ys[i];
                for (int k = 0; k < nc; k++)
                    if (live[k]) lh += (dxl[k * nc + i] - dxg[k * nc + i]) * r[k];
                z_bar[(long)i * n + c] = -lh;
            }
        }
        if (P_bar) P_bar[c] = pb;
        lnphi_kij_vjp(f, a, b, aij, P[c], T[c], xs, Zl[c], wl, kij_bar);
        lnphi_kij_vjp(f, a, b, aij, P[c], T[c], ys, Zg[c], wg, kij_bar);
    }
    return singular;
}
