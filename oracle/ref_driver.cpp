/* C entry points into the reference simulator compiled unmodified from its
 * own sources (test infrastructure only: oracle/_ref/libosiris_ref.so).
 *
 * Each entry point sets the reference's global state the way its own
 * initialisation does, calls the reference function, and copies the
 * results out into flat arrays.  Nothing here re-implements reference
 * arithmetic; the restated oracle lives in oracle/flash_oracle.c.
 *
 * Layout of the flat arrays (shared with the restated oracle and the CUDA
 * library): per-cell scalars are [n]; per-component fields are
 * component-major [nc][n]. */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include "Functions.h"

namespace {

int g_alloc_nc = -1;

/* Allocate the reference's global arrays for a 1x1x1 grid with nc
 * components, through the reference's own Allocation()
 * (compsim/Data_Input.cpp:1351).  Called once per component count. */
void ensure_single_cell(int nc) {
    if (g_alloc_nc == nc) return;
    Nx = Ny = Nz = 1;
    PNc = nc;
    UNc = 0;
    Nc = nc;
    Nswt = 2;
    Nsgt = 2;
    wellNO = 0;
    NOOptionsDB = 0;
    MPIsize = 1;
    MPIRank = 0;
    Allocation();
    g_alloc_nc = nc;
}

/* Component table and binary interaction: fluidProp columns as set by the
 * COMPNAME library (compsim/Data_Input.cpp:653-952), bic = 1 - kij as the
 * BIC keyword stores it (compsim/Data_Input.cpp:977-990). */
void set_fluid(int nc, int eos, const double *tc, const double *pc, const double *acf, const double *kij) {
    PR = (eos == 0);
    SRK = (eos != 0);
    for (int i = 0; i < nc; i++) {
        for (int c = 0; c < COMP_PROPS; c++) fluidProp[i][c] = 0;
        fluidProp[i][TCRIT] = tc[i];
        fluidProp[i][PCRIT] = pc[i];
        fluidProp[i][AC] = acf[i];
        fluidProp[i][MW] = 100.0;
        fluidProp[i][ZCRIT] = 0.28;
        for (int j = 0; j < nc; j++) bic[i][j] = 1 - kij[i * nc + j];
    }
}

/* EOS_Init divides VCRIT by 1e6 on every call (compsim/Init_Calcs.cpp:75),
 * so the driver restores it before each per-temperature call. */
void eos_at(int nc, double T) {
    for (int i = 0; i < nc; i++) fluidProp[i][VCRIT] = 300.0;
    resTemp = T;
    EOS_Init();
}

}  // namespace

extern "C" {

/* Flash n independent cells with the reference's SuccFalsh
 * (compsim/Init_Calcs.cpp:571-738): Wilson K, successive substitution with an
 * inner Rachford-Rice Newton, phase label from L.  Water saturation is 0, so
 * sat_o/sat_g are the hydrocarbon volume fractions.  kij is [nc][nc]. */
int ref_flash_batch(int nc, int eos, const double *tc, const double *pc, const double *acf, const double *kij,
                    long n, const double *P, const double *T, const double *z, double *x, double *y,
                    signed char *label, double *sat_o, double *sat_g, double *rho_o, double *rho_g) {
    if (nc < 1 || nc > 64) return -1;
    ensure_single_cell(nc);
    set_fluid(nc, eos, tc, pc, acf, kij);
    double lastT = -1;
    for (long c = 0; c < n; c++) {
        if (T[c] != lastT) {
            eos_at(nc, T[c]);
            lastT = T[c];
        }
        ::P[1][1][1][1] = P[c];
        sat[0][0][0][0] = 0;
        for (int i = 0; i < nc; i++) {
            comp[0][0][0][i][2] = z[(long)i * n + c];
            comp[0][0][0][i][0] = 0;
            comp[0][0][0][i][1] = 0;
        }
        SuccFalsh(0, 0, 0);
        for (int i = 0; i < nc; i++) {
            x[(long)i * n + c] = comp[0][0][0][i][0];
            y[(long)i * n + c] = comp[0][0][0][i][1];
        }
        label[c] = phaseStat[0][0][0];
        sat_o[c] = sat[0][0][0][1];
        sat_g[c] = sat[0][0][0][2];
        rho_o[c] = blockFProps[0][0][0][RO][0];
        rho_g[c] = blockFProps[0][0][0][RO][1];
    }
    return 0;
}

/* The reference's cubic root rule (compsim/Globals.cpp:212-264), exposed for
 * the root-selection tests. */
double ref_solve_z(double a1, double a2, double a3, int gas) { return Solve_Z(a1, a2, a3, gas ? 'g' : 'l'); }

/* EOS parameters a_i(T), b_i from the reference's EOS_Init
 * (compsim/Init_Calcs.cpp:66-97). */
int ref_eos_params(int nc, int eos, const double *tc, const double *pc, const double *acf, double T, double *a,
                   double *b) {
    if (nc < 1 || nc > 64) return -1;
    ensure_single_cell(nc);
    double zero[64 * 64] = {0};
    set_fluid(nc, eos, tc, pc, acf, zero);
    eos_at(nc, T);
    for (int i = 0; i < nc; i++) {
        a[i] = fluidProp[i][EOS_A];
        b[i] = fluidProp[i][EOS_B];
    }
    return 0;
}

}  // extern "C"
